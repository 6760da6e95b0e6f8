"""The C-ABI library loads and exports every entry point of include/rspi.h
(no GPU needed: only host-side calls)."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, 'include', 'rspi.h')


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(rspi_\w+)\s*\(', text)))


@pytest.fixture(scope='module')
def lib():
    from rspi import lib as rlib
    return rlib.load()


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert 'rspi_loglike' in syms and 'rspi_maxlp_pattern' in syms
    assert len(syms) >= 15


def test_every_declared_symbol_is_exported(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_bindings_cover_header():
    from rspi import lib as rlib
    assert sorted(rlib.SIGNATURES) == declared_symbols()


def test_version_and_status_strings(lib):
    assert lib.rspi_version().decode().startswith('rspi')
    assert lib.rspi_status_string(0).decode() == 'ok'
    assert 'argument' in lib.rspi_status_string(-1).decode()


def test_argument_errors_without_launch(lib):
    # bad sizes are rejected on the host before any launch
    assert lib.rspi_loglike_max_tile(24928, 1) == 1
    assert lib.rspi_loglike_max_tile(7392, 1) == 3
    assert lib.rspi_loglike_max_tile(10 ** 6, 1) == 0
    null = ctypes.c_void_p(0)
    assert lib.rspi_mean(null, 0, null, null) == -1
    assert lib.rspi_frame_reduce(null, 1, 0, 0, null, null, null, null) == -1


def test_bindings_match_header_argument_counts():
    """Every ctypes signature in rspi/lib.py has as many arguments as its
    declaration in include/rspi.h."""
    import re
    from rspi.lib import SIGNATURES
    with open(os.path.join(REPO, 'include', 'rspi.h')) as f:
        h = re.sub(r'/\*.*?\*/', '', f.read(), flags=re.S)
    seen = 0
    for m in re.finditer(r'\b(?:int|long long|const char \*)\s*(rspi_\w+)\s*\(([^)]*)\)\s*;', h):
        name, args = m.group(1), m.group(2).strip()
        n = 0 if args in ('', 'void') else len(args.split(','))
        assert name in SIGNATURES, name
        assert len(SIGNATURES[name][1]) == n, (name, len(SIGNATURES[name][1]), n)
        seen += 1
    assert seen == len(SIGNATURES)
