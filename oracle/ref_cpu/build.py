"""Build the reference's own kernels.cu for the CPU into ``oracle/_ref/``.

Recipe (test infrastructure only): ``g++ -O2 -shared -fPIC`` over
``launch.cpp``, which includes ``kernels.cu`` from the reference tree where it
lies, with ``shim/`` standing in for ``<cupy/complex.cuh>`` and
``<math_constants.h>`` and ``shim/cuda_cpu.h`` force-included for the CUDA
built-ins.  Nothing from the reference tree is copied: the output is only the
shared library ``oracle/_ref/libref_kernels_cpu.so``.

Usage: ``python oracle/ref_cpu/build.py [--ref-root DIR]``.  When the
reference tree is absent the build is skipped (the library, if built before,
is used as is).
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(os.path.dirname(HERE), '_ref')
LIB = os.path.join(OUT_DIR, 'libref_kernels_cpu.so')
DEFAULT_REF = os.environ.get('RSPI_REFERENCE_ROOT', '/root/reference')


def build(ref_root=DEFAULT_REF, quiet=False):
    src = os.path.join(ref_root, 'kernels.cu')
    if not os.path.exists(src):
        if not quiet:
            print('reference tree absent: skipping the CPU build of kernels.cu')
        return LIB if os.path.exists(LIB) else None
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ['g++', '-O2', '-std=c++17', '-shared', '-fPIC', '-w',
           '-ffp-contract=off',
           '-I', os.path.join(HERE, 'shim'), '-I', ref_root,
           '-include', os.path.join(HERE, 'shim', 'cuda_cpu.h'),
           os.path.join(HERE, 'launch.cpp'), '-o', LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref-root', default=DEFAULT_REF)
    args = ap.parse_args()
    out = build(args.ref_root)
    print(out)
    sys.exit(0 if out else 1)
