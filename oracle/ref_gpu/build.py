"""Build the reference's own kernels.cu for the GPU into ``oracle/_ref/``.

Recipe (test and baseline infrastructure only): ``nvcc -shared`` over
``launch.cu``, which includes ``kernels.cu`` from the reference tree where it
lies, with ``shim/`` standing in for ``<cupy/complex.cuh>`` (the toolkit
provides ``<math_constants.h>``).  Nothing from the reference tree is copied:
the output is only ``oracle/_ref/libref_kernels_gpu.so`` (sm_100a).

Usage: ``python oracle/ref_gpu/build.py [--ref-root DIR]``.  Without the
reference tree the build is skipped and a library built before is kept.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(os.path.dirname(HERE), '_ref')
LIB = os.path.join(OUT_DIR, 'libref_kernels_gpu.so')
DEFAULT_REF = os.environ.get('RSPI_REFERENCE_ROOT', '/root/reference')


def build(ref_root=DEFAULT_REF, quiet=False):
    src = os.path.join(ref_root, 'kernels.cu')
    if not os.path.exists(src):
        if not quiet:
            print('reference tree absent: skipping the GPU build of kernels.cu')
        return LIB if os.path.exists(LIB) else None
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [os.environ.get('NVCC', 'nvcc'), '-gencode', 'arch=compute_100a,code=sm_100a', '-O3',
           '-std=c++17', '-shared', '-Xcompiler', '-fPIC', '-cudart', 'static', '-w',
           '-I', os.path.join(HERE, 'shim'), '-I', ref_root,
           os.path.join(HERE, 'launch.cu'), '-o', LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref-root', default=DEFAULT_REF)
    args = ap.parse_args()
    out = build(args.ref_root)
    print(out)
    sys.exit(0 if out else 1)
