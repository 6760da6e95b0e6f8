"""Build librspi.so (the sm_100a kernels behind include/rspi.h) in-tree.

``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` per source,
then one shared library with the CUDA runtime linked statically, written to
``refspi-maxlp_b200/rspi/librspi.so``.  Sources are rebuilt only when they
(or the headers) are newer than their object files.

Usage: ``python refspi-maxlp_b200/csrc/build.py [-v] [--force]``.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
INCLUDE = os.path.join(REPO, 'include')
OBJ_DIR = os.path.join(HERE, '_build')
LIB = os.path.join(PKG, 'rspi', 'librspi.so')
NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC',
         '-I', INCLUDE, '-I', HERE]


def _newer(src, dst, deps):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(f) > t for f in [src] + deps)


def build(verbose=False, force=False, ptxas_info=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(HERE, '*.cu')))
    deps = glob.glob(os.path.join(HERE, '*.cuh')) + glob.glob(os.path.join(INCLUDE, '*.h'))
    jobs = []
    for src in sources:
        obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + '.o')
        if force or ptxas_info or _newer(src, obj, deps):
            cmd = [NVCC] + ARCH + FLAGS + (['-Xptxas', '-v'] if ptxas_info else []) + \
                ['-c', src, '-o', obj]
            jobs.append((src, cmd))
    objs = [os.path.join(OBJ_DIR, os.path.basename(s)[:-3] + '.o') for s in sources]

    def run(job):
        src, cmd = job
        if verbose:
            print(' '.join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for src, r in ex.map(run, jobs):
            if r.returncode != 0 or (ptxas_info and r.stderr):
                sys.stderr.write(r.stderr)
            if r.returncode != 0:
                raise RuntimeError('nvcc failed on %s' % src)
    if jobs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ['-shared', '-cudart', 'static', '-o', LIB] + objs
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('-v', '--verbose', action='store_true')
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--ptxas-info', action='store_true')
    a = ap.parse_args()
    print(build(a.verbose, a.force, a.ptxas_info))
