"""
Build libpyrecon_cuda.so in-tree (pyrecon_b200/lib/) with nvcc for sm_100a.

    python -m pyrecon_b200.build          # incremental
    python -m pyrecon_b200.build --force  # rebuild everything

Objects go to pyrecon_b200/_build/; the shared library is what travels with the tree.
"""
import os
import sys
import subprocess
import argparse
import concurrent.futures

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIBDIR = os.path.join(HERE, 'lib')
LIBNAME = 'libpyrecon_cuda.so'
SOURCES = ['cic.cu', 'fft.cu', 'multigrid.cu', 'misc.cu']
HEADERS = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cuh')) + \
    [os.path.join(ROOT, 'include', 'pyrecon_cuda.h')]

NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
         '--expt-relaxed-constexpr', '-I' + os.path.join(ROOT, 'include')]


def library_path():
    return os.path.join(LIBDIR, LIBNAME)


def _stale(target, deps):
    if not os.path.isfile(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra=()):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
    path = os.path.join(CSRC, src)
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + ['-c', path, '-o', obj]
    subprocess.run(cmd, check=True)
    return obj


def build(force=False, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    todo = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
        objs.append(obj)
        if force or _stale(obj, [os.path.join(CSRC, src)] + HEADERS):
            todo.append(src)
    if todo:
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(todo)) as ex:
            for _ in ex.map(lambda s: _compile(s, extra), todo):
                pass
    lib = library_path()
    if force or todo or _stale(lib, objs):
        cmd = [NVCC] + ARCH + ['-shared', '-o', lib] + objs + ['-cudart', 'static']
        subprocess.run(cmd, check=True)
        if verbose:
            print('built', lib)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--ptxas-verbose', action='store_true', help='print register / shared memory use per kernel')
    args = ap.parse_args(argv)
    extra = ['-Xptxas', '-v'] if args.ptxas_verbose else []
    build(force=args.force or args.ptxas_verbose, verbose=True, extra=extra)


if __name__ == '__main__':
    sys.exit(main())
