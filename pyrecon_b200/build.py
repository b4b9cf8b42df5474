"""
Build libpyrecon_cuda.so in-tree (pyrecon_b200/lib/) with nvcc for sm_100a.

    python -m pyrecon_b200.build          # incremental
    python -m pyrecon_b200.build --force  # rebuild everything

Objects go to pyrecon_b200/_build/; the shared library is what travels with the tree.

Variants: the same library with some build-time knobs changed (VARIANTS), linked from a
rebuilt fft.cu and the regular objects into lib/libpyrecon_cuda_<name>.so.  The tests load
them in a subprocess (PRC_LIBRARY) to check that each variant computes the same bits.
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
SOURCES = ['cic.cu', 'fft.cu', 'multigrid.cu', 'misc.cu', 'tune.cu']
HEADERS = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cuh')) + \
    [os.path.join(ROOT, 'include', 'pyrecon_cuda.h')]

NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
         '--expt-relaxed-constexpr', '-I' + os.path.join(ROOT, 'include')]


# name -> (source rebuilt, extra nvcc flags).  'nopp': every TMA-fed FFT pass with two barriers per
# shared-memory exchange instead of the ping-pong buffers (same arithmetic, same order).
VARIANTS = {
    'nopp': ('fft.cu', ['-DPRC_STRIDED_PP=0', '-DPRC_KSPACE_PP=0', '-DPRC_HESS_PP=0', '-DPRC_C2R_PP=0']),
    # every radix-8 twiddle read from the pass table (7 loads per butterfly instead of 3 and 4 products)
    'twload': ('fft.cu', ['-DPRC_TW_RECUR=0']),
    # the z passes' row transforms with block barriers instead of warp barriers (same arithmetic, same order)
    'rowblock': ('fft.cu', ['-DPRC_ROW_WARP_SYNC=0']),
}


def library_path(variant=None):
    if variant is None:
        return os.path.join(LIBDIR, LIBNAME)
    return os.path.join(LIBDIR, 'libpyrecon_cuda_{}.so'.format(variant))


def _stale(target, deps):
    if not os.path.isfile(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra=(), obj=None):
    obj = obj or os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
    path = os.path.join(CSRC, src)
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + ['-c', path, '-o', obj]
    subprocess.run(cmd, check=True)
    return obj


def _link(lib, objs):
    subprocess.run([NVCC] + ARCH + ['-shared', '-o', lib] + objs + ['-cudart', 'static'], check=True)


def build(force=False, verbose=False, extra=(), variants=True):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    jobs = []          # (source, extra flags, object)
    objs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
        objs.append(obj)
        if force or _stale(obj, [os.path.join(CSRC, src)] + HEADERS):
            jobs.append((src, list(extra), obj))
    variant_objs = {}
    for name, (src, flags) in (VARIANTS.items() if variants else []):
        obj = os.path.join(BUILD, '{}_{}.o'.format(os.path.splitext(src)[0], name))
        variant_objs[name] = (src, obj)
        if force or _stale(obj, [os.path.join(CSRC, src)] + HEADERS):
            jobs.append((src, list(extra) + flags, obj))
    if jobs:
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            for _ in ex.map(lambda j: _compile(j[0], j[1], j[2]), jobs):
                pass
    lib = library_path()
    if force or jobs or _stale(lib, objs):
        _link(lib, objs)
        if verbose:
            print('built', lib)
    for name, (src, vobj) in variant_objs.items():
        vlib = library_path(name)
        base = os.path.splitext(src)[0] + '.o'
        vobjs = [vobj if os.path.basename(o) == base else o for o in objs]
        if force or _stale(vlib, vobjs):
            _link(vlib, vobjs)
            if verbose:
                print('built', vlib)
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
