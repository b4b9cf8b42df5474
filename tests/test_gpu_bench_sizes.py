"""
Parity at the sizes the benchmarks run: the compile-time FFT instances for 128-512 points (TMA-fed
strided, k-space, Hessian and inverse-z passes, whose persistent grids re-arm their copy stages when
tiles outnumber resident CTAs) and the whole pipelines at nmesh 256 and 512 against the FP64 oracle.

Tolerances: shifted positions within 1e-6 Mpc/h of the FP64 oracle in the
all-FP64 mode ('f8'), within 1e-3 Mpc/h in the FP32 mode ('f4').  Every pipeline case prints its
density-contrast, displacement (psi or phi) and shifted-position errors.
"""
import os

import numpy as np
import pytest

from oracle import pipeline
from _util import maxrel, maxabs

pytestmark = pytest.mark.gpu

CORES = os.cpu_count() or 1


def _rfftn(x):
    import scipy.fft
    return scipy.fft.rfftn(x, workers=CORES)


def _fft_roundtrip(nmesh, dtype, seed=8):
    """(spectrum error, round-trip error) of prc_rfft3d / prc_irfft3d against scipy's FP64 rfftn."""
    import torch
    from pyrecon_b200 import _lib as L
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(nmesh, dtype='f8').astype(dtype)
    ref = _rfftn(x.astype('f8'))
    cdt = torch.complex64 if dtype == 'f4' else torch.complex128
    rdt = torch.float32 if dtype == 'f4' else torch.float64
    dx = torch.from_numpy(x).cuda()
    spec = torch.empty((nmesh[0], nmesh[1], nmesh[2] // 2 + 1), dtype=cdt, device='cuda')
    nm, st = L.i3(nmesh), L.stream_of(torch.device('cuda'))
    L.call('prc_rfft3d_' + L.suffix(dtype), L.ptr(dx), np.dtype(dtype).itemsize, L.ptr(spec), nm, st)
    got = spec.cpu().numpy()
    # relative to the largest mode (the zero mode of a standard normal field is ~sqrt(N))
    e_spec = float(np.abs(got - ref).max() / np.abs(ref).max())
    del got, ref
    back = torch.empty(nmesh, dtype=rdt, device='cuda')
    L.call('prc_irfft3d_' + L.suffix(dtype), L.ptr(spec), L.ptr(back), nm, st)
    e_back = maxrel(back.cpu().numpy(), x)
    assert L.load().prc_device_fault_flags(1) == 0
    return e_spec, e_back


# 96, 192 and 384 run the register kernels' radix-3 form (three sub-transforms and a radix-3 step)
FFT_SIZES = [(128, 128, 128), (192, 192, 192), (256, 256, 256), (384, 384, 384), (512, 512, 512), (512, 256, 128),
             (128, 512, 256), (96, 96, 96), (96, 384, 192), (384, 192, 96)]


@pytest.mark.parametrize('nmesh', FFT_SIZES)
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_fft_bench_sizes(nmesh, dtype):
    e_spec, e_back = _fft_roundtrip(nmesh, dtype)
    tol = 2e-6 if dtype == 'f4' else 1e-13
    print('fft {} {}: spectrum {:.2e}, round trip {:.2e}'.format(nmesh, dtype, e_spec, e_back))
    assert e_spec < tol and e_back < tol, (e_spec, e_back)


def _subprocess(code, **env):
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, '-c', "import sys; sys.path.insert(0, '.'); sys.path.insert(0, 'tests');" + code],
                         cwd=root, env=dict(os.environ, **env), capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-3000:]
    return res.stdout


def test_fft_bench_sizes_without_tma():
    """The register-prefetch strided passes (PRC_FFT_TMA=0) at the bench sizes."""
    _subprocess("import test_gpu_bench_sizes as T; "
                "[T.test_fft_bench_sizes(n, d) for n in [(256, 256, 256), (512, 256, 128), (384, 192, 96)] "
                "for d in ['f4', 'f8']]",
                PRC_FFT_TMA='0')


# ---------------------------------------------------------------------------------------------
# Whole pipelines against the FP64 oracle
# ---------------------------------------------------------------------------------------------

ALGOS = {'iterative_fft': 'IterativeFFTReconstruction', 'multigrid': 'MultiGridReconstruction',
         'plane_parallel_fft': 'PlaneParallelFFTReconstruction'}


def _catalogues(algorithm, nmesh, pos_dtype=None):
    """Seeded lognormal data and uniform randoms (a reduced count of the benchmark's catalogues, with
    randoms dense enough that no smoothed-randoms cell sits within rounding of the ran_min threshold,
    where FP32 and FP64 would mask it differently); multigrid takes FP64 positions and weights
    U[0.5, 1.5] as in its benchmark, the FFT algorithms FP32 positions and unit weights."""
    from pyrecon_b200 import mocks
    boxsize, boxcenter = 2000., 2000.
    pos_dtype = pos_dtype or ('f8' if algorithm == 'multigrid' else 'f4')
    nd, nr = (400_000, 1_600_000) if nmesh <= 256 else (2_000_000, 12_000_000)
    data = mocks.lognormal_positions_numpy(nd, nmesh, boxsize, boxcenter, seed=2100 + nmesh, field_seed=1100 + nmesh,
                                           dtype=pos_dtype)
    randoms = mocks.uniform_positions_numpy(nr, boxsize, boxcenter, seed=3100 + nmesh, dtype=pos_dtype)
    wd = wr = None
    if algorithm == 'multigrid':
        wd = mocks.weights_numpy(nd, seed=4100 + nmesh)
        wr = mocks.weights_numpy(nr, seed=4200 + nmesh)
    return dict(data=data, randoms=randoms, wdata=wd, wrandoms=wr, boxsize=boxsize, boxcenter=boxcenter)


def _los(algorithm):
    return 'z' if algorithm == 'plane_parallel_fft' else None


_ORACLE = {}


def _oracle(algorithm, nmesh, pos_dtype=None):
    """FP64 oracle (the reference's C kernels compiled from source with OpenMP when built, else the C
    restatement; pocketfft on all host cores) on the case's catalogues, positions as the GPU run reads
    them (rounded to `pos_dtype`); cached per case."""
    rounded = 'f4' if 'f4' in (pos_dtype, 'f8' if algorithm == 'multigrid' else 'f4') else 'f8'
    key = (algorithm, nmesh, rounded)
    if key not in _ORACLE:
        _ORACLE.clear()
        c = _catalogues(algorithm, nmesh)
        if pos_dtype is not None:
            c = dict(c, data=c['data'].astype(pos_dtype), randoms=c['randoms'].astype(pos_dtype))
        kernels = 'reference' if pipeline.reference_kernels_available() else 'oracle'
        rec = pipeline.OracleReconstruction(algorithm, f=0.8, bias=2., los=_los(algorithm), nmesh=nmesh,
                                            boxsize=c['boxsize'], boxcenter=c['boxcenter'], dtype='f8', kernels=kernels,
                                            fft_engine='scipy', nthreads=CORES)
        data, randoms = c['data'].astype('f8'), c['randoms'].astype('f8')
        rec.assign_data(data, c['wdata'])
        rec.assign_randoms(randoms, c['wrandoms'])
        rec.set_density_contrast(smoothing_radius=15.)
        out = dict(delta=rec.mesh_delta.copy())
        rec.run()
        if algorithm == 'multigrid':
            out['field'] = rec.mesh_phi
        else:
            out['field'] = np.stack(rec.mesh_psi)
        out['shifted_data'] = rec.read_shifted_positions(data)
        out['shifted_randoms'] = rec.read_shifted_positions(randoms)
        _ORACLE[key] = (c, out)
    return _ORACLE[key]


def _gpu(algorithm, nmesh, dtype, c, **kwargs):
    import pyrecon_b200
    Cls = getattr(pyrecon_b200, ALGOS[algorithm])
    rec = Cls(f=0.8, bias=2., los=_los(algorithm), nmesh=nmesh, boxsize=c['boxsize'], boxcenter=c['boxcenter'],
              dtype=dtype, **kwargs)
    data, randoms = c['data'].astype(dtype), c['randoms'].astype(dtype)
    rec.assign_data(data, c['wdata'])
    rec.assign_randoms(randoms, c['wrandoms'])
    rec.set_density_contrast(smoothing_radius=15.)
    out = dict(delta=np.asarray(rec.mesh_delta).copy())
    rec.run()
    if algorithm == 'multigrid':
        out['field'] = np.asarray(rec.mesh_phi)
    else:
        out['field'] = np.stack([np.asarray(p) for p in rec.mesh_psi])
    out['shifted_data'] = rec.read_shifted_positions(data)
    out['shifted_randoms'] = rec.read_shifted_positions(randoms)
    return out


PIPELINES = [('iterative_fft', 128, 'f4'), ('iterative_fft', 256, 'f4'), ('iterative_fft', 256, 'f8'),
             ('multigrid', 256, 'f4'), ('multigrid', 256, 'f8'), ('plane_parallel_fft', 256, 'f4'),
             ('plane_parallel_fft', 256, 'f8'), ('iterative_fft', 512, 'f4'), ('iterative_fft', 512, 'f8'),
             ('multigrid', 512, 'f4'), ('iterative_fft', 192, 'f8'), ('iterative_fft', 192, 'f4'),
             ('plane_parallel_fft', 192, 'f4'), ('iterative_fft', 384, 'f4')]


@pytest.mark.parametrize('algorithm,nmesh,dtype', PIPELINES)
def test_pipeline_against_fp64_oracle(algorithm, nmesh, dtype, record_property):
    c, ref = _oracle(algorithm, nmesh, pos_dtype=dtype)
    got = _gpu(algorithm, nmesh, dtype, c)
    errs = dict(delta=maxrel(got['delta'], ref['delta']), field=maxrel(got['field'], ref['field']),
                shifted_data_mpc=maxabs(got['shifted_data'], ref['shifted_data']),
                shifted_randoms_mpc=maxabs(got['shifted_randoms'], ref['shifted_randoms']))
    for k, v in errs.items():
        record_property(k, v)
    print('{} nmesh {} {}: delta {:.2e} (rel), {} {:.2e} (rel), shifted data {:.2e} / randoms {:.2e} Mpc/h'.format(
        algorithm, nmesh, dtype, errs['delta'], 'phi' if algorithm == 'multigrid' else 'psi', errs['field'],
        errs['shifted_data_mpc'], errs['shifted_randoms_mpc']))
    assert got['shifted_data'].dtype == np.dtype(dtype)
    tol = 1e-6 if dtype == 'f8' else 1e-3
    assert errs['shifted_data_mpc'] < tol and errs['shifted_randoms_mpc'] < tol, errs
    if dtype == 'f8':
        assert errs['delta'] < 1e-9 and errs['field'] < 1e-8, errs
    else:
        assert errs['delta'] < 1e-3 and errs['field'] < 2e-3, errs


def _gpu_outputs(path, algorithm, nmesh, dtype):
    """Run one pipeline on the GPU and save its outputs (called in a subprocess for library variants)."""
    c = _catalogues(algorithm, nmesh)
    np.savez(path, **_gpu(algorithm, nmesh, dtype, c))


def _fft_outputs(path, nmesh, dtype):
    import torch
    from pyrecon_b200 import _lib as L
    x = np.random.default_rng(8).standard_normal(nmesh, dtype='f8').astype(dtype)
    cdt = torch.complex64 if dtype == 'f4' else torch.complex128
    spec = torch.empty((nmesh[0], nmesh[1], nmesh[2] // 2 + 1), dtype=cdt, device='cuda')
    dx = torch.from_numpy(x).cuda()
    st = L.stream_of(torch.device('cuda'))
    L.call('prc_rfft3d_' + L.suffix(dtype), L.ptr(dx), np.dtype(dtype).itemsize, L.ptr(spec), L.i3(nmesh), st)
    back = torch.empty_like(dx)
    L.call('prc_irfft3d_' + L.suffix(dtype), L.ptr(spec.clone()), L.ptr(back), L.i3(nmesh), st)
    np.savez(path, spec=spec.cpu().numpy(), back=back.cpu().numpy())


@pytest.mark.parametrize('variant', ['nopp', 'rowblock'])
def test_library_variant_same_bits(variant, tmp_path):
    """The library built with the ping-pong exchanges switched off (two barriers per exchange), or with the
    z passes' row exchanges synchronised per block instead of per warp, gives the same bits as the default
    build on the nmesh-256 iterative pipeline and a 512^3 FFT round trip: the exchanges change only which
    shared-memory buffer a pass reads and which threads wait for it."""
    from pyrecon_b200 import build
    assert os.path.isfile(build.library_path(variant)), 'variant {} not built'.format(variant)
    for kind, args in [('pipeline', ('iterative_fft', 256, 'f4')), ('fft', ((512, 512, 512), 'f4'))]:
        path = str(tmp_path / '{}_{}.npz'.format(variant, kind))
        fn = '_gpu_outputs' if kind == 'pipeline' else '_fft_outputs'
        _subprocess('import test_gpu_bench_sizes as T; T.{}({!r}, *{!r})'.format(fn, path, args), PRC_LIBRARY=variant)
        ref = str(tmp_path / 'default_{}.npz'.format(kind))
        globals()[fn](ref, *args)
        a, b = np.load(path), np.load(ref)
        for k in b.files:
            assert np.array_equal(a[k], b[k]), (kind, k)


def _iterative_psi(nmesh, dtype, fuse):
    """psi of prc_iterative_fft (local line of sight, 3 iterations) with the inverse z pass handing its
    rows to the next forward z transform (fuse) or storing and reloading them."""
    import torch
    from pyrecon_b200 import _lib as L
    item = np.dtype(dtype).itemsize
    x = np.random.default_rng(11).standard_normal(nmesh, dtype='f8').astype(dtype)
    delta = torch.from_numpy(x).cuda()
    psi4 = torch.empty(tuple(nmesh) + (4,), dtype=delta.dtype, device='cuda')
    nm = L.i3(nmesh)
    ws = torch.empty(L.load().prc_iterative_fft_workspace_bytes(nm, item, 1), dtype=torch.uint8, device='cuda')
    psis = [L.c_void_p(psi4.data_ptr() + a * item) for a in range(3)]
    L.tune_set('fft_fuse_z', 0, int(fuse))
    try:
        L.call('prc_iterative_fft_' + L.suffix(dtype), L.ptr(delta), nm, L.d3([1000., 1200., 900.]),
               L.d3([0., 100., 2000.]), 0.4, None, 3, *psis, 4, L.ptr(ws), ws.numel(), L.stream_of(torch.device('cuda')))
        torch.cuda.synchronize()
    finally:
        L.tune_set('fft_fuse_z', 0, -1)
    assert L.load().prc_device_fault_flags(1) == 0
    return psi4.cpu().numpy()


@pytest.mark.parametrize('nmesh', [(256, 256, 256), (64, 32, 128), (32, 64, 16), (96, 192, 384)])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_fused_z_passes_same_bits(nmesh, dtype):
    """The local-line-of-sight iteration's inverse z pass transforms its new density rows forward at once
    (the next iteration's r2c z pass, the same arithmetic), instead of storing them and reading them back:
    the displacements are the same bits."""
    assert np.array_equal(_iterative_psi(nmesh, dtype, True), _iterative_psi(nmesh, dtype, False))
