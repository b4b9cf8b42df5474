"""
Kernel-level parity of libpyrecon_cuda.so against the CPU oracle, called through the C ABI.

Bit-exact: cell keys and their stable sort order, CIC gathers (same arithmetic, same order,
no FMA contraction).  FP64 sums: painted meshes to 1e-13 relative (order of summation only).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle import pipeline  # noqa: E402
from _util import maxrel  # noqa: E402


def torch():
    import torch as t
    return t


def dev(x):
    return torch().from_numpy(np.ascontiguousarray(x)).cuda()


def lib():
    from pyrecon_b200 import _lib
    return _lib


def stream():
    return lib().stream_of(torch().device('cuda'))


def flags():
    return torch().zeros(1, dtype=torch().int32, device='cuda')


def ws(nbytes):
    return torch().empty(max(int(nbytes), 256), dtype=torch().uint8, device='cuda')


def catalog(n, boxsize, boxcenter, seed=0, dtype='f8'):
    rng = np.random.default_rng(seed)
    return (np.asarray(boxcenter) + rng.uniform(-0.5, 0.5, (n, 3)) * np.asarray(boxsize)).astype(dtype)


@pytest.mark.parametrize('nmesh,npos,pos_dtype,mesh_dtype,wrap', [
    ((8, 8, 8), 200000, 'f8', 'f8', False),         # ~390 particles per cell: long runs of equal keys
    ((64, 48, 40), 300000, 'f4', 'f4', False),
    ((16, 12, 20), 50000, 'f4', 'f8', True),
    ((512, 512, 512), 100000, 'f8', 'f4', False),    # 27-bit keys: three 9-bit digit passes
])
def test_cell_order_bit_exact(nmesh, npos, pos_dtype, mesh_dtype, wrap):
    L = lib()
    boxsize, boxcenter = np.array([1000., 900., 800.]), np.array([100., -200., 3000.])
    pos = catalog(npos, boxsize * (1.3 if wrap else 1.), boxcenter, seed=1, dtype=pos_dtype)
    geom = pipeline.Geometry(nmesh, boxsize, boxcenter, dtype=mesh_dtype)
    key, order = pipeline.sorted_cell_order(pos, geom, wrap=wrap)
    t = torch()
    k = t.empty(npos, dtype=t.int32, device='cuda')
    o = t.empty(npos, dtype=t.int32, device='cuda')
    fl = flags()
    nm, bs, bc = L.i3(geom.nmesh), L.d3(geom.boxsize), L.d3(geom.boxcenter)
    w = ws(L.load().prc_assign_cic_workspace_bytes(nm, npos, np.dtype(mesh_dtype).itemsize))
    dpos = dev(pos)
    L.call('prc_cic_cell_order', L.ptr(k), L.ptr(o), nm, bs, bc, np.dtype(mesh_dtype).itemsize, L.ptr(dpos),
           np.dtype(pos_dtype).itemsize, npos, int(wrap), L.ptr(fl), L.ptr(w), w.numel(), stream())
    assert int(fl.item()) == 0
    np.testing.assert_array_equal(k.cpu().numpy().view(np.uint32).astype('i8'), key[order])
    np.testing.assert_array_equal(o.cpu().numpy().view(np.uint32).astype('i8'), order)


def _cell_order(pos, geom, wrap=False):
    L = lib()
    t = torch()
    npos = len(pos)
    k = t.empty(npos, dtype=t.int32, device='cuda')
    o = t.empty(npos, dtype=t.int32, device='cuda')
    fl = flags()
    nm, bs, bc = L.i3(geom.nmesh), L.d3(geom.boxsize), L.d3(geom.boxcenter)
    w = ws(L.load().prc_assign_cic_workspace_bytes(nm, npos, geom.dtype.itemsize))
    dpos = dev(pos)
    L.call('prc_cic_cell_order', L.ptr(k), L.ptr(o), nm, bs, bc, geom.dtype.itemsize, L.ptr(dpos),
           pos.dtype.itemsize, npos, int(wrap), L.ptr(fl), L.ptr(w), w.numel(), stream())
    assert int(fl.item()) == 0
    return k.cpu().numpy(), o.cpu().numpy()


@pytest.mark.parametrize('nmesh,npos', [
    ((8, 8, 8), 200000),           # few digits: long runs, every tile waits on the same digits
    ((512, 512, 512), 20_000_000), # the bench's randoms: 4883 tiles, three passes
    ((64, 48, 40), 4096),          # exactly one tile
    ((16, 12, 20), 4097),          # one item in the second tile
    ((100, 90, 80), 1),
])
def test_sort_one_sweep_equals_reduce_then_scan(nmesh, npos):
    """The paint's sort with one kernel per digit (tiles find their offsets by looking back over the tiles
    before them) gives the keys and the order of the reduce-then-scan passes (histogram, scan, scatter)."""
    L = lib()
    boxsize, boxcenter = np.array([1000., 900., 800.]), np.array([100., -200., 3000.])
    pos = catalog(npos, boxsize, boxcenter, seed=3, dtype='f4')
    geom = pipeline.Geometry(nmesh, boxsize, boxcenter, dtype='f4')
    one = _cell_order(pos, geom)
    L.tune_set('sort_onesweep', 0, 0)
    try:
        rts = _cell_order(pos, geom)
    finally:
        L.tune_set('sort_onesweep', 0, -1)
    np.testing.assert_array_equal(one[0], rts[0])
    np.testing.assert_array_equal(one[1], rts[1])


def gpu_paint(pos, weights, geom, wrap=False, accumulate_into=None):
    L = lib()
    t = torch()
    n = geom.shape
    mesh = accumulate_into if accumulate_into is not None else t.zeros(n, dtype=t.float64, device='cuda')
    colsums = t.zeros(n[0] * n[1], dtype=t.float64, device='cuda')
    fl = flags()
    nm, bs, bc = L.i3(geom.nmesh), L.d3(geom.boxsize), L.d3(geom.boxcenter)
    w = ws(L.load().prc_assign_cic_workspace_bytes(nm, len(pos), geom.dtype.itemsize))
    wt = dev(weights) if weights is not None else None
    dpos = dev(pos) if len(pos) else None
    L.call('prc_assign_cic', L.ptr(mesh), L.ptr(colsums), nm, bs, bc, geom.dtype.itemsize, L.ptr(dpos),
           pos.dtype.itemsize, L.ptr(wt), 0 if weights is None else weights.dtype.itemsize, len(pos), int(wrap),
           int(accumulate_into is not None), L.ptr(fl), L.ptr(w), w.numel(), stream())
    return mesh, colsums, int(fl.item())


@pytest.mark.parametrize('mesh_dtype', ['f4', 'f8'])
def test_paint_matches_oracle(mesh_dtype):
    boxsize, boxcenter = 1000., 0.
    geom = pipeline.Geometry((16, 12, 20), boxsize, boxcenter, dtype=mesh_dtype)
    pos = catalog(100000, [boxsize] * 3, [boxcenter] * 3, seed=2, dtype=mesh_dtype)
    pos[0] = [500., -500., 500.]          # exactly on the upper / lower faces: index == n and 0
    weights = np.random.default_rng(3).uniform(0.5, 1.5, len(pos)).astype(mesh_dtype)
    ref = np.zeros(geom.shape, dtype='f8')
    k = pipeline._Kernels('f8')
    k.assign_cic(ref, geom.nmesh, geom.to_index(pos).astype('f8'), weights.astype('f8'))
    mesh, colsums, fl = gpu_paint(pos, weights, geom)
    assert fl == 0
    m = mesh.cpu().numpy()
    tol = 1e-13 if mesh_dtype == 'f8' else 1e-6   # f4: CIC fractions computed in float, as the reference does
    assert maxrel(m, ref) < tol
    np.testing.assert_allclose(colsums.cpu().numpy().reshape(m.shape[:2]), m.sum(axis=2), rtol=1e-12, atol=1e-9)
    # deterministic: a second run gives the same bits
    mesh2, _, _ = gpu_paint(pos, weights, geom)
    assert torch().equal(mesh, mesh2)
    # accumulation over two calls equals one call over both halves (up to FP64 rounding)
    half = len(pos) // 2
    acc, _, _ = gpu_paint(pos[:half], weights[:half], geom)
    acc, _, _ = gpu_paint(pos[half:], weights[half:], geom, accumulate_into=acc)
    assert maxrel(acc.cpu().numpy(), m) < 1e-13


def test_paint_empty_and_unit_weights():
    geom = pipeline.Geometry(8, 100., 0.)
    mesh, colsums, fl = gpu_paint(np.zeros((0, 3)), None, geom)
    assert fl == 0 and float(mesh.abs().sum()) == 0.
    pos = catalog(1000, [100.] * 3, [0.] * 3, seed=4)
    mesh, _, _ = gpu_paint(pos, None, geom)
    assert abs(float(mesh.sum()) - 1000.) < 1e-9


def test_paint_flags_leave_mesh_untouched():
    geom = pipeline.Geometry(8, 100., 0.)
    pos = catalog(1000, [100.] * 3, [0.] * 3, seed=5)
    t = torch()
    base = t.full(geom.shape, 7., dtype=t.float64, device='cuda')
    bad = pos.copy()
    bad[10, 1] = 60.                     # outside [-50, 50]
    mesh, _, fl = gpu_paint(bad, None, geom, accumulate_into=base.clone())
    assert fl & lib().PRC_FLAG_OUT_OF_BOX
    assert torch().equal(mesh, base)
    bad = pos.copy()
    bad[3, 0] = np.nan
    mesh, _, fl = gpu_paint(bad, None, geom, wrap=True, accumulate_into=base.clone())
    assert fl & lib().PRC_FLAG_NONFINITE
    assert torch().equal(mesh, base)


def test_paint_flags_zero_a_fresh_mesh():
    """A non-accumulating paint of a bad catalogue writes zeros over whatever the buffer held."""
    geom = pipeline.Geometry(8, 100., 0.)
    pos = catalog(1000, [100.] * 3, [0.] * 3, seed=5)
    pos[10, 1] = 60.
    L, t = lib(), torch()
    n = geom.shape
    mesh = t.full(n, 7., dtype=t.float64, device='cuda')
    colsums = t.full((n[0] * n[1],), 3., dtype=t.float64, device='cuda')
    fl = flags()
    nm, bs, bc = L.i3(geom.nmesh), L.d3(geom.boxsize), L.d3(geom.boxcenter)
    w = ws(L.load().prc_assign_cic_workspace_bytes(nm, len(pos), 8))
    dpos = dev(pos)
    L.call('prc_assign_cic', L.ptr(mesh), L.ptr(colsums), nm, bs, bc, 8, L.ptr(dpos), 8, None, 0, len(pos), 0, 0,
           L.ptr(fl), L.ptr(w), w.numel(), stream())
    assert int(fl.item()) & L.PRC_FLAG_OUT_OF_BOX
    assert float(mesh.abs().max()) == 0. and float(colsums.abs().max()) == 0.


@pytest.mark.parametrize('mesh_dtype,pos_dtype', [('f8', 'f8'), ('f4', 'f4'), ('f4', 'f8')])
def test_gathers_bit_exact(mesh_dtype, pos_dtype):
    L = lib()
    geom = pipeline.Geometry((16, 12, 20), 1000., 0., dtype=mesh_dtype)
    rng = np.random.default_rng(6)
    mesh = rng.standard_normal(geom.shape).astype(mesh_dtype)
    pos = catalog(20000, [1000.] * 3, [0.] * 3, seed=7, dtype=pos_dtype)
    k = pipeline._Kernels(mesh_dtype)
    idx = geom.to_index(pos)
    ref_read = k.read_cic(mesh, geom.nmesh, idx).astype(pos_dtype)
    ref_fd = k.read_finite_difference_cic(mesh, geom.nmesh, geom.boxsize, idx).astype(pos_dtype)
    t = torch()
    out = t.empty(len(pos), dtype=t.float32 if pos_dtype == 'f4' else t.float64, device='cuda')
    out3 = t.empty((len(pos), 3), dtype=out.dtype, device='cuda')
    fl = flags()
    nm, bs, bc = L.i3(geom.nmesh), L.d3(geom.boxsize), L.d3(geom.boxcenter)
    sfx = L.suffix(mesh_dtype)
    dm, dp = dev(mesh), dev(pos)
    L.call('prc_read_cic_' + sfx, L.ptr(dm), nm, bs, bc, L.ptr(dp), pos.dtype.itemsize, len(pos), 0, L.ptr(out), L.ptr(fl), stream())
    L.call('prc_read_finite_difference_cic_' + sfx, L.ptr(dm), nm, bs, bc, L.ptr(dp), pos.dtype.itemsize, len(pos), 0,
           L.ptr(out3), L.ptr(fl), stream())
    np.testing.assert_array_equal(out.cpu().numpy(), ref_read)
    np.testing.assert_array_equal(out3.cpu().numpy(), ref_fd)


@pytest.mark.parametrize('nmesh', [(8, 8, 8), (16, 12, 20), (18, 14, 10), (64, 64, 64), (96, 48, 24), (7, 5, 6)])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_fft_against_numpy(nmesh, dtype):
    L = lib()
    t = torch()
    rng = np.random.default_rng(8)
    x = rng.standard_normal(nmesh).astype(dtype)
    ref = np.fft.rfftn(x.astype('f8'))
    cdt = t.complex64 if dtype == 'f4' else t.complex128
    spec = t.empty((nmesh[0], nmesh[1], nmesh[2] // 2 + 1), dtype=cdt, device='cuda')
    nm = L.i3(nmesh)
    sfx = L.suffix(dtype)
    dx = dev(x)
    L.call('prc_rfft3d_' + sfx, L.ptr(dx), np.dtype(dtype).itemsize, L.ptr(spec), nm, stream())
    tol = 1e-5 if dtype == 'f4' else 1e-13
    assert maxrel(spec.cpu().numpy(), ref) < tol
    back = t.empty(nmesh, dtype=t.float32 if dtype == 'f4' else t.float64, device='cuda')
    L.call('prc_irfft3d_' + sfx, L.ptr(spec), L.ptr(back), nm, stream())
    assert maxrel(back.cpu().numpy(), x) < tol


def test_fft_supported_sizes():
    L = lib()
    assert L.load().prc_fft_supported(L.i3((16, 16, 16))) == 1
    assert L.load().prc_fft_supported(L.i3((11, 16, 16))) == 1     # prime factor 11
    assert L.load().prc_fft_supported(L.i3((16, 16, 15))) == 1     # odd last axis
    assert L.load().prc_fft_supported(L.i3((2048, 16, 16))) == 1   # above the register kernels' 1024
    assert L.load().prc_fft_supported(L.i3((2049, 16, 16))) == 0   # above 2048
    assert L.load().prc_fft_supported(L.i3((16, 1, 16))) == 0


@pytest.mark.parametrize('nmesh', [(13, 11, 9), (17, 19, 23), (125, 125, 125), (1021, 4, 6), (6, 4, 1021),
                                   (2048, 8, 8), (8, 6, 2048), (9, 2046, 5), (3, 2, 3), (22, 26, 34)])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_fft_any_size_against_numpy(nmesh, dtype):
    """Every axis length the reference's FFT engines take (up to 2048): prime factors above 7 by direct
    summation, odd last axes as full-length transforms, powers of two above 1024 on the shared-memory kernels."""
    L = lib()
    t = torch()
    rng = np.random.default_rng(18)
    x = rng.standard_normal(nmesh).astype(dtype)
    ref = np.fft.rfftn(x.astype('f8'))
    cdt = t.complex64 if dtype == 'f4' else t.complex128
    spec = t.empty((nmesh[0], nmesh[1], nmesh[2] // 2 + 1), dtype=cdt, device='cuda')
    nm = L.i3(nmesh)
    dx = dev(x)
    L.call('prc_rfft3d_' + L.suffix(dtype), L.ptr(dx), np.dtype(dtype).itemsize, L.ptr(spec), nm, stream())
    tol = 5e-5 if dtype == 'f4' else 1e-12
    got = spec.cpu().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() < tol
    back = t.empty(nmesh, dtype=t.float32 if dtype == 'f4' else t.float64, device='cuda')
    L.call('prc_irfft3d_' + L.suffix(dtype), L.ptr(spec), L.ptr(back), nm, stream())
    assert maxrel(back.cpu().numpy(), x) < tol


@pytest.mark.parametrize('los', [None, [0., 0., 1.], [0.3, -0.5, 0.8]])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_multigrid_components(los, dtype):
    L = lib()
    t = torch()
    n = (16, 12, 20)
    boxsize, boxcenter, beta = np.array([800., 600., 1000.]), np.array([1600., 0., 300.]), 0.4
    if los is not None:
        los = np.asarray(los) / np.linalg.norm(los)
    rng = np.random.default_rng(9)
    v = rng.standard_normal(n).astype(dtype)
    f = rng.standard_normal(n).astype(dtype)
    lib_o = pipeline._Kernels(dtype)._mesh
    import ctypes
    from numpy import ctypeslib
    ct = ctypeslib.as_ctypes_type(np.dtype(dtype))
    arr = lambda a: np.ascontiguousarray(a, dtype=dtype)
    nn = np.array(n, dtype='i8')
    losp = None if los is None else arr(los).ctypes.data_as(ctypes.POINTER(ct))
    # residual
    r_ref = np.empty(n, dtype=dtype)
    fn = lib_o.oracle_mg_residual
    fn.argtypes = None
    fn(arr(v).ctypes.data_as(ctypes.c_void_p), arr(f).ctypes.data_as(ctypes.c_void_p), r_ref.ctypes.data_as(ctypes.c_void_p),
       nn.ctypes.data_as(ctypes.c_void_p), arr(boxsize).ctypes.data_as(ctypes.c_void_p),
       arr(boxcenter).ctypes.data_as(ctypes.c_void_p), ct(beta), losp)
    sfx = L.suffix(dtype)
    r = t.empty(n, dtype=t.float32 if dtype == 'f4' else t.float64, device='cuda')
    los_arg = L.opt_d3(None if los is None else list(arr(los)))
    dv0, df = dev(v), dev(f)     # keep the device copies alive until the kernels have run
    L.call('prc_mg_residual_' + sfx, L.ptr(dv0), L.ptr(df), L.ptr(r), L.i3(n), L.d3(boxsize), L.d3(boxcenter),
           beta, los_arg, stream())
    tol = 1e-12 if dtype == 'f8' else 2e-5
    assert maxrel(r.cpu().numpy(), r_ref) < tol
    # jacobi, 3 sweeps
    vj = arr(v).copy()
    fn = lib_o.oracle_mg_jacobi
    fn(vj.ctypes.data_as(ctypes.c_void_p), arr(f).ctypes.data_as(ctypes.c_void_p), nn.ctypes.data_as(ctypes.c_void_p),
       arr(boxsize).ctypes.data_as(ctypes.c_void_p), arr(boxcenter).ctypes.data_as(ctypes.c_void_p), ct(beta), ct(0.4),
       ctypes.c_int(3), losp)
    dv = dev(v)
    scratch = t.empty_like(dv)
    L.call('prc_mg_jacobi_' + sfx, L.ptr(dv), L.ptr(df), L.ptr(scratch), L.i3(n), L.d3(boxsize), L.d3(boxcenter),
           beta, 0.4, 3, los_arg, stream())
    assert maxrel(dv.cpu().numpy(), vj) < tol
    # reduce / prolong
    c_ref = np.empty((8, 6, 10), dtype=dtype)
    lib_o.oracle_mg_reduce(arr(v).ctypes.data_as(ctypes.c_void_p), c_ref.ctypes.data_as(ctypes.c_void_p),
                           nn.ctypes.data_as(ctypes.c_void_p))
    c = t.empty((8, 6, 10), dtype=r.dtype, device='cuda')
    L.call('prc_mg_reduce_' + sfx, L.ptr(dv0), L.ptr(c), L.i3(n), stream())
    assert maxrel(c.cpu().numpy(), c_ref) < tol
    p_ref = np.empty(n, dtype=dtype)
    nc = np.array([8, 6, 10], dtype='i8')
    lib_o.oracle_mg_prolong(c_ref.ctypes.data_as(ctypes.c_void_p), p_ref.ctypes.data_as(ctypes.c_void_p),
                            nc.ctypes.data_as(ctypes.c_void_p))
    pr = t.empty(n, dtype=r.dtype, device='cuda')
    dc = dev(c_ref)
    L.call('prc_mg_prolong_' + sfx, L.ptr(dc), L.ptr(pr), L.i3((8, 6, 10)), stream())
    assert maxrel(pr.cpu().numpy(), p_ref) < tol


@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_prod_sum(dtype):
    L = lib()
    rng = np.random.default_rng(10)
    shape = (4, 3, 10)
    mesh = rng.uniform(0.5, 1.5, shape).astype(dtype)
    coords = rng.uniform(1., 2., sum(shape)).astype(dtype)
    ref = mesh.copy()
    pipeline._Kernels(dtype).prod_sum(ref.reshape(-1), shape, coords, -1)
    d, dc = dev(mesh), dev(coords)
    L.call('prc_prod_sum_' + L.suffix(dtype), L.ptr(d), L.i3(shape), L.ptr(dc), -1, stream())
    assert maxrel(d.cpu().numpy(), ref) < (1e-15 if dtype == 'f8' else 1e-6)


def test_sum_deterministic():
    L = lib()
    t = torch()
    x = t.randn(1000003, dtype=t.float64, device='cuda')
    out = t.empty(2, dtype=t.float64, device='cuda')
    w = ws(L.load().prc_sum_workspace_bytes(x.numel()))
    L.call('prc_sum_f64', L.ptr(x), x.numel(), L.ptr(out), L.ptr(w), w.numel(), stream())
    L.call('prc_sum_f64', L.ptr(x), x.numel(), L.c_void_p(out.data_ptr() + 8), L.ptr(w), w.numel(), stream())
    o = out.cpu().numpy()
    assert o[0] == o[1]
    assert abs(o[0] - x.double().sum().item()) < 1e-9


def _smooth(dtype, mesh, nmesh, boxsize, radius):
    L = lib()
    t = torch()
    nm = L.i3(nmesh)
    w = ws(L.load().prc_fft_workspace_bytes(nm, np.dtype(dtype).itemsize, 1))
    out = t.empty(nmesh, dtype=t.float32 if dtype == 'f4' else t.float64, device='cuda')
    L.call('prc_smooth_gaussian_' + L.suffix(dtype), L.ptr(mesh), mesh.element_size(), L.ptr(out), nm,
           L.d3(boxsize), L.d3(radius), L.ptr(w), w.numel(), stream())
    return out.double().cpu().numpy()


@pytest.mark.parametrize('nmesh', [(16, 16, 16), (32, 32, 32), (64, 32, 16), (24, 20, 18)])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
@pytest.mark.parametrize('randoms', [True, False])
def test_density_contrast_batched(nmesh, dtype, randoms):
    """Data and randoms smoothed in one batched pass equal two separate smoothings + the formula
    of set_density_contrast (pyrecon/recon.py:227-247)."""
    L = lib()
    t = torch()
    rng = np.random.default_rng(11)
    md = dev(rng.uniform(0.5, 1.5, nmesh))
    mr = dev(rng.uniform(0.2, 1.8, nmesh))
    sums = t.tensor([float(md.sum()), float(mr.sum())], dtype=t.float64, device='cuda')
    boxsize, radius, bias, ran_min = [800., 700., 600.], [30.] * 3, 2., 0.01
    ncell = int(np.prod(nmesh))
    size_randoms = ran_min * float(mr.sum()) / 1.0   # threshold = 1.0: about half the cells masked
    nm = L.i3(nmesh)
    w = ws(L.load().prc_density_contrast_workspace_bytes(nm, np.dtype(dtype).itemsize, int(randoms)))
    delta = t.empty(nmesh, dtype=t.float32 if dtype == 'f4' else t.float64, device='cuda')
    L.call('prc_density_contrast_' + L.suffix(dtype), L.ptr(md), L.ptr(mr) if randoms else None, L.ptr(sums), nm,
           L.d3(boxsize), L.d3(radius), bias, ran_min, size_randoms, L.ptr(delta), L.ptr(w), w.numel(), stream())
    got = delta.double().cpu().numpy()
    d = _smooth(dtype, md, nmesh, boxsize, radius)
    s = sums.cpu().numpy()
    if randoms:
        r = _smooth(dtype, mr, nmesh, boxsize, radius)
        alpha = s[0] / s[1]
        threshold = ran_min * s[1] / size_randoms
        mask = r > threshold
        assert 0.1 < mask.mean() < 0.9
        ref = np.where(mask, (d - alpha * r) / (bias * alpha * np.where(mask, r, 1.)), 0.)
        ok = np.abs(r - threshold) > 1e-4      # cells on the threshold may flip between precisions
    else:
        ref = (d / (s[0] / ncell) - 1.) / bias
        ok = np.ones(nmesh, dtype=bool)
    tol = 2e-5 if dtype == 'f4' else 1e-12
    assert np.abs(got - ref)[ok].max() < tol * max(np.abs(ref).max(), 1.)


def test_generic_fft_path_on_power_of_two_sizes():
    """The mixed-radix kernels also serve power-of-two sizes when forced (PRC_FFT_GENERIC=1)."""
    import subprocess
    import sys
    import os
    code = ("import sys; sys.path.insert(0, '.'); sys.path.insert(0, 'tests');"
            "import test_gpu_kernels as T; T.test_fft_against_numpy((64, 32, 16), 'f4'); "
            "T.test_fft_against_numpy((16, 16, 16), 'f8'); T.test_density_contrast_batched((32, 32, 32), 'f4', True)")
    env = dict(os.environ, PRC_FFT_GENERIC='1')
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, '-c', code], cwd=root, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr


def test_register_fft_path_without_tma():
    """PRC_FFT_TMA=0 keeps the register-prefetch strided and k-space kernels (the ones user-laid-out
    FP32 spectra with odd rows always take) checked on the composite entry points too."""
    import subprocess
    import sys
    import os
    code = ("import sys; sys.path.insert(0, '.'); sys.path.insert(0, 'tests');"
            "import test_gpu_kernels as T; T.test_fft_against_numpy((16, 16, 16), 'f8'); "
            "T.test_density_contrast_batched((32, 32, 32), 'f4', True); "
            "T.test_density_contrast_batched((64, 32, 16), 'f8', True)")
    env = dict(os.environ, PRC_FFT_TMA='0')
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, '-c', code], cwd=root, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr


def test_no_device_faults_after_kernels():
    """The FFT kernels' bounded waits never ran out in this process."""
    from pyrecon_b200 import _lib
    import torch
    torch.cuda.synchronize()
    assert _lib.load().prc_device_fault_flags(0) == 0


def test_bounded_wait_gives_up_and_is_reported():
    """The failure path of the bounded barrier waits, without a GPU fault: a barrier armed for bytes that
    no copy delivers (none is issued) makes the wait run out after 2 ms; the kernel sets the fault bit
    and returns, the next read-out of a reconstruction raises ReconstructionError (clearing the word),
    and the context stays usable: the read-out after it succeeds with the same result as before."""
    import time
    import pyrecon_b200
    from pyrecon_b200 import _lib as L
    t = torch()
    assert L.load().prc_device_fault_flags(1) == 0
    out = t.zeros(1, dtype=t.int32, device='cuda')
    t0 = time.perf_counter()
    L.call('prc_debug_wait_timeout', 2_000_000, L.ptr(out), stream())
    t.cuda.synchronize()
    assert time.perf_counter() - t0 < 5.
    assert int(out.item()) == 1
    assert L.load().prc_device_fault_flags(0) & L.PRC_FAULT_WAIT_TIMEOUT
    assert L.load().prc_debug_wait_timeout(0, L.ptr(out), stream()) == L.PRC_ERR_ARG
    pos = catalog(5000, [1000.] * 3, [2000.] * 3, seed=12)
    rec = pyrecon_b200.IterativeFFTReconstruction(f=0.8, bias=2., nmesh=16, boxsize=1000., boxcenter=2000., dtype='f8')
    rec.assign_data(pos)
    rec.set_density_contrast(smoothing_radius=15.)
    rec.run()
    with pytest.raises(pyrecon_b200.ReconstructionError):
        rec.read_shifted_positions(pos)
    assert L.load().prc_device_fault_flags(0) == 0
    first = rec.read_shifted_positions(pos)
    L.call('prc_debug_wait_timeout', 1_000_000, L.ptr(out), stream())
    with pytest.raises(pyrecon_b200.ReconstructionError):
        rec.read_shifted_positions(pos)
    np.testing.assert_array_equal(rec.read_shifted_positions(pos), first)


def mg_solve(dtype, mixed, nmesh=(32, 32, 32), los=None, calls=1):
    """phi of prc_multigrid_* on a fixed random right-hand side, `calls` times on the same buffers."""
    L, t = lib(), torch()
    rng = np.random.default_rng(21)
    delta = dev(rng.standard_normal(nmesh).astype(dtype))
    phi = t.empty(nmesh, dtype=delta.dtype, device='cuda')
    nm, bs, bc = L.i3(nmesh), L.d3([800.] * 3), L.d3([0., 0., 1500.])
    w = ws(L.load().prc_multigrid_workspace_bytes(nm, np.dtype(dtype).itemsize, int(mixed)))
    args = [L.ptr(delta), L.ptr(phi), nm, bs, bc, 0.4, 0.4, 5, 6, L.opt_d3(los)]
    if dtype == 'f4':
        args.append(int(mixed))
    out = []
    for _ in range(calls):
        L.call('prc_multigrid_' + L.suffix(dtype), *args, L.ptr(w), w.numel(), stream())
        t.cuda.synchronize()
        out.append(phi.cpu().numpy().copy())
    return out


@pytest.mark.parametrize('dtype,mixed', [('f8', False), ('f4', True), ('f4', False)])
def test_multigrid_graph_replay_equals_direct_launches(dtype, mixed, tmp_path):
    """A solve is captured into a CUDA graph on its first call and replayed on the next call with the
    same buffers; both give the bits of the same solve launched kernel by kernel (PRC_MG_GRAPH=0)."""
    import subprocess
    import sys
    import os
    L = lib()
    n0 = L.launch_count()
    first, second = mg_solve(dtype, mixed, calls=2)
    assert np.array_equal(first, second)
    assert L.launch_count() - n0 > 100          # replayed kernels are counted
    path = str(tmp_path / 'phi.npy')
    code = ("import sys, numpy; sys.path.insert(0, '.'); sys.path.insert(0, 'tests');"
            "import test_gpu_kernels as T; numpy.save({!r}, T.mg_solve({!r}, {!r})[0])".format(path, dtype, mixed))
    env = dict(os.environ, PRC_MG_GRAPH='0')
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, '-c', code], cwd=root, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert np.array_equal(np.load(path), first)


@pytest.mark.parametrize('dtype,mixed,los', [('f8', False, None), ('f4', True, None), ('f4', False, [0., 0., 1.]),
                                             ('f8', False, [0.3, -0.5, 0.8])])
def test_multigrid_batch_equals_separate_solves(dtype, mixed, los):
    """prc_multigrid_batch_*: three problems in one batched solve give the bits of three separate solves."""
    L, t = lib(), torch()
    nmesh = (24, 16, 32)
    rng = np.random.default_rng(31)
    deltas = [dev(rng.standard_normal(nmesh).astype(dtype)) for _ in range(3)]
    nm, bs, bc = L.i3(nmesh), L.d3([800., 600., 900.]), L.d3([0., 100., 1500.])
    sfx, item = L.suffix(dtype), np.dtype(dtype).itemsize
    tail = [nm, bs, bc, 0.4, 0.4, 5, 6, L.opt_d3(los)] + ([int(mixed)] if dtype == 'f4' else [])
    alone = []
    for d in deltas:
        phi = t.empty_like(d)
        w = ws(L.load().prc_multigrid_workspace_bytes(nm, item, int(mixed)))
        L.call('prc_multigrid_' + sfx, L.ptr(d), L.ptr(phi), *tail, L.ptr(w), w.numel(), stream())
        alone.append(phi.cpu().numpy())
    phis = [t.empty_like(d) for d in deltas]
    w = ws(L.load().prc_multigrid_batch_workspace_bytes(nm, item, int(mixed), 3))
    L.call('prc_multigrid_batch_' + sfx, L.pointer_array(deltas), L.pointer_array(phis), 3, *tail, L.ptr(w), w.numel(),
           stream())
    for a, p in zip(alone, phis):
        assert np.array_equal(a, p.cpu().numpy())


@pytest.mark.parametrize('dtype,mixed', [('f8', False), ('f4', True), ('f4', False)])
@pytest.mark.parametrize('axis', [0, 1, 2])
def test_multigrid_axis_stencil_same_bits(dtype, mixed, axis):
    """A line of sight along one axis runs the 7-point form of the operator (the terms it drops are exact
    zeros of the 19-point form): the solve agrees with the 19-point kernels (mg_axis_stencil = 0) to the
    rounding of the multiply-adds the compiler forms from the kept terms."""
    L = lib()
    los = [0., 0., 0.]
    los[axis] = 1.
    nmesh = (32, 24, 16)
    fast = mg_solve(dtype, mixed, nmesh=nmesh, los=los)[0]
    L.tune_set('mg_axis_stencil', 0, 0)
    try:
        full = mg_solve(dtype, mixed, nmesh=nmesh, los=los)[0]
    finally:
        L.tune_set('mg_axis_stencil', 0, -1)
    assert np.isfinite(fast).all()
    assert maxrel(fast, full) < (2e-6 if dtype == 'f4' else 1e-13)


@pytest.mark.parametrize('dtype,mixed', [('f8', False), ('f4', True)])
@pytest.mark.parametrize('los,nmesh', [(None, (32, 32, 32)), ([0., 0., 1.], (64, 32, 48)), ([0.3, -0.5, 0.8], (24, 24, 24)),
                                       (None, (48, 48, 48))])
def test_multigrid_small_levels_in_one_block(dtype, mixed, los, nmesh):
    """The V-cycles of the levels of at most 16^3 cells run as one block per visit (vcycle_small, shared
    memory); the solve agrees with every step launched as its own kernel (mg_small_cells = 0) to rounding."""
    L = lib()
    if los is not None:
        los = list(np.asarray(los) / np.linalg.norm(los))
    n0 = L.launch_count()
    fused = mg_solve(dtype, mixed, nmesh=nmesh, los=los)[0]
    fused_launches = L.launch_count() - n0
    L.tune_set('mg_small_cells', 0, 0)
    try:
        n0 = L.launch_count()
        steps = mg_solve(dtype, mixed, nmesh=nmesh, los=los)[0]
        step_launches = L.launch_count() - n0
    finally:
        L.tune_set('mg_small_cells', 0, -1)
    assert np.isfinite(fused).all()
    assert fused_launches < step_launches
    assert maxrel(fused, steps) < (1e-5 if dtype == 'f4' else 1e-12)


def _smooth_real_gpu(value, radius_box, nsigmas, dtype):
    L = lib()
    t = torch()
    nm = L.i3(value.shape)
    src = dev(value.astype(dtype))
    out = t.empty_like(src)
    nbytes = L.load().prc_smooth_gaussian_real_workspace_bytes(nm, L.d3(radius_box), float(nsigmas), np.dtype(dtype).itemsize)
    assert nbytes > 0
    w = ws(nbytes)
    L.call('prc_smooth_gaussian_real_' + L.suffix(dtype), L.ptr(src), L.ptr(out), nm, L.d3(radius_box),
           float(nsigmas), L.ptr(w), w.numel(), stream())
    return out.cpu().numpy()


@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_real_space_smoothing_bit_exact(dtype):
    """RealMesh.smooth_gaussian(method='real') equals the reference's output bit for bit (golden
    vectors: isotropic, anisotropic, and a kernel wider than the mesh), twice in a row."""
    import json
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, 'mesh_kernels.npz'))
    for i, c in enumerate(json.loads(str(z['smooth_cases']))):
        radius = pipeline._array3(c['radius'], dtype) / pipeline._array3(c['boxsize'], dtype)
        nsig = np.dtype(dtype).type(c['nsigmas'])
        ref = z['smooth_real_{}_{:d}'.format(dtype, i)]
        for _ in range(2):
            out = _smooth_real_gpu(z['smooth_in_{:d}'.format(i)], radius, nsig, dtype)
            assert out.dtype == ref.dtype
            np.testing.assert_array_equal(out, ref, err_msg=str(c))


@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_real_space_smoothing_matches_oracle_noncubic(dtype):
    """Non-cubic mesh, widths differing per axis, tiles cut by the mesh edge: bit-exact against the C oracle."""
    rng = np.random.default_rng(7)
    nmesh = (37, 30, 45)
    value = rng.uniform(-1., 3., nmesh).astype(dtype)
    radius = np.array([0.09, 0.12, 0.07], dtype=dtype)
    k = pipeline._Kernels(dtype)
    ref = value.copy()
    k.smooth_gaussian(ref, np.array(nmesh), radius, 2.5)
    out = _smooth_real_gpu(value, radius, np.dtype(dtype).type(2.5), dtype)
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize('dtype', ['f4', 'f8'])
@pytest.mark.parametrize('randoms', [True, False])
def test_density_contrast_original_matches_numpy(dtype, randoms):
    """Martin's density contrast (before smoothing) against its numpy restatement in FP64."""
    L = lib()
    t = torch()
    rng = np.random.default_rng(11)
    nmesh = (48, 40, 36)
    d = rng.gamma(2., 1., nmesh)
    r = rng.gamma(1.5, 0.6, nmesh) * (rng.uniform(size=nmesh) > 0.2) if randoms else None
    bias, ran_min = 1.7, 0.75
    if randoms:
        mask = r >= ran_min
        dd = np.where((r > 0) & (r < ran_min), 0., d)
        alpha = dd.sum() / r[mask].sum()
        ref = np.where(mask, (dd / (alpha * np.where(mask, r, 1.)) - 1.) / bias, 0.).astype(dtype)
        nz = ref != 0
        ref[nz] = (ref[nz].astype('f8') - ref[nz].astype('f8').mean()).astype(dtype)
    else:
        ref = ((d / d.mean() - 1.) / bias).astype(dtype)
    out = t.empty(nmesh, dtype=t.float32 if dtype == 'f4' else t.float64, device='cuda')
    w = ws(L.load().prc_density_contrast_original_workspace_bytes())
    d_dev, r_dev = dev(d), (dev(r) if randoms else None)        # kept alive until the kernel has run
    L.call('prc_density_contrast_original_' + L.suffix(dtype), L.ptr(d_dev), L.ptr(r_dev), L.i3(nmesh), bias, ran_min,
           L.ptr(out), L.ptr(w), w.numel(), stream())
    out = out.cpu().numpy()
    assert np.array_equal(out == 0, ref == 0)
    tol = 1e-12 if dtype == 'f8' else 1e-6
    assert maxrel(out, ref) < tol


def _jacobi(dtype, nmesh, niter, los, slab, seed=41):
    """prc_mg_jacobi_* with the tuning table's "mg_jacobi" entry for this n0 set to `slab` (0: one sweep
    per pass, s > 0: two sweeps per pass in slabs of s planes)."""
    L, t = lib(), torch()
    rng = np.random.default_rng(seed)
    v = dev(rng.standard_normal(nmesh).astype(dtype))
    f = dev(rng.standard_normal(nmesh).astype(dtype))
    scratch = t.empty_like(v)
    knob = 'mg_jacobi' if dtype == 'f4' else 'mg_jacobi_f64'
    L.tune_set(knob, nmesh[0], slab)
    try:
        L.call('prc_mg_jacobi_' + L.suffix(dtype), L.ptr(v), L.ptr(f), L.ptr(scratch), L.i3(nmesh),
               L.d3([800., 600., 1000.]), L.d3([1600., 0., 300.]), 0.4, 0.4, niter, L.opt_d3(los), stream())
        return v.cpu().numpy()
    finally:
        L.tune_set(knob, nmesh[0], -1)


@pytest.mark.parametrize('nmesh', [(16, 12, 20), (24, 16, 32), (8, 8, 8), (64, 48, 40), (128, 64, 96), (96, 200, 68)])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
@pytest.mark.parametrize('los', [None, [0.3, -0.5, 0.8]])
def test_jacobi_two_sweeps_per_pass(nmesh, dtype, los):
    """Temporal blocking (two damped-Jacobi sweeps per pass, shared-memory plane rings, x-marching slabs)
    gives the result of one sweep per pass: odd sweep counts, slabs longer and shorter than the mesh,
    tiles cut by the mesh edge and tiles larger than the mesh.  Both evaluate each cell with the same
    function; FP64 agrees bit for bit, FP32 to a few units of the last place (the compiler may fuse a
    multiply-add differently in the two kernels)."""
    if los is not None:
        los = list(np.asarray(los) / np.linalg.norm(los))
    ref = _jacobi(dtype, nmesh, 5, los, 0)
    for slab in [1, 3, 8, 64]:
        got = _jacobi(dtype, nmesh, 5, los, slab)
        if dtype == 'f8':
            assert np.array_equal(got, ref), (nmesh, dtype, slab, np.abs(got - ref).max())
        else:
            assert maxrel(got, ref) < 2e-6, (nmesh, dtype, slab, maxrel(got, ref))


@pytest.mark.parametrize('dtype,mixed', [('f8', False), ('f4', True), ('f4', False)])
def test_multigrid_solve_with_temporal_blocking(dtype, mixed):
    """A whole solve (graph-captured) with two sweeps per pass on every level gives the solve with one
    sweep per pass (FP64 bit for bit, FP32 to rounding); the tuning change makes the solve capture a
    new graph."""
    L = lib()
    nmesh = (32, 32, 32)
    knob = 'mg_jacobi' if dtype == 'f4' else 'mg_jacobi_f64'
    for n in [32, 16, 8]:
        L.tune_set(knob, n, 0)
    try:
        ref = mg_solve(dtype, mixed, nmesh=nmesh)[0]
        for n in [32, 16, 8]:
            L.tune_set(knob, n, 4)
        got = mg_solve(dtype, mixed, nmesh=nmesh)[0]
    finally:
        for n in [32, 16, 8]:
            L.tune_set(knob, n, -1)
    if dtype == 'f8' or mixed:
        assert np.array_equal(got, ref) if dtype == 'f8' else maxrel(got, ref) < 1e-5
    else:
        assert maxrel(got, ref) < 1e-4
