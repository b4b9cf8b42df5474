"""
End-to-end parity of the CUDA reconstruction against the reference's own outputs
(golden fixtures) and the FP64 oracle, through the public Python API.

Tolerances (stated by the north-star contract): shifted positions within 1e-6 Mpc/h of the
FP64 oracle in the all-FP64 mode ('f8'), within 1e-3 Mpc/h in the FP32 mode ('f4').
Intermediate meshes are compared relative to their maximum.
"""
import numpy as np
import pytest

from conftest import golden_cases
from _util import load_golden, run_oracle, run_gpu, maxrel, maxabs

pytestmark = pytest.mark.gpu

F8_CASES = [c for c in golden_cases() if load_golden(c)['meta']['dtype'] == 'f8']


@pytest.mark.parametrize('name', F8_CASES)
def test_f8_matches_reference(name):
    g = load_golden(name)
    out, rec = run_gpu(g)
    for key, tol in [('mesh_data', 1e-13), ('mesh_randoms', 1e-13), ('mesh_delta', 1e-10), ('mesh_phi', 1e-9),
                     ('mesh_psi', 1e-9)]:
        if key in g:        # the large-mesh fixtures keep inputs and shifts only
            assert maxrel(out[key], g[key]) < tol, (name, key)
    for k in ['shifts_disp', 'shifts_rsd', 'shifted_data', 'shifted_randoms', 'shifts_data_disp', 'shifts_data_rsd',
              'shifted_data_str']:
        if k in g:
            assert out[k].dtype == g[k].dtype, k
            assert maxabs(out[k], g[k]) < 1e-6, (name, k, maxabs(out[k], g[k]))


@pytest.mark.parametrize('name', golden_cases())
def test_f4_within_1e3_of_f8_oracle(name):
    """FP32 mode (FP64 paint sums / normalisation / multigrid defects) against the FP64 oracle."""
    g = load_golden(name)
    for k in ['data', 'randoms']:
        if k in g:
            g[k] = g[k].astype('f4')
    ref = run_oracle(g, dtype='f8')
    out, rec = run_gpu(g, dtype='f4')
    # float index coordinates, as the reference's f4: a CIC fraction is off by up to ~n 2^-24
    tol = max(1e-5, 3. * max(np.broadcast_to(g['meta']['nmesh'], 3)) * 2. ** -24)
    assert maxrel(out['mesh_data'], ref['mesh_data']) < tol
    for k in ['shifted_data', 'shifted_randoms', 'shifted_data_str']:
        if k in ref:
            assert out[k].dtype == np.float32
            assert maxabs(out[k], ref[k]) < 1e-3, (name, k, maxabs(out[k], ref[k]))


def test_f4_multigrid_mixed_and_plain():
    """Both FP32 multigrid variants stay within tolerance; the FP64-defect one is the closer."""
    g = load_golden('mg_f8_local')
    ref = run_oracle(g, dtype='f8')
    errs = {}
    for mixed in [True, False]:
        out, _ = run_gpu(g, dtype='f4', mixed_precision=mixed)
        errs[mixed] = maxabs(out['shifted_data'], ref['shifted_data'])
        assert errs[mixed] < 1e-3
    assert errs[True] <= errs[False] * 1.5 + 1e-6


def test_repeatable_bitwise():
    """Same inputs, same bits: the deterministic paint makes the whole pipeline reproducible."""
    g = load_golden('ifft_f8_local')
    a, _ = run_gpu(g)
    b, _ = run_gpu(g)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize('dtype,nmesh', [('f4', (48, 32, 64)), ('f8', (32, 32, 32)), ('f4', (192, 192, 192))])
def test_plane_parallel_run_batch_equals_separate_runs(dtype, nmesh):
    """plane_parallel_fft.run_batch: three reconstructions (a pair sharing the FFT passes, then one) give
    the displacements and shifted positions of three separate runs, bit for bit."""
    import pyrecon_b200
    from pyrecon_b200 import mocks
    from pyrecon_b200.plane_parallel_fft import run_batch
    cats = [mocks.lognormal_positions_numpy(20000 + 4000 * i, 32, 1000., 500., seed=130 + i, field_seed=140 + i)
            for i in range(3)]

    def prepared(data):
        rec = pyrecon_b200.PlaneParallelFFTReconstruction(f=0.8, bias=2., los='y', nmesh=nmesh, boxsize=1000.,
                                                           boxcenter=500., wrap=True, dtype=dtype)
        rec.assign_data(data.astype(dtype))
        rec.set_density_contrast(smoothing_radius=15.)
        return rec

    alone = []
    for data in cats:
        rec = prepared(data)
        rec.run()
        alone.append((rec._psi4.cpu().numpy(), rec.read_shifted_positions(data.astype(dtype))))
    recs = [prepared(data) for data in cats]
    run_batch(recs)
    for rec, data, (psi, shifted) in zip(recs, cats, alone):
        assert np.array_equal(rec._psi4.cpu().numpy(), psi)
        assert np.array_equal(rec.read_shifted_positions(data.astype(dtype)), shifted)


@pytest.mark.parametrize('kind', ['numpy', 'pinned', 'pageable'])
def test_chunked_host_readout_equals_device_readout(kind):
    """Host positions read out in overlapping chunks (copy in / kernel / copy out on separate
    streams) give the same bits as one read-out of the same positions resident on the device."""
    import torch
    g = load_golden('ifft_f8_local')
    out, rec = run_gpu(g)
    data = g['data']
    ref = rec.read_shifted_positions(torch.from_numpy(data).cuda()).cpu().numpy()
    rec._read_chunk = 97                      # many chunks, a ragged last one
    if kind == 'numpy':
        pos = data
    else:
        pos = torch.from_numpy(data)
        if kind == 'pinned':
            pos = pos.pin_memory()
    got = rec.read_shifted_positions(pos)
    got = got if kind == 'numpy' else got.numpy()
    assert got.dtype == ref.dtype and got.shape == ref.shape
    assert np.array_equal(got, ref)
    disp = rec.read_shifts(pos, field='disp')
    disp = disp if kind == 'numpy' else disp.numpy()
    assert np.array_equal(disp, out['shifts_disp'])


@pytest.mark.parametrize('name', ['ifft_f4_local', 'mg_f8_local', 'ifftp_f8_local', 'ifftp_f4_local', 'pp_f8_box_wrap',
                                  'mg_f8_box_wrap', 'mg_f4_local'])
def test_readout_in_paint_order_equals_plain_readout(name):
    """Device catalogues are read out in the cell order of their paint, from the cell-ordered copy of the
    positions the paint kept; a copy of the same positions (no order remembered) gives the same bits,
    and so does the read-out after the catalogue was modified in place (the kept copy is then stale and
    not used)."""
    import torch
    import pyrecon_b200
    from _util import ALGOS
    g = load_golden(name)
    m = g['meta']
    Cls = getattr(pyrecon_b200, ALGOS[m['algorithm']])
    rec = Cls(f=m['f'], bias=m['bias'], los=m['los'], nmesh=m['nmesh'], boxsize=m['boxsize'],
              boxcenter=m['boxcenter'], dtype=m['dtype'], wrap=m['wrap'])
    data = torch.from_numpy(g['data']).cuda()
    rec.assign_data(data, None if g['wdata'] is None else torch.from_numpy(g['wdata']).cuda())
    randoms = None
    if m['randoms']:
        randoms = torch.from_numpy(g['randoms']).cuda()
        rec.assign_randoms(randoms, None if g['wrandoms'] is None else torch.from_numpy(g['wrandoms']).cuda())
    rec.set_density_contrast(smoothing_radius=m['smoothing_radius'])
    rec.run()
    assert rec._order_for(data) is not None
    assert (rec._sorted_for(data) is not None) == (m['algorithm'] != 'iterative_fft_particle')
    for cat in [data] + ([randoms] if randoms is not None else []):
        ordered = rec.read_shifted_positions(cat)
        plain = rec.read_shifted_positions(cat.clone())
        assert torch.equal(ordered, plain)
        assert torch.equal(rec.read_shifts(cat, field='rsd'), rec.read_shifts(cat.clone(), field='rsd'))
    # an in-place change of the catalogue: the order is still used (any order gives the same bits), the
    # kept cell-ordered positions are not
    data[:10] = data[10:20].clone()
    assert rec._sorted_for(data) is None and rec._order_for(data) is not None
    assert torch.equal(rec.read_shifted_positions(data), rec.read_shifted_positions(data.clone()))
    # the painted tensor freed and another catalogue of the same length created in its place (same
    # address from the caching allocator, version counter 0 again): the kept positions are not its own
    shape, ptr = tuple(data.shape), data.data_ptr()
    other = np.ascontiguousarray(np.flip(g['data'], axis=0))
    del data, ordered, plain, cat
    torch.cuda.synchronize()
    fresh = torch.from_numpy(other).cuda()
    if fresh.data_ptr() == ptr and tuple(fresh.shape) == shape:
        assert rec._sorted_for(fresh) is None
    assert torch.equal(rec.read_shifted_positions(fresh), rec.read_shifted_positions(fresh.clone()))


def test_sky_conversions_on_device():
    """utils.cartesian_to_sky / sky_to_cartesian on CUDA tensors agree with the numpy (reference) path."""
    import torch
    from pyrecon_b200 import utils
    rng = np.random.default_rng(3)
    for dtype, tol in [('f8', 1e-12), ('f4', 2e-6)]:
        pos = (rng.normal(size=(10000, 3)) * 800.).astype(dtype)
        t = torch.from_numpy(pos).cuda()
        ref = utils.cartesian_to_sky(pos)
        out = utils.cartesian_to_sky(t)
        for a, b in zip(out, ref):
            assert a.is_cuda
            assert maxrel(a.cpu().numpy(), b) < tol
        xyz = utils.sky_to_cartesian(*out)
        assert xyz.is_cuda and maxrel(xyz.cpu().numpy(), pos) < 10 * tol


def test_mesh_numpy_interop():
    """numpy ufuncs on meshes return meshes of the same kind (booleans and reductions return arrays),
    arithmetic and comparisons run on the device, FFT-engine settings are accepted."""
    import torch
    from pyrecon_b200 import RealMesh
    rng = np.random.default_rng(5)
    value = rng.uniform(0.5, 2., (8, 6, 4))
    mesh = RealMesh(value, boxsize=100., boxcenter=0., dtype='f8')
    e = np.exp(mesh)
    assert isinstance(e, RealMesh) and np.allclose(np.asarray(e), np.exp(value))
    assert np.allclose(np.asarray(mesh ** 2), value ** 2) and np.allclose(np.asarray(2. ** mesh), 2. ** value)
    gt = mesh > 1.
    assert isinstance(gt, torch.Tensor) and gt.dtype == torch.bool
    assert np.array_equal(gt.cpu().numpy(), value > 1.)
    assert isinstance(np.greater(mesh, 1.), np.ndarray)
    assert np.isclose(np.mean(mesh), value.mean())
    mesh.set_fft_engine('fftw', nthreads=4)
    mesh.set_num_threads(4)
    c = mesh.to_complex()
    assert np.allclose(c.fundamental_freq, 2 * np.pi / 100.) and c.hshape == (8, 6, 3)
