"""
Pin the CPU oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py).  No GPU needed: this is what makes the oracle
trustworthy as the checker of the CUDA path.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from oracle import pipeline


def load(name):
    z = np.load(os.path.join(GOLDEN, name + '.npz'))
    out = {k: z[k] for k in z.files}
    out['meta'] = json.loads(str(out['meta']))
    return out


def run_oracle(g, kernels='oracle', dtype=None):
    m = g['meta']
    rec = pipeline.OracleReconstruction(m['algorithm'], f=m['f'], bias=m['bias'], los=m['los'], nmesh=m['nmesh'],
                                        boxsize=m['boxsize'], boxcenter=m['boxcenter'], dtype=dtype or m['dtype'],
                                        wrap=m['wrap'], kernels=kernels)
    out = {}
    rec.assign_data(g['data'], g['wdata'])
    out['mesh_data'] = rec.mesh_data.copy()
    key, order = pipeline.sorted_cell_order(g['data'], rec.geom, wrap=m['wrap'])
    out['keys_data'] = key
    if m['randoms']:
        rec.assign_randoms(g['randoms'], g['wrandoms'])
        out['mesh_randoms'] = rec.mesh_randoms.copy()
    rec.set_density_contrast(smoothing_radius=m['smoothing_radius'], **m.get('density_kwargs', {}))
    out['mesh_delta'] = rec.mesh_delta.copy()
    rec.run()
    if m['algorithm'] in ('multigrid', 'multigrid_original'):
        out['mesh_phi'] = rec.mesh_phi
    else:
        out['mesh_psi'] = np.stack(rec.mesh_psi)
    out['shifts_disp'] = rec.read_shifts(g['data'], field='disp')
    out['shifts_rsd'] = rec.read_shifts(g['data'], field='rsd')
    out['shifted_data'] = rec.read_shifted_positions(g['data'])
    if m['randoms']:
        out['shifted_randoms'] = rec.read_shifted_positions(g['randoms'])
    if m['algorithm'] == 'iterative_fft_particle':
        out['shifts_data_disp'] = rec.read_shifts('data', field='disp')
        out['shifts_data_rsd'] = rec.read_shifts('data', field='rsd')
        out['shifted_data_str'] = rec.read_shifted_positions('data')
    return out


def tolerances(dtype):
    # The restatement differs from the reference only in the summation order of the multigrid
    # stencils (the FFT-path cases agree bit for bit): ~1e-15 relative in f8, ~1e-6 in f4.
    return dict(rtol=1e-12, atol=1e-12) if dtype == 'f8' else dict(rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize('name', golden_cases())
def test_oracle_matches_reference_golden(name):
    g = load(name)
    out = run_oracle(g)
    tol = tolerances(g['meta']['dtype'])
    if 'keys_data' in g:
        np.testing.assert_array_equal(out['keys_data'], g['keys_data'])   # cell indices: bit-exact
    for key in ['mesh_data', 'mesh_randoms', 'mesh_delta', 'mesh_phi', 'mesh_psi', 'shifts_disp', 'shifts_rsd',
                'shifted_data', 'shifted_randoms', 'shifts_data_disp', 'shifts_data_rsd', 'shifted_data_str']:
        if key not in g:
            continue
        ref = g[key]
        scale = max(np.abs(ref).max(), 1e-30)
        assert out[key].dtype == ref.dtype, key
        np.testing.assert_allclose(out[key], ref, rtol=tol['rtol'], atol=tol['atol'] * scale, err_msg='{} {}'.format(name, key))


@pytest.mark.skipif(not pipeline.reference_kernels_available(), reason='reference C kernels not compiled here')
@pytest.mark.parametrize('name', ['mg_f8_local', 'ifft_f8_local', 'pp_f8_losz', 'omg_f8_local', 'mg_f8_real'])
def test_reference_kernel_backend_matches_golden(name):
    """The CPU-baseline back-end (reference C compiled from source, oracle/_ref) reproduces the golden run."""
    g = load(name)
    out = run_oracle(g, kernels='reference')
    for key in ['mesh_data', 'mesh_delta', 'shifted_data']:
        np.testing.assert_allclose(out[key], g[key], rtol=1e-12, atol=1e-12 * np.abs(g[key]).max())


def test_mesh_kernels_golden():
    z = np.load(os.path.join(GOLDEN, 'mesh_kernels.npz'))
    for dtype in ['f4', 'f8']:
        geom = pipeline.Geometry([16, 12, 20], 1000., 0., dtype=dtype)
        k = pipeline._Kernels(dtype)
        mesh = np.zeros(geom.shape, dtype=dtype)
        pos = z['positions'].astype(dtype)
        k.assign_cic(mesh, geom.nmesh, geom.to_index(pos), z['weights'].astype(dtype))
        tol = dict(rtol=1e-12, atol=1e-12) if dtype == 'f8' else dict(rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(mesh, z['assign_' + dtype], **tol)
        rp = z['readpos'].astype(dtype)
        np.testing.assert_allclose(k.read_cic(mesh, geom.nmesh, geom.to_index(rp)), z['read_' + dtype], **tol)
        fd = k.read_finite_difference_cic(mesh, geom.nmesh, geom.boxsize, geom.to_index(rp))
        np.testing.assert_allclose(fd.ravel(), z['fd_' + dtype].ravel(), **tol)
        # ComplexMesh defaults to a Hermitian (half last axis) layout: last axis from rfftfreq
        d = 1. / np.array([4, 3, 5])
        arrays = [1. + 2 * np.pi * np.fft.fftfreq(4, d=d[0]), 1. + 2 * np.pi * np.fft.fftfreq(3, d=d[1]),
                  1. + 2 * np.pi * np.fft.rfftfreq(5, d=d[2])]
        val = z['prod_in_' + dtype].copy()
        rec = pipeline.OracleReconstruction.__new__(pipeline.OracleReconstruction)
        rec.dtype, rec.kernels = np.dtype(dtype), k
        rec._prod_sum_complex(val, arrays, exp=-1)
        np.testing.assert_allclose(val, z['prod_out_' + dtype], **tol)


def smooth_cases():
    z = np.load(os.path.join(GOLDEN, 'mesh_kernels.npz'))
    return z, json.loads(str(z['smooth_cases']))


@pytest.mark.parametrize('kernels', ['oracle', 'reference'])
@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_real_space_smoothing_bit_exact(dtype, kernels):
    """RealMesh.smooth_gaussian(method='real'): the C restatement (and the reference C compiled here)
    equal the reference's output bit for bit, kernels wider than the mesh included."""
    if kernels == 'reference' and not pipeline.reference_kernels_available():
        pytest.skip('reference C kernels not compiled here')
    z, cases = smooth_cases()
    for i, c in enumerate(cases):
        geom = pipeline.Geometry(c['nmesh'], c['boxsize'], 0., dtype=dtype)
        rec = pipeline.OracleReconstruction.__new__(pipeline.OracleReconstruction)
        rec.geom, rec.dtype, rec.kernels = geom, geom.dtype, pipeline._Kernels(dtype, source=kernels)
        out = rec.smooth_gaussian(z['smooth_in_{:d}'.format(i)].astype(dtype), c['radius'], method='real',
                                  nsigmas=c['nsigmas'])
        ref = z['smooth_real_{}_{:d}'.format(dtype, i)]
        assert out.dtype == ref.dtype
        np.testing.assert_array_equal(out, ref, err_msg=str(c))


def test_cell_order_is_stable_sort():
    g = load('mg_f8_local')
    geom = pipeline.Geometry(16, 800., 1600.)
    key, order = pipeline.sorted_cell_order(g['data'], geom)
    assert np.all(np.diff(key[order]) >= 0)
    same = np.diff(key[order]) == 0
    assert np.all(np.diff(order)[same] > 0)   # ties keep input order
