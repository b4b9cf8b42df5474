"""
Generate the golden fixtures in this directory by running the REFERENCE
implementation (cosmodesi/pyrecon 1.0.0) on small seeded inputs.

This script runs only where the reference source tree is available (its
path in the environment variable PYRECON_REFERENCE, required); it copies the
tree to a temporary directory, builds its C kernels there with the system
gcc (the reference's own src/Makefile), imports it and stores, per case,
the inputs and every intermediate the drop-in exposes:

  mesh_data, mesh_randoms   painted meshes (before smoothing)
  keys_data                 base-cell index of every data particle, from the
                            reference's own index transform (mesh.py:554-555,
                            mesh.c:35-37)
  mesh_delta                density contrast after set_density_contrast
  mesh_phi / mesh_psi       solver output (multigrid / FFT algorithms)
  shifts_{disp,rsd}, shifted_data, shifted_randoms

plus mesh-level kernel outputs in mesh_kernels.npz.  The fixtures are small
(nmesh <= 24, a few thousand particles) so the oracle reproduces them in
seconds.  Usage:  python tests/golden/make_golden.py [name ...]   (all by default)
"""

import os
import sys
import json
import shutil
import tempfile
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pyrecon_b200 import mocks  # noqa: E402


def import_reference(tmp):
    src = os.environ.get('PYRECON_REFERENCE')
    if not src or not os.path.isfile(os.path.join(src, 'pyrecon', 'recon.py')):
        raise SystemExit('set PYRECON_REFERENCE to the root of the reference source tree (holding pyrecon/ and src/); '
                         'got {!r}'.format(src))
    dst = os.path.join(tmp, 'reference')
    shutil.copytree(src, dst)
    subprocess.run(['make', '-s', '-C', os.path.join(dst, 'src'), 'CC=/usr/bin/gcc',
                    'LIBDIR={}'.format(os.path.join(dst, 'pyrecon', 'lib'))], check=True)
    sys.path.insert(0, dst)
    import pyrecon
    return pyrecon


CASES = [
    # name, algorithm, dtype, los, nmesh, boxsize, boxcenter, wrap, with randoms, run kwargs, smoothing radius
    dict(name='mg_f8_local', algorithm='multigrid', dtype='f8', los=None, nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='mg_f4_local', algorithm='multigrid', dtype='f4', los=None, nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='mg_f8_losx', algorithm='multigrid', dtype='f8', los='x', nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='mg_f8_local_n24', algorithm='multigrid', dtype='f8', los=None, nmesh=24, boxsize=800., boxcenter=1600.),
    dict(name='mg_f8_noncubic', algorithm='multigrid', dtype='f8', los=[1., 1., 1.], nmesh=[16, 12, 20],
         boxsize=[800., 600., 1000.], boxcenter=[1600., 0., 300.]),
    dict(name='mg_f8_box_wrap', algorithm='multigrid', dtype='f8', los='z', nmesh=16, boxsize=800., boxcenter=400.,
         wrap=True, randoms=False),
    dict(name='ifft_f8_local', algorithm='iterative_fft', dtype='f8', los=None, nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='ifft_f4_local', algorithm='iterative_fft', dtype='f4', los=None, nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='ifft_f8_losvec', algorithm='iterative_fft', dtype='f8', los=[0.3, -0.5, 0.8], nmesh=16, boxsize=800.,
         boxcenter=1600.),
    dict(name='ifft_f8_radix', algorithm='iterative_fft', dtype='f8', los=None, nmesh=[12, 18, 20],
         boxsize=[600., 900., 1000.], boxcenter=[1600., 100., -200.]),
    dict(name='ifft_f8_box_wrap', algorithm='iterative_fft', dtype='f8', los='z', nmesh=16, boxsize=800., boxcenter=400.,
         wrap=True, randoms=False),
    dict(name='pp_f8_losz', algorithm='plane_parallel_fft', dtype='f8', los='z', nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='pp_f4_losx', algorithm='plane_parallel_fft', dtype='f4', los='x', nmesh=16, boxsize=800., boxcenter=1600.),
    dict(name='pp_f8_box_wrap', algorithm='plane_parallel_fft', dtype='f8', los=[1., 2., 2.], nmesh=16, boxsize=800.,
         boxcenter=400., wrap=True, randoms=False),
    dict(name='ifftp_f8_local', algorithm='iterative_fft_particle', dtype='f8', los=None, nmesh=16, boxsize=800.,
         boxcenter=1600.),
    dict(name='ifftp_f4_local', algorithm='iterative_fft_particle', dtype='f4', los=None, nmesh=16, boxsize=800.,
         boxcenter=1600.),
    dict(name='ifftp_f8_losvec', algorithm='iterative_fft_particle', dtype='f8', los=[0.3, -0.5, 0.8], nmesh=16,
         boxsize=800., boxcenter=1600.),
    dict(name='ifftp_f8_box_wrap', algorithm='iterative_fft_particle', dtype='f8', los='z', nmesh=16, boxsize=800.,
         boxcenter=400., wrap=True, randoms=False),
    # OriginalMultiGridReconstruction: Martin's density contrast (multigrid.py:49-97)
    dict(name='omg_f8_local', algorithm='multigrid_original', dtype='f8', los=None, nmesh=16, boxsize=800.,
         boxcenter=1600.),
    dict(name='omg_f4_local', algorithm='multigrid_original', dtype='f4', los=None, nmesh=16, boxsize=800.,
         boxcenter=1600.),
    dict(name='omg_f8_box_wrap', algorithm='multigrid_original', dtype='f8', los='z', nmesh=16, boxsize=800.,
         boxcenter=400., wrap=True, randoms=False),
    dict(name='omg_f8_real', algorithm='multigrid_original', dtype='f8', los=None, nmesh=16, boxsize=800.,
         boxcenter=1600., density_kwargs=dict(method='real')),
    # base density contrast with real-space smoothing (recon.py:220-226, mesh.py:684-695)
    dict(name='mg_f8_real', algorithm='multigrid', dtype='f8', los=None, nmesh=16, boxsize=800., boxcenter=1600.,
         density_kwargs=dict(method='real')),
    dict(name='ifft_f4_real', algorithm='iterative_fft', dtype='f4', los=None, nmesh=16, boxsize=800., boxcenter=1600.,
         density_kwargs=dict(method='real', nsigmas=3.)),
    # mesh sizes with prime factors above 7 and odd last axes (any size the reference's FFT engines take)
    dict(name='ifft_f8_prime', algorithm='iterative_fft', dtype='f8', los=None, nmesh=[13, 11, 9],
         boxsize=[650., 550., 450.], boxcenter=[1600., 100., -200.]),
    dict(name='ifft_f4_prime', algorithm='iterative_fft', dtype='f4', los=None, nmesh=[13, 11, 9],
         boxsize=[650., 550., 450.], boxcenter=[1600., 100., -200.]),
    dict(name='mg_f8_prime', algorithm='multigrid', dtype='f8', los=None, nmesh=[13, 11, 9],
         boxsize=[650., 550., 450.], boxcenter=[1600., 100., -200.]),
    dict(name='pp_f8_odd', algorithm='plane_parallel_fft', dtype='f8', los='z', nmesh=[15, 22, 21],
         boxsize=[750., 1100., 1050.], boxcenter=[1600., 0., 300.]),
    dict(name='ifftp_f8_prime', algorithm='iterative_fft_particle', dtype='f8', los=None, nmesh=[17, 12, 19],
         boxsize=[850., 600., 950.], boxcenter=[1600., 100., -200.]),
    # 125^3 (5^3: odd on every axis): inputs and shifts only (the meshes would make a 100 MB fixture)
    dict(name='ifft_f8_n125', algorithm='iterative_fft', dtype='f8', los=None, nmesh=125, boxsize=1000.,
         boxcenter=1600., light=True),
    dict(name='mg_f8_n125', algorithm='multigrid', dtype='f8', los=None, nmesh=125, boxsize=1000., boxcenter=1600.,
         light=True),
]

NDATA, NRANDOMS = 1500, 4000
SMOOTHING = 30.


def make_inputs(case, seed):
    nmesh = np.broadcast_to(np.asarray(case['nmesh']), 3)
    boxsize = np.broadcast_to(np.asarray(case['boxsize'], dtype='f8'), 3)
    boxcenter = np.broadcast_to(np.asarray(case['boxcenter'], dtype='f8'), 3)
    # lognormal field on a cube covering the largest side, then rescaled per axis into the box
    unit = mocks.lognormal_positions_numpy(NDATA, 16, 800., 0., seed=2000 + seed, field_seed=1000 + seed) / 800.
    data = boxcenter + unit * boxsize * 0.98
    randoms = boxcenter + (np.random.default_rng(3000 + seed).uniform(-0.49, 0.49, (NRANDOMS, 3))) * boxsize
    wdata = mocks.weights_numpy(NDATA, seed=4000 + seed)
    wrandoms = mocks.weights_numpy(NRANDOMS, seed=5000 + seed)
    if case.get('wrap', False):
        # periodic box: push a few points one box length outside on each side
        data[:50] += boxsize
        data[50:100] -= boxsize
        randoms[:50] += boxsize
    dtype = case['dtype']
    if dtype == 'f4':
        data, randoms = data.astype('f4'), randoms.astype('f4')
    return data, wdata, randoms, wrandoms


def run_case(pyrecon, case, seed):
    Cls = {'multigrid': pyrecon.MultiGridReconstruction, 'iterative_fft': pyrecon.IterativeFFTReconstruction,
           'multigrid_original': pyrecon.multigrid.OriginalMultiGridReconstruction,
           'plane_parallel_fft': pyrecon.PlaneParallelFFTReconstruction,
           'iterative_fft_particle': pyrecon.IterativeFFTParticleReconstruction}[case['algorithm']]
    data, wdata, randoms, wrandoms = make_inputs(case, seed)
    with_randoms = case.get('randoms', True)
    wrap = case.get('wrap', False)
    recon = Cls(f=0.8, bias=2., los=case['los'], nmesh=case['nmesh'], boxsize=case['boxsize'],
                boxcenter=case['boxcenter'], dtype=case['dtype'], wrap=wrap, nthreads=1)
    out = dict(data=data, wdata=wdata)
    recon.assign_data(data, wdata)
    out['mesh_data'] = np.array(recon.mesh_data.value)
    info = recon.mesh_data.info
    pos = info.wrap(data) if wrap else data
    idx = (((pos - info.boxcenter) / info.boxsize + 0.5) * info.nmesh).astype(recon.mesh_data._type_float)
    n = info.nmesh.astype('i8')
    cell = np.trunc(idx).astype('i8') % n
    out['keys_data'] = (cell[:, 0] * n[1] + cell[:, 1]) * n[2] + cell[:, 2]
    if with_randoms:
        out.update(randoms=randoms, wrandoms=wrandoms)
        recon.assign_randoms(randoms, wrandoms)
        out['mesh_randoms'] = np.array(recon.mesh_randoms.value)
    recon.set_density_contrast(smoothing_radius=SMOOTHING, **case.get('density_kwargs', {}))
    out['mesh_delta'] = np.array(recon.mesh_delta.value)
    recon.run()
    if case['algorithm'] in ('multigrid', 'multigrid_original'):
        out['mesh_phi'] = np.array(recon.mesh_phi.value)
    else:
        out['mesh_psi'] = np.stack([np.array(p.value) for p in recon.mesh_psi])
    if case.get('light', False):
        for k in ['mesh_data', 'mesh_randoms', 'mesh_delta', 'mesh_phi', 'mesh_psi', 'keys_data']:
            out.pop(k, None)
    out['shifts_disp'] = recon.read_shifts(data, field='disp')
    out['shifts_rsd'] = recon.read_shifts(data, field='rsd')
    out['shifted_data'] = recon.read_shifted_positions(data)
    if with_randoms:
        out['shifted_randoms'] = recon.read_shifted_positions(randoms)
    if case['algorithm'] == 'iterative_fft_particle':
        # the data at their own reconstructed real-space positions (iterative_fft_particle.py:176-186)
        out['shifts_data_disp'] = recon.read_shifts('data', field='disp')
        out['shifts_data_rsd'] = recon.read_shifts('data', field='rsd')
        out['shifted_data_str'] = recon.read_shifted_positions('data')
    meta = dict(case)
    meta.update(f=0.8, bias=2., smoothing_radius=SMOOTHING, randoms=with_randoms, wrap=wrap,
                reference_version=pyrecon.__version__)
    out['meta'] = np.array(json.dumps(meta))
    return out


def mesh_kernels(pyrecon):
    """assign_cic / read_cic / read_finite_difference_cic / prod_sum on one mesh, f4 and f8
    (the reference's own mesh tests, pyrecon/tests/test_mesh.py:42-80 and :173-190, at fixture size)."""
    out = {}
    rng = np.random.default_rng(42)
    positions = rng.uniform(-400., 400., (3000, 3))
    weights = rng.uniform(0.5, 1., 3000)
    readpos = rng.uniform(-400., 400., (2000, 3))
    # edge cases: a coordinate exactly on the upper box face and on the lower one
    positions[0] = [500., 0., -500.]
    positions[1] = [-500., 500., 499.999999]
    out['positions'], out['weights'], out['readpos'] = positions, weights, readpos
    for dtype in ['f4', 'f8']:
        mesh = pyrecon.RealMesh(boxsize=1000., boxcenter=0., nmesh=[16, 12, 20], dtype=dtype)
        mesh.assign_cic(positions.astype(dtype), weights.astype(dtype))
        out['assign_' + dtype] = np.array(mesh.value)
        out['read_' + dtype] = mesh.read_cic(readpos.astype(dtype))
        out['fd_' + dtype] = mesh.read_finite_difference_cic(readpos.astype(dtype))
        cmesh = pyrecon.ComplexMesh(value=1., boxsize=1., boxcenter=0., nmesh=(4, 3, 5), dtype='c8' if dtype == 'f4' else 'c16')
        arrays = [1. + c for c in cmesh.coords()]
        cmesh.value = (rng.uniform(0, 1, cmesh.shape) + 1j * rng.uniform(0, 1, cmesh.shape)).astype(cmesh.dtype)
        out['prod_in_' + dtype] = np.array(cmesh.value)
        cmesh.prod_sum(arrays, exp=-1)
        out['prod_out_' + dtype] = np.array(cmesh.value)
    # real-space Gaussian smoothing (mesh.py:684-695): isotropic, anisotropic, and a kernel wider
    # than the mesh (neighbour indices wrap through the C code's unsigned arithmetic)
    rng = np.random.default_rng(43)
    smooth = [dict(nmesh=16, boxsize=1000., radius=90., nsigmas=2.5),
              dict(nmesh=16, boxsize=1000., radius=[70., 90., 80.], nsigmas=3.),
              dict(nmesh=6, boxsize=600., radius=250., nsigmas=2.5)]
    out['smooth_cases'] = np.array(json.dumps(smooth))
    for i, c in enumerate(smooth):
        value = rng.uniform(-1., 3., (c['nmesh'],) * 3)
        out['smooth_in_{:d}'.format(i)] = value
        for dtype in ['f4', 'f8']:
            mesh = pyrecon.RealMesh(boxsize=c['boxsize'], boxcenter=0., nmesh=c['nmesh'], dtype=dtype)
            mesh.value = value.astype(dtype)
            mesh.smooth_gaussian(c['radius'], method='real', nsigmas=c['nsigmas'])
            out['smooth_real_{}_{:d}'.format(dtype, i)] = np.array(mesh.value)
    return out


def distance_of_z(z):
    """A smooth distance-redshift relation for the DistanceToRedshift fixture."""
    return 2997.92458 * z / (1. + 0.6 * z) ** 0.5


def utils_fixture(pyrecon):
    """pyrecon.utils conversions: sky <-> Cartesian (f4, f8), DistanceToRedshift, random_box_positions."""
    from pyrecon import utils
    out = {}
    rng = np.random.default_rng(44)
    for dtype in ['f4', 'f8']:
        pos = (rng.normal(size=(500, 3)) * 800.).astype(dtype)
        out['pos_' + dtype] = pos
        for degree in [True, False]:
            for wrap in [True, False]:
                d, ra, dec = utils.cartesian_to_sky(pos, wrap=wrap, degree=degree)
                tag = '{}_{:d}{:d}'.format(dtype, degree, wrap)
                out['dist_' + tag], out['ra_' + tag], out['dec_' + tag] = d, ra, dec
            d, ra, dec = utils.cartesian_to_sky(pos, degree=degree)
            out['xyz_{}_{:d}'.format(dtype, degree)] = utils.sky_to_cartesian(d, ra, dec, degree=degree)
    d2z = utils.DistanceToRedshift(distance_of_z)
    r = np.linspace(0., 5000., 301)
    out['d2z_r'], out['d2z_z'] = r, d2z(r)
    out['box'] = utils.random_box_positions(1000., boxcenter=[100., 0., -50.], size=200, seed=42, dtype='f4')
    out['box_nbar'] = utils.random_box_positions([10., 20., 30.], nbar=0.5, seed=7)
    return out


def main(names=None):
    """Write every fixture, or only those named (case names, 'mesh_kernels')."""
    with tempfile.TemporaryDirectory() as tmp:
        pyrecon = import_reference(tmp)
        if not names or 'mesh_kernels' in names:
            np.savez_compressed(os.path.join(HERE, 'mesh_kernels.npz'), **mesh_kernels(pyrecon))
        if not names or 'utils' in names:
            np.savez_compressed(os.path.join(HERE, 'utils.npz'), **utils_fixture(pyrecon))
        for seed, case in enumerate(CASES):
            if names and case['name'] not in names:
                continue
            out = run_case(pyrecon, case, seed)
            np.savez_compressed(os.path.join(HERE, case['name'] + '.npz'), **out)
            print('wrote', case['name'])


if __name__ == '__main__':
    main(sys.argv[1:])
