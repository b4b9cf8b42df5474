"""Shared helpers for the test-suite (golden fixtures, oracle runs, GPU runs)."""
import json
import os

import numpy as np

from conftest import GOLDEN
from oracle import pipeline

ALGOS = {'multigrid': 'MultiGridReconstruction', 'iterative_fft': 'IterativeFFTReconstruction',
         'plane_parallel_fft': 'PlaneParallelFFTReconstruction',
         'iterative_fft_particle': 'IterativeFFTParticleReconstruction',
         'multigrid_original': 'OriginalMultiGridReconstruction'}


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + '.npz'))
    out = {k: z[k] for k in z.files}
    out['meta'] = json.loads(str(out['meta']))
    return out


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def run_oracle(g, dtype=None, kernels='oracle'):
    """Oracle run on a golden case's inputs, returning the same keys as the fixture."""
    m = g['meta']
    rec = pipeline.OracleReconstruction(m['algorithm'], f=m['f'], bias=m['bias'], los=m['los'], nmesh=m['nmesh'],
                                        boxsize=m['boxsize'], boxcenter=m['boxcenter'], dtype=dtype or m['dtype'],
                                        wrap=m['wrap'], kernels=kernels)
    data = g['data'].astype(dtype) if dtype else g['data']
    out = {}
    rec.assign_data(data, g['wdata'])
    out['mesh_data'] = rec.mesh_data.copy()
    if m['randoms']:
        randoms = g['randoms'].astype(dtype) if dtype else g['randoms']
        rec.assign_randoms(randoms, g['wrandoms'])
        out['mesh_randoms'] = rec.mesh_randoms.copy()
    rec.set_density_contrast(smoothing_radius=m['smoothing_radius'], **m.get('density_kwargs', {}))
    out['mesh_delta'] = rec.mesh_delta.copy()
    rec.run()
    if m['algorithm'] in ('multigrid', 'multigrid_original'):
        out['mesh_phi'] = rec.mesh_phi
    else:
        out['mesh_psi'] = np.stack(rec.mesh_psi)
    out['shifts_disp'] = rec.read_shifts(data, field='disp')
    out['shifts_rsd'] = rec.read_shifts(data, field='rsd')
    out['shifted_data'] = rec.read_shifted_positions(data)
    if m['randoms']:
        out['shifted_randoms'] = rec.read_shifted_positions(randoms)
    if m['algorithm'] == 'iterative_fft_particle':
        out['shifts_data_disp'] = rec.read_shifts('data', field='disp')
        out['shifts_data_rsd'] = rec.read_shifts('data', field='rsd')
        out['shifted_data_str'] = rec.read_shifted_positions('data')
    return out


def run_gpu(g, dtype=None, **kwargs):
    """The CUDA pipeline on a golden case's inputs (numpy in, numpy out, as a user calls it)."""
    import pyrecon_b200
    m = g['meta']
    Cls = getattr(pyrecon_b200, ALGOS[m['algorithm']])
    rec = Cls(f=m['f'], bias=m['bias'], los=m['los'], nmesh=m['nmesh'], boxsize=m['boxsize'],
              boxcenter=m['boxcenter'], dtype=dtype or m['dtype'], wrap=m['wrap'], **kwargs)
    data = g['data'].astype(dtype) if dtype else g['data']
    out = {}
    rec.assign_data(data, g['wdata'])
    out['mesh_data'] = rec.mesh_data._accum.cpu().numpy()
    if m['randoms']:
        randoms = g['randoms'].astype(dtype) if dtype else g['randoms']
        rec.assign_randoms(randoms, g['wrandoms'])
        out['mesh_randoms'] = rec.mesh_randoms._accum.cpu().numpy()
    rec.set_density_contrast(smoothing_radius=m['smoothing_radius'], **m.get('density_kwargs', {}))
    out['mesh_delta'] = np.asarray(rec.mesh_delta)
    rec.run()
    if m['algorithm'] in ('multigrid', 'multigrid_original'):
        out['mesh_phi'] = np.asarray(rec.mesh_phi)
    else:
        out['mesh_psi'] = np.stack([np.asarray(p) for p in rec.mesh_psi])
    out['shifts_disp'] = rec.read_shifts(data, field='disp')
    out['shifts_rsd'] = rec.read_shifts(data, field='rsd')
    out['shifted_data'] = rec.read_shifted_positions(data)
    if m['randoms']:
        out['shifted_randoms'] = rec.read_shifted_positions(randoms)
    if m['algorithm'] == 'iterative_fft_particle':
        out['shifts_data_disp'] = rec.read_shifts('data', field='disp')
        out['shifts_data_rsd'] = rec.read_shifts('data', field='rsd')
        out['shifted_data_str'] = rec.read_shifted_positions('data')
    return out, rec


def maxrel(a, b):
    a = np.asarray(a, dtype='f8')
    b = np.asarray(b, dtype='f8')
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def maxabs(a, b):
    return np.abs(np.asarray(a, dtype='f8') - np.asarray(b, dtype='f8')).max()
