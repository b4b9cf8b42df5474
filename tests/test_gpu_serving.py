"""
The request loop (pyrecon_b200.serving): requests that run concurrently, on their own streams,
give the same bits as the same requests run alone, one after the other; admission keeps the
requests in flight within the HBM budget.
"""
import numpy as np
import pytest

from pyrecon_b200 import mocks

pytestmark = pytest.mark.gpu


def _requests():
    from pyrecon_b200.serving import ReconstructionRequest
    reqs = []
    # periodic boxes, global line of sight, no randoms (plane-parallel and multigrid)
    for i, (algo, nmesh, dtype) in enumerate([('PlaneParallelFFTReconstruction', 64, 'f4'),
                                              ('MultiGridReconstruction', 48, 'f4'),
                                              ('PlaneParallelFFTReconstruction', 32, 'f8'),
                                              ('MultiGridReconstruction', 32, 'f8')]):
        data = mocks.lognormal_positions_numpy(20000 + 5000 * i, nmesh, 1000., 500., seed=50 + i, field_seed=60 + i)
        reqs.append(ReconstructionRequest(algo, data=data, f=0.8, bias=2., los='z', nmesh=nmesh, boxsize=1000.,
                                          boxcenter=500., wrap=True, dtype=dtype,
                                          density_kwargs=dict(smoothing_radius=15.)))
    # survey-like: local line of sight with randoms
    for i, (algo, dtype) in enumerate([('IterativeFFTReconstruction', 'f4'), ('MultiGridReconstruction', 'f4'),
                                       ('IterativeFFTReconstruction', 'f8')]):
        data = mocks.lognormal_positions_numpy(30000, 32, 1000., 2000., seed=70 + i, field_seed=80 + i)
        randoms = mocks.uniform_positions_numpy(90000, 1000., 2000., seed=90 + i)
        reqs.append(ReconstructionRequest(algo, data=data, randoms=randoms, f=0.8, bias=2., los=None, nmesh=32,
                                          boxsize=1000., boxcenter=2000., dtype=dtype,
                                          density_kwargs=dict(smoothing_radius=15.)))
    return reqs


def _same(a, b):
    assert set(a) == set(b)
    for k in a:
        assert a[k].dtype == b[k].dtype and np.array_equal(a[k], b[k]), k


def test_results_alone_equal_results_in_the_mix():
    from pyrecon_b200.serving import ReconstructionServer, run_request
    reqs = _requests()
    alone = [run_request(r) for r in reqs]
    with ReconstructionServer(slots=4) as server:
        futures = [server.submit(r) for r in reqs]
        mixed = [f.result(timeout=300) for f in futures]
        stats = server.stats()
    assert stats['completed'] == len(reqs) and stats['peak_active'] > 1
    assert stats['p50_ms'] is not None and stats['p99_ms'] >= stats['p50_ms']
    for a, b in zip(alone, mixed):
        _same(a, b)


def test_admission_keeps_requests_within_the_budget():
    from pyrecon_b200.serving import ReconstructionServer, estimate_device_bytes
    reqs = [_requests()[0] for _ in range(3)]                     # three requests of the same size
    budget = 1.5 * estimate_device_bytes(reqs[0])                 # room for one at a time
    with ReconstructionServer(slots=4, hbm_budget=budget) as server:
        futures = [server.submit(r) for r in reqs]
        for f in futures:
            f.result(timeout=300)
        assert server.peak_active == 1
    with ReconstructionServer(slots=2, hbm_budget=budget) as server:
        with pytest.raises(ValueError):
            big = _requests()[4]
            big.kwargs['nmesh'] = 1024
            server.submit(big)


@pytest.mark.parametrize('algorithm,dtype', [('MultiGridReconstruction', 'f4'), ('PlaneParallelFFTReconstruction', 'f4'),
                                             ('PlaneParallelFFTReconstruction', 'f8')])
def test_batched_requests_equal_requests_alone(algorithm, dtype):
    """Queued multigrid or plane-parallel requests of the same mesh and settings run as one job with a
    batched run (one solve, or FFT passes shared by pairs of meshes); each result has the bits of the
    same request run alone."""
    from pyrecon_b200.serving import ReconstructionRequest, ReconstructionServer, run_request, batch_key
    reqs = []
    for i in range(5):
        data = mocks.lognormal_positions_numpy(10000 + 3000 * i, 32, 1000., 500., seed=100 + i, field_seed=110 + i)
        reqs.append(ReconstructionRequest(algorithm, data=data, f=0.8, bias=2., los='z', nmesh=32,
                                          boxsize=1000., boxcenter=500., wrap=True, dtype=dtype,
                                          density_kwargs=dict(smoothing_radius=15.)))
    assert len(set(batch_key(r) for r in reqs)) == 1
    alone = [run_request(r) for r in reqs]
    with ReconstructionServer(slots=1, max_batch=4) as server:
        futures = [server.submit(r) for r in reqs]
        mixed = [f.result(timeout=300) for f in futures]
        assert server.peak_active >= 2          # at least one batch of several requests
    for a, b in zip(alone, mixed):
        _same(a, b)
