"""
CPU-only tests: the C ABI library loads and exports every entry point of
include/pyrecon_cuda.h (no compute call without a GPU), and the host-side logic of the
drop-in (geometry, nmesh selection, line of sight, argument checks) matches the reference.
"""
import os
import re
import ctypes
import warnings

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, 'include', 'pyrecon_cuda.h')).read()
    return sorted(set(re.findall(r'^PRC_API [^(]*?\b(prc_\w+)\(', text, flags=re.M)))


def test_library_exports_every_header_symbol():
    from pyrecon_b200 import _lib
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 40
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding declares a signature for every entry point, and nothing else
    assert sorted(_lib.exported_symbols()) == names
    # exported with default visibility from the .so itself
    out = os.popen('nm -D --defined-only {}'.format(_lib.library_path())).read()
    for name in names:
        assert re.search(r'\bT {}\b'.format(name), out), name


def test_host_only_entry_points():
    from pyrecon_b200 import _lib
    lib = _lib.load()
    assert lib.prc_version().startswith(b'pyrecon_b200')
    assert _lib.status_string(2) == 'workspace too small'
    assert lib.prc_fft_supported(_lib.i3((512, 512, 512))) == 1
    assert lib.prc_fft_supported(_lib.i3((384, 192, 320))) == 1
    assert lib.prc_fft_supported(_lib.i3((13, 16, 15))) == 1      # any size: prime factors, odd last axis
    assert lib.prc_fft_supported(_lib.i3((2049, 16, 16))) == 0    # above 2048
    assert lib.prc_assign_cic_workspace_bytes(_lib.i3((512, 512, 512)), 25_000_000, 4) > 25_000_000 * 16
    assert lib.prc_iterative_fft_workspace_bytes(_lib.i3((512, 512, 512)), 4, 1) > 7 * 512 * 512 * 257 * 8
    assert lib.prc_multigrid_workspace_bytes(_lib.i3((64, 64, 64)), 4, 1) > 64 ** 3 * 8 * 2
    # argument checks run before anything touches a device
    assert lib.prc_assign_cic(None, None, _lib.i3((8, 8, 8)), _lib.d3([1.] * 3), _lib.d3([0.] * 3), 8, None, 8, None, 0,
                              0, 0, 0, None, None, 0, None) == 1
    # real-space smoothing: taps of a half-width (2.5 * 0.09 * 64 + 1 -> 15 cells) stored as rows + weights
    nm64 = _lib.i3((64, 64, 64))
    small = lib.prc_smooth_gaussian_real_workspace_bytes(nm64, _lib.d3([0.09] * 3), 2.5, 4)
    assert 4 * 4 * 31 * 31 * 0.5 < small < 256 + 16 * 31 * 31 + 4 * 31 ** 3
    assert lib.prc_smooth_gaussian_real_workspace_bytes(nm64, _lib.d3([0.09] * 3), 2.5, 8) > small
    assert lib.prc_smooth_gaussian_real_workspace_bytes(nm64, _lib.d3([40.] * 3), 2.5, 4) == 0      # too wide
    assert lib.prc_smooth_gaussian_real_workspace_bytes(nm64, _lib.d3([0., 0.1, 0.1]), 2.5, 4) == 0  # no radius
    buf = ctypes.c_void_p(4096)
    assert lib.prc_smooth_gaussian_real_f32(buf, buf, nm64, _lib.d3([0.09] * 3), 2.5, None, 0, None) == 1  # in place
    assert lib.prc_density_contrast_original_workspace_bytes() >= 4 * 8
    assert lib.prc_density_contrast_original_f64(None, None, nm64, 2., 0.75, None, None, 0, None) == 1


def test_meshinfo_semantics():
    from pyrecon_b200 import MeshInfo, MeshError
    info = MeshInfo(boxsize=1000., boxcenter=0., nmesh=64)
    assert np.all(info.boxsize == 1000)
    info.boxsize = 2000.
    assert np.all(info.boxsize == 2000)
    assert info.nmesh.dtype == np.int32
    info = MeshInfo(boxsize=1000., boxcenter=0., nmesh=64, dtype='f4')
    assert info.boxsize.dtype == np.float32
    pos = np.random.default_rng(0).uniform(-100, 100, (1000, 3))
    info = MeshInfo(positions=pos, nmesh=32, boxpad=2.)
    np.testing.assert_allclose(info.boxsize, 2. * (pos.max(axis=0) - pos.min(axis=0)))
    with pytest.raises(MeshError):
        MeshInfo(nmesh=32)
    with pytest.raises(MeshError):
        MeshInfo(positions=pos, boxsize=10., nmesh=32)
    info = MeshInfo(positions=pos, cellsize=10., boxsize=300.)
    assert np.all(info.nmesh == 30)
    w = ((pos + 1000.) - info.offset) % info.boxsize + info.offset
    np.testing.assert_allclose(info.wrap(pos + 1000.), w)


def test_select_nmesh_matches_reference_rule():
    from pyrecon_b200.multigrid import OriginalMultiGridReconstruction as MG
    sel = MG._select_nmesh
    assert list(sel(np.array([12, 13, 17]))) == [12, 14, 20]
    assert list(sel(np.array([512, 500, 384]))) == [512, 512, 384]
    assert list(sel(np.array([64, 65, 100]))) == [64, 80, 112]


def test_reconstruction_needs_gpu_or_raises():
    """No silent CPU path: without a CUDA device the constructor raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    from pyrecon_b200 import MultiGridReconstruction
    from pyrecon_b200._lib import LibraryError
    with pytest.raises(LibraryError):
        MultiGridReconstruction(f=0.8, bias=2., nmesh=16, boxsize=100., boxcenter=0.)


def test_fft_engine_kwargs_accepted():
    """The reference's FFTW / threading keywords are accepted (and ignored) by the constructor signature."""
    import inspect
    from pyrecon_b200 import BaseReconstruction
    params = inspect.signature(BaseReconstruction.__init__).parameters
    for name in ['f', 'bias', 'los', 'fft_engine', 'fft_wisdom', 'save_fft_wisdom', 'fft_plan', 'wrap']:
        assert name in params


def _replica_worker(rank, world, port, out):
    import os
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        # rank r "timed" 10 (r + 1) ms: every rank must see the slowest one, as bench.py reports it
        ms = bench.reduce_max(10. * (rank + 1), world, 'cpu')
        dist.barrier()
        out[rank] = ms
    finally:
        dist.destroy_process_group()


def test_replicas_timing_is_the_max_over_ranks_gloo():
    """The N>1 host logic of bench.py (independent replicas, max over ranks) on two gloo ranks."""
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context('spawn')
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(out) == {0: 20., 1: 20.}


def _utils_fixture():
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, 'utils.npz'))
    return {k: z[k] for k in z.files}


def test_sky_cartesian_match_reference():
    """cartesian_to_sky / sky_to_cartesian equal the reference's outputs (numpy, f4 and f8)."""
    from pyrecon_b200 import utils
    g = _utils_fixture()
    for dtype in ['f4', 'f8']:
        pos = g['pos_' + dtype]
        for degree in [True, False]:
            for wrap in [True, False]:
                tag = '{}_{:d}{:d}'.format(dtype, degree, wrap)
                d, ra, dec = utils.cartesian_to_sky(pos, wrap=wrap, degree=degree)
                for name, v in zip(['dist_', 'ra_', 'dec_'], [d, ra, dec]):
                    assert v.dtype == g[name + tag].dtype
                    np.testing.assert_array_equal(v, g[name + tag])
            d, ra, dec = utils.cartesian_to_sky(pos, degree=degree)
            xyz = utils.sky_to_cartesian(d, ra, dec, degree=degree)
            ref = g['xyz_{}_{:d}'.format(dtype, degree)]
            assert xyz.dtype == ref.dtype
            np.testing.assert_array_equal(xyz, ref)


def test_distance_to_redshift_and_box_positions_match_reference():
    from pyrecon_b200 import utils
    g = _utils_fixture()
    d2z = utils.DistanceToRedshift(lambda z: 2997.92458 * z / (1. + 0.6 * z) ** 0.5)
    np.testing.assert_allclose(d2z(g['d2z_r']), g['d2z_z'], rtol=1e-12, atol=1e-14)
    box = utils.random_box_positions(1000., boxcenter=[100., 0., -50.], size=200, seed=42, dtype='f4')
    assert box.dtype == g['box'].dtype
    np.testing.assert_array_equal(box, g['box'])
    np.testing.assert_array_equal(utils.random_box_positions([10., 20., 30.], nbar=0.5, seed=7), g['box_nbar'])
    with pytest.raises(ValueError):
        utils.random_box_positions(10.)


def test_memory_monitor_and_mkdir(tmp_path, capsys):
    from pyrecon_b200 import utils
    d = str(tmp_path / 'a' / 'b')
    utils.mkdir(d)
    utils.mkdir(d)                      # existing: no error
    assert os.path.isdir(d)
    with utils.MemoryMonitor() as mem:
        mem('step')
    out = capsys.readouterr().out
    assert '[step] using' in out and 'increase of' in out


def test_serving_admission_counts_resident_slot_memory():
    """The request loop's admission: each slot's stream keeps (at least) the largest job it ran, so a job
    goes to a free slot only if every slot's resident memory, that slot grown to the job, fits the budget;
    a slot that already holds enough is preferred (it adds nothing)."""
    import types
    from pyrecon_b200.serving import ReconstructionServer
    srv = types.SimpleNamespace(hbm_budget=100., _resident=[60., 0., 0.], _free_streams=[0, 1, 2])
    assert ReconstructionServer._pick_slot(srv, 30.) == (0, 70.)      # slot 0 holds 60 >= 30; may grow to 100
    srv._free_streams = [1, 2]                                        # slot 0 busy with its 60
    assert ReconstructionServer._pick_slot(srv, 50.) == (None, 0.)    # 60 + 50 > 100
    assert ReconstructionServer._pick_slot(srv, 40.) == (1, 0.)
    srv._resident = [60., 10., 30.]
    assert ReconstructionServer._pick_slot(srv, 20.) == (2, 10.)      # slot 2 holds 30: nothing added


def test_serving_batch_keys():
    """Queued multigrid and plane-parallel requests of the same mesh and settings share a batch key (one
    batched run); another mesh, other settings, catalogue-derived geometry or another algorithm do not."""
    from pyrecon_b200.serving import ReconstructionRequest, batch_key
    cat = np.zeros((10, 3))
    box = dict(f=0.8, bias=2., los='z', boxsize=1000., boxcenter=500., wrap=True, dtype='f4',
               density_kwargs=dict(smoothing_radius=15.))

    def req(algo, **kw):
        args = dict(box, **kw)
        return ReconstructionRequest(algo, data=cat, **args)

    for algo in ['MultiGridReconstruction', 'PlaneParallelFFTReconstruction']:
        a, b = req(algo, nmesh=64), req(algo, nmesh=64)
        assert batch_key(a) is not None and batch_key(a) == batch_key(b)
        assert batch_key(req(algo, nmesh=128)) != batch_key(a)
        assert batch_key(req(algo, nmesh=64, f=0.7)) != batch_key(a)
        assert batch_key(ReconstructionRequest(algo, data=cat, positions=cat, **box)) is None
    assert batch_key(req('MultiGridReconstruction', nmesh=64)) != batch_key(req('PlaneParallelFFTReconstruction',
                                                                               nmesh=64))
    assert batch_key(req('IterativeFFTReconstruction', nmesh=64)) is None


def test_flag_words_map_to_mesh_errors():
    """Every PRC_FLAG_* bit the kernels can raise (box, NaN/inf, a bounded device wait that gave up) turns
    into MeshError on the host; the header and the binding agree on the values."""
    from pyrecon_b200 import _lib, MeshError
    from pyrecon_b200.mesh import _Flags
    text = open(os.path.join(ROOT, 'include', 'pyrecon_cuda.h')).read()
    for name in ['PRC_FLAG_OUT_OF_BOX', 'PRC_FLAG_NONFINITE', 'PRC_FLAG_DEVICE_WAIT']:
        value = int(re.search(r'#define {}\s+(\d+)'.format(name), text).group(1))
        assert getattr(_lib, name) == value
        fl = _Flags('cpu')
        fl.t[0] = value
        with pytest.raises(MeshError):
            fl.raise_if_set(0., 1.)
    fl = _Flags('cpu')
    fl.raise_if_set(0., 1.)
