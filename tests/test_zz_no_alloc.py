"""
The allocation-free paint, prc_assign_cic_noalloc, for callers that cannot allocate device
memory: it must give the same mesh as prc_assign_cic (to the FP64 rounding of its chunked
accumulation, the 1e-13 the paint tests use) on consecutive calls that share its built-in
scratch, and refuse meshes beyond its stated maximum.  Collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    from pyrecon_b200 import _lib
    return torch, _lib


def _catalog(n, seed, dtype):
    rng = np.random.default_rng(seed)
    pos = (rng.uniform(-0.5, 0.5, (n, 3)) * np.array([1000., 900., 800.]) + np.array([100., 0., 2000.])).astype(dtype)
    w = rng.uniform(0.5, 1.5, n).astype(dtype)
    return pos, w


def _paint(name, pos, w, nmesh, mesh_bytes, accumulate_into=None):
    torch, L = _setup()
    n = tuple(nmesh)
    mesh = accumulate_into.clone() if accumulate_into is not None else torch.zeros(n, dtype=torch.float64, device='cuda')
    colsums = torch.zeros(n[0] * n[1], dtype=torch.float64, device='cuda')
    flags = torch.zeros(1, dtype=torch.int32, device='cuda')
    dpos = torch.from_numpy(pos).cuda()
    dw = torch.from_numpy(w).cuda()
    nm, bs, bc = L.i3(n), L.d3([1000., 900., 800.]), L.d3([100., 0., 2000.])
    st = L.stream_of(torch.device('cuda'))
    args = [L.ptr(mesh), L.ptr(colsums), nm, bs, bc, mesh_bytes, L.ptr(dpos), pos.dtype.itemsize, L.ptr(dw),
            w.dtype.itemsize, len(pos), 0, int(accumulate_into is not None), L.ptr(flags)]
    if name == 'prc_assign_cic':
        ws = torch.empty(L.load().prc_assign_cic_workspace_bytes(nm, len(pos), mesh_bytes), dtype=torch.uint8,
                         device='cuda')
        args += [L.ptr(ws), ws.numel()]
    L.call(name, *args, st)
    torch.cuda.synchronize()
    assert int(flags.item()) == 0
    return mesh, colsums


@pytest.mark.parametrize('dtype', ['f4', 'f8'])
def test_noalloc_paint_matches_workspace_paint_twice(dtype):
    torch, _ = _setup()
    nmesh = (64, 48, 40)
    mesh_bytes = np.dtype(dtype).itemsize
    for call, (npos, seed) in enumerate([(700_000, 1), (150_000, 2)]):   # 3 chunks, then 1 chunk
        pos, w = _catalog(npos, seed, dtype)
        ref, ref_cols = _paint('prc_assign_cic', pos, w, nmesh, mesh_bytes)
        got, got_cols = _paint('prc_assign_cic_noalloc', pos, w, nmesh, mesh_bytes)
        scale = float(ref.abs().max())
        assert float((got - ref).abs().max()) <= 1e-13 * scale, call
        assert float((got_cols - ref_cols).abs().max()) <= 1e-12 * float(ref_cols.abs().max()), call
    # accumulating into an existing mesh, as repeated assign_* calls do
    base = ref
    acc_ref, _ = _paint('prc_assign_cic', pos, w, nmesh, mesh_bytes, accumulate_into=base)
    acc_got, _ = _paint('prc_assign_cic_noalloc', pos, w, nmesh, mesh_bytes, accumulate_into=base)
    assert float((acc_got - acc_ref).abs().max()) <= 1e-13 * float(acc_ref.abs().max())


def test_noalloc_paint_rejects_oversized_mesh():
    torch, L = _setup()
    mesh = torch.zeros(1, dtype=torch.float64, device='cuda')
    flags = torch.zeros(1, dtype=torch.int32, device='cuda')
    st = L.stream_of(torch.device('cuda'))
    status = L.load().prc_assign_cic_noalloc(L.ptr(mesh), None, L.i3((2048, 1024, 8)), L.d3([1.] * 3), L.d3([0.] * 3),
                                             8, None, 8, None, 0, 0, 0, 0, L.ptr(flags), st)
    assert status == 4   # PRC_ERR_UNSUPPORTED: more than 2^20 (x, y) columns


def test_noalloc_paint_at_the_stated_maximum():
    """2^20 (x, y) columns in FP64, more particles than one chunk: the largest mesh the built-in scratch
    serves gives the workspace paint's mesh; one more cell along z than 4096 is rejected."""
    torch, L = _setup()
    nmesh = (1024, 1024, 8)
    pos, w = _catalog(600_000, 3, 'f8')
    ref, ref_cols = _paint('prc_assign_cic', pos, w, nmesh, 8)
    got, got_cols = _paint('prc_assign_cic_noalloc', pos, w, nmesh, 8)
    assert float((got - ref).abs().max()) <= 1e-13 * float(ref.abs().max())
    assert float((got_cols - ref_cols).abs().max()) <= 1e-12 * float(ref_cols.abs().max())
    mesh = torch.zeros(1, dtype=torch.float64, device='cuda')
    flags = torch.zeros(1, dtype=torch.int32, device='cuda')
    st = L.stream_of(torch.device('cuda'))
    status = L.load().prc_assign_cic_noalloc(L.ptr(mesh), None, L.i3((8, 8, 4104)), L.d3([1.] * 3), L.d3([0.] * 3),
                                             8, None, 8, None, 0, 0, 0, 0, L.ptr(flags), st)
    assert status == 4   # PRC_ERR_UNSUPPORTED: n2 above 4096
