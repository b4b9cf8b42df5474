"""Eisenstein et al. 2007 plane-parallel reconstruction (pyrecon/plane_parallel_fft.py) on CUDA."""
from . import _lib
from .mesh import RealMesh, MeshError, torch_dtype
from .recon import BaseReconstruction, ReconstructionError, FFTShiftsMixin


class PlaneParallelFFTReconstruction(FFTShiftsMixin, BaseReconstruction):
    r"""
    :math:`\psi_a = \mathrm{IFFT}(i k_a \delta_k / (k^2 (1 + \beta \mu^2)))` with a global line of sight
    (Eisenstein et al. 2007, section 3; pyrecon/plane_parallel_fft.py:41-55).
    """

    def __init__(self, los=None, **kwargs):
        super(PlaneParallelFFTReconstruction, self).__init__(los=los, **kwargs)

    def set_los(self, los=None):
        super(PlaneParallelFFTReconstruction, self).set_los(los=los)
        if self.los is None:
            raise ReconstructionError('A (global) line-of-sight must be provided')

    def run(self):
        """Compute the Zeldovich displacements :attr:`mesh_psi`."""
        import torch
        with self._stream_ctx():
            nm, bs, _ = self.info.c_geometry()
            lib = _lib.load()
            psi4, psis = self._new_psi()
            ws = self._ws.get(lib.prc_plane_parallel_workspace_bytes(nm, self.info.dtype.itemsize))
            _lib.call('prc_plane_parallel_fft_' + _lib.suffix(self.info.dtype), _lib.ptr(self.mesh_delta.value), nm, bs,
                      float(self.beta), _lib.d3([float(x) for x in self.los]), *self._psi_pointers(psi4), 4,
                      _lib.ptr(ws), ws.numel(), _lib.stream_of(self.device), error=MeshError)
            del self.mesh_delta
            self._psi4 = psi4
            self.mesh_psi = psis


def run_batch(recons):
    """:meth:`PlaneParallelFFTReconstruction.run` of several reconstructions at once, on the first one's stream
    and workspace: the meshes share the launches of every FFT pass, two at a time.  They must share the mesh
    (nmesh, boxsize, dtype), the line of sight, beta and the device, and have their density contrast set.
    Results equal separate :meth:`~PlaneParallelFFTReconstruction.run` calls."""
    import torch
    recons = list(recons)
    if not recons:
        return
    r0 = recons[0]
    key = lambda r: (tuple(r.info.nmesh), tuple(r.info.boxsize), r.info.dtype, tuple(float(x) for x in r.los),
                     float(r.beta), str(r.device))
    for r in recons:
        if not isinstance(r, PlaneParallelFFTReconstruction):
            raise ValueError('run_batch takes plane-parallel reconstructions')
        if key(r) != key(r0):
            raise ValueError('run_batch needs the same mesh, line of sight, beta and device')
        if getattr(r, 'mesh_delta', None) is None:
            raise ReconstructionError('set_density_contrast must be called before run')
    streams = [r.stream if r.stream is not None else torch.cuda.current_stream(r.device) for r in recons]
    with r0._stream_ctx():
        st0 = streams[0]
        for st in streams[1:]:
            if st != st0:
                st0.wait_stream(st)         # the other reconstructions' density contrasts are done
        nm, bs, _ = r0.info.c_geometry()
        lib = _lib.load()
        count = len(recons)
        outs = [r._new_psi() for r in recons]
        # component a of every interleaved psi (psi_stride 4)
        comp = lambda a: (_lib.c_void_p * count)(*[psi4.data_ptr() + a * psi4.element_size() for psi4, _ in outs])
        ws = r0._ws.get(lib.prc_plane_parallel_batch_workspace_bytes(nm, r0.info.dtype.itemsize, count))
        _lib.call('prc_plane_parallel_fft_batch_' + _lib.suffix(r0.info.dtype),
                  _lib.pointer_array([r.mesh_delta.value for r in recons]),
                  comp(0), comp(1), comp(2), count, nm, bs, float(r0.beta),
                  _lib.d3([float(x) for x in r0.los]), 4, _lib.ptr(ws), ws.numel(), _lib.stream_of(r0.device),
                  error=MeshError)
        for r, st, (psi4, psis) in zip(recons, streams, outs):
            if st != st0:
                st.wait_stream(st0)         # later work on that reconstruction's stream sees its psi
                psi4.record_stream(st)
            del r.mesh_delta
            r._psi4 = psi4
            r.mesh_psi = psis
