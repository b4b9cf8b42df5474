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
