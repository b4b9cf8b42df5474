"""Burden et al. 2015 field-level iterative reconstruction (pyrecon/iterative_fft.py) on CUDA."""
from . import _lib
from .mesh import RealMesh, MeshError, torch_dtype
from .recon import BaseReconstruction, FFTShiftsMixin


class IterativeFFTReconstruction(FFTShiftsMixin, BaseReconstruction):
    """
    Field-level iterative reconstruction (Burden et al. 2015, https://arxiv.org/abs/1504.02591, eqs. 12, 22, 24):
    ``niterations`` RSD-removal iterations on the density contrast, then
    :math:`\\psi_a = \\mathrm{IFFT}(i k_a \\delta_k / k^2)` (pyrecon/iterative_fft.py:12-82).
    """

    def run(self, niterations=3):
        """Compute the Zeldovich displacements :attr:`mesh_psi`."""
        import torch
        with self._stream_ctx():
            nm, bs, bc = self.info.c_geometry()
            lib = _lib.load()
            psi4, psis = self._new_psi()
            self.log_info('Running {:d} iterations.'.format(niterations))
            ws = self._ws.get(lib.prc_iterative_fft_workspace_bytes(nm, self.info.dtype.itemsize, int(self.los is None)))
            _lib.call('prc_iterative_fft_' + _lib.suffix(self.info.dtype), _lib.ptr(self.mesh_delta.value), nm, bs, bc,
                      float(self.beta), self._los_arg(), int(niterations), *self._psi_pointers(psi4), 4,
                      _lib.ptr(ws), ws.numel(), _lib.stream_of(self.device), error=MeshError)
            self._iter = int(niterations)
            del self.mesh_delta
            self._psi4 = psi4
            self.mesh_psi = psis
