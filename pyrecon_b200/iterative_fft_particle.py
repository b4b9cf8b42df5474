"""
IterativeFFTParticleReconstruction (Bautista et al. 2018) on CUDA (pyrecon/iterative_fft_particle.py).

The reconstruction iterates on the data positions: every iteration paints the current
reconstructed real-space data positions (after the first), smooths them, forms the density
contrast against the smoothed randoms, solves for the Zeldovich displacement and moves the
data by the RSD part of it.  Paint, smoothing, displacement and the particle update are this
library's kernels; the positions stay on the device between iterations.
"""
import numpy as np

from . import _lib
from .mesh import RealMesh, MeshError, Particles, torch_dtype, _array3
from .recon import BaseReconstruction, ReconstructionError, FFTShiftsMixin, ALLOWED_FIELDS


class OriginalIterativeFFTParticleReconstruction(FFTShiftsMixin, BaseReconstruction):
    """
    Iterative reconstruction on the data particles (pyrecon/iterative_fft_particle.py:9-244).
    ``read_shifts('data')`` / ``read_shifted_positions('data')`` give the data at their own
    reconstructed real-space positions.
    """

    # its read-outs gather through prc_ifftp_read (cell order only): no sorted copy of the catalogues
    _sorted_positions = False

    def assign_data(self, positions, weights=None, check=True):
        """Paint data and keep positions and weights for :meth:`run` (iterative_fft_particle.py:16-33)."""
        import torch
        with self._stream_ctx():
            p = Particles(positions, self.device, weights=weights, weight_dtype=None)
            w = p.weights
            if w is None:
                w = torch.ones(p.size, dtype=p.pos.dtype, device=self.device)
            if getattr(self, '_positions_data', None) is None:
                self._positions_data, self._weights_data = p.pos, w
                self._data_kind = p
            else:
                self._positions_data = torch.cat([self._positions_data, p.pos.to(self._positions_data.dtype)], dim=0)
                self._weights_data = torch.cat([self._weights_data, w.to(self._weights_data.dtype)], dim=0)
            order, _ = self._new_order(positions)
            self.mesh_data.assign_cic(p.pos, weights=w, wrap=self.wrap, check=check, order_out=order)
            self._keep_order(positions, order)

    def set_density_contrast(self, ran_min=0.01, smoothing_radius=15., check=False, **kwargs):
        """Keep ``ran_min`` and ``smoothing_radius`` for :meth:`run` and set :attr:`mesh_delta` from the
        meshes as they are (run smooths them first; iterative_fft_particle.py:35-63)."""
        import torch
        self.ran_min = ran_min
        self.smoothing_radius = smoothing_radius
        if not self.mesh_data.is_set:
            raise ReconstructionError('assign_data must be called before set_density_contrast')
        with self._stream_ctx():
            sums = self._sums_of(self.mesh_data._accum, self.mesh_randoms._accum if self.has_randoms else None)
            self.mesh_delta = self._delta(self.mesh_data._accum, self.mesh_randoms._accum if self.has_randoms else None,
                                          sums)

    # -- device steps --

    def _sums_of(self, data, randoms):
        import torch
        lib = _lib.load()
        st = _lib.stream_of(self.device)
        sums = torch.zeros(2, dtype=torch.float64, device=self.device)
        ws = self._ws.get(lib.prc_sum_workspace_bytes(0))
        for i, m in enumerate([data, randoms]):
            if m is None:
                continue
            name = 'prc_sum_f64' if m.dtype == torch.float64 else 'prc_sum_f32'
            _lib.call(name, _lib.ptr(m), m.numel(), _lib.c_void_p(sums.data_ptr() + 8 * i), _lib.ptr(ws), ws.numel(), st)
        return sums

    def _delta(self, data, randoms, sums):
        import torch
        nm, _, _ = self.info.c_geometry()
        delta = RealMesh(info=self.info, device=self.device)
        delta.__dict__['value'] = torch.empty(self.info.shape, dtype=torch_dtype(self.info.dtype), device=self.device)
        _lib.call('prc_delta_from_meshes_' + _lib.suffix(self.info.dtype), _lib.ptr(data), _lib.ptr(randoms),
                  data.element_size(), _lib.ptr(sums), nm, float(self.bias), float(self.ran_min),
                  float(self._size_randoms), _lib.ptr(delta.value), _lib.stream_of(self.device), error=MeshError)
        return delta

    def _smooth(self, accum):
        import torch
        lib = _lib.load()
        nm, bs, _ = self.info.c_geometry()
        out = torch.empty(self.info.shape, dtype=torch_dtype(self.info.dtype), device=self.device)
        ws = self._ws.get(lib.prc_fft_workspace_bytes(nm, self.info.dtype.itemsize, 1))
        radius = _array3(self.smoothing_radius, self.info._type_float)
        _lib.call('prc_smooth_gaussian_' + _lib.suffix(self.info.dtype), _lib.ptr(accum), accum.element_size(),
                  _lib.ptr(out), nm, bs, _lib.d3(radius), _lib.ptr(ws), ws.numel(), _lib.stream_of(self.device),
                  error=MeshError)
        return out

    def _paint_reconstructed(self):
        """Fresh mesh of the reconstructed data positions, always wrapped (iterative_fft_particle.py:86-93)."""
        import torch
        from .mesh import paint
        accum = torch.empty(self.info.shape, dtype=torch.float64, device=self.device)
        colsums = torch.empty(int(self.info.nmesh[0]) * int(self.info.nmesh[1]), dtype=torch.float64,
                              device=self.device)
        p = Particles(self._positions_rec_data, self.device, weights=self._weights_data)
        paint(self.info, accum, colsums, p, True, False, self._ws, self._flags, check=False)
        return accum

    def run(self, niterations=3):
        """Iterate (iterative_fft_particle.py:65-146); sets :attr:`mesh_psi` (last iteration's displacement)."""
        import torch
        if not hasattr(self, 'smoothing_radius'):
            self.ran_min, self.smoothing_radius = 0.01, 15.
        lib = _lib.load()
        nm, bs, bc = self.info.c_geometry()
        with self._stream_ctx():
            st = _lib.stream_of(self.device)
            data_s = self._smooth(self.mesh_data._accum)
            randoms_s = self._smooth(self.mesh_randoms._accum) if self.has_randoms else None
            sums = self._sums_of(data_s, randoms_s)
            self._positions_rec_data = self._positions_data.clone()
            pbytes = self._positions_data.element_size()
            psi4 = None
            for it in range(niterations):
                if it > 0:
                    data_s = self._smooth(self._paint_reconstructed())
                    sums = self._sums_of(data_s, randoms_s)
                delta = self._delta(data_s, randoms_s, sums)
                psi4, meshes = self._new_psi()
                ws = self._ws.get(lib.prc_zeldovich_psi_workspace_bytes(nm, self.info.dtype.itemsize))
                _lib.call('prc_zeldovich_psi_' + _lib.suffix(self.info.dtype), _lib.ptr(delta.value), nm, bs,
                          *self._psi_pointers(psi4), 4, _lib.ptr(ws), ws.numel(), st, error=MeshError)
                _lib.call('prc_ifftp_update_' + _lib.suffix(self.info.dtype), _lib.ptr(psi4), nm, bs, bc,
                          _lib.ptr(self._positions_data), _lib.ptr(self._positions_rec_data), pbytes,
                          len(self._positions_data), float(self.f), float(self.beta), int(it == 0), self._los_arg(),
                          int(self.wrap), self._flags.ptr, st, error=MeshError)
            if psi4 is not None:
                self._psi4, self.mesh_psi = psi4, meshes
            self.__dict__.pop('mesh_delta', None)
            self.mesh_randoms = RealMesh(info=self.info, device=self.device)

    # -- shifts (iterative_fft_particle.py:148-244) --

    def _read(self, positions, field, shifted):
        import torch
        field = field.lower()
        if field not in ALLOWED_FIELDS:
            raise ReconstructionError('Unknown field {}. Choices are {}'.format(field, ALLOWED_FIELDS))
        if not hasattr(self, '_psi4'):
            raise ReconstructionError('run() must be called before reading shifts')
        nm, bs, bc = self._geometry_args()
        data_mode = isinstance(positions, str)
        if data_mode and positions != 'data':
            raise ReconstructionError('positions must be an array or "data"')
        with self._stream_ctx():
            order = None
            if data_mode:
                pos, rec, kind = self._positions_data, self._positions_rec_data, self._data_kind
                n, pbytes = len(pos), pos.element_size()
            else:
                kind = Particles(positions, self.device)
                pos, rec, n, pbytes = kind.pos, None, kind.size, kind.pos_bytes
                order = self._order_for(positions)
            obytes = max(pbytes, self.info.dtype.itemsize) if (shifted and self.wrap) else pbytes
            out = torch.empty((n, 3), dtype=torch_dtype('f4' if obytes == 4 else 'f8'), device=self.device)
            _lib.call('prc_ifftp_read_' + _lib.suffix(self.info.dtype), _lib.ptr(self._psi4), nm, bs, bc, _lib.ptr(pos),
                      _lib.ptr(rec), pbytes, n, float(self.f), self._los_arg(), _lib.FIELDS[field], int(shifted),
                      int(self.wrap), _lib.ptr(out), obytes, self._flags.ptr, _lib.ptr(order),
                      _lib.stream_of(self.device), error=MeshError)
            low, high = self.info.boxcenter - self.info.boxsize / 2., self.info.boxcenter + self.info.boxsize / 2.
            self._flags.raise_if_set(low, high)
            _lib.check_device_faults(ReconstructionError)
            return kind.output(out)


class IterativeFFTParticleReconstruction(OriginalIterativeFFTParticleReconstruction):
    """Any update / test / improvement upon original algorithm (iterative_fft_particle.py:241-244)."""
