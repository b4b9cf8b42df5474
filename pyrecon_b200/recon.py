"""
BaseReconstruction: the reference's pipeline (pyrecon/recon.py) on one CUDA device.

    recon = MultiGridReconstruction(f=0.8, bias=2.0, los=None, nmesh=512, boxsize=1000., boxcenter=2000.)
    recon.assign_data(positions_data, weights_data)
    recon.assign_randoms(positions_randoms, weights_randoms)
    recon.set_density_contrast()
    recon.run()
    positions_rec_data = recon.read_shifted_positions(positions_data)

Positions and weights may be numpy arrays, CPU torch tensors (pinned memory makes the
host-to-device copies asynchronous) or CUDA tensors; results come back in the same kind of
container.  ``dtype='f4'`` runs the FP32 pipeline with FP64 cloud-in-cell sums, FP64
normalisation and (multigrid) FP64 defect correction; ``dtype='f8'`` runs everything in FP64.
"""
import weakref

import numpy as np

from . import _lib
from .mesh import (MeshInfo, RealMesh, MeshError, Particles, _Workspace, _Flags, _device_of, torch_dtype, paint,
                   _array3)
from .utils import BaseClass, distance


class ReconstructionError(Exception):
    """Error raised when issue with reconstruction."""


ALLOWED_FIELDS = ['disp', 'rsd', 'disp+rsd']


class BaseReconstruction(BaseClass):
    """Base template reconstruction class (pyrecon/recon.py:15-325).  Algorithms implement :meth:`run`."""

    _needs_fft_mesh = True
    # keep the cell-ordered copy of painted device catalogues for the read-out (prc_assign_cic_sorted)
    _sorted_positions = True

    @staticmethod
    def _select_nmesh(nmesh):
        return nmesh.copy()

    def __init__(self, f=0., bias=1., los=None, fft_engine='numpy', fft_wisdom=None, save_fft_wisdom=None,
                 fft_plan='measure', wrap=False, device=None, mixed_precision=True, stream=None, workspace=None,
                 **kwargs):
        """
        Parameters are the reference's (recon.py:66-120): growth rate ``f``, ``bias``, line of sight
        ``los`` (None / 'local' for a varying one, 'x' / 'y' / 'z' or a 3-vector), ``wrap`` and the
        mesh keywords nmesh, boxsize, boxcenter, cellsize, positions, boxpad, dtype.  ``fft_engine`` and
        ``nthreads`` are accepted for compatibility and ignored (the FFTs are this library's CUDA kernels).
        ``fft_wisdom``, ``save_fft_wisdom`` and ``fft_plan`` keep their meaning for this library's
        autotuner (:mod:`pyrecon_b200.tuning`): ``fft_wisdom`` (a path or dict) is applied to the kernel
        launchers' tuning table; with ``save_fft_wisdom`` (True for the default file name, or a path) that
        file is loaded if it exists, the knobs it lacks for this mesh are timed on the device unless
        ``fft_plan='estimate'``, and the result is saved there.

        Extra: ``device`` (CUDA device, default current), ``mixed_precision`` (dtype 'f4' multigrid
        with FP64 defect correction, default True), ``stream`` (torch.cuda.Stream to enqueue on),
        ``workspace`` (a scratch buffer object kept from an earlier reconstruction, so successive
        reconstructions reuse the same device scratch; see :mod:`pyrecon_b200.serving`).
        """
        import torch
        self.set_cosmo(f=f, bias=bias)
        self.wrap = bool(wrap)
        kwargs.pop('nthreads', None)
        self.info = MeshInfo(select_nmesh=self._select_nmesh, **kwargs)
        self.device = _device_of(device)
        self.stream = stream
        self.mixed_precision = bool(mixed_precision)
        self.set_los(los)
        _lib.load()
        if not _lib.load().prc_fft_supported(_lib.i3(self.info.nmesh)):
            raise MeshError('nmesh {} is not supported by the CUDA FFT (each axis must be between 2 and 2048)'.format(
                self.info.nmesh))
        self.fft_engine = 'cuda'
        from . import tuning
        self.fft_wisdom = tuning.setup(self.info.nmesh, self.info.dtype, fft_wisdom=fft_wisdom,
                                       save_fft_wisdom=save_fft_wisdom, fft_plan=fft_plan,
                                       los=None if self.los is None else list(self.los), device=self.device)
        self._ws = workspace if workspace is not None else _Workspace(self.device)
        self._flags = _Flags(self.device)
        self._size_randoms = 0
        with self._stream_ctx():
            self.mesh_data = self._new_paint_mesh()
            self.mesh_randoms = self._new_paint_mesh()
        self.log_info('Using mesh {}.'.format(self.mesh_data))
        del torch

    def _stream_ctx(self):
        import torch
        if self.stream is None:
            return torch.cuda.device(self.device)
        return torch.cuda.stream(self.stream)

    def _new_paint_mesh(self):
        mesh = RealMesh(info=self.info, device=self.device)
        mesh._ws = self._ws
        mesh._fl = self._flags
        return mesh

    @property
    def beta(self):
        r""":math:`\beta = f / b`."""
        return self.f / self.bias

    def set_cosmo(self, f=None, bias=None, beta=None):
        """recon.py:127-147."""
        if bias is None:
            bias = self.bias
        if beta is not None:
            f = beta * bias
        if f is None:
            f = self.f
        self.f = f
        self.bias = bias

    def set_los(self, los=None):
        """recon.py:149-170: None / 'local' -> local; 'x', 'y', 'z' or a 3-vector -> unit vector."""
        if los is None or (isinstance(los, str) and los == 'local'):
            self.los = None
        else:
            if isinstance(los, str):
                los = 'xyz'.index(los)
            if np.ndim(los) == 0:
                ilos = los
                los = np.zeros(3, dtype=self.info._type_float)
                los[ilos] = 1.
            los = np.array(los, dtype=self.info._type_float)
            self.los = los / distance(los)

    # -- geometry shortcuts (recon.py:328-338) --
    boxsize = property(lambda self: self.info.boxsize)
    boxcenter = property(lambda self: self.info.boxcenter)
    nmesh = property(lambda self: self.info.nmesh)
    offset = property(lambda self: self.info.offset)
    cellsize = property(lambda self: self.info.cellsize)

    # -- painting (recon.py:172-196) --

    def assign_data(self, positions, weights=None, check=True):
        """Paint data (accumulates over calls, e.g. slab by slab).  ``check=False`` defers the
        box / NaN check (no host synchronisation)."""
        with self._stream_ctx():
            order, spos = self._new_order(positions)
            self.mesh_data.assign_cic(positions, weights=weights, wrap=self.wrap, check=check, order_out=order,
                                      sorted_out=spos)
            self._keep_order(positions, order, spos)

    def assign_randoms(self, positions, weights=None, check=True):
        """Same as :meth:`assign_data`, for randoms."""
        if not self.mesh_randoms.is_set:
            self._size_randoms = 0
        with self._stream_ctx():
            order, spos = self._new_order(positions)
            self.mesh_randoms.assign_cic(positions, weights=weights, wrap=self.wrap, check=check, order_out=order,
                                         sorted_out=spos)
            self._keep_order(positions, order, spos)
        self._size_randoms += len(positions)

    # Device-resident catalogues keep the cell order their paint used: a later read-out of the same
    # tensor visits the particles in that order, so the gathers of neighbouring threads hit
    # neighbouring cells.  Any permutation gives the same results; the key (address, length) only
    # picks which one.  The paint also keeps the positions in that order, which the read-out streams
    # instead of gathering them through the permutation, only for the very tensor object that was
    # painted (a weak reference: a new tensor that the allocator places at the same address is not
    # it) and as long as it has not been modified in place since (its version counter is unchanged).

    @staticmethod
    def _order_key(positions):
        import torch
        if isinstance(positions, torch.Tensor) and positions.is_cuda and positions.ndim == 2:
            return (positions.data_ptr(), int(positions.shape[0]))
        return None

    def _new_order(self, positions):
        import torch
        if self._order_key(positions) is None or len(positions) == 0:
            return None, None
        order = torch.empty(len(positions), dtype=torch.int32, device=self.device)
        spos = None
        if self._sorted_positions and positions.shape[-1] == 3 and positions.dtype in (torch.float32, torch.float64):
            spos = torch.empty(positions.shape, dtype=positions.dtype, device=self.device)
        return order, spos

    def _keep_order(self, positions, order, spos=None):
        if order is not None:
            if not hasattr(self, '_orders'):
                self._orders = {}
            self._orders[self._order_key(positions)] = (order, spos, positions._version, weakref.ref(positions))

    def _order_for(self, positions):
        key = self._order_key(positions)
        kept = None if key is None else getattr(self, '_orders', {}).get(key)
        return None if kept is None else kept[0]

    def _sorted_for(self, positions):
        key = self._order_key(positions)
        kept = None if key is None else getattr(self, '_orders', {}).get(key)
        if kept is None or kept[1] is None or kept[3]() is not positions or positions._version != kept[2]:
            return None
        return kept[1]

    @property
    def has_randoms(self):
        return self.mesh_randoms.is_set

    # -- density contrast (recon.py:198-249) --

    def set_density_contrast(self, ran_min=0.01, smoothing_radius=15., check=False, **kwargs):
        r"""Smooth data and randoms, then :math:`\delta = (d - \alpha r) / (b \alpha r)` where the smoothed
        randoms exceed ``ran_min`` times their mean weight, else 0 (no randoms: :math:`d / \bar{d} - 1`, / b)."""
        import torch
        method = kwargs.pop('method', 'fft')
        if method != 'fft':
            return self._density_contrast_real(ran_min, smoothing_radius, check, **kwargs)
        with self._stream_ctx():
            nm, bs, _ = self.info.c_geometry()
            radius = _array3(smoothing_radius, self.info._type_float)
            lib = _lib.load()
            st = _lib.stream_of(self.device)
            if not self.mesh_data.is_set:
                raise ReconstructionError('assign_data must be called before set_density_contrast')
            sums = torch.zeros(2, dtype=torch.float64, device=self.device)
            sws = torch.empty(lib.prc_sum_workspace_bytes(0), dtype=torch.uint8, device=self.device)
            ncol = int(self.info.nmesh[0]) * int(self.info.nmesh[1])
            _lib.call('prc_sum_f64', _lib.ptr(self.mesh_data._colsums), ncol, _lib.ptr(sums), _lib.ptr(sws),
                      sws.numel(), st)
            has_randoms = self.has_randoms
            if has_randoms:
                _lib.call('prc_sum_f64', _lib.ptr(self.mesh_randoms._colsums), ncol, _lib.c_void_p(sums.data_ptr() + 8),
                          _lib.ptr(sws), sws.numel(), st)
                if check:
                    nnonzero = int((self.mesh_randoms._accum > 0.).sum())
                    if nnonzero < 2:
                        raise ValueError('Very few randoms!')
            delta = RealMesh(info=self.info, device=self.device)
            delta.__dict__['value'] = torch.empty(self.info.shape, dtype=torch_dtype(self.info.dtype), device=self.device)
            ws = self._ws.get(lib.prc_density_contrast_workspace_bytes(nm, self.info.dtype.itemsize, int(has_randoms)))
            _lib.call('prc_density_contrast_' + _lib.suffix(self.info.dtype), _lib.ptr(self.mesh_data._accum),
                      _lib.ptr(self.mesh_randoms._accum) if has_randoms else None, _lib.ptr(sums), nm, bs,
                      _lib.d3(radius), float(self.bias), float(ran_min), float(self._size_randoms),
                      _lib.ptr(delta.value), _lib.ptr(ws), ws.numel(), st, error=MeshError)
            if check and has_randoms:
                s = sums.cpu().numpy()
                threshold = ran_min * s[1] / self._size_randoms
                self.log_info('Smoothed random threshold is (ran_min * mean weight) = {:.4f}.'.format(threshold))
            self._sums = sums
            self.mesh_delta = delta
            del self.mesh_data
            del self.mesh_randoms

    def _density_contrast_real(self, ran_min, smoothing_radius, check, nsigmas=2.5, **kwargs):
        """set_density_contrast with real-space smoothing (recon.py:220-249, mesh.py:684-695): both meshes
        smoothed in the mesh dtype by the truncated convolution, then the contrast from their sums."""
        import torch
        with self._stream_ctx():
            if not self.mesh_data.is_set:
                raise ReconstructionError('assign_data must be called before set_density_contrast')
            lib = _lib.load()
            st = _lib.stream_of(self.device)
            nm, _, _ = self.info.c_geometry()
            self.mesh_data.smooth_gaussian(smoothing_radius, method='real', nsigmas=nsigmas)
            data, randoms = self.mesh_data.value, None
            if self.has_randoms:
                if check and int((self.mesh_randoms.value > 0.).sum()) < 2:
                    raise ValueError('Very few randoms!')
                self.mesh_randoms.smooth_gaussian(smoothing_radius, method='real', nsigmas=nsigmas)
                randoms = self.mesh_randoms.value
            sums = torch.zeros(2, dtype=torch.float64, device=self.device)
            ws = self._ws.get(lib.prc_sum_workspace_bytes(0))
            for i, m in enumerate([data, randoms]):
                if m is not None:
                    _lib.call('prc_sum_' + _lib.suffix(self.info.dtype), _lib.ptr(m), m.numel(),
                              _lib.c_void_p(sums.data_ptr() + 8 * i), _lib.ptr(ws), ws.numel(), st)
            delta = RealMesh(info=self.info, device=self.device)
            delta.__dict__['value'] = torch.empty(self.info.shape, dtype=torch_dtype(self.info.dtype), device=self.device)
            _lib.call('prc_delta_from_meshes_' + _lib.suffix(self.info.dtype), _lib.ptr(data), _lib.ptr(randoms),
                      data.element_size(), _lib.ptr(sums), nm, float(self.bias), float(ran_min),
                      float(self._size_randoms), _lib.ptr(delta.value), st, error=MeshError)
            self._sums = sums
            self.mesh_delta = delta
            del self.mesh_data
            del self.mesh_randoms

    def run(self, *args, **kwargs):
        raise NotImplementedError('Implement method "run" in your "{}"-inherited algorithm'.format(self.__class__.__name__))

    # -- shifts (recon.py:255-325) --

    def _shift_call(self, particles, field, shifted, out, out_bytes):
        raise NotImplementedError

    # particles per chunk of a read-out from host memory (copies in, kernel, copies out overlap)
    _read_chunk = 1 << 21

    def _read(self, positions, field, shifted):
        import torch
        field = field.lower()
        if field not in ALLOWED_FIELDS:
            raise ReconstructionError('Unknown field {}. Choices are {}'.format(field, ALLOWED_FIELDS))
        host = not (isinstance(positions, torch.Tensor) and positions.is_cuda)
        if host and len(positions) > self._read_chunk:
            return self._read_pipelined(positions, field, shifted)
        with self._stream_ctx():
            p = Particles(positions, self.device)
            p.order = self._order_for(positions)
            p.sorted = self._sorted_for(positions) if p.order is not None else None
            pbytes = p.pos_bytes
            obytes = max(pbytes, self.info.dtype.itemsize) if (shifted and self.wrap) else pbytes
            out = torch.empty((p.size, 3), dtype=torch_dtype('f4' if obytes == 4 else 'f8'), device=self.device)
            self._shift_call(p, _lib.FIELDS[field], int(shifted), out, obytes)
            low, high = self.info.boxcenter - self.info.boxsize / 2., self.info.boxcenter + self.info.boxsize / 2.
            self._flags.raise_if_set(low, high)
            _lib.check_device_faults(ReconstructionError)
            return p.output(out)

    def _copy_streams(self):
        import torch
        if getattr(self, '_streams', None) is None:
            self._streams = (torch.cuda.Stream(self.device), torch.cuda.Stream(self.device))
        return self._streams

    def _read_pipelined(self, positions, field, shifted):
        """Read-out of host positions in chunks: the host-to-device copy of chunk i + 1, the kernel on
        chunk i and the device-to-host copy of chunk i - 1 run at once (two copy streams, events
        between them; the kernels stay on the reconstruction's stream).  Same results as one call."""
        import torch
        numpy_in = not isinstance(positions, torch.Tensor)
        if numpy_in:
            arr = np.asarray(positions)
            if arr.dtype not in (np.float32, np.float64):
                arr = arr.astype('f8')
            host = torch.from_numpy(np.ascontiguousarray(arr))
        else:
            host = positions if positions.dtype in (torch.float32, torch.float64) else positions.double()
            host = host.contiguous()
        if host.ndim != 2 or host.shape[1] != 3:
            raise MeshError('positions must be of shape (N, 3)')
        n, pbytes = int(host.shape[0]), host.element_size()
        obytes = max(pbytes, self.info.dtype.itemsize) if (shifted and self.wrap) else pbytes
        odt = torch_dtype('f4' if obytes == 4 else 'f8')
        out_host = torch.empty((n, 3), dtype=odt, pin_memory=True)
        chunk = self._read_chunk
        s_in, s_out = self._copy_streams()
        with self._stream_ctx():
            compute = torch.cuda.current_stream(self.device)
            nbuf = 2
            din = [torch.empty((chunk, 3), dtype=host.dtype, device=self.device) for _ in range(nbuf)]
            dout = [torch.empty((chunk, 3), dtype=odt, device=self.device) for _ in range(nbuf)]
            for k in range(nbuf):
                din[k].record_stream(s_in)
                dout[k].record_stream(s_out)
            read_done, copied_out = [None] * nbuf, [None] * nbuf

            class _Chunk(object):
                pass

            for i, a in enumerate(range(0, n, chunk)):
                k, b = i % nbuf, min(n, a + chunk)
                m = b - a
                with torch.cuda.stream(s_in):
                    if read_done[k] is not None:
                        s_in.wait_event(read_done[k])
                    din[k][:m].copy_(host[a:b], non_blocking=True)
                    arrived = torch.cuda.Event()
                    arrived.record(s_in)
                compute.wait_event(arrived)
                if copied_out[k] is not None:
                    compute.wait_event(copied_out[k])
                c = _Chunk()
                c.pos, c.size, c.pos_bytes = din[k], m, pbytes
                self._shift_call(c, _lib.FIELDS[field], int(shifted), dout[k], obytes)
                read_done[k] = torch.cuda.Event()
                read_done[k].record(compute)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(read_done[k])
                    out_host[a:b].copy_(dout[k][:m], non_blocking=True)
                    copied_out[k] = torch.cuda.Event()
                    copied_out[k].record(s_out)
            s_out.synchronize()
            low, high = self.info.boxcenter - self.info.boxsize / 2., self.info.boxcenter + self.info.boxsize / 2.
            self._flags.raise_if_set(low, high)
            _lib.check_device_faults(ReconstructionError)
        return out_host.numpy() if numpy_in else out_host

    def read_shifts(self, positions, field='disp+rsd'):
        """Displacements at ``positions``: 'disp' (Zeldovich), 'rsd' or 'disp+rsd'."""
        return self._read(positions, field, False)

    def read_shifted_positions(self, positions, field='disp+rsd'):
        """``positions - read_shifts(positions, field)``, wrapped into the box if :attr:`wrap`."""
        return self._read(positions, field, True)

    def _geometry_args(self):
        return self.info.c_geometry()

    def _los_arg(self):
        return _lib.opt_d3(None if self.los is None else [float(x) for x in self.los])


class FFTShiftsMixin(object):
    """Displacements stored interleaved, (psi_x, psi_y, psi_z, 0) per cell, so the CIC read-out does
    one vector load per corner; ``mesh_psi`` are the three component views (recon.py:255-302)."""

    def _new_psi(self):
        import torch
        psi4 = torch.empty(self.info.shape + (4,), dtype=torch_dtype(self.info.dtype), device=self.device)
        meshes = []
        for a in range(3):
            m = RealMesh(info=self.info, device=self.device)
            m.__dict__['value'] = psi4[..., a]
            meshes.append(m)
        return psi4, meshes

    @staticmethod
    def _psi_pointers(psi4):
        base = psi4.data_ptr()
        item = psi4.element_size()
        return [_lib.c_void_p(base), _lib.c_void_p(base + item), _lib.c_void_p(base + 2 * item)]

    def _shift_call(self, p, field, shifted, out, obytes):
        if not hasattr(self, 'mesh_psi'):
            raise ReconstructionError('run() must be called before reading shifts')
        nm, bs, bc = self._geometry_args()
        _lib.call('prc_read_shifts_psi_' + _lib.suffix(self.info.dtype), *self._psi_pointers(self._psi4), 4, nm, bs,
                  bc, _lib.ptr(p.pos), p.pos_bytes, p.size, _lib.ptr(getattr(p, 'order', None)), float(self.f),
                  self._los_arg(), field, shifted,
                  int(self.wrap), _lib.ptr(out), obytes, self._flags.ptr, _lib.stream_of(self.device),
                  _lib.ptr(getattr(p, 'sorted', None)), error=MeshError)
