"""Full-multigrid reconstruction after M. J. White's recon_code (pyrecon/multigrid.py) on CUDA."""
import numpy as np

from . import _lib
from .mesh import RealMesh, MeshError, torch_dtype
from .recon import BaseReconstruction


class OriginalMultiGridReconstruction(BaseReconstruction):
    """
    Solves the RSD-modified Poisson equation for the displacement potential :attr:`mesh_phi` with the
    reference's fixed full-multigrid schedule of damped-Jacobi V-cycles (pyrecon/multigrid.py:13-158,
    src/multigrid.c), and reads shifts as its finite-difference gradient.
    """

    @staticmethod
    def _select_nmesh(nmesh):
        """Smallest size >= n of the form 2^k, 3 2^k, 5 2^k or 7 2^k (multigrid.py:24-36)."""
        out = []
        for n in nmesh:
            nbits = int(n).bit_length() - 1
            ntries = [2 ** nbits, 3 * 2 ** (nbits - 1), 5 * 2 ** (nbits - 2), 7 * 2 ** (nbits - 2), 2 ** (nbits + 1)]
            mindiff, iclosest = n, None
            for itry, ntry in enumerate(ntries):
                diff = ntry - n
                if 0 <= diff < mindiff:
                    mindiff, iclosest = diff, itry
            out.append(ntries[iclosest])
        return np.array(out, dtype='i8')

    def set_density_contrast(self, ran_min=0.75, smoothing_radius=15., **kwargs):
        r"""Martin's density contrast (multigrid.py:49-97): cells whose (unsmoothed) randoms are below
        ``ran_min`` get :math:`\delta = 0` (their data is left out of the normalisation where randoms are
        positive), elsewhere :math:`\delta = (d / (\alpha r) - 1) / b`; the mean of the non-zero
        :math:`\delta` is removed, then :math:`\delta` is smoothed (``kwargs``: :meth:`RealMesh.smooth_gaussian`).
        Without randoms :math:`\delta = (d / \bar{d} - 1) / b`, smoothed."""
        import torch
        with self._stream_ctx():
            if not self.mesh_data.is_set:
                from .recon import ReconstructionError
                raise ReconstructionError('assign_data must be called before set_density_contrast')
            lib = _lib.load()
            nm, _, _ = self.info.c_geometry()

            def fp64(mesh):
                return mesh._accum if mesh._accum is not None else mesh.value.to(torch.float64)

            has_randoms = self.has_randoms
            data = fp64(self.mesh_data)
            randoms = fp64(self.mesh_randoms) if has_randoms else None
            delta = RealMesh(info=self.info, device=self.device)
            delta._ws = self._ws
            delta.__dict__['value'] = torch.empty(self.info.shape, dtype=torch_dtype(self.info.dtype), device=self.device)
            ws = self._ws.get(lib.prc_density_contrast_original_workspace_bytes())
            _lib.call('prc_density_contrast_original_' + _lib.suffix(self.info.dtype), _lib.ptr(data),
                      _lib.ptr(randoms), nm, float(self.bias), float(ran_min), _lib.ptr(delta.value), _lib.ptr(ws),
                      ws.numel(), _lib.stream_of(self.device), error=MeshError)
            if has_randoms:
                del self.mesh_data
                del self.mesh_randoms
            delta.smooth_gaussian(smoothing_radius, **kwargs)
            self.mesh_delta = delta

    def run(self, jacobi_damping_factor=0.4, jacobi_niterations=5, vcycle_niterations=6):
        """Compute the displacement potential :attr:`mesh_phi` (multigrid.py:99-135)."""
        import torch
        with self._stream_ctx():
            nm, bs, bc = self.info.c_geometry()
            lib = _lib.load()
            phi = RealMesh(info=self.info, device=self.device)
            phi.__dict__['value'] = torch.empty(self.info.shape, dtype=torch_dtype(self.info.dtype), device=self.device)
            self.log_info('Computing displacement potential.')
            f32 = self.info.dtype.itemsize == 4
            ws = self._ws.get(lib.prc_multigrid_workspace_bytes(nm, self.info.dtype.itemsize, int(self.mixed_precision)))
            tail = [nm, bs, bc, float(self.beta), float(jacobi_damping_factor), int(jacobi_niterations),
                    int(vcycle_niterations), self._los_arg()]
            self._phi64 = None
            if f32 and self.mixed_precision:
                # the FP64 iterate of the refinement is kept for the finite-difference read-out
                self._phi64 = torch.empty(self.info.shape, dtype=torch.float64, device=self.device)
                _lib.call('prc_multigrid_mixed_f32', _lib.ptr(self.mesh_delta.value), _lib.ptr(phi.value),
                          _lib.ptr(self._phi64), *tail, _lib.ptr(ws), ws.numel(), _lib.stream_of(self.device),
                          error=MeshError)
            else:
                args = [_lib.ptr(self.mesh_delta.value), _lib.ptr(phi.value)] + tail + ([0] if f32 else [])
                _lib.call('prc_multigrid_' + _lib.suffix(self.info.dtype), *args, _lib.ptr(ws), ws.numel(),
                          _lib.stream_of(self.device), error=MeshError)
            del self.mesh_delta
            self.mesh_phi = phi

    def _shift_call(self, p, field, shifted, out, obytes):
        if not hasattr(self, 'mesh_phi'):
            from .recon import ReconstructionError
            raise ReconstructionError('run() must be called before reading shifts')
        nm, bs, bc = self._geometry_args()
        phi64 = getattr(self, '_phi64', None)
        if phi64 is not None:
            # mixed precision: the gradient of the FP64 iterate (the FP32 mesh_phi would add its rounding)
            name, mesh = 'prc_read_shifts_phi_f64', phi64
        else:
            name, mesh = 'prc_read_shifts_phi_' + _lib.suffix(self.info.dtype), self.mesh_phi.value
        _lib.call(name, _lib.ptr(mesh), nm, bs, bc,
                  _lib.ptr(p.pos), p.pos_bytes, p.size, _lib.ptr(getattr(p, 'order', None)), float(self.f),
                  self._los_arg(), field, shifted, int(self.wrap),
                  _lib.ptr(out), obytes, self._flags.ptr, _lib.stream_of(self.device),
                  _lib.ptr(getattr(p, 'sorted', None)), error=MeshError)


def run_batch(recons, jacobi_damping_factor=0.4, jacobi_niterations=5, vcycle_niterations=6):
    """:meth:`OriginalMultiGridReconstruction.run` of several reconstructions at once: one batched solve
    (every kernel of the multigrid schedule runs over all of them in one launch), on the first
    reconstruction's stream and workspace.  They must share the mesh (nmesh, boxsize, boxcenter, dtype),
    the line of sight, beta, the precision mode and the device, and have their density contrast set.
    Results equal separate :meth:`run` calls."""
    import torch
    recons = list(recons)
    if not recons:
        return
    r0 = recons[0]
    key = lambda r: (tuple(r.info.nmesh), tuple(r.info.boxsize), tuple(r.info.boxcenter), r.info.dtype,
                     None if r.los is None else tuple(float(x) for x in r.los), float(r.beta),
                     bool(r.mixed_precision), str(r.device))
    for r in recons:
        if not isinstance(r, OriginalMultiGridReconstruction):
            raise ValueError('run_batch takes multigrid reconstructions')
        if key(r) != key(r0):
            raise ValueError('run_batch needs the same mesh, line of sight, beta, precision and device')
        if getattr(r, 'mesh_delta', None) is None:
            from .recon import ReconstructionError
            raise ReconstructionError('set_density_contrast must be called before run')
    streams = [r.stream if r.stream is not None else torch.cuda.current_stream(r.device) for r in recons]
    with r0._stream_ctx():
        st0 = streams[0]
        for st in streams[1:]:
            if st != st0:
                st0.wait_stream(st)         # the other reconstructions' density contrasts are done
        nm, bs, bc = r0.info.c_geometry()
        lib = _lib.load()
        item = r0.info.dtype.itemsize
        count = len(recons)
        deltas = [r.mesh_delta.value for r in recons]
        phis = []
        for r in recons:
            phi = RealMesh(info=r.info, device=r.device)
            phi.__dict__['value'] = torch.empty(r.info.shape, dtype=torch_dtype(r.info.dtype), device=r.device)
            phis.append(phi)
        ws = r0._ws.get(lib.prc_multigrid_batch_workspace_bytes(nm, item, int(r0.mixed_precision), count))
        tail = [count, nm, bs, bc, float(r0.beta), float(jacobi_damping_factor), int(jacobi_niterations),
                int(vcycle_niterations), r0._los_arg()]
        mixed = item == 4 and r0.mixed_precision
        phis64 = [torch.empty(r.info.shape, dtype=torch.float64, device=r.device) for r in recons] if mixed else None
        if mixed:
            _lib.call('prc_multigrid_batch_mixed_f32', _lib.pointer_array(deltas),
                      _lib.pointer_array([p.value for p in phis]), _lib.pointer_array(phis64), *tail, _lib.ptr(ws),
                      ws.numel(), _lib.stream_of(r0.device), error=MeshError)
        else:
            args = [_lib.pointer_array(deltas), _lib.pointer_array([p.value for p in phis])] + tail + \
                ([0] if item == 4 else [])
            _lib.call('prc_multigrid_batch_' + _lib.suffix(r0.info.dtype), *args, _lib.ptr(ws), ws.numel(),
                      _lib.stream_of(r0.device), error=MeshError)
        for i, (r, st, phi) in enumerate(zip(recons, streams, phis)):
            if st != st0:
                st.wait_stream(st0)         # later work on that reconstruction's stream sees its phi
                phi.value.record_stream(st)
                if mixed:
                    phis64[i].record_stream(st)
            del r.mesh_delta
            r.mesh_phi = phi
            r._phi64 = phis64[i] if mixed else None


class MultiGridReconstruction(OriginalMultiGridReconstruction):
    """Multigrid reconstruction with the base class's density contrast (multigrid.py:161-167)."""

    def set_density_contrast(self, *args, **kwargs):
        BaseReconstruction.set_density_contrast(self, *args, **kwargs)
