"""
Mesh geometry and device meshes, with the reference's names and semantics
(pyrecon/mesh.py): :class:`MeshInfo`, :class:`RealMesh`, :class:`ComplexMesh`,
:class:`MeshError`.

Mesh values live in CUDA memory as torch tensors; every computation goes through
libpyrecon_cuda.so (no CPU fallback).  ``numpy.asarray(mesh)`` copies to the host.
"""
import copy
import numbers
import warnings

import numpy as np

from . import _lib
from .utils import BaseClass


class MeshError(Exception):
    """Exception raised when issue with mesh."""


def _array3(value, dtype):
    out = np.empty(3, dtype=dtype)
    out[...] = value
    return out


def _torch():
    import torch
    return torch


def _to_numpy(x):
    torch = _torch()
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


class MeshInfo(BaseClass):
    """Mesh geometry: dtype, nmesh, boxsize, boxcenter (pyrecon/mesh.py:322-483)."""

    _attrs = ['dtype', 'nmesh', 'boxsize', 'boxcenter']

    def __init__(self, nmesh=None, boxsize=None, boxcenter=None, cellsize=None, value=None, positions=None, boxpad=1.5,
                 select_nmesh=None, dtype=None):
        if value is not None:
            shape = tuple(value.shape)
            if dtype is None:
                dtype = _to_numpy(value.reshape(-1)[:0]).dtype
            if nmesh is None:
                nmesh = shape
        dtype = np.dtype(dtype if dtype is not None else 'f8')
        if boxsize is None or boxcenter is None:
            if positions is None:
                raise MeshError('positions must be provided if boxsize or boxcenter are not specified')
            pos = positions
            torch = _torch()
            if isinstance(pos, torch.Tensor):
                pos_min, pos_max = [t.double().cpu().numpy() for t in (pos.min(dim=0).values, pos.max(dim=0).values)]
            else:
                pos_min, pos_max = pos.min(axis=0), pos.max(axis=0)
            delta = np.abs(pos_max - pos_min)
            if boxcenter is None:
                boxcenter = 0.5 * (pos_min + pos_max)
            if boxsize is None:
                if cellsize is not None and nmesh is not None:
                    boxsize = nmesh * cellsize
                else:
                    boxsize = delta * boxpad
            if (boxsize < delta).any():
                raise MeshError('boxsize too small to contain all data')
        boxsize = _array3(boxsize, 'f8')
        if nmesh is None:
            if cellsize is not None:
                cellsize = _array3(cellsize, 'f8')
                nmesh = np.ceil(boxsize / cellsize).astype('i8')
                if select_nmesh is not None:
                    nmesh = select_nmesh(nmesh)
                boxsize = nmesh * cellsize
            else:
                raise MeshError('nmesh (or cellsize) must be specified')
        self.__dict__['dtype'] = np.dtype(dtype)
        self.boxsize = boxsize
        self.boxcenter = boxcenter
        self.nmesh = nmesh
        if select_nmesh is not None:
            recommended = select_nmesh(self.nmesh)
            if not np.all(recommended == self.nmesh):
                warnings.warn('Recommended nmesh is {}, provided nmesh is {}'.format(recommended, self.nmesh))

    def __setattr__(self, name, value):
        # boxsize / boxcenter are stored in the mesh dtype, nmesh as int32 (mesh.py:447-460)
        if name == 'dtype':
            self.__dict__['dtype'] = np.dtype(value)
            self.boxsize = self.boxsize
            self.boxcenter = self.boxcenter
            return
        if name in ('boxsize', 'boxcenter'):
            value = _array3(value, self._type_float)
        elif name == 'nmesh':
            value = _array3(value, np.int32)
        super(MeshInfo, self).__setattr__(name, value)

    @property
    def _type_float(self):
        return np.empty(0, dtype=self.dtype).real.dtype

    @property
    def offset(self):
        """Coordinates of the (0, 0, 0) corner of the box."""
        return self.boxcenter - self.boxsize / 2.

    @property
    def cellsize(self):
        return self.boxsize / self.nmesh

    @property
    def ndim(self):
        return 3

    @property
    def shape(self):
        return tuple(int(n) for n in self.nmesh)

    def wrap(self, positions):
        """((p - offset) % boxsize) + offset (mesh.py:477-479); numpy or torch."""
        torch = _torch()
        if isinstance(positions, torch.Tensor):
            off = torch.as_tensor(self.offset, device=positions.device)
            bs = torch.as_tensor(self.boxsize, device=positions.device)
            return torch.remainder(positions - off, bs) + off
        return ((positions - self.offset) % self.boxsize) + self.offset

    def clone(self, **kwargs):
        for name in self._attrs:
            kwargs.setdefault(name, getattr(self, name))
        return self.__class__(**kwargs)

    def deepcopy(self):
        return copy.deepcopy(self)

    # arguments of the C ABI
    def c_geometry(self):
        return _lib.i3(self.nmesh), _lib.d3(self.boxsize), _lib.d3(self.boxcenter)

    def __repr__(self):
        return 'MeshInfo(dtype={}, nmesh={}, boxsize={}, boxcenter={})'.format(self.dtype, self.nmesh, self.boxsize,
                                                                              self.boxcenter)


def _device_of(device):
    torch = _torch()
    if device is None:
        if not torch.cuda.is_available():
            raise _lib.LibraryError('pyrecon_b200 needs a CUDA device (there is no CPU fallback)')
        return torch.device('cuda', torch.cuda.current_device())
    device = torch.device(device)
    if device.type != 'cuda':
        raise _lib.LibraryError('pyrecon_b200 runs on CUDA devices only, got {}'.format(device))
    if device.index is None:
        device = torch.device('cuda', torch.cuda.current_device())
    return device


def torch_dtype(dtype):
    torch = _torch()
    return {4: torch.float32, 8: torch.float64}[np.dtype(dtype).itemsize]


_copy_streams = {}


def _upload(t, device):
    """Device copy of `t`.  From pinned host memory the copy runs on a copy stream of the device, so it
    overlaps the kernels already queued on the current stream (e.g. the paint of the previous
    catalogue); the current stream waits for it before any later use."""
    torch = _torch()
    if t.is_cuda or not t.is_pinned():
        return t.to(device, non_blocking=True).contiguous()
    t = t.contiguous()
    compute = torch.cuda.current_stream(device)
    copy = _copy_streams.get(device)
    if copy is None:
        copy = _copy_streams[device] = torch.cuda.Stream(device)
    with torch.cuda.stream(copy):
        out = torch.empty(t.shape, dtype=t.dtype, device=device)     # from the copy stream's pool
        out.copy_(t, non_blocking=True)
        done = torch.cuda.Event()
        done.record(copy)
    compute.wait_event(done)
    out.record_stream(compute)          # not reused before the current stream's work on it is done
    return out


class Particles(object):
    """Positions (and optional weights) resident on the device, with how to return results."""

    def __init__(self, positions, device, weights=None, weight_dtype=None):
        torch = _torch()
        self.kind = 'torch' if isinstance(positions, torch.Tensor) else 'numpy'
        self.host_device = positions.device if self.kind == 'torch' else None
        if self.kind == 'numpy':
            positions = np.asarray(positions)
            if positions.dtype not in (np.float32, np.float64):
                positions = positions.astype('f8')
            self.np_dtype = positions.dtype
            t = torch.from_numpy(np.ascontiguousarray(positions))
        else:
            t = positions
            if t.dtype not in (torch.float32, torch.float64):
                t = t.double()
            self.np_dtype = np.dtype('f4') if t.dtype == torch.float32 else np.dtype('f8')
        if t.ndim != 2 or t.shape[1] != 3:
            raise MeshError('positions must be of shape (N, 3)')
        self.size = int(t.shape[0])
        self.pos = _upload(t, device)
        self.weights = None
        if weights is not None:
            w = weights if isinstance(weights, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(weights))
            if w.dtype not in (torch.float32, torch.float64):
                w = w.to(torch_dtype(weight_dtype or 'f8'))
            if w.shape[0] != self.size:
                raise MeshError('weights must have the same length as positions')
            self.weights = _upload(w.reshape(-1), device)

    @property
    def pos_bytes(self):
        return self.np_dtype.itemsize

    def output(self, t):
        """Return a device result in the caller's container type (host tensors: pinned memory)."""
        if self.kind == 'numpy':
            return t.cpu().numpy()
        if self.host_device is not None and self.host_device.type != 'cuda':
            torch = _torch()
            out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            out.copy_(t, non_blocking=True)
            torch.cuda.current_stream(t.device).synchronize()
            return out
        return t


class _Workspace(object):
    """Grow-only device scratch owned by one mesh or reconstruction."""

    def __init__(self, device):
        self.device = device
        self.buf = None

    def get(self, nbytes):
        torch = _torch()
        nbytes = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = None
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self.buf

    def release(self):
        self.buf = None


class _Flags(object):
    """Device status word written by the kernels (PRC_FLAG_*)."""

    def __init__(self, device):
        torch = _torch()
        self.t = torch.zeros(1, dtype=torch.int32, device=device)

    @property
    def ptr(self):
        return _lib.ptr(self.t)

    def raise_if_set(self, low, high, what='positions'):
        v = int(self.t.item())
        if v & _lib.PRC_FLAG_OUT_OF_BOX:
            raise MeshError('{} not in box range {} - {}'.format(what, low, high))
        if v & _lib.PRC_FLAG_NONFINITE:
            raise MeshError('Some positions or weights are NaN/inf')
        if v & _lib.PRC_FLAG_DEVICE_WAIT:
            raise MeshError('a bounded wait on the device gave up (sort look-back); the mesh was not painted')


class BaseMesh(BaseClass):
    """Common part of real and complex device meshes."""

    def __init__(self, value=None, info=None, device=None, attrs=None, **kwargs):
        if info is None:
            info = MeshInfo(value=value, **kwargs)
        elif kwargs:
            info = info.clone(**kwargs)
        self.info = info
        self.device = _device_of(device if device is not None else (value.device if _is_cuda_tensor(value) else None))
        self.attrs = attrs or {}
        self.value = value

    @property
    def dtype(self):
        return self.info.dtype

    @property
    def nmesh(self):
        return self.info.nmesh

    @property
    def boxsize(self):
        return self.info.boxsize

    @property
    def boxcenter(self):
        return self.info.boxcenter

    @property
    def offset(self):
        return self.info.offset

    @property
    def cellsize(self):
        return self.info.cellsize

    @property
    def ndim(self):
        return 3

    @property
    def size(self):
        return int(np.prod(self.shape))

    def __array__(self, dtype=None, copy=None):
        out = self.value.detach().cpu().numpy()
        return out.astype(dtype) if dtype is not None else out

    def __getitem__(self, index):
        return self.value.__getitem__(index)

    def __setitem__(self, index, value):
        self.value.__setitem__(index, value)

    def mean(self, axis=None, dtype=None, out=None, **kwargs):
        return float(self.value.double().mean()) if axis is None else self.value.mean(dim=axis)

    def sum(self, axis=None, dtype=None, out=None, **kwargs):
        return float(self.value.double().sum()) if axis is None else self.value.sum(dim=axis)

    def std(self, axis=None, dtype=None, out=None, ddof=0, **kwargs):
        return float(self.value.double().std(correction=ddof))

    def _binary(self, other, op):
        o = other.value if isinstance(other, BaseMesh) else other
        new = self.deepcopy(copy_value=False)
        new.value = op(self.value, o).to(self.value.dtype)
        return new

    def __add__(self, other): return self._binary(other, lambda a, b: a + b)
    def __radd__(self, other): return self._binary(other, lambda a, b: b + a)
    def __sub__(self, other): return self._binary(other, lambda a, b: a - b)
    def __rsub__(self, other): return self._binary(other, lambda a, b: b - a)
    def __mul__(self, other): return self._binary(other, lambda a, b: a * b)
    def __rmul__(self, other): return self._binary(other, lambda a, b: b * a)
    def __truediv__(self, other): return self._binary(other, lambda a, b: a / b)
    def __rtruediv__(self, other): return self._binary(other, lambda a, b: b / a)
    def __neg__(self): return self._binary(0, lambda a, b: -a)

    def __pow__(self, other): return self._binary(other, lambda a, b: a ** b)
    def __rpow__(self, other): return self._binary(other, lambda a, b: b ** a)

    # comparisons give boolean device tensors (the reference's ufuncs give boolean arrays, not meshes)
    def _compare(self, other, op):
        return op(self.value, other.value if isinstance(other, BaseMesh) else other)

    def __gt__(self, other): return self._compare(other, lambda a, b: a > b)
    def __ge__(self, other): return self._compare(other, lambda a, b: a >= b)
    def __lt__(self, other): return self._compare(other, lambda a, b: a < b)
    def __le__(self, other): return self._compare(other, lambda a, b: a <= b)

    __array_priority__ = 100

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        """numpy ufuncs on meshes (mesh.py:185-225): evaluated on host copies of the values; a result of the
        mesh's shape that is not boolean comes back as a mesh of this kind, anything else as an array."""
        if kwargs.get('out'):
            return NotImplemented
        args = [np.asarray(x) if isinstance(x, BaseMesh) else x for x in inputs]
        result = getattr(ufunc, method)(*args, **kwargs)

        def cast(r):
            if not isinstance(r, np.ndarray) or r.dtype == np.bool_ or r.shape != tuple(self.shape):
                return r
            new = self.deepcopy(copy_value=False)
            new.value = r
            return new

        return tuple(cast(r) for r in result) if isinstance(result, tuple) else cast(result)

    # FFT-engine and thread-count settings of the reference's CPU meshes: accepted, without effect
    # (the transforms are this library's CUDA kernels)
    nthreads = None

    def set_num_threads(self, nthreads=None):
        self.nthreads = nthreads

    def get_fft_engine(self, engine='numpy', **kwargs):
        return engine

    def set_fft_engine(self, engine='numpy', **kwargs):
        self.fft_engine = self.get_fft_engine(engine=engine, **kwargs)

    def __iadd__(self, other):
        self.value += other.value if isinstance(other, BaseMesh) else other
        return self

    def __isub__(self, other):
        self.value -= other.value if isinstance(other, BaseMesh) else other
        return self

    def __imul__(self, other):
        self.value *= other.value if isinstance(other, BaseMesh) else other
        return self

    def __itruediv__(self, other):
        self.value /= other.value if isinstance(other, BaseMesh) else other
        return self

    def deepcopy(self, copy_value=True):
        new = self.__class__.__new__(self.__class__)
        new.__dict__.update(self.__dict__)
        new.info = self.info.deepcopy()
        new.attrs = dict(self.attrs)
        if copy_value and self.value is not None:
            new.__dict__['value'] = self.value.clone()
        if '_accum' in new.__dict__:
            # the copy owns its values; a later paint into it starts a new FP64 accumulator from them
            new.__dict__['_accum'] = None
            new.__dict__['_colsums'] = None
        return new

    def __repr__(self):
        return '{}(dtype={}, nmesh={}, boxsize={}, boxcenter={})'.format(self.__class__.__name__, self.dtype, self.nmesh,
                                                                         self.boxsize, self.boxcenter)


def _is_cuda_tensor(x):
    try:
        import torch
        return isinstance(x, torch.Tensor) and x.is_cuda
    except ImportError:
        return False


class RealMesh(BaseMesh):
    """3D real mesh on a CUDA device (pyrecon/mesh.py:486-736)."""

    def __init__(self, value=None, dtype=None, info=None, device=None, nthreads=None, attrs=None, **kwargs):
        if dtype is None and (value is None or np.ndim(value) == 0) and info is None:
            dtype = 'f8'
        if dtype is not None:
            kwargs['dtype'] = dtype
        if info is None and value is not None and np.ndim(value) == 3:
            kwargs.setdefault('nmesh', tuple(value.shape))              # mesh shape from the values (mesh.py:384-389)
            kwargs.setdefault('dtype', _to_numpy(value.reshape(-1)[:0]).dtype if hasattr(value, 'reshape') else 'f8')
        super(RealMesh, self).__init__(value=None, info=info, device=device, attrs=attrs, **kwargs)
        if 'float' not in self.dtype.name:
            raise MeshError('Provide float dtype')
        self._accum = None     # FP64 paint accumulator
        self.value = value

    @property
    def shape(self):
        return self.info.shape

    def __getattr__(self, name):
        # An FP32 mesh filled by assign_cic keeps its FP64 sums (what set_density_contrast reads); its
        # FP32 `value` is made from them on first access only.
        if name == 'value':
            accum = self.__dict__.get('_accum')
            if accum is None:
                return None
            value = accum.to(_torch().float32)
            self.__dict__['value'] = value
            return value
        raise AttributeError(name)

    @property
    def is_set(self):
        """Whether the mesh holds values (painted or assigned), without materialising them."""
        return self.__dict__.get('value') is not None or self.__dict__.get('_accum') is not None

    def __setattr__(self, name, value):
        if name == 'value' and value is not None:
            torch = _torch()
            tdt = torch_dtype(self.dtype)
            if isinstance(value, torch.Tensor):
                value = value.to(self.device, tdt).reshape(self.shape).contiguous()
            elif isinstance(value, np.ndarray) and value.size == int(np.prod(self.shape)):
                value = torch.from_numpy(np.ascontiguousarray(value).astype(self.dtype).reshape(self.shape)).to(self.device)
            else:
                value = torch.full(self.shape, float(value), dtype=tdt, device=self.device)
        super(RealMesh, self).__setattr__(name, value)

    def zeros_like(self):
        torch = _torch()
        new = self.deepcopy(copy_value=False)
        new.__dict__['value'] = torch.zeros(self.shape, dtype=torch_dtype(self.dtype), device=self.device)
        return new

    def empty_like(self):
        torch = _torch()
        new = self.deepcopy(copy_value=False)
        new.__dict__['value'] = torch.empty(self.shape, dtype=torch_dtype(self.dtype), device=self.device)
        return new

    def coords(self):
        """Node coordinates along each axis (mesh.py:522-527)."""
        return tuple(o + d * np.arange(n) for n, o, d in zip(self.nmesh, self.offset, self.boxsize / self.nmesh))

    # -- particles --

    def _check_positions_geometry(self):
        low, high = self.boxcenter - self.boxsize / 2., self.boxcenter + self.boxsize / 2.
        return low, high

    def assign_cic(self, positions, weights=None, wrap=False, check=True, order_out=None, sorted_out=None):
        """Paint positions with CIC, accumulating (mesh.py:529-568); FP64 sums, deterministic.
        ``order_out``: optional int32 device tensor of len(positions) that receives the particles'
        indices in the (cell-sorted) order the paint summed them; ``sorted_out`` (with ``order_out``):
        optional device tensor shaped like the positions that receives them in that order."""
        torch = _torch()
        p = Particles(positions, self.device, weights=weights, weight_dtype=self.dtype)
        accumulate = True
        if self._accum is None:
            # a fresh mesh is written (not added to) by the paint, which covers every cell and column sum
            self._accum = torch.empty(self.shape, dtype=torch.float64, device=self.device)
            self._colsums = torch.empty(int(self.nmesh[0]) * int(self.nmesh[1]), dtype=torch.float64, device=self.device)
            if self.value is not None:
                self._accum.copy_(self.value)
            else:
                accumulate = False
        paint(self.info, self._accum, self._colsums, p, wrap, accumulate, self._workspace(), self._flags(), check=check,
              order_out=order_out, sorted_out=sorted_out)
        if self.dtype.itemsize == 8:
            self.__dict__['value'] = self._accum
        else:
            self.__dict__.pop('value', None)

    def _workspace(self):
        if getattr(self, '_ws', None) is None:
            self._ws = _Workspace(self.device)
        return self._ws

    def _flags(self):
        if getattr(self, '_fl', None) is None:
            self._fl = _Flags(self.device)
        return self._fl

    def read_cic(self, positions, wrap=False):
        """CIC interpolation at positions (mesh.py:570-610)."""
        torch = _torch()
        p = Particles(positions, self.device)
        out = torch.empty(p.size, dtype=p.pos.dtype, device=self.device)
        fl = self._flags()
        nm, bs, bc = self.info.c_geometry()
        _lib.call('prc_read_cic_' + _lib.suffix(self.dtype), _lib.ptr(self.value), nm, bs, bc, _lib.ptr(p.pos),
                  p.pos_bytes, p.size, int(bool(wrap)), _lib.ptr(out), fl.ptr, _lib.stream_of(self.device), error=MeshError)
        fl.raise_if_set(*self._check_positions_geometry())
        if not wrap and not bool(torch.isfinite(p.pos).all()):
            warnings.warn('Some positions are NaN/inf')
        return p.output(out)

    def read_finite_difference_cic(self, positions, wrap=False):
        """Finite-difference gradient, CIC-interpolated at positions (mesh.py:612-653)."""
        torch = _torch()
        p = Particles(positions, self.device)
        out = torch.empty((p.size, 3), dtype=p.pos.dtype, device=self.device)
        fl = self._flags()
        nm, bs, bc = self.info.c_geometry()
        _lib.call('prc_read_finite_difference_cic_' + _lib.suffix(self.dtype), _lib.ptr(self.value), nm, bs, bc,
                  _lib.ptr(p.pos), p.pos_bytes, p.size, int(bool(wrap)), _lib.ptr(out), fl.ptr,
                  _lib.stream_of(self.device), error=MeshError)
        fl.raise_if_set(*self._check_positions_geometry())
        return p.output(out)

    # -- spectral --

    def smooth_gaussian(self, radius, method='fft', nsigmas=2.5, **kwargs):
        """Gaussian smoothing (mesh.py:655-695): by FFT (``method='fft'``), else by the real-space
        convolution truncated at ``nsigmas``, whose output equals the reference's bit for bit."""
        torch = _torch()
        radius_ = _array3(radius, self.info._type_float)
        nm, bs, _ = self.info.c_geometry()
        lib = _lib.load()
        out = torch.empty(self.shape, dtype=torch_dtype(self.dtype), device=self.device)
        if method == 'fft':
            src = self._accum if self._accum is not None else self.value
            ws = self._workspace().get(lib.prc_fft_workspace_bytes(nm, self.dtype.itemsize, 1))
            _lib.call('prc_smooth_gaussian_' + _lib.suffix(self.dtype), _lib.ptr(src), src.element_size(), _lib.ptr(out),
                      nm, bs, _lib.d3(radius_), _lib.ptr(ws), ws.numel(), _lib.stream_of(self.device), error=MeshError)
        else:
            src = self.value                                   # in the mesh dtype, as the reference smooths it
            box = radius_ / self.info.boxsize                  # box units, in the mesh dtype (mesh.py:685)
            nsig = float(self.info._type_float.type(nsigmas))
            nbytes = lib.prc_smooth_gaussian_real_workspace_bytes(nm, _lib.d3(box), nsig, self.dtype.itemsize)
            if nbytes == 0:
                raise MeshError('smooth_gaussian: invalid radius {} or nsigmas {}'.format(radius, nsigmas))
            ws = self._workspace().get(nbytes)
            _lib.call('prc_smooth_gaussian_real_' + _lib.suffix(self.dtype), _lib.ptr(src), _lib.ptr(out), nm,
                      _lib.d3(box), nsig, _lib.ptr(ws), ws.numel(), _lib.stream_of(self.device), error=MeshError)
        self._accum = None
        self._colsums = None
        self.__dict__['value'] = out

    def to_complex(self):
        """Forward FFT (Hermitian half spectrum, numpy's rfftn convention)."""
        torch = _torch()
        cdt = torch.complex64 if self.dtype.itemsize == 4 else torch.complex128
        n = self.shape
        out = torch.empty((n[0], n[1], n[2] // 2 + 1), dtype=cdt, device=self.device)
        nm, _, _ = self.info.c_geometry()
        _lib.call('prc_rfft3d_' + _lib.suffix(self.dtype), _lib.ptr(self.value), self.value.element_size(),
                  _lib.ptr(out), nm, _lib.stream_of(self.device), error=MeshError)
        return ComplexMesh(out, info=self.info, device=self.device, attrs=self.attrs)

    def prod_sum(self, arrays, exp=1):
        """mesh *= (a0[:, None, None] + a1[None, :, None] + a2[None, None, :]) ** exp (mesh.py:707-736)."""
        torch = _torch()
        if len(arrays) != 3:
            raise MeshError('Provide a sequence of 3 arrays')
        coords = np.concatenate([np.asarray(a, dtype=self.info._type_float) for a in list(arrays)[::-1]], axis=0)
        if coords.size != sum(self.shape):
            raise MeshError('Length of input arrays must match shape')
        c = torch.from_numpy(coords).to(self.device)
        _lib.call('prc_prod_sum_' + _lib.suffix(self.dtype), _lib.ptr(self.value), _lib.i3(self.shape), _lib.ptr(c),
                  int(exp), _lib.stream_of(self.device), error=MeshError)


class ComplexMesh(BaseMesh):
    """Hermitian half spectrum on a CUDA device (shape n0 x n1 x (n2 // 2 + 1))."""

    def __init__(self, value=None, info=None, device=None, attrs=None, hermitian=True, **kwargs):
        if not hermitian:
            raise MeshError('pyrecon_b200 stores spectra of real meshes as Hermitian halves (hermitian=True)')
        self.hermitian = True
        super(ComplexMesh, self).__init__(value=value, info=info, device=device, attrs=attrs, **kwargs)

    @property
    def shape(self):
        n = self.info.shape
        return (n[0], n[1], n[2] // 2 + 1)

    @property
    def hshape(self):
        """Shape of the Hermitian half (the stored shape)."""
        return self.shape

    @property
    def fundamental_freq(self):
        """Fundamental frequency 2 pi / boxsize along each axis (mesh.py:806-810)."""
        return 2 * np.pi / self.boxsize

    def coords(self):
        """Wavenumbers along each axis, fftfreq / rfftfreq (mesh.py:812-820)."""
        out = []
        for idim, (n, d) in enumerate(zip(self.nmesh, self.boxsize / self.nmesh)):
            out.append(2 * np.pi * (np.fft.fftfreq(n, d=d) if idim < 2 else np.fft.rfftfreq(n, d=d)))
        return tuple(out)

    def to_real(self):
        """Inverse FFT (divided by the number of cells); the spectrum is consumed."""
        torch = _torch()
        out = torch.empty(self.info.shape, dtype=torch_dtype(self.info._type_float), device=self.device)
        nm, _, _ = self.info.c_geometry()
        work = self.value.clone()
        _lib.call('prc_irfft3d_' + _lib.suffix(self.info._type_float), _lib.ptr(work), _lib.ptr(out), nm,
                  _lib.stream_of(self.device), error=MeshError)
        return RealMesh(out, info=self.info, device=self.device, attrs=self.attrs)


def paint(info, accum, colsums, particles, wrap, accumulate, workspace, flags, check=True, order_out=None,
          sorted_out=None):
    """Deterministic CIC paint of ``particles`` into the FP64 ``accum`` mesh (C ABI prc_assign_cic)."""
    nm, bs, bc = info.c_geometry()
    lib = _lib.load()
    ws = workspace.get(lib.prc_assign_cic_workspace_bytes(nm, particles.size, info.dtype.itemsize))
    w = particles.weights
    args = [_lib.ptr(accum), _lib.ptr(colsums), nm, bs, bc, info.dtype.itemsize, _lib.ptr(particles.pos),
            particles.pos_bytes, _lib.ptr(w), 0 if w is None else w.element_size(), particles.size, int(bool(wrap)),
            int(bool(accumulate)), flags.ptr, _lib.ptr(ws), ws.numel(), _lib.stream_of(accum.device)]
    if order_out is not None and sorted_out is not None:
        _lib.call('prc_assign_cic_sorted', *args, _lib.ptr(order_out), _lib.ptr(sorted_out), error=MeshError)
    elif order_out is not None:
        _lib.call('prc_assign_cic_order', *args, _lib.ptr(order_out), error=MeshError)
    else:
        _lib.call('prc_assign_cic', *args, error=MeshError)
    if check:
        low, high = info.boxcenter - info.boxsize / 2., info.boxcenter + info.boxsize / 2.
        flags.raise_if_set(low, high)
