"""
Small utilities with the reference's names (pyrecon/utils.py): per-class loggers,
``distance``, ``broadcast_arrays``, ``setup_logging``.  They accept numpy arrays and
torch tensors alike.
"""
import sys
import time
import logging

import numpy as np

logger = logging.getLogger('pyrecon_b200')


def setup_logging(level=logging.INFO, stream=sys.stdout, filename=None, filemode='w', **kwargs):
    """Configure the root logger with elapsed-time prefixes (pyrecon/utils.py:26-70)."""
    if isinstance(level, str):
        level = {'info': logging.INFO, 'debug': logging.DEBUG, 'warning': logging.WARNING}[level.lower()]
    for handler in logging.root.handlers:
        logging.root.removeHandler(handler)
    t0 = time.time()

    class _Formatter(logging.Formatter):
        def format(self, record):
            self._style._fmt = '[%09.2f] ' % (time.time() - t0) + ' %(asctime)s %(name)-28s %(levelname)-8s %(message)s'
            return super(_Formatter, self).format(record)

    fmt = _Formatter(datefmt='%m-%d %H:%M ')
    handler = logging.FileHandler(filename, mode=filemode) if filename is not None else logging.StreamHandler(stream=stream)
    handler.setFormatter(fmt)
    logging.basicConfig(level=level, handlers=[handler], **kwargs)


class BaseMetaClass(type):
    """Gives every class a logger named after it and log_<level> class methods (pyrecon/utils.py:81-108)."""

    def __new__(meta, name, bases, class_dict):
        cls = super().__new__(meta, name, bases, class_dict)
        cls.logger = logging.getLogger(name)

        def make(level):
            @classmethod
            def log(cls, *args, **kwargs):
                getattr(cls.logger, level)(*args, **kwargs)
            return log

        for level in ['debug', 'info', 'warning', 'error', 'critical']:
            setattr(cls, 'log_{}'.format(level), make(level))
        return cls


class BaseClass(object, metaclass=BaseMetaClass):
    """Base class with shallow ``copy``."""

    def __copy__(self):
        new = self.__class__.__new__(self.__class__)
        new.__dict__.update(self.__dict__)
        return new

    def copy(self):
        return self.__copy__()


def broadcast_arrays(*arrays):
    """N 1D arrays -> N arrays of shape (n1, 1, ...), (1, n2, ...), ... (pyrecon/utils.py:125-143)."""
    out = []
    for iaxis, array in enumerate(arrays):
        sl = [None] * len(arrays)
        sl[iaxis] = slice(None)
        out.append(array[tuple(sl)])
    return tuple(out)


def distance(position):
    """Cartesian distance along the last axis (pyrecon/utils.py:146-148)."""
    try:
        import torch
        if isinstance(position, torch.Tensor):
            return torch.sqrt((position ** 2).sum(dim=-1))
    except ImportError:
        pass
    return np.sqrt((position ** 2).sum(axis=-1))


def mkdir(dirname):
    """Create ``dirname`` (and parents); an existing directory is not an error (pyrecon/utils.py:73-78)."""
    import os
    try:
        os.makedirs(dirname)
    except OSError:
        return


def _is_tensor(x):
    try:
        import torch
        return isinstance(x, torch.Tensor)
    except ImportError:
        return False


def cartesian_to_sky(position, wrap=True, degree=True):
    """Distance, RA, Dec of Cartesian positions of shape (N, 3) (pyrecon/utils.py:151-182): RA from
    arctan2(y, x), wrapped into [0, 2 pi) if ``wrap``, Dec = arcsin(z / distance); angles in degrees if
    ``degree``.  Torch tensors are transformed where they are (e.g. on the GPU)."""
    dist = distance(position)
    if _is_tensor(position):
        import torch
        ra = torch.atan2(position[:, 1], position[:, 0])
        if wrap:
            ra = torch.remainder(ra, 2. * np.pi)
        dec = torch.asin(position[:, 2] / dist)
    else:
        ra = np.arctan2(position[:, 1], position[:, 0])
        if wrap:
            ra %= 2. * np.pi
        dec = np.arcsin(position[:, 2] / dist)
    conversion = np.pi / 180. if degree else 1.
    return dist, ra / conversion, dec / conversion


def sky_to_cartesian(dist, ra, dec, degree=True, dtype=None):
    """Cartesian positions, shape (N, 3), of distance, RA, Dec (pyrecon/utils.py:185-217); ``dtype`` of the
    unit vectors as numpy's ``array(..., dtype)``.  Torch tensors are transformed where they are."""
    conversion = np.pi / 180. if degree else 1.
    if _is_tensor(dist) or _is_tensor(ra) or _is_tensor(dec):
        import torch
        ra, dec = torch.as_tensor(ra), torch.as_tensor(dec)
        cos_dec = torch.cos(dec * conversion)
        unit = torch.stack([cos_dec * torch.cos(ra * conversion), cos_dec * torch.sin(ra * conversion),
                            torch.sin(dec * conversion)])
        if dtype is not None:
            from .mesh import torch_dtype
            unit = unit.to(torch_dtype(dtype))
        return (torch.as_tensor(dist, device=unit.device) * unit).T
    cos_dec = np.cos(dec * conversion)
    unit = np.array([cos_dec * np.cos(ra * conversion), cos_dec * np.sin(ra * conversion), np.sin(dec * conversion)],
                    dtype=dtype)
    return (dist * unit).T


class DistanceToRedshift(object):
    """Redshift as a function of distance (pyrecon/utils.py:220-256): ``distance(z)`` tabulated on z = 0
    and ``nz`` log-spaced redshifts from 1e-8 to ``zmax``, inverted by an interpolating spline of order
    ``interp_order`` through (distance, z)."""

    def __init__(self, distance, zmax=100., nz=2048, interp_order=3):
        from scipy import interpolate
        self.distance = distance
        self.zmax = zmax
        self.nz = nz
        self.zgrid = np.concatenate([[0.], np.logspace(-8, np.log10(self.zmax), self.nz)])
        self.rgrid = self.distance(self.zgrid)
        self.interp = interpolate.UnivariateSpline(self.rgrid, self.zgrid, k=interp_order, s=0)

    def __call__(self, distance):
        """Redshift at ``distance`` (scalar, array, or tensor: evaluated on the host, returned alike)."""
        if _is_tensor(distance):
            import torch
            z = self(distance.detach().cpu().numpy())
            return torch.as_tensor(z).to(distance.device)
        distance = np.asarray(distance)
        return self.interp(distance).astype(distance.dtype, copy=False)


def random_box_positions(boxsize, boxcenter=0., size=None, nbar=None, rng=None, seed=None, dtype=None):
    """Uniform positions of shape (size, 3) in a box (pyrecon/utils.py:266-310); ``size`` defaults to the
    nearest integer to ``nbar`` times the box volume.  Same draws as the reference for the same ``seed``
    (numpy RandomState)."""
    if rng is None:
        rng = np.random.RandomState(seed=seed)
    boxsize_ = np.empty(3, dtype=dtype)
    boxsize_[...] = boxsize
    if size is None:
        if nbar is None:
            raise ValueError('Provide either size or nbar')
        size = int(nbar * np.prod(boxsize_) + 0.5)
    positions = rng.uniform(0., 1., size=(size, 3)).astype(dtype)
    boxsize_ = boxsize_.astype(dtype)
    boxcenter_ = np.empty(3, dtype=positions.dtype)
    boxcenter_[...] = boxcenter
    return positions * boxsize_ + (boxcenter_ - boxsize_ / 2.)


class MemoryMonitor(object):
    """Host memory (RSS, MB) and wall time since the last call, printed on creation and every call; with
    ``device``, also the CUDA device memory allocated by torch (pyrecon/utils.py:313-352).

    >>> with MemoryMonitor() as mem:
    ...     mem('painted')
    """

    def __init__(self, pid=None, device=None):
        import os
        import psutil
        self.proc = psutil.Process(os.getpid() if pid is None else pid)
        self.device = device
        self.mem = self.proc.memory_info().rss / 1e6
        self.time = time.time()
        print('using {}'.format(self._usage()), flush=True)

    def _usage(self):
        msg = '{:.3f} [Mb]'.format(self.mem)
        if self.device is not None:
            import torch
            msg += ', device {:.3f} [Mb]'.format(torch.cuda.memory_allocated(self.device) / 1e6)
        return msg

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self()

    def __call__(self, log=None):
        mem = self.proc.memory_info().rss / 1e6
        t = time.time()
        msg = 'using {:.3f} [Mb] (increase of {:.3f} [Mb]) after {:.3f} [s]'.format(mem, mem - self.mem, t - self.time)
        if self.device is not None:
            import torch
            msg += ', device {:.3f} [Mb]'.format(torch.cuda.memory_allocated(self.device) / 1e6)
        if log:
            msg = '[{}] {}'.format(log, msg)
        print(msg, flush=True)
        self.mem, self.time = mem, t
