"""
Autotuner of the library's run-time knobs, with its choices kept as JSON wisdom.

The reference plans its FFTW transforms with a planner effort (``fft_plan``: 'estimate' ..
'exhaustive') and keeps the planner's wisdom for later runs (``fft_wisdom`` / ``save_fft_wisdom`` of
the reconstruction classes, pyrecon/mesh.py:1050-1081).  Here the CUDA launchers read integer knobs
from a run-time table (``prc_tune_set``); :func:`autotune` times the candidate values of each knob on
the device at hand for one mesh and keeps the fastest, and :class:`Wisdom` stores the choices per
device name as JSON, so a later run (or another process) applies them without timing anything.

Knobs:

* ``mg_jacobi`` (FP32 sweeps) and ``mg_jacobi_f64`` (FP64 sweeps), keyed by a multigrid level's n0:
  0 = one damped-Jacobi sweep per pass over the mesh, s > 0 = two sweeps per pass (temporal blocking),
  each block marching through slabs of s planes along x.  Unset levels use the library's default.
"""
import json
import os

import numpy as np

from . import _lib

FORMAT = 'pyrecon_b200 wisdom 1'
MG_SLABS = (0, 4, 8, 16, 32, 64)


def device_name(device=None):
    import torch
    return torch.cuda.get_device_name(device)


def mg_levels(nmesh):
    """The multigrid hierarchy's level shapes (coarsened while every axis is even and above 4,
    src/multigrid.c:303-328)."""
    n = [int(x) for x in nmesh]
    levels = [tuple(n)]
    while all(x > 4 and x % 2 == 0 for x in n):
        n = [x // 2 for x in n]
        levels.append(tuple(n))
    return levels


def _knob(dtype):
    return 'mg_jacobi' if np.dtype(dtype).itemsize == 4 else 'mg_jacobi_f64'


def _time_jacobi(shape, dtype, los, slab, device, repeats, sweeps=4):
    """Median CUDA-event time of `sweeps` damped-Jacobi sweeps at `shape` with the knob at `slab`."""
    import torch
    knob = _knob(dtype)
    tdt = torch.float32 if np.dtype(dtype).itemsize == 4 else torch.float64
    g = torch.Generator(device=device).manual_seed(7)
    v = torch.rand(shape, generator=g, device=device, dtype=tdt)
    f = torch.rand(shape, generator=g, device=device, dtype=tdt)
    tmp = torch.empty_like(v)
    st = torch.cuda.current_stream(device)
    args = (_lib.ptr(v), _lib.ptr(f), _lib.ptr(tmp), _lib.i3(shape), _lib.d3([2000.] * 3), _lib.d3([2000.] * 3), 0.4,
            0.4, sweeps, _lib.opt_d3(los), _lib.c_void_p(st.cuda_stream))
    name = 'prc_mg_jacobi_' + _lib.suffix(dtype)
    old = _lib.tune_get(knob, shape[0], -1)
    _lib.tune_set(knob, shape[0], slab)
    try:
        _lib.call(name, *args)      # warm-up
        times = []
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            _lib.call(name, *args)
            b.record(st)
            b.synchronize()
            times.append(a.elapsed_time(b))
    finally:
        _lib.tune_set(knob, shape[0], old)
    return float(np.median(times))


def autotune(nmesh, dtype='f4', los=None, device=None, repeats=5, candidates=MG_SLABS, mixed_precision=True):
    """Time every candidate of every knob for a mesh of shape `nmesh` and precision `dtype` on `device`
    (current by default); returns {knob: {key: best value}} and {knob: {key: {value: ms}}}.  FP32
    meshes with mixed precision run their sweeps in FP32 (the FP64 defect correction has no sweeps)."""
    import torch
    device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
    dtype = np.dtype(dtype)
    knob = _knob(dtype)
    best, timings = {knob: {}}, {knob: {}}
    for shape in mg_levels(nmesh):
        if shape[2] % 4 != 0:
            continue            # the one-cell kernels: nothing to choose
        ms = {}
        for slab in candidates:
            if slab > 0 and slab > 2 * shape[0]:
                continue
            ms[slab] = _time_jacobi(shape, dtype, los, slab, device, repeats)
        timings[knob][shape[0]] = ms
        best[knob][shape[0]] = int(min(ms, key=ms.get))
    return best, timings


class Wisdom(object):
    """Tuning choices per device name: {device: {knob: {key: value}}}, kept as JSON."""

    def __init__(self, entries=None):
        self.entries = {}
        if entries:
            for dev, knobs in entries.items():
                for knob, kv in knobs.items():
                    for key, value in kv.items():
                        self.entries.setdefault(dev, {}).setdefault(knob, {})[int(key)] = int(value)

    @classmethod
    def load(cls, source):
        """From a path, a JSON string's parsed dict, or another Wisdom."""
        if isinstance(source, Wisdom):
            return cls(source.entries)
        if isinstance(source, dict):
            return cls(source.get('devices', source))
        with open(source) as fh:
            data = json.load(fh)
        if data.get('format') != FORMAT:
            raise ValueError('{} is not {} wisdom'.format(source, FORMAT))
        return cls(data['devices'])

    def save(self, path):
        data = dict(format=FORMAT, devices={dev: {knob: {str(k): v for k, v in sorted(kv.items())}
                                                  for knob, kv in knobs.items()} for dev, knobs in self.entries.items()})
        tmp = '{}.tmp{}'.format(path, os.getpid())
        with open(tmp, 'w') as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)

    def update(self, device, best):
        for knob, kv in best.items():
            self.entries.setdefault(device, {}).setdefault(knob, {}).update({int(k): int(v) for k, v in kv.items()})

    def covers(self, device, nmesh, dtype):
        """True if every tunable level of this mesh has an entry for `device`."""
        knob = _knob(dtype)
        have = self.entries.get(device, {}).get(knob, {})
        return all(shape[0] in have for shape in mg_levels(nmesh) if shape[2] % 4 == 0)

    def apply(self, device):
        """Set this device's entries in the library's tuning table; returns how many."""
        count = 0
        for knob, kv in self.entries.get(device, {}).items():
            for key, value in kv.items():
                _lib.tune_set(knob, key, value)
                count += 1
        return count


def default_wisdom_path(nmesh, dtype, device=None):
    """Named like the reference's default FFTW wisdom file (pyrecon/mesh.py:1056-1058)."""
    name = device_name(device).replace(' ', '_')
    return 'wisdom.shape-{:d}-{:d}-{:d}.type-{}.device-{}.json'.format(*[int(n) for n in nmesh], np.dtype(dtype).str[1:],
                                                                       name)


def setup(nmesh, dtype, fft_wisdom=None, save_fft_wisdom=None, fft_plan='measure', los=None, device=None):
    """The reconstruction classes' wisdom arguments: apply `fft_wisdom` (path, dict or Wisdom); with
    `save_fft_wisdom` (True for the default path, or a path), load that file if it exists, autotune what it
    lacks for this mesh unless fft_plan is 'estimate', apply and save it.  Returns the Wisdom in use or None."""
    wisdom = None
    if fft_wisdom is None and (save_fft_wisdom is None or save_fft_wisdom is False):
        return None
    dev = device_name(device)
    if fft_wisdom is not None:
        try:
            wisdom = Wisdom.load(fft_wisdom)
        except (OSError, ValueError, TypeError, KeyError, AttributeError) as exc:
            # the reference's FFTW wisdom (a tuple, or a .npy file) means nothing to these kernels
            import warnings
            warnings.warn('fft_wisdom ignored: not {} wisdom ({})'.format(FORMAT, exc))
        else:
            wisdom.apply(dev)
    if save_fft_wisdom is not None and save_fft_wisdom is not False:
        path = default_wisdom_path(nmesh, dtype, device) if save_fft_wisdom is True else str(save_fft_wisdom)
        saved = Wisdom.load(path) if os.path.isfile(path) else Wisdom()
        if wisdom is not None:
            saved.entries = {**wisdom.entries, **saved.entries}
        if not saved.covers(dev, nmesh, dtype) and str(fft_plan).lower() != 'estimate':
            best, _ = autotune(nmesh, dtype, los=los, device=device)
            saved.update(dev, best)
        saved.apply(dev)
        saved.save(path)
        wisdom = saved
    return wisdom
