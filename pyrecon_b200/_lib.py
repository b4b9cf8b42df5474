"""
ctypes binding of libpyrecon_cuda.so (include/pyrecon_cuda.h).

The library is built in-tree by ``python -m pyrecon_b200.build``; there is no CPU
fallback: if the library or a CUDA device is missing, every entry point raises.
"""
import os
import ctypes
import threading

import numpy as np

from . import build as _build

c_int, c_i64, c_size, c_double, c_void_p = ctypes.c_int, ctypes.c_int64, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p
I3 = ctypes.c_int32 * 3
D3 = ctypes.c_double * 3
DP = ctypes.POINTER(ctypes.c_double)   # optional 3-vector (NULL = local line of sight)

PRC_OK = 0
PRC_FLAG_OUT_OF_BOX = 1
PRC_FLAG_NONFINITE = 2
PRC_FLAG_DEVICE_WAIT = 4
PRC_ERR_ARG = 1
PRC_ERR_TIMEOUT = 5
PRC_FAULT_WAIT_TIMEOUT = 1
FIELDS = {'disp': 0, 'rsd': 1, 'disp+rsd': 2}

_lock = threading.Lock()
_lib = None

_p = c_void_p
_SIGNATURES = {
    'prc_version': (ctypes.c_char_p, []),
    'prc_status_string': (ctypes.c_char_p, [c_int]),
    'prc_launch_count': (ctypes.c_ulonglong, []),
    'prc_profile_enable': (None, [c_int]),
    'prc_profile_collect': (c_int, [ctypes.c_char_p, c_size]),
    'prc_fft_supported': (c_int, [I3]),
    'prc_sum_f32': (c_int, [_p, c_i64, _p, _p, c_size, _p]),
    'prc_zeldovich_psi_workspace_bytes': (c_size, [I3, c_int]),
    'prc_device_fault_flags': (ctypes.c_uint, [c_int]),
    'prc_debug_wait_timeout': (c_int, [c_i64, _p, _p]),
    'prc_tune_set': (c_int, [ctypes.c_char_p, c_int, c_int]),
    'prc_tune_get': (c_int, [ctypes.c_char_p, c_int, c_int]),
    'prc_tune_clear': (None, []),
    'prc_assign_cic_workspace_bytes': (c_size, [I3, c_i64, c_int]),
    'prc_assign_cic': (c_int, [_p, _p, I3, D3, D3, c_int, _p, c_int, _p, c_int, c_i64, c_int, c_int, _p, _p, c_size, _p]),
    'prc_assign_cic_order': (c_int, [_p, _p, I3, D3, D3, c_int, _p, c_int, _p, c_int, c_i64, c_int, c_int, _p, _p, c_size,
                                     _p, _p]),
    'prc_assign_cic_sorted': (c_int, [_p, _p, I3, D3, D3, c_int, _p, c_int, _p, c_int, c_i64, c_int, c_int, _p, _p, c_size,
                                      _p, _p, _p]),
    'prc_cic_cell_order': (c_int, [_p, _p, I3, D3, D3, c_int, _p, c_int, c_i64, c_int, _p, _p, c_size, _p]),
    'prc_assign_cic_noalloc': (c_int, [_p, _p, I3, D3, D3, c_int, _p, c_int, _p, c_int, c_i64, c_int, c_int, _p, _p]),
    'prc_sum_workspace_bytes': (c_size, [c_i64]),
    'prc_sum_f64': (c_int, [_p, c_i64, _p, _p, c_size, _p]),
    'prc_fft_workspace_bytes': (c_size, [I3, c_int, c_int]),
    'prc_density_contrast_workspace_bytes': (c_size, [I3, c_int, c_int]),
    'prc_plane_parallel_workspace_bytes': (c_size, [I3, c_int]),
    'prc_iterative_fft_workspace_bytes': (c_size, [I3, c_int, c_int]),
    'prc_multigrid_workspace_bytes': (c_size, [I3, c_int, c_int]),
    'prc_smooth_gaussian_real_workspace_bytes': (c_size, [I3, D3, c_double, c_int]),
    'prc_density_contrast_original_workspace_bytes': (c_size, []),
}
for _s in ['f32', 'f64']:
    _SIGNATURES.update({
        'prc_read_cic_' + _s: (c_int, [_p, I3, D3, D3, _p, c_int, c_i64, c_int, _p, _p, _p]),
        'prc_read_finite_difference_cic_' + _s: (c_int, [_p, I3, D3, D3, _p, c_int, c_i64, c_int, _p, _p, _p]),
        'prc_read_shifts_psi_' + _s: (c_int, [_p, _p, _p, c_int, I3, D3, D3, _p, c_int, c_i64, _p, c_double, DP,
                                              c_int, c_int, c_int, _p, c_int, _p, _p, _p]),
        'prc_read_shifts_phi_' + _s: (c_int, [_p, I3, D3, D3, _p, c_int, c_i64, _p, c_double, DP, c_int, c_int, c_int,
                                              _p, c_int, _p, _p, _p]),
        'prc_delta_from_meshes_' + _s: (c_int, [_p, _p, c_int, _p, I3, c_double, c_double, c_double, _p, _p]),
        'prc_zeldovich_psi_' + _s: (c_int, [_p, I3, D3, _p, _p, _p, c_int, _p, c_size, _p]),
        'prc_ifftp_update_' + _s: (c_int, [_p, I3, D3, D3, _p, _p, c_int, c_i64, c_double, c_double, c_int, DP, c_int,
                                           _p, _p]),
        'prc_ifftp_read_' + _s: (c_int, [_p, I3, D3, D3, _p, _p, c_int, c_i64, c_double, DP, c_int, c_int, c_int, _p,
                                         c_int, _p, _p, _p]),
        'prc_rfft3d_' + _s: (c_int, [_p, c_int, _p, I3, _p]),
        'prc_irfft3d_' + _s: (c_int, [_p, _p, I3, _p]),
        'prc_smooth_gaussian_' + _s: (c_int, [_p, c_int, _p, I3, D3, D3, _p, c_size, _p]),
        'prc_smooth_gaussian_real_' + _s: (c_int, [_p, _p, I3, D3, c_double, _p, c_size, _p]),
        'prc_density_contrast_original_' + _s: (c_int, [_p, _p, I3, c_double, c_double, _p, _p, c_size, _p]),
        'prc_density_contrast_' + _s: (c_int, [_p, _p, _p, I3, D3, D3, c_double, c_double, c_double, _p, _p, c_size, _p]),
        'prc_plane_parallel_fft_' + _s: (c_int, [_p, I3, D3, c_double, D3, _p, _p, _p, c_int, _p, c_size, _p]),
        'prc_iterative_fft_' + _s: (c_int, [_p, I3, D3, D3, c_double, DP, c_int, _p, _p, _p, c_int, _p, c_size, _p]),
        'prc_prod_sum_' + _s: (c_int, [_p, I3, _p, c_int, _p]),
        'prc_mg_jacobi_' + _s: (c_int, [_p, _p, _p, I3, D3, D3, c_double, c_double, c_int, DP, _p]),
        'prc_mg_residual_' + _s: (c_int, [_p, _p, _p, I3, D3, D3, c_double, DP, _p]),
        'prc_mg_reduce_' + _s: (c_int, [_p, _p, I3, _p]),
        'prc_mg_prolong_' + _s: (c_int, [_p, _p, I3, _p]),
    })
_SIGNATURES['prc_multigrid_f32'] = (c_int, [_p, _p, I3, D3, D3, c_double, c_double, c_int, c_int, DP, c_int, _p, c_size, _p])
_SIGNATURES['prc_multigrid_f64'] = (c_int, [_p, _p, I3, D3, D3, c_double, c_double, c_int, c_int, DP, _p, c_size, _p])
_SIGNATURES['prc_multigrid_batch_workspace_bytes'] = (c_size, [I3, c_int, c_int, c_int])
_SIGNATURES['prc_plane_parallel_batch_workspace_bytes'] = (c_size, [I3, c_int, c_int])
for _s in ('f32', 'f64'):
    _SIGNATURES['prc_plane_parallel_fft_batch_' + _s] = (c_int, [_p, _p, _p, _p, c_int, I3, D3, c_double, D3, c_int, _p,
                                                                 c_size, _p])
_SIGNATURES['prc_multigrid_mixed_f32'] = (c_int, [_p, _p, _p, I3, D3, D3, c_double, c_double, c_int, c_int, DP, _p,
                                                  c_size, _p])
_SIGNATURES['prc_multigrid_batch_mixed_f32'] = (c_int, [_p, _p, _p, c_int, I3, D3, D3, c_double, c_double, c_int,
                                                        c_int, DP, _p, c_size, _p])
_SIGNATURES['prc_multigrid_batch_f32'] = (c_int, [_p, _p, c_int, I3, D3, D3, c_double, c_double, c_int, c_int, DP, c_int,
                                                  _p, c_size, _p])
_SIGNATURES['prc_multigrid_batch_f64'] = (c_int, [_p, _p, c_int, I3, D3, D3, c_double, c_double, c_int, c_int, DP, _p,
                                                  c_size, _p])


def pointer_array(tensors):
    """Host array of the device pointers of `tensors` (a `const T* const*` argument)."""
    return (c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


class LibraryError(RuntimeError):
    """The CUDA library is missing, or a call into it failed."""


def library_path():
    """The in-tree library, or the build variant named by PRC_LIBRARY (a path, or a variant name such as
    'nopp' for lib/libpyrecon_cuda_nopp.so)."""
    alt = os.environ.get('PRC_LIBRARY')
    if alt:
        return alt if os.sep in alt else _build.library_path(alt)
    return _build.library_path()


def load():
    """Load the CUDA library (raises LibraryError if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            path = library_path()
            if not os.path.isfile(path):
                raise LibraryError('{} not found: build it with `python -m pyrecon_b200.build` '
                                   '(there is no CPU fallback)'.format(path))
            lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
            for name, (restype, argtypes) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _lib = lib
    return _lib


def exported_symbols():
    return sorted(_SIGNATURES)


def status_string(status):
    return load().prc_status_string(int(status)).decode()


def i3(v):
    return I3(*[int(x) for x in v])


def d3(v):
    return D3(*[float(x) for x in v])


def opt_d3(v):
    """Optional 3-vector argument (a double[3], or NULL when v is None)."""
    return None if v is None else d3(v)


def ptr(t):
    return None if t is None else c_void_p(t.data_ptr())


def stream_of(device):
    import torch
    return c_void_p(torch.cuda.current_stream(device).cuda_stream)


def call(name, *args, error=None):
    """Call entry point `name`; raise `error` (an exception class) with the status text on failure."""
    fn = getattr(load(), name)
    status = fn(*args)
    if status != PRC_OK:
        exc = error or LibraryError
        raise exc('{} failed: {} (status {})'.format(name, status_string(status), status))
    return status


def tune_set(name, key, value):
    """Set knob `name` for key `key` (a mesh axis length) of the run-time tuning table; value < 0 removes it."""
    call('prc_tune_set', name.encode(), int(key), int(value))


def tune_get(name, key, default=-1):
    return int(load().prc_tune_get(name.encode(), int(key), int(default)))


def tune_clear():
    load().prc_tune_clear()


def launch_count():
    """Kernels launched by the library so far."""
    return int(load().prc_launch_count())


def profile_enable(on=True):
    load().prc_profile_enable(int(bool(on)))


def profile_collect():
    """{kernel name: (launches, total device ms)} of the launches since profile_enable(True)."""
    import json
    buf = ctypes.create_string_buffer(1 << 16)
    load().prc_profile_collect(buf, len(buf))
    return {k: tuple(v) for k, v in json.loads(buf.value.decode()).items()}


def check_device_faults(error=RuntimeError):
    """Raise ``error`` if a kernel on the current device gave up a bounded wait (the device fault
    word, cleared here); synchronises with the device."""
    flags = load().prc_device_fault_flags(1)
    if flags:
        raise error('{} (device fault flags {:#x})'.format(status_string(PRC_ERR_TIMEOUT), flags))


def suffix(dtype):
    return 'f32' if np.dtype(dtype).itemsize == 4 else 'f64'
