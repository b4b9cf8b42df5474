"""
TEST INFRASTRUCTURE ONLY -- not part of the product.

CPU oracle for the reconstruction hot path: a numpy restatement of the
reference's Python glue (pyrecon/recon.py, pyrecon/mesh.py,
pyrecon/iterative_fft.py, pyrecon/plane_parallel_fft.py,
pyrecon/multigrid.py) driving C kernels through ctypes.  Two C back-ends:

* ``kernels='oracle'``: our own C restatement (oracle/oracle_mesh.c,
  oracle/oracle_multigrid.c), built by ``make -C oracle``;
* ``kernels='reference'``: the reference's own C sources compiled unchanged
  into oracle/_ref/ by ``make -C oracle ref`` (same ABI as the reference's
  mesh_{float,double}.so / multigrid_{float,double}.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, always as the checker or the timed CPU baseline, never as the
product path.

Every step keeps the reference's dtype semantics: meshes are stored in the
mesh dtype ('f4' or 'f8') after every mesh operation, FFTs are full complex
(c2c) transforms whose inverse keeps ``.real`` (pyrecon/recon.py:117,
pyrecon/mesh.py:842, :978-988), and k-space multipliers are built from
``2 pi fftfreq`` in float64.
"""

import os
import ctypes

import numpy as np
from numpy import ctypeslib

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, '_build')
REF_DIR = os.path.join(HERE, '_ref')


class OracleError(Exception):
    """Raised for the conditions the reference raises MeshError / ReconstructionError on."""


def build(reference_src=None):
    """Compile the oracle C restatement and, given the reference's ``src/`` directory (argument, or the
    environment variable PYRECON_REFERENCE_SRC), the reference kernels into oracle/_ref."""
    import subprocess
    subprocess.run(['make', '-s', '-C', HERE, 'all'], check=True)
    src = reference_src or os.environ.get('PYRECON_REFERENCE_SRC')
    if src is None:
        print('oracle: reference kernels not built (no reference src/ given: set PYRECON_REFERENCE_SRC)')
        return
    if not os.path.isfile(os.path.join(src, 'mesh.c')):
        raise OracleError('{} is not the reference\'s src/ directory (no mesh.c)'.format(src))
    subprocess.run(['make', '-s', '-C', HERE, 'ref', 'REFERENCE_SRC={}'.format(src)], check=True)


def reference_kernels_available():
    return all(os.path.isfile(os.path.join(REF_DIR, '{}_{}.so'.format(k, p)))
               for k in ['mesh', 'multigrid'] for p in ['float', 'double'])


# ----------------------------------------------------------------------------------------------
# C back-ends
# ----------------------------------------------------------------------------------------------

class _Kernels(object):
    """ctypes wrapper over one precision of either C back-end."""

    def __init__(self, dtype, source='oracle'):
        self.dtype = np.dtype(dtype)
        self.source = source
        ctype = ctypeslib.as_ctypes_type(self.dtype)
        self._ctype = ctype
        if source == 'oracle':
            name = os.path.join(BUILD_DIR, 'liboracle_{}.so'.format('f32' if self.dtype.itemsize == 4 else 'f64'))
            if not os.path.isfile(name):
                build()
            lib = ctypes.CDLL(name, mode=ctypes.RTLD_LOCAL)
            self._mesh, self._mg = lib, lib
            self._names = dict(assign='oracle_assign_cic', read='oracle_read_cic',
                               fd='oracle_read_finite_difference_cic', prod='oracle_prod_sum', fmg='oracle_fmg',
                               smooth='oracle_smooth_gaussian')
        elif source == 'reference':
            prec = 'float' if self.dtype.itemsize == 4 else 'double'
            self._mesh = ctypes.CDLL(os.path.join(REF_DIR, 'mesh_{}.so'.format(prec)), mode=ctypes.RTLD_LOCAL)
            self._mg = ctypes.CDLL(os.path.join(REF_DIR, 'multigrid_{}.so'.format(prec)), mode=ctypes.RTLD_LOCAL)
            self._names = dict(assign='assign_cic', read='read_cic', fd='read_finite_difference_cic',
                               prod='prod_sum', fmg='fmg', smooth='smooth_gaussian')
        else:
            raise ValueError('unknown kernel source {}'.format(source))

    def set_num_threads(self, nthreads):
        if self.source == 'reference' and nthreads:
            self._mesh.set_num_threads.argtypes = (ctypes.c_int,)
            # one libgomp per process: this also sets the thread count multigrid.c runs with
            self._mesh.set_num_threads(int(nthreads))

    def _ptr(self, n):
        return ctypeslib.ndpointer(dtype=self.dtype, shape=n, flags='C')

    @staticmethod
    def _sizes(nmesh):
        return np.ascontiguousarray(nmesh, dtype=np.uint64)

    def assign_cic(self, mesh, nmesh, pos, weights):
        f = getattr(self._mesh, self._names['assign'])
        f.argtypes = (self._ptr(mesh.size), ctypeslib.ndpointer(np.uint64, shape=3), self._ptr(pos.size),
                      self._ptr(weights.size), ctypes.c_size_t)
        f.restype = ctypes.c_int
        flat = mesh.reshape(-1)
        if f(flat, self._sizes(nmesh), pos, weights, len(weights)) != 0:
            raise OracleError('assign_cic failed')

    def read_cic(self, mesh, nmesh, pos):
        out = np.empty(pos.size // 3, dtype=self.dtype)
        f = getattr(self._mesh, self._names['read'])
        f.argtypes = (self._ptr(mesh.size), ctypeslib.ndpointer(np.uint64, shape=3), self._ptr(pos.size),
                      self._ptr(out.size), ctypes.c_size_t)
        f.restype = ctypes.c_int
        if f(np.ascontiguousarray(mesh).reshape(-1), self._sizes(nmesh), pos, out, out.size) != 0:
            raise OracleError('read_cic failed')
        return out

    def read_finite_difference_cic(self, mesh, nmesh, boxsize, pos):
        out = np.empty(pos.size, dtype=self.dtype)
        f = getattr(self._mesh, self._names['fd'])
        f.argtypes = (self._ptr(mesh.size), ctypeslib.ndpointer(np.uint64, shape=3), self._ptr(3),
                      self._ptr(pos.size), self._ptr(out.size), ctypes.c_size_t)
        f.restype = ctypes.c_int
        if f(np.ascontiguousarray(mesh).reshape(-1), self._sizes(nmesh), np.ascontiguousarray(boxsize, dtype=self.dtype),
             pos, out, pos.size // 3) != 0:
            raise OracleError('read_finite_difference_cic failed')
        return out.reshape(-1, 3)

    def prod_sum(self, flat_real, shape, coords, exp):
        f = getattr(self._mesh, self._names['prod'])
        f.argtypes = (self._ptr(flat_real.size), ctypeslib.ndpointer(np.uint64, shape=3), self._ptr(coords.size), ctypes.c_int)
        f.restype = ctypes.c_int
        f(flat_real, self._sizes(shape), coords, int(exp))

    def smooth_gaussian(self, mesh, nmesh, radius, nsigmas):
        """In-place real-space smoothing; radius in box units (mesh.py:684-695, mesh.c:117-143)."""
        f = getattr(self._mesh, self._names['smooth'])
        f.argtypes = (self._ptr(mesh.size), ctypeslib.ndpointer(np.uint64, shape=3), self._ptr(3), self._ctype)
        f.restype = ctypes.c_int
        flat = mesh.reshape(-1)
        if f(flat, self._sizes(nmesh), np.ascontiguousarray(radius, dtype=self.dtype), self.dtype.type(nsigmas)) != 0:
            raise OracleError('smooth_gaussian failed')

    def fmg(self, delta, nmesh, boxsize, boxcenter, beta, damping, jacobi_niterations, vcycle_niterations, los):
        phi = np.zeros(delta.size, dtype=self.dtype)
        f = getattr(self._mg, self._names['fmg'])
        ptr = ctypes.POINTER(self._ctype)
        f.argtypes = (self._ptr(delta.size), self._ptr(delta.size), ctypeslib.ndpointer(np.uint64, shape=3),
                      self._ptr(3), self._ptr(3), self._ctype, self._ctype, ctypes.c_int, ctypes.c_int,
                      ptr if los is None else self._ptr(3))
        if self.source == 'oracle':
            f.restype = ctypes.c_int
        losarg = ptr() if los is None else np.ascontiguousarray(los, dtype=self.dtype)
        f(np.ascontiguousarray(delta, dtype=self.dtype).reshape(-1), phi, self._sizes(nmesh),
          np.ascontiguousarray(boxsize, dtype=self.dtype), np.ascontiguousarray(boxcenter, dtype=self.dtype),
          beta, damping, int(jacobi_niterations), int(vcycle_niterations), losarg)
        return phi.reshape(tuple(nmesh))


# ----------------------------------------------------------------------------------------------
# FFT engines: full complex transforms, forward unnormalised, backward divided by the size
# ----------------------------------------------------------------------------------------------

class FFT(object):
    """``engine='numpy'`` is the reference's default (pyrecon/mesh.py:974-988); ``'scipy'`` is the same
    pocketfft algorithm with ``workers`` threads, standing in for the reference's multithreaded FFTW engine."""

    def __init__(self, engine='numpy', workers=1):
        self.engine = engine
        self.workers = workers

    def forward(self, value, ctype):
        if self.engine == 'scipy':
            import scipy.fft
            return scipy.fft.fftn(value, workers=self.workers).astype(ctype, copy=False)
        return np.fft.fftn(value).astype(ctype, copy=False)

    def backward(self, value, ctype):
        if self.engine == 'scipy':
            import scipy.fft
            return scipy.fft.ifftn(value, workers=self.workers).astype(ctype, copy=False)
        return np.fft.ifftn(value).astype(ctype, copy=False)


# ----------------------------------------------------------------------------------------------
# Geometry (pyrecon/mesh.py:342-483)
# ----------------------------------------------------------------------------------------------

def _array3(value, dtype):
    """A length-3 array of ``dtype`` filled from a scalar or a 3-sequence (mesh.py:15-19)."""
    out = np.empty(3, dtype=dtype)
    out[...] = value
    return out


class Geometry(object):

    def __init__(self, nmesh, boxsize, boxcenter, dtype='f8'):
        self.dtype = np.dtype(dtype)
        self.nmesh = _array3(nmesh, np.int32)                          # mesh.py:460 (ctypes.c_int)
        self.boxsize = _array3(_array3(boxsize, 'f8'), self.dtype)     # mesh.py:403 then :450
        self.boxcenter = _array3(boxcenter, self.dtype)                # mesh.py:455
        self.ctype = np.dtype('c{:d}'.format(2 * self.dtype.itemsize))

    @property
    def shape(self):
        return tuple(int(n) for n in self.nmesh)

    @property
    def offset(self):
        return self.boxcenter - self.boxsize / 2.

    def wrap(self, positions):
        """mesh.py:477-479."""
        return ((positions - self.offset) % self.boxsize) + self.offset

    def check_in_box(self, positions):
        low, high = self.boxcenter - self.boxsize / 2., self.boxcenter + self.boxsize / 2.
        if not np.all((positions >= low) & (positions <= high)):
            raise OracleError('positions not in box range {} - {}'.format(low, high))

    def to_index(self, positions):
        """Index-space coordinates handed to C (mesh.py:554-555, :598-599, :640-641)."""
        positions = ((positions - self.boxcenter) / self.boxsize + 0.5) * self.nmesh
        return positions.astype(self.dtype, copy=False).ravel(order='C')

    def real_coords(self):
        """RealMesh.coords (mesh.py:522-527)."""
        return tuple(o + d * np.arange(n) for n, o, d in zip(self.nmesh, self.offset, self.boxsize / self.nmesh))

    def k_coords(self):
        """ComplexMesh.coords for a non-Hermitian mesh (mesh.py:812-820)."""
        return tuple(2 * np.pi * np.fft.fftfreq(n, d=d) for n, d in zip(self.nmesh, self.boxsize / self.nmesh))


def broadcast(*arrays):
    """utils.broadcast_arrays (pyrecon/utils.py:125-143)."""
    out = []
    for i, a in enumerate(arrays):
        sl = [None] * len(arrays)
        sl[i] = slice(None)
        out.append(a[tuple(sl)])
    return tuple(out)


def distance(positions):
    """utils.distance (pyrecon/utils.py:146-148)."""
    return np.sqrt((positions ** 2).sum(axis=-1))


def sorted_cell_order(positions, geom, wrap=False):
    """Linear base-cell index of every particle and the stable order that sorts them, from the
    index-space coordinates the reference's paint kernel sees (mesh.py:554-555, mesh.c:35-37).
    This is what the CUDA paint's radix sort must reproduce bit for bit."""
    if wrap:
        positions = geom.wrap(positions)
    p = geom.to_index(positions).reshape(-1, 3)
    n = geom.nmesh.astype(np.int64)
    cell = (p.astype(np.int64) if p.dtype.kind == 'i' else np.trunc(p).astype(np.int64)) % n
    key = (cell[:, 0] * n[1] + cell[:, 1]) * n[2] + cell[:, 2]
    return key, np.argsort(key, kind='stable')


# ----------------------------------------------------------------------------------------------
# The pipeline (pyrecon/recon.py and the three algorithm modules)
# ----------------------------------------------------------------------------------------------

class OracleReconstruction(object):
    """One reconstruction, step by step as the reference runs it.

    algorithm: 'multigrid' (MultiGridReconstruction, pyrecon/multigrid.py:99-167), 'multigrid_original'
    (OriginalMultiGridReconstruction, pyrecon/multigrid.py:13-158, Martin's density contrast),
    'iterative_fft' (pyrecon/iterative_fft.py:12-82), 'plane_parallel_fft'
    (pyrecon/plane_parallel_fft.py:27-55) or 'iterative_fft_particle'
    (IterativeFFTParticleReconstruction, pyrecon/iterative_fft_particle.py:9-244).
    """

    def __init__(self, algorithm, f=0., bias=1., los=None, nmesh=None, boxsize=None, boxcenter=None,
                 dtype='f8', wrap=False, kernels='oracle', fft_engine='numpy', nthreads=1):
        self.algorithm = algorithm
        self.f, self.bias = f, bias
        self.wrap = wrap
        self.geom = Geometry(nmesh, boxsize, boxcenter, dtype=dtype)
        self.dtype = self.geom.dtype
        self.kernels = _Kernels(self.dtype, source=kernels)
        self.kernels.set_num_threads(nthreads)
        self.fft = FFT(fft_engine, workers=nthreads)
        self.set_los(los)
        if algorithm == 'plane_parallel_fft' and self.los is None:
            raise OracleError('A (global) line-of-sight must be provided')
        self.mesh_data = None
        self.mesh_randoms = None
        self._size_randoms = 0

    @property
    def beta(self):
        return self.f / self.bias

    def set_los(self, los):
        """recon.py:149-170."""
        if los is None or (isinstance(los, str) and los == 'local'):
            self.los = None
            return
        if isinstance(los, str):
            los = 'xyz'.index(los)
        if np.ndim(los) == 0:
            ilos = los
            los = np.zeros(3, dtype=self.dtype)
            los[ilos] = 1.
        los = np.array(los, dtype=self.dtype)
        self.los = los / distance(los)

    # -- painting (recon.py:172-192, mesh.py:529-568) --

    def _assign(self, mesh, positions, weights):
        g = self.geom
        size = len(positions)
        if weights is None:
            weights = np.ones(size, dtype=self.dtype)
        if self.wrap:
            positions = g.wrap(positions)
        else:
            g.check_in_box(positions)
        if not (np.isfinite(positions).all() and np.isfinite(weights).all()):
            raise OracleError('Some positions or weights are NaN/inf')
        pos = g.to_index(positions)
        w = np.ascontiguousarray(weights).astype(self.dtype, copy=False).ravel(order='C')
        if mesh is None:
            mesh = np.zeros(g.shape, dtype=self.dtype)
        self.kernels.assign_cic(mesh, g.nmesh, pos, w)
        return mesh

    def assign_data(self, positions, weights=None):
        if self.algorithm == 'iterative_fft_particle':
            # keeps the (wrapped) positions and weights for run (iterative_fft_particle.py:16-33)
            if weights is None:
                weights = np.ones_like(positions, shape=(len(positions),))
            if self.wrap:
                positions = self.geom.wrap(positions)
            if self.mesh_data is None:
                self._positions_data, self._weights_data = positions, weights
            else:
                self._positions_data = np.concatenate([self._positions_data, positions], axis=0)
                self._weights_data = np.concatenate([self._weights_data, weights], axis=0)
        self.mesh_data = self._assign(self.mesh_data, positions, weights)

    def assign_randoms(self, positions, weights=None):
        if self.mesh_randoms is None:
            self._size_randoms = 0
        self.mesh_randoms = self._assign(self.mesh_randoms, positions, weights)
        self._size_randoms += len(positions)

    @property
    def has_randoms(self):
        return self.mesh_randoms is not None

    # -- FFT helpers --

    def _cast(self, value):
        """A mesh operation's result stored back in the mesh dtype (mesh.py:236-244)."""
        return np.asarray(value).astype(self.dtype, copy=False)

    def _ccast(self, value):
        return np.asarray(value).astype(self.geom.ctype, copy=False)

    def _to_complex(self, value):
        return self.fft.forward(value, self.geom.ctype)

    def _to_real(self, valuek):
        return self._cast(self.fft.backward(valuek, self.geom.ctype).real)

    def smooth_gaussian(self, value, radius, method='fft', nsigmas=2.5):
        """RealMesh.smooth_gaussian (mesh.py:655-695): by FFT, or (method='real') by the C convolution."""
        radius_ = np.empty_like(self.geom.boxsize, order='C')
        radius_[:] = radius
        if method != 'fft':
            out = np.array(value, dtype=self.dtype, order='C')
            self.kernels.smooth_gaussian(out, self.geom.nmesh, radius_ / self.geom.boxsize, nsigmas)
            return out
        valuek = self._to_complex(value)
        k2 = sum(-0.5 * (r * k) ** 2 for r, k in zip(radius_, broadcast(*self.geom.k_coords())))
        valuek *= np.exp(k2)
        return self._to_real(valuek)

    # -- density contrast (recon.py:198-249) --

    def set_density_contrast(self, ran_min=None, smoothing_radius=15., **kwargs):
        if self.algorithm == 'multigrid_original':
            self._density_contrast_original(0.75 if ran_min is None else ran_min, smoothing_radius, **kwargs)
            return
        if ran_min is None:
            ran_min = 0.01
        if self.algorithm == 'iterative_fft_particle':
            # the meshes are smoothed by run (iterative_fft_particle.py:35-63)
            self.ran_min, self.smoothing_radius = ran_min, smoothing_radius
            self._delta_from_meshes()
            return
        data = self.smooth_gaussian(self.mesh_data, smoothing_radius, **kwargs)
        if self.has_randoms:
            randoms = self.smooth_gaussian(self.mesh_randoms, smoothing_radius, **kwargs)
            sum_data, sum_randoms = np.sum(data), np.sum(randoms)
            alpha = sum_data * 1. / sum_randoms
            delta = self._cast(data - alpha * randoms)
            threshold = ran_min * sum_randoms / self._size_randoms
            mask = randoms > threshold
            delta[mask] /= (self.bias * alpha * randoms[mask])
            delta[~mask] = 0.
        else:
            delta = self._cast(data / np.mean(data) - 1.)
            delta = self._cast(delta / self.bias)
        self.mesh_delta = delta
        self.mesh_data = self.mesh_randoms = None

    def _density_contrast_original(self, ran_min, smoothing_radius, **kwargs):
        """OriginalMultiGridReconstruction.set_density_contrast, Martin's recipe (multigrid.py:49-97)."""
        data = self.mesh_data.copy()
        if not self.has_randoms:
            delta = self._cast(data / np.mean(data) - 1.)
            delta = self._cast(delta / self.bias)
        else:
            randoms = self.mesh_randoms
            mask = randoms >= ran_min
            data[(randoms > 0) & (randoms < ran_min)] = 0.
            alpha = np.sum(data) / np.sum(randoms[mask])
            data[mask] /= alpha * randoms[mask]
            delta = data
            delta -= 1
            delta[~mask] = 0.
            delta /= self.bias
            mask = delta != 0.
            delta[mask] -= np.mean(delta[mask])
        self.mesh_delta = self.smooth_gaussian(delta, smoothing_radius, **kwargs)
        self.mesh_data = self.mesh_randoms = None

    def _delta_from_meshes(self):
        """OriginalIterativeFFTParticleReconstruction.set_density_contrast body, on the current meshes."""
        data = self.mesh_data
        if self.has_randoms:
            randoms = self.mesh_randoms
            sum_data, sum_randoms = np.sum(data), np.sum(randoms)
            alpha = sum_data * 1. / sum_randoms
            delta = self._cast(data - alpha * randoms)
            threshold = self.ran_min * sum_randoms / self._size_randoms
            mask = randoms > threshold
            delta[mask] /= (self.bias * alpha * randoms[mask])
            delta[~mask] = 0.
        else:
            delta = self._cast(data / np.mean(data) - 1.)
            delta = self._cast(delta / self.bias)
        self.mesh_delta = delta

    def _read_cic_wrap(self, mesh, positions):
        """RealMesh.read_cic(positions, wrap=True) (mesh.py:570-610)."""
        g = self.geom
        dtype = positions.dtype
        values = self.kernels.read_cic(mesh, g.nmesh, g.to_index(g.wrap(positions)))
        return values.astype(dtype, copy=False)

    def _run_iterative_fft_particle(self, niterations=3):
        """OriginalIterativeFFTParticleReconstruction.run/_iterate (iterative_fft_particle.py:65-146)."""
        self._iter = 0
        self.mesh_data = self.smooth_gaussian(self.mesh_data, self.smoothing_radius)
        if self.has_randoms:
            self.mesh_randoms = self.smooth_gaussian(self.mesh_randoms, self.smoothing_radius)
        self._positions_rec_data = self._positions_data.copy()
        for it in range(niterations):
            self.mesh_psi = self._iterate_particle(return_psi=it == niterations - 1)

    def _iterate_particle(self, return_psi=False):
        g = self.geom
        if self._iter > 0:
            wrap = self.wrap
            self.wrap = True                               # painting always wraps here
            self.mesh_data = self._assign(None, self._positions_rec_data, self._weights_data)
            self.wrap = wrap
            self.mesh_data = self.smooth_gaussian(self.mesh_data, self.smoothing_radius)
        self._delta_from_meshes()
        self.mesh_data = None
        delta_k = self._to_complex(self.mesh_delta)
        self.mesh_delta = None
        kc = g.k_coords()
        k = broadcast(*kc)
        self._prod_sum_complex(delta_k, [kk ** 2 for kk in kc], exp=-1)
        delta_k[0, 0, 0] = 0.
        shifts = np.empty_like(self._positions_rec_data)
        psis = []
        for iaxis in range(3):
            if not return_psi and self.los is not None and self.los[iaxis] == 0:
                shifts[:, iaxis] = 0.
                continue
            psi = self._to_real(self._ccast(delta_k * 1j * k[iaxis]))
            shifts[:, iaxis] = self._read_cic_wrap(psi, self._positions_rec_data)
            if return_psi:
                psis.append(psi)
        if self.los is None:
            los = self._positions_data / distance(self._positions_data)[:, None]
        else:
            los = self.los
        if self._iter == 0:
            shifts -= self.beta / (1 + self.beta) * np.sum(shifts * los, axis=-1)[:, None] * los
        self._positions_rec_data = self._positions_data - self.f * np.sum(shifts * los, axis=-1)[:, None] * los
        self._iter += 1
        if return_psi:
            return psis

    def _read_shifts_particle(self, positions, field):
        """OriginalIterativeFFTParticleReconstruction.read_shifts (iterative_fft_particle.py:148-218)."""
        g = self.geom

        def read(pos, wrap):
            shifts = np.empty_like(pos)
            for iaxis, psi in enumerate(self.mesh_psi):
                if wrap:
                    shifts[:, iaxis] = self._read_cic_wrap(psi, pos)
                else:
                    shifts[:, iaxis] = self._read_cic(psi, pos)
            return shifts

        if isinstance(positions, str) and positions == 'data':
            shifts = read(self._positions_rec_data, True)
            if field == 'disp':
                return shifts
            rsd = self._positions_data - self._positions_rec_data
            if field == 'rsd':
                return rsd
            shifts += rsd
            return shifts
        if self.wrap:
            positions = g.wrap(positions)
        shifts = read(positions, False)
        if field == 'disp':
            return shifts
        los = positions / distance(positions)[:, None] if self.los is None else self.los
        rsd = self.f * np.sum(shifts * los, axis=-1)[:, None] * los
        if field == 'rsd':
            return rsd
        real_positions = positions - rsd
        shifts = read(real_positions, True)
        return shifts + rsd

    # -- solvers --

    def run(self, **kwargs):
        return getattr(self, '_run_' + self.algorithm)(**kwargs)

    def _prod_sum_complex(self, valuek, arrays, exp):
        """ComplexMesh.prod_sum (mesh.py:846-883) through the C kernel on the interleaved view."""
        arrays = list(arrays)
        arrays[-1] = np.repeat(arrays[-1], 2)
        coords = np.concatenate([np.asarray(a, dtype=self.dtype) for a in arrays[::-1]], axis=0)
        shape = list(valuek.shape)
        shape[-1] *= 2
        flat = valuek.reshape(-1).view(self.dtype)
        self.kernels.prod_sum(flat, shape, coords, exp)

    def _run_iterative_fft(self, niterations=3):
        """IterativeFFTReconstruction.run/_iterate/_compute_psi (iterative_fft.py:12-82)."""
        delta_real = self.mesh_delta.copy()
        beta = self.beta
        for it in range(niterations):
            delta_k = self._to_complex(delta_real)
            kc = self.geom.k_coords()
            k = broadcast(*kc)
            self._prod_sum_complex(delta_k, [kk ** 2 for kk in kc], exp=-1)
            delta_k[0, 0, 0] = 0.
            delta_real = self.mesh_delta.copy()
            if self.los is not None:
                disp_deriv_k = self._ccast(sum(kk * ll for ll, kk in zip(k, self.los)) ** 2 * delta_k)
                delta_rsd = self._to_real(disp_deriv_k)
                factor = beta
                if it == 0:
                    factor /= (1. + beta)
                delta_real = self._cast(delta_real - self._cast(factor * delta_rsd))
            else:
                x = broadcast(*self.geom.real_coords())
                x2 = sum(x_ ** 2 for x_ in x)
                for i in range(3):
                    for j in range(i, 3):
                        disp_deriv_k = self._ccast(k[i] * k[j] * delta_k)
                        delta_rsd = self._cast(self._cast(x[i] * x[j] * self._to_real(disp_deriv_k)) / x2)
                        factor = (1. + (i != j)) * beta
                        if it == 0:
                            factor /= (1. + beta)
                        delta_real = self._cast(delta_real - self._cast(factor * delta_rsd))
        self.mesh_delta_real = delta_real
        delta_k = self._to_complex(delta_real)
        k = broadcast(*self.geom.k_coords())
        k2 = sum(kk ** 2 for kk in k)
        k2[0, 0, 0] = 1.
        delta_k /= k2
        delta_k[0, 0, 0] = 0.
        self.mesh_psi = [self._to_real(self._ccast(1j * k[i] * delta_k)) for i in range(3)]
        self.mesh_delta = None

    def _run_plane_parallel_fft(self):
        """PlaneParallelFFTReconstruction.run (plane_parallel_fft.py:41-55)."""
        delta_k = self._to_complex(self.mesh_delta)
        self.mesh_delta = None
        k = broadcast(*self.geom.k_coords())
        k2 = sum(kk ** 2 for kk in k)
        k2[0, 0, 0] = 1.
        delta_k /= k2
        mu2 = sum(kk * ll for ll, kk in zip(k, self.los)) ** 2 / k2
        psis = []
        for i in range(3):
            tmp = self._ccast(self._ccast(1j * k[i] * delta_k) / (1. + self.beta * mu2))
            psis.append(self._to_real(tmp))
        self.mesh_psi = psis

    def _run_multigrid(self, jacobi_damping_factor=0.4, jacobi_niterations=5, vcycle_niterations=6):
        """OriginalMultiGridReconstruction.run (multigrid.py:99-135) -> fmg (multigrid.c:303-328)."""
        g = self.geom
        self.mesh_phi = self.kernels.fmg(self.mesh_delta, g.nmesh, g.boxsize, g.boxcenter, self.beta,
                                         jacobi_damping_factor, jacobi_niterations, vcycle_niterations, self.los)
        self.mesh_delta = None

    _run_multigrid_original = _run_multigrid

    # -- shifts (recon.py:255-325, multigrid.py:137-158, mesh.py:570-653) --

    def _read_cic(self, mesh, positions):
        g = self.geom
        dtype = positions.dtype
        g.check_in_box(positions)
        values = self.kernels.read_cic(mesh, g.nmesh, g.to_index(positions))
        return values.astype(dtype, copy=False)

    def read_shifts(self, positions, field='disp+rsd'):
        field = field.lower()
        if field not in ['disp', 'rsd', 'disp+rsd']:
            raise OracleError('Unknown field {}'.format(field))
        if self.algorithm == 'iterative_fft_particle':
            return self._read_shifts_particle(positions, field)
        g = self.geom
        if self.algorithm in ('multigrid', 'multigrid_original'):
            dtype = positions.dtype
            p = g.wrap(positions) if self.wrap else positions
            if not self.wrap:
                g.check_in_box(p)
            shifts = self.kernels.read_finite_difference_cic(self.mesh_phi, g.nmesh, g.boxsize, g.to_index(p))
            shifts = shifts.astype(dtype, copy=False)
            los_pos = positions                       # unwrapped (multigrid.py:149-151)
        else:
            shifts = np.empty_like(positions)
            if self.wrap:
                positions = g.wrap(positions)        # recon.py:288
            for iaxis, psi in enumerate(self.mesh_psi):
                shifts[:, iaxis] = self._read_cic(psi, positions)
            los_pos = positions
        if field == 'disp':
            return shifts
        los = los_pos / distance(los_pos)[:, None] if self.los is None else self.los
        rsd = self.f * np.sum(shifts * los, axis=-1)[:, None] * los
        if field == 'rsd':
            return rsd
        shifts += rsd
        return shifts

    def read_shifted_positions(self, positions, field='disp+rsd'):
        shifts = self.read_shifts(positions, field=field)
        if isinstance(positions, str) and positions == 'data':
            positions = self._positions_data
        positions = positions - shifts
        if self.wrap:
            positions = self.geom.wrap(positions)
        return positions
