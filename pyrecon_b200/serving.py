"""
Serving many reconstructions on one GPU: continuous batching of independent requests.

    server = ReconstructionServer(slots=8, hbm_budget=150e9)
    fut = server.submit(ReconstructionRequest('PlaneParallelFFTReconstruction', data=positions,
                                              nmesh=256, boxsize=1000., boxcenter=500., los='z', wrap=True))
    shifted = fut.result()['shifted_data']
    print(server.stats())          # throughput, p50 / p99 latency, peak concurrency
    server.close()

Requests are admitted in arrival order as soon as a slot (a CUDA stream with its own resident device
scratch) is free and their estimated device memory fits in what the budget has left; each admitted
request runs the plain
pipeline (constructor, assign_data, assign_randoms, set_density_contrast, run,
read_shifted_positions) on its own stream from a worker thread, so the kernels of the requests
in flight overlap on the device while requests keep arriving.  Queued multigrid or plane-parallel
requests of the same mesh and settings are admitted together (up to max_batch) and run as one batched
run: every kernel of the multigrid schedule covers all the solves in one launch, every plane-parallel FFT
pass two meshes at a time.  A request's result does not depend on what else is running: every kernel is
deterministic, requests share no device buffers and a batched run gives each problem the bits of its own
run.
"""
import threading
import time
import collections
import concurrent.futures

import numpy as np

from . import _lib
from .mesh import _device_of


class ReconstructionRequest(object):
    """One reconstruction: the algorithm class name, its constructor keywords (f, bias, los, nmesh,
    boxsize, boxcenter, wrap, dtype, ...), the catalogues (numpy arrays or torch tensors), the
    keywords of set_density_contrast and of run."""

    def __init__(self, algorithm, data, data_weights=None, randoms=None, randoms_weights=None,
                 density_kwargs=None, run_kwargs=None, keep_output=True, **kwargs):
        self.algorithm = algorithm
        # keep_output=False: the shifted positions are computed and then dropped (the future's result
        # holds their shapes only), so a long stream of requests on device catalogues does not pile up
        # outputs in device memory
        self.keep_output = bool(keep_output)
        self.data, self.data_weights = data, data_weights
        self.randoms, self.randoms_weights = randoms, randoms_weights
        self.density_kwargs = dict(density_kwargs or {})
        self.run_kwargs = dict(run_kwargs or {})
        self.kwargs = dict(kwargs)
        self.submitted = None


def _size(x):
    return 0 if x is None else int(len(x))


def estimate_device_bytes(request):
    """Device memory a request holds at its peak (meshes, workspaces, catalogues, outputs), from the
    library's own workspace queries; used for admission."""
    import pyrecon_b200
    from .multigrid import OriginalMultiGridReconstruction
    from .mesh import MeshInfo
    lib = _lib.load()
    cls = getattr(pyrecon_b200, request.algorithm)
    kw = dict(request.kwargs)
    geometry = ('nmesh', 'boxsize', 'boxcenter', 'cellsize', 'positions', 'boxpad', 'dtype')
    info = MeshInfo(select_nmesh=cls._select_nmesh, **{k: kw[k] for k in geometry if k in kw})
    n = int(np.prod(info.nmesh))
    item = info.dtype.itemsize
    nm = _lib.i3(info.nmesh)
    npart = _size(request.data) + _size(request.randoms)
    nmeshes = 2 if request.randoms is not None else 1
    total = 8 * n * nmeshes + 8 * int(info.nmesh[0] * info.nmesh[1]) * nmeshes           # FP64 paint meshes
    total += lib.prc_assign_cic_workspace_bytes(nm, max(_size(request.data), _size(request.randoms)), item)
    total += lib.prc_density_contrast_workspace_bytes(nm, item, int(request.randoms is not None))
    total += n * item                                                                     # delta
    if issubclass(cls, OriginalMultiGridReconstruction):
        total += lib.prc_multigrid_workspace_bytes(nm, item, 1) + n * item                # hierarchy, phi
        if item == 4:
            total += 8 * n                                                                # FP64 phi (mixed)
    elif request.algorithm == 'IterativeFFTReconstruction':
        total += lib.prc_iterative_fft_workspace_bytes(nm, item, int(kw.get('los') is None)) + 4 * n * item
    else:
        total += lib.prc_plane_parallel_workspace_bytes(nm, item) + 4 * n * item
    total += npart * 3 * 8 * 3                                                            # positions, outputs
    return int(total)


def prepare_request(request, device=None, stream=None, workspace=None):
    """Constructor, paints and density contrast of one request on `stream`; returns the reconstruction."""
    import pyrecon_b200
    cls = getattr(pyrecon_b200, request.algorithm)
    rec = cls(device=device, stream=stream, workspace=workspace, **request.kwargs)
    rec.assign_data(request.data, request.data_weights)
    if request.randoms is not None:
        rec.assign_randoms(request.randoms, request.randoms_weights)
    rec.set_density_contrast(**request.density_kwargs)
    return rec


def finish_request(request, rec):
    """The shifted positions of a request whose reconstruction has run (their shapes only when the
    request does not keep its output)."""
    out = {'shifted_data': rec.read_shifted_positions(request.data)}
    if request.randoms is not None:
        out['shifted_randoms'] = rec.read_shifted_positions(request.randoms)
    if not request.keep_output:
        out = {k: tuple(v.shape) for k, v in out.items()}
    return out


def run_request(request, device=None, stream=None, workspace=None):
    """The plain pipeline for one request on `stream`; returns {'shifted_data', 'shifted_randoms'}.
    `workspace`: scratch kept across requests (a slot's), so its address, and with it the multigrid
    solve's captured CUDA graph, is reused."""
    rec = prepare_request(request, device=device, stream=stream, workspace=workspace)
    rec.run(**request.run_kwargs)
    return finish_request(request, rec)


def batch_key(request):
    """Requests with the same key can share one batched run: a multigrid solve or the plane-parallel FFT
    passes (same algorithm, mesh, line of sight, cosmology, precision and solver settings; the catalogues
    may differ); None: not batchable."""
    import pyrecon_b200
    from .multigrid import OriginalMultiGridReconstruction
    from .plane_parallel_fft import PlaneParallelFFTReconstruction
    cls = getattr(pyrecon_b200, request.algorithm)
    kw = request.kwargs
    if not issubclass(cls, (OriginalMultiGridReconstruction, PlaneParallelFFTReconstruction)) or 'positions' in kw:
        return None
    if not all(k in kw for k in ('nmesh', 'boxsize', 'boxcenter')) and not ('cellsize' in kw and 'boxsize' in kw):
        return None
    norm = lambda d: repr(sorted((k, np.asarray(v).tolist() if isinstance(v, (list, tuple, np.ndarray)) else v)
                                 for k, v in d.items()))
    return (request.algorithm, norm(kw), norm(request.density_kwargs), norm(request.run_kwargs))


def run_batch_requests(requests, device=None, stream=None, workspace=None):
    """Several batchable requests (same batch_key) on one stream: each is prepared, their runs go as one
    batched run (multigrid solve or plane-parallel FFT passes), then each is read out; returns their outputs
    in order."""
    from . import multigrid, plane_parallel_fft
    recs = [prepare_request(r, device=device, stream=stream, workspace=workspace) for r in requests]
    if isinstance(recs[0], plane_parallel_fft.PlaneParallelFFTReconstruction):
        plane_parallel_fft.run_batch(recs)
    else:
        multigrid.run_batch(recs, **requests[0].run_kwargs)
    return [finish_request(r, rec) for r, rec in zip(requests, recs)]


class ReconstructionServer(object):
    """Continuous-batching request loop on one GPU (see the module docstring).

    slots: jobs in flight at most (one CUDA stream each).  hbm_budget: bytes of device memory the
    requests in flight may hold together (default: 90% of the free memory at start).  max_batch:
    queued multigrid requests with the same mesh and settings (batch_key) are taken together as one
    job of up to this many, whose solves run as one batched solve (a power of two, so the slot's
    captured solves are reused); 1 disables.  batch_algorithms: the algorithm classes whose requests are
    batched (default: the multigrid and plane-parallel ones).
    """

    def __init__(self, device=None, slots=8, hbm_budget=None, max_batch=8, batch_algorithms=None):
        import torch
        self.device = _device_of(device)
        _lib.load()
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = 0.9 * free
        self.hbm_budget = float(hbm_budget)
        self.max_batch = max(1, int(max_batch))
        self.batch_algorithms = None if batch_algorithms is None else set(batch_algorithms)
        from .mesh import _Workspace
        self._streams = [torch.cuda.Stream(self.device) for _ in range(slots)]
        # device scratch resident per slot: reused by every request the slot runs
        self._workspaces = [_Workspace(self.device) for _ in range(slots)]
        self._free_streams = list(range(slots))
        # device memory each slot's stream keeps: torch's caching allocator pools freed blocks per stream,
        # so a slot holds (at least) the largest job it has run; admission counts these, not only the
        # jobs in flight
        self._resident = [0.] * slots
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=slots)
        self._cv = threading.Condition()
        self._queue = collections.deque()
        self._in_use = 0.
        self._active = 0
        self.peak_active = 0
        self.latencies = []
        self._first_submit = None
        self._last_done = None
        self._closed = False
        self._dispatcher = threading.Thread(target=self._loop, name='pyrecon-b200-dispatch', daemon=True)
        self._dispatcher.start()

    def submit(self, request):
        """Queue a request; returns a concurrent.futures.Future of run_request's result."""
        need = estimate_device_bytes(request)
        if need > self.hbm_budget:
            raise ValueError('request needs ~{:.1f} GB, above the HBM budget of {:.1f} GB'.format(need / 1e9,
                                                                                                self.hbm_budget / 1e9))
        fut = concurrent.futures.Future()
        with self._cv:
            if self._closed:
                raise RuntimeError('server is closed')
            request.submitted = time.perf_counter()
            if self._first_submit is None:
                self._first_submit = request.submitted
            batched = self.max_batch > 1 and (self.batch_algorithms is None or request.algorithm in self.batch_algorithms)
            self._queue.append((request, need, fut, batch_key(request) if batched else None))
            self._cv.notify_all()
        return fut

    def _pick_slot(self, need):
        """A free slot whose stream can take a job of `need` bytes within the budget (preferring one that
        already holds that much), and the budget left for the job beyond `need`; (None, 0) if none fits."""
        total = sum(self._resident)
        best = None
        for s in self._free_streams:
            grown = max(self._resident[s], need)
            left = self.hbm_budget - (total - self._resident[s] + grown)
            if left < 0:
                continue
            # fewest bytes added to the resident total, then the smallest resident slot
            score = (grown - self._resident[s], self._resident[s])
            if best is None or score < best[0]:
                best = (score, s, left + (grown - need))
        return (None, 0.) if best is None else (best[1], best[2])

    def _loop(self):
        while True:
            with self._cv:
                while True:
                    if self._queue and self._free_streams:
                        slot, room = self._pick_slot(self._queue[0][1])
                        if slot is not None:
                            break
                    if self._closed and not self._queue:
                        return
                    self._cv.wait()
                job = [self._queue.popleft()]
                key = job[0][3]
                if key is not None:
                    # queued requests of the same batch key join, while the slot's budget allows
                    for item in list(self._queue):
                        if len(job) >= self.max_batch:
                            break
                        if item[3] == key and item[1] <= room:
                            job.append(item)
                            room -= item[1]
                    n = 1
                    while 2 * n <= len(job):
                        n *= 2
                    job = job[:n]
                    for item in job[1:]:
                        self._queue.remove(item)
                self._free_streams.remove(slot)
                need = sum(item[1] for item in job)
                self._resident[slot] = max(self._resident[slot], need)
                self._in_use += need
                self._active += len(job)
                self.peak_active = max(self.peak_active, self._active)
            self._pool.submit(self._work, job, need, slot)

    def _work(self, job, need, slot):
        import torch
        stream = self._streams[slot]
        requests = [item[0] for item in job]
        try:
            with torch.cuda.device(self.device):
                if len(requests) == 1:
                    outs = [run_request(requests[0], device=self.device, stream=stream,
                                        workspace=self._workspaces[slot])]
                else:
                    outs = run_batch_requests(requests, device=self.device, stream=stream,
                                              workspace=self._workspaces[slot])
                stream.synchronize()
        except BaseException as exc:
            for item in job:
                item[2].set_exception(exc)
        else:
            done = time.perf_counter()
            with self._cv:
                for r in requests:
                    self.latencies.append(done - r.submitted)
                self._last_done = done
            for item, out in zip(job, outs):
                item[2].set_result(out)
        finally:
            with self._cv:
                self._in_use -= need
                self._active -= len(job)
                self._free_streams.append(slot)
                self._cv.notify_all()

    def reset_stats(self):
        """Forget the latencies and the throughput window so far (e.g. after a warm-up)."""
        with self._cv:
            self.latencies = []
            self._first_submit = None
            self._last_done = None
            self.peak_active = self._active

    def stats(self):
        """Throughput (completed requests / s from the first submission to the last completion) and
        latency percentiles (submission to result, ms)."""
        with self._cv:
            lat = sorted(self.latencies)
            span = (self._last_done - self._first_submit) if lat else 0.
        pct = lambda q: 1e3 * lat[min(len(lat) - 1, int(round(q / 100. * (len(lat) - 1))))] if lat else None
        return dict(completed=len(lat), recons_per_s=len(lat) / span if span > 0 else None, p50_ms=pct(50),
                    p99_ms=pct(99), peak_active=self.peak_active)

    def close(self, wait=True):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            self._dispatcher.join()
            self._pool.shutdown(wait=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
