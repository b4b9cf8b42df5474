"""
Reconstructions per second of the pyrecon hot path on B200.

    python bench.py [--gpus N --steps K --warmup W] [--workload iterative_fft_512] [--impl ours|reference]

One step = one complete reconstruction of the workload (constructor, assign_data, assign_randoms,
set_density_contrast, run, read_shifted_positions of data and of randoms), as the reference's
own timing of a reconstruction goes from the constructor to both read_shifted_positions calls.

* value: steps/s with the catalogues resident in HBM (device-side CUDA-event timing, max over
  ranks, N ranks run independent replicas: "replicas only", weak scaling).
* e2e: the same reconstruction through the public API from pinned HOST tensors: every step copies
  the catalogues host->device and the shifted positions device->host.
* roofline: the kernel with the largest device time in the timed region, its compulsory bytes
  (reported by the library per launch) / its event-timed duration, against MEASURED_PEAKS.json.
* shift_err_mpc: max |shifted positions - those of the all-FP64 mode (dtype f8) of the same
  reconstruction| over data and randoms, checked outside the timed region (the FP64 mode is pinned
  to the FP64 oracle by the parity tests at nmesh 128-512).
* baseline_metric: the metric's comparison with the plain GPU path: 64 batched periodic mocks and
  500 Poisson-arriving requests through the request loop against the same requests run one at a time
  (skipped with --no-multi or when N > 1).
* --impl reference: the reference package itself (pip-installed unmodified into baseline/_ref, its C
  kernels built from source with OpenMP on all host cores) running the full workload through its own
  classes, fft_engine 'fftw' when pyfftw imports, else 'numpy'; 1 warm-up + 2 timed reconstructions
  at most (each a few minutes on the CPU).
* cpu_baseline (GPU arm): the reference's C kernels (oracle/_ref, OpenMP on all host cores) driven by
  the oracle's restatement of its numpy glue with pocketfft on all cores, on a 1/8-scale sample of the
  workload (nmesh/2 per axis, 1/8 of the particles), scaled x8.
"""
import os
import sys
import json
import time
import argparse
import subprocess
import statistics

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'recons/s + p50/p99 latency vs plain GPU path, nmesh 512, shift err<1e-3 Mpc/h'

WORKLOADS = {
    # the metric's workload: IterativeFFTReconstruction nmesh=512, boxsize=2000, niterations=3, f=0.8, bias=2, local los,
    # smoothing_radius=15, 5M lognormal data, 20M uniform randoms, float32 positions
    'iterative_fft_512': dict(algorithm='IterativeFFTReconstruction', nmesh=512, boxsize=2000., boxcenter=2000.,
                              los=None, ndata=5_000_000, nrandoms=20_000_000, pos_dtype='f4', dtype='f4',
                              weights=None, run_kwargs=dict(niterations=3)),
    # multigrid workload: MultiGridReconstruction nmesh=256, boxsize=2000, local los, 2M data, 10M randoms,
    # weights uniform in [0.5, 1.5]; FP32 stencils with FP64 residual refinement
    'multigrid_256': dict(algorithm='MultiGridReconstruction', nmesh=256, boxsize=2000., boxcenter=2000., los=None,
                          ndata=2_000_000, nrandoms=10_000_000, pos_dtype='f8', dtype='f4', weights=(0.5, 1.5),
                          run_kwargs={}),
    # small case of the same pipeline for ncu captures (spectra of 134 MB, above L2)
    'iterative_fft_256': dict(algorithm='IterativeFFTReconstruction', nmesh=256, boxsize=2000., boxcenter=2000.,
                              los=None, ndata=1_000_000, nrandoms=4_000_000, pos_dtype='f4', dtype='f4',
                              weights=None, run_kwargs=dict(niterations=3)),
    'multigrid_512': dict(algorithm='MultiGridReconstruction', nmesh=512, boxsize=2000., boxcenter=2000., los=None,
                          ndata=5_000_000, nrandoms=20_000_000, pos_dtype='f4', dtype='f4', weights=None, run_kwargs={}),
    'plane_parallel_512': dict(algorithm='PlaneParallelFFTReconstruction', nmesh=512, boxsize=2000., boxcenter=2000.,
                               los='z', ndata=5_000_000, nrandoms=20_000_000, pos_dtype='f4', dtype='f4', weights=None,
                               run_kwargs={}),
    'iterative_fft_particle_512': dict(algorithm='IterativeFFTParticleReconstruction', nmesh=512, boxsize=2000.,
                                       boxcenter=2000., los=None, ndata=5_000_000, nrandoms=20_000_000, pos_dtype='f4',
                                       dtype='f4', weights=None, run_kwargs=dict(niterations=3)),
    # OriginalMultiGridReconstruction (Martin's density contrast) with the real-space (truncated convolution)
    # smoothing, on the multigrid_256 catalogues; the reference sample runs at full size (the convolution's
    # cost grows with the cube of the mesh size at a fixed radius, so a smaller mesh would not scale)
    'original_multigrid_real_256': dict(algorithm='OriginalMultiGridReconstruction', nmesh=256, boxsize=2000.,
                                        boxcenter=2000., los=None, ndata=2_000_000, nrandoms=10_000_000,
                                        pos_dtype='f8', dtype='f4', weights=(0.5, 1.5), run_kwargs={},
                                        density_kwargs=dict(method='real'), reference_scale=1),
}
DEFAULT_WORKLOAD = 'iterative_fft_512'

# Many requests at once through the request loop (pyrecon_b200.serving), against the same requests run one
# after the other on one stream (the plain path).  A step is the whole set of requests.
MULTI_WORKLOADS = {
    # batched mocks: 64 periodic-box mocks, plane-parallel and multigrid mixed, los='z', nmesh in
    # {128, 192, 256}, boxsize 1000, 0.3M-2M lognormal data each, no randoms
    'batched_mocks': dict(kind='batched', nrequests=64, algorithms=['PlaneParallelFFTReconstruction',
                                                                    'MultiGridReconstruction'],
                          nmesh=[128, 192, 256], ndata=(300_000, 2_000_000), randoms_factor=0, boxsize=1000.,
                          boxcenter=500., los='z', wrap=True, dtype='f4', slots=2, max_batch=8, passes=5),
    # serving: 500 requests with Poisson arrivals at 20 req/s, the three algorithms, nmesh in
    # {128, 256, 384, 512}, 0.5M-8M data with 4x randoms, 150 GB admission budget.  Two slots: measured
    # p50 / p99 19.5-19.9 / 162-171 ms with 2, 21.3 / 174 with 1, 20.1 / 201 with 4 (the device is ~43 %
    # busy at this rate; more concurrent requests stretch the long ones)
    'serving': dict(kind='serving', nrequests=500, rate=20., algorithms=['MultiGridReconstruction',
                                                                        'IterativeFFTReconstruction',
                                                                        'PlaneParallelFFTReconstruction'],
                    nmesh=[128, 256, 384, 512], ndata=(500_000, 8_000_000), randoms_factor=4, boxsize=2000.,
                    boxcenter=2000., los=None, wrap=False, dtype='f4', slots=2, max_batch=8, hbm_budget=150e9),
}

for _name, _w in MULTI_WORKLOADS.items():
    _w['name'] = _name


def workload_name(w):
    name = '{algorithm} nmesh={nmesh} boxsize={boxsize:g} boxcenter={boxcenter:g} los={los} f=0.8 bias=2.0 ' \
           'smoothing_radius=15 data={ndata} lognormal randoms={nrandoms} uniform positions={pos_dtype}'.format(**w)
    if w.get('density_kwargs'):
        name += ' ' + ' '.join('{}={}'.format(k, v) for k, v in sorted(w['density_kwargs'].items()))
    return name


def dist_env():
    return int(os.environ.get('RANK', 0)), int(os.environ.get('LOCAL_RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))


# ---------------------------------------------------------------------------------------------
# CPU reference arm
# ---------------------------------------------------------------------------------------------

def reference_sample(w, seed=0):
    """Time the reference's CPU path on a 1/8-scale sample of workload `w`; returns (seconds, info)."""
    import numpy as np
    from oracle import pipeline
    from pyrecon_b200 import mocks
    cores = os.cpu_count() or 1
    kernels = 'reference' if pipeline.reference_kernels_available() else 'oracle'
    scale = w.get('reference_scale', 8)
    n = w['nmesh'] // (2 if scale == 8 else 1)
    nd, nr = w['ndata'] // scale, w['nrandoms'] // scale
    algo = {'IterativeFFTReconstruction': 'iterative_fft', 'MultiGridReconstruction': 'multigrid',
            'PlaneParallelFFTReconstruction': 'plane_parallel_fft',
            'IterativeFFTParticleReconstruction': 'iterative_fft_particle',
            'OriginalMultiGridReconstruction': 'multigrid_original'}[w['algorithm']]
    data = mocks.lognormal_positions_numpy(nd, n, w['boxsize'], w['boxcenter'], seed=2002 + seed,
                                           field_seed=1002 + seed, dtype=w['pos_dtype'])
    randoms = mocks.uniform_positions_numpy(nr, w['boxsize'], w['boxcenter'], seed=3002 + seed, dtype=w['pos_dtype'])
    wd = wr = None
    if w['weights'] is not None:
        wd = mocks.weights_numpy(nd, *w['weights'], seed=4002 + seed)
        wr = mocks.weights_numpy(nr, *w['weights'], seed=4003 + seed)
    t0 = time.perf_counter()
    rec = pipeline.OracleReconstruction(algo, f=0.8, bias=2., los=w['los'], nmesh=n, boxsize=w['boxsize'],
                                        boxcenter=w['boxcenter'], dtype=w['dtype'], kernels=kernels,
                                        fft_engine='scipy', nthreads=cores)
    rec.assign_data(data, wd)
    rec.assign_randoms(randoms, wr)
    rec.set_density_contrast(smoothing_radius=15., **w.get('density_kwargs', {}))
    rec.run(**w['run_kwargs'])
    rec.read_shifted_positions(data)
    rec.read_shifted_positions(randoms)
    dt = time.perf_counter() - t0
    what = '1/8 sample: nmesh {} and {} + {} particles, time x8'.format(n, nd, nr) if scale == 8 else \
        'full-size run: nmesh {} and {} + {} particles'.format(n, nd, nr)
    info = dict(cores=cores, kind='reference' if kernels == 'reference' else 'port', scale=scale,
                sample='reference CPU path ({} C kernels with OpenMP x{}, numpy glue, scipy pocketfft x{}) on a {}'.format(
                    'reference' if kernels == 'reference' else 'restated', cores, cores, what))
    return dt, info


REFERENCE_PACKAGE = os.path.join(ROOT, 'baseline', '_ref')


def import_reference_package():
    """(pyrecon, None) from the unmodified reference installed in baseline/_ref, or (None, why)."""
    if not os.path.isfile(os.path.join(REFERENCE_PACKAGE, 'pyrecon', '__init__.py')):
        return None, 'baseline/_ref holds no install of the reference (pip install --target baseline/_ref)'
    if REFERENCE_PACKAGE not in sys.path:
        sys.path.insert(0, REFERENCE_PACKAGE)
    try:
        import pyrecon
    except Exception as exc:       # the reference's own import failing (missing C libraries, ...)
        return None, 'the reference in baseline/_ref does not import: {}'.format(exc)
    if not os.path.abspath(pyrecon.__file__).startswith(REFERENCE_PACKAGE):
        return None, 'pyrecon imported from {}, not baseline/_ref'.format(pyrecon.__file__)
    return pyrecon, None


def reference_catalogs(w):
    """The GPU arm's catalogues of rank 0 (same generators and seeds, drawn on the GPU when there is one),
    as numpy arrays."""
    import torch
    if torch.cuda.is_available():
        cats = make_catalogs(w, torch.device('cuda', 0), 0)
        out = [None if t is None else t.cpu().numpy() for t in cats]
        del cats
        torch.cuda.empty_cache()
        return out, 'the GPU arm\'s catalogues (rank 0 seeds)'
    from pyrecon_b200 import mocks
    data = mocks.lognormal_positions_numpy(w['ndata'], w['nmesh'], w['boxsize'], w['boxcenter'], seed=2003,
                                           field_seed=1003, dtype=w['pos_dtype'])
    randoms = mocks.uniform_positions_numpy(w['nrandoms'], w['boxsize'], w['boxcenter'], seed=3003,
                                            dtype=w['pos_dtype'])
    wd = wr = None
    if w['weights'] is not None:
        wd = mocks.weights_numpy(w['ndata'], *w['weights'], seed=4003, dtype=w['pos_dtype'])
        wr = mocks.weights_numpy(w['nrandoms'], *w['weights'], seed=4004, dtype=w['pos_dtype'])
    return [data, wd, randoms, wr], 'numpy draws of the same distributions (no GPU)'


def run_reference_arm(args, w):
    """The reference's own classes on the full workload, timed from the constructor to both
    read_shifted_positions calls (catalogue generation excluded), on all host cores."""
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    pyrecon, why = import_reference_package()
    if pyrecon is None:
        print(json.dumps({'impl': 'reference', 'unavailable': why}), flush=True)
        return 0
    cores = os.cpu_count() or 1
    try:
        import pyfftw  # noqa: F401
        engine = 'fftw'
    except ImportError:
        engine = 'numpy'
    (data, wd, randoms, wr), source = reference_catalogs(w)
    Cls = getattr(pyrecon, w['algorithm'])

    def one():
        t0 = time.perf_counter()
        rec = Cls(f=0.8, bias=2., los=w['los'], nmesh=w['nmesh'], boxsize=w['boxsize'], boxcenter=w['boxcenter'],
                  dtype=w['dtype'], fft_engine=engine, nthreads=cores)
        rec.assign_data(data, wd)
        rec.assign_randoms(randoms, wr)
        rec.set_density_contrast(smoothing_radius=15., **w.get('density_kwargs', {}))
        rec.run(**w['run_kwargs'])
        rec.read_shifted_positions(data)
        rec.read_shifted_positions(randoms)
        return time.perf_counter() - t0

    budget = float(os.environ.get('PRC_REFERENCE_BUDGET_S', 1500.))
    nwarm, nsteps = min(args.warmup, 1), max(1, min(args.steps, 2))
    t_start = time.perf_counter()
    warm = [one() for _ in range(nwarm)]
    times = []
    for _ in range(nsteps):
        last = (times or warm or [0.])[-1]
        if times and time.perf_counter() - t_start + last > budget:
            break
        times.append(one())
    sec = statistics.median(times)
    value = 1. / sec
    sample = ('the reference package {} (baseline/_ref, unmodified) through its {} on the full workload, '
              'fft_engine={!r}{}, nthreads={} (OpenMP C kernels), {}; {} warm-up + {} timed reconstructions, '
              'median').format(pyrecon.__version__, w['algorithm'], engine,
                               '' if engine == 'fftw' else ' (pyfftw absent: single-threaded numpy FFTs)', cores,
                               source, len(warm), len(times))
    line = dict(metric=METRIC, value=value, unit='recons/s', n_gpus=args.gpus, steps=len(times), warmup=len(warm),
                steps_requested=args.steps, warmup_requested=args.warmup, ms_per_step=sec * 1e3,
                step_seconds=[round(t, 2) for t in times], warmup_seconds=[round(t, 2) for t in warm],
                higher_is_better=True, scaling='weak', vs_baseline=None, dtype=w['dtype'],
                data='synthetic seeded lognormal data + uniform randoms', config=dict(workload=workload_name(w)),
                impl='reference', same_config=True,
                cpu_baseline=dict(value=value, unit='recons/s', cores=cores, kind='reference', sample=sample),
                e2e=dict(value=value, unit='recons/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------

class ClockSampler(object):
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile
        try:
            fd, self.path = tempfile.mkstemp(prefix='prc_clocks_rank{}_'.format(self.index), suffix='.csv')
            self.fh = os.fdopen(fd, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '200'], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or self.path is None or not os.path.isfile(self.path):
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=['nvidia-smi unavailable'])
        sms, maxs, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        with open(self.path) as fh:
            lines = fh.readlines()
        os.remove(self.path)
        self.path = None
        for line in lines:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxs.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == 'active':
                    reasons.add(name)
        if not sms:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=['no samples'])
        return dict(sm_mhz=statistics.median(sms), sm_max_mhz=max(maxs), reasons=sorted(reasons), samples=len(sms))


def make_catalogs(w, device, rank):
    import torch
    from pyrecon_b200 import mocks
    g = dict(device=device)
    data = mocks.lognormal_positions_torch(w['ndata'], w['nmesh'], w['boxsize'], w['boxcenter'], seed=2003 + rank,
                                           field_seed=1003 + rank, dtype=w['pos_dtype'], **g)
    randoms = mocks.uniform_positions_torch(w['nrandoms'], w['boxsize'], w['boxcenter'], seed=3003 + rank,
                                            dtype=w['pos_dtype'], **g)
    wd = wr = None
    if w['weights'] is not None:
        wd = mocks.weights_torch(w['ndata'], *w['weights'], seed=4003 + rank, dtype=w['pos_dtype'], **g)
        wr = mocks.weights_torch(w['nrandoms'], *w['weights'], seed=4004 + rank, dtype=w['pos_dtype'], **g)
    torch.cuda.synchronize(device)
    return data, wd, randoms, wr


def reconstruct(w, device, data, wd, randoms, wr, check):
    import pyrecon_b200
    Cls = getattr(pyrecon_b200, w['algorithm'])
    rec = Cls(f=0.8, bias=2., los=w['los'], nmesh=w['nmesh'], boxsize=w['boxsize'], boxcenter=w['boxcenter'],
              dtype=w['dtype'], device=device)
    rec.assign_data(data, wd, check=check)
    rec.assign_randoms(randoms, wr, check=check)
    rec.set_density_contrast(smoothing_radius=15., **w.get('density_kwargs', {}))
    rec.run(**w['run_kwargs'])
    out_d = rec.read_shifted_positions(data)
    out_r = rec.read_shifted_positions(randoms)
    return out_d, out_r


# ncu DRAM-traffic summaries (profiles/): per kernel, DRAM bytes per launch over the algorithmic bytes of the
# same launches; the nmesh-512 capture of the FFT passes first, the nmesh-256 capture of the whole pipeline
# (particle kernels included) for the rest
TRAFFIC_PROFILES = [os.path.join(ROOT, 'profiles', 'traffic_iterative_fft_512.md'),
                    os.path.join(ROOT, 'profiles', 'traffic_iterative_fft_256.md')]


def traffic_ratio(kernel):
    """(ratio, profile file name) of the first summary with a row for `kernel`, or (None, None)."""
    for path in TRAFFIC_PROFILES:
        try:
            with open(path) as fh:
                for line in fh:
                    cells = [c.strip() for c in line.strip().strip('|').split('|')]
                    if len(cells) >= 5 and cells[0] == kernel:
                        return float(cells[4]), os.path.basename(path)
        except (OSError, ValueError):
            continue
    return None, None


def load_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.isfile(path):
        with open(path) as fh:
            p = json.load(fh)
        return float(p['hbm_gbs']), 'measured'
    return 6650., 'fallback'


def timed_loop(fn, steps, device):
    """Per-step CUDA events on the current stream; returns (total ms, per-step ms list)."""
    import torch
    st = torch.cuda.current_stream(device)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(st)
    for i in range(steps):
        fn()
        evs[i + 1].record(st)
    torch.cuda.synchronize(device)
    per = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
    return evs[0].elapsed_time(evs[-1]), per


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q / 100.
    f, c = int(k), min(int(k) + 1, len(xs) - 1)
    return xs[f] + (xs[c] - xs[f]) * (k - f)


def reduce_max(x, world, device):
    """Max of a per-rank number over the ranks of the default process group (the timing of an N-replica run is
    the slowest rank's); the tensor lives on `device` (the GPU for NCCL, the CPU for gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_gpu_arm(args, w):
    import torch
    import torch.distributed as dist
    from pyrecon_b200 import _lib
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device('cuda', local_rank)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300), device_id=device)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(x, world, device)

    data, wd, randoms, wr = make_catalogs(w, device, rank)
    step = lambda: reconstruct(w, device, data, wd, randoms, wr, check=False)
    # correctness of the measured configuration: a checked run first (raises on bad inputs), whose shifted
    # positions are compared with the all-FP64 mode after the timed region
    checked = reconstruct(w, device, data, wd, randoms, wr, check=True)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(device)

    # --- device-resident timed region ---
    barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(local_rank) as clocks:
        time.sleep(1.0)                     # let nvidia-smi start sampling before the timed region
        barrier()
        torch.cuda.synchronize(device)
        launches0 = _lib.launch_count()
        _lib.profile_enable(True)
        total_ms, per_step = timed_loop(step, args.steps, device)
    prof = _lib.profile_collect()
    _lib.profile_enable(False)
    launches = _lib.launch_count() - launches0
    barrier()
    total_ms = max_over_ranks(total_ms)
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms / 1e3)

    # --- accuracy of the measured configuration: the all-FP64 mode on the same catalogues ---
    shift_err = None
    if w['dtype'] == 'f4' and not args.no_check:
        d8 = lambda t: None if t is None else t.double()
        ref = reconstruct(dict(w, dtype='f8'), device, d8(data), d8(wd), d8(randoms), d8(wr), check=False)
        errs = [float((a.double() - b).abs().max()) for a, b in zip(checked, ref)]
        shift_err = dict(max_abs=max(errs), data=errs[0], randoms=errs[1], unit='Mpc/h', tolerance=1e-3,
                         vs='the all-FP64 mode (dtype f8) of the same reconstruction on the same catalogues; the '
                            'FP64 mode is pinned to the FP64 oracle by the parity tests at nmesh 128-512')
        del ref
    del checked

    # --- end to end through the public API from pinned host memory ---
    e2e = None
    if not args.no_e2e:
        pin = lambda t: None if t is None else t.cpu().pin_memory()
        hd, hwd, hr, hwr = pin(data), pin(wd), pin(randoms), pin(wr)
        # positions cross twice: to the device for the paint, and again (in chunks, overlapped with the
        # kernel and the copy back) for the read-out of the host catalogues
        h2d = sum(t.numel() * t.element_size() for t in [hd, hwd, hr, hwr] if t is not None)
        h2d += (hd.numel() + hr.numel()) * hd.element_size()
        d2h = (hd.numel() + hr.numel()) * hd.element_size()
        e2e_step = lambda: reconstruct(w, device, hd, hwd, hr, hwr, check=False)
        e2e_step()
        barrier()
        e_ms, _ = timed_loop(e2e_step, max(1, args.steps), device)
        barrier()
        e_ms = max_over_ranks(e_ms)
        e2e = dict(value=world * max(1, args.steps) / (e_ms / 1e3), unit='recons/s', h2d_bytes_per_step=int(h2d),
                   d2h_bytes_per_step=int(d2h), ms_per_step=e_ms / max(1, args.steps))

    # --- roofline of the dominant kernel ---
    peak, peak_kind = load_peaks()
    name, (nl, kms, kbytes) = max(prof.items(), key=lambda kv: kv[1][1])
    achieved = (kbytes / 1e9) / (kms / 1e3) if kms > 0 else 0.
    kernels = {k: dict(launches=v[0], ms=round(v[1], 3), share=round(v[1] / max(sum(x[1] for x in prof.values()), 1e-9), 4),
                       gbs=round((v[2] / 1e9) / (v[1] / 1e3), 1) if v[1] > 0 else None) for k, v in prof.items()}
    ratio, tsrc = traffic_ratio(name) if w['algorithm'] == 'IterativeFFTReconstruction' else (None, None)
    traffic = None if ratio is None else ratio * kbytes / nl
    roofline = dict(bound='hbm', kernel=name, achieved=round(achieved, 1), peak=peak, unit='GB/s',
                    frac=round(achieved / peak, 4), traffic=traffic,
                    traffic_source=None if ratio is None else
                    'ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this kernel '
                    '(profiles/{}), ratio {:.3f} to its algorithmic bytes, applied to this launch'.format(tsrc, ratio),
                    bytes_per_launch=kbytes / nl, launch_ms=kms / nl, peak_source=peak_kind + ' (MEASURED_PEAKS.json hbm_gbs)')

    # --- the metric's comparison with the plain GPU path: many requests through the request loop ---
    # (the single-request workload's catalogues and cached scratch are released first)
    pos_mb = (data.numel() + randoms.numel()) * data.element_size() / 1e6
    del data, wd, randoms, wr, step
    if e2e is not None:
        del hd, hwd, hr, hwr, e2e_step
    import gc
    gc.collect()
    torch.cuda.empty_cache()
    baseline_metric = None
    if world == 1 and not args.no_multi:
        baseline_metric = {}
        for name in ['batched_mocks', 'serving']:
            m = multi_workload(args, MULTI_WORKLOADS[name], device, rank)
            keep = ['served_vs_plain', 'served', 'plain', 'config', 'gpu_launches', 'clocks']
            baseline_metric[name] = {k: m[k] for k in keep}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sec, info = reference_sample(w)
        cpu = dict(value=1. / (info['scale'] * sec), unit='recons/s', cores=info['cores'], kind=info['kind'], sample=info['sample'])

    if rank == 0:
        line = dict(metric=METRIC, value=value, unit='recons/s', n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms_per_step, higher_is_better=True, scaling='weak', vs_baseline=None, dtype=w['dtype'],
                    data='synthetic: seeded lognormal data (sigma_G=0.8, P(k)~k^-1.5 exp(-(8k)^2)) + uniform randoms',
                    config=dict(workload=workload_name(w), parallelism='replicas (one independent reconstruction per GPU)',
                                precision='f4 mesh pipeline, FP64 CIC sums and normalisation',
                                l2='inputs larger than L2 (positions {:.0f} MB)'.format(pos_mb)),
                    latency_ms=dict(p50=percentile(per_step, 50), p99=percentile(per_step, 99)),
                    shift_err_mpc=shift_err, baseline_metric=baseline_metric,
                    e2e=e2e, roofline=roofline, cpu_baseline=cpu, gpu_launches=int(launches),
                    clocks=clocks.summary(), kernels=kernels)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def multi_requests(w, device, seed=0):
    """The request list of a multi-request workload: catalogues drawn once per nmesh on the device (a request
    takes a prefix of them, itself a random sample), sizes and algorithms from a seeded generator."""
    import numpy as np
    from pyrecon_b200 import mocks
    from pyrecon_b200.serving import ReconstructionRequest
    rng = np.random.default_rng(5000 + seed)
    pool = {}
    nmax = w['ndata'][1]
    for i, n in enumerate(w['nmesh']):
        data = mocks.lognormal_positions_torch(nmax, n, w['boxsize'], w['boxcenter'], seed=6000 + i, field_seed=7000 + i,
                                               dtype='f4', device=device)
        randoms = None
        if w['randoms_factor']:
            randoms = mocks.uniform_positions_torch(w['randoms_factor'] * nmax, w['boxsize'], w['boxcenter'],
                                                    seed=8000 + i, dtype='f4', device=device)
        pool[n] = (data, randoms)
    reqs = []
    for r in range(w['nrequests']):
        algo = w['algorithms'][int(rng.integers(len(w['algorithms'])))]
        n = int(w['nmesh'][int(rng.integers(len(w['nmesh'])))])
        nd = int(rng.integers(w['ndata'][0], w['ndata'][1] + 1))
        data, randoms = pool[n]
        los = w['los']
        if algo == 'PlaneParallelFFTReconstruction' and los is None:
            los = 'z'
        reqs.append(ReconstructionRequest(algo, data=data[:nd],
                                          randoms=None if randoms is None else randoms[:w['randoms_factor'] * nd],
                                          f=0.8, bias=2., los=los, nmesh=n, boxsize=w['boxsize'],
                                          boxcenter=w['boxcenter'], wrap=w['wrap'], dtype=w['dtype'],
                                          density_kwargs=dict(smoothing_radius=15.), keep_output=False))
    return reqs


def run_multi_arm(args, w):
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    line = multi_workload(args, w, torch.device('cuda', local_rank), rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def multi_workload(args, w, device, rank):
    """Throughput and latency of a multi-request workload: the plain path (requests one after the other on one
    stream) and the request loop (continuous batching on `slots` streams; for 'serving', submitted at Poisson
    arrival times, where throughput is bounded by the arrival rate and the comparison is the latency against
    the plain path serving the same arrivals first come, first served).  Both warmed up by one pass over the
    requests.  Wall clock with the device synchronised on both sides.  Returns the JSON line."""
    import gc
    import torch
    import numpy as np
    from pyrecon_b200 import _lib
    from pyrecon_b200.serving import ReconstructionServer, run_request
    world = dist_env()[2]
    reqs = multi_requests(w, device, seed=rank)
    # warm-up of the plain path: every request once (kernels, multigrid graphs, allocator)
    for r in reqs:
        run_request(r, device=device)
    torch.cuda.synchronize(device)
    # plain path (kernel times recorded: how busy the device is when requests run one at a time).  A
    # workload whose requests all arrive at once is timed `passes` times (one pass takes a fraction of a
    # second and varies by 10-20 % run to run): the median pass, its latencies and kernel times are kept.
    passes = int(w.get('passes', 1)) if w['kind'] != 'serving' else 1
    runs = []
    for _ in range(passes):
        lat = []
        _lib.profile_enable(True)
        t0 = time.perf_counter()
        for r in reqs:
            t = time.perf_counter()
            run_request(r, device=device)
            torch.cuda.synchronize(device)
            lat.append(time.perf_counter() - t)
        runs.append((time.perf_counter() - t0, lat, _lib.profile_collect()))
        _lib.profile_enable(False)
    plain_all = sorted(x[0] for x in runs)
    plain_s, lat_plain, prof = sorted(runs, key=lambda x: x[0])[len(runs) // 2]
    plain_kernel_ms = sum(v[1] for v in prof.values())
    top = sorted(prof.items(), key=lambda kv: -kv[1][1])[:6]
    # request loop
    rng = np.random.default_rng(9000 + rank)
    arrivals = np.cumsum(rng.exponential(1. / w['rate'], len(reqs))) if w['kind'] == 'serving' else np.zeros(len(reqs))
    # the plain path serving the same arrivals one request at a time (first come, first served): latency =
    # waiting + its measured service time
    fifo, free_at = [], 0.
    for at, dt in zip(arrivals, lat_plain):
        free_at = max(free_at, at) + dt
        fifo.append(free_at - at)
    launches0 = None
    # the admission budget cannot exceed what the device has free once the plain path's cached scratch is
    # released (torch's allocator keeps freed blocks per stream, and the slots run on their own streams)
    gc.collect()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info(device)
    budget = min(w.get('hbm_budget') or float('inf'), 0.75 * free)
    with ClockSampler(device.index or 0) as clocks:
        server = ReconstructionServer(device=device, slots=w['slots'], hbm_budget=budget,
                                      max_batch=w.get('max_batch', 1), batch_algorithms=w.get('batch_algorithms'))
        # warm-up of the request loop: the whole request set once, all at once (each slot's scratch and
        # multigrid graphs, the streams' allocator pools), as a long-running server would be
        for f in [server.submit(r) for r in reqs]:
            f.result()
        served_runs = []
        for _ in range(passes):
            server.reset_stats()
            launches0 = _lib.launch_count()
            torch.cuda.synchronize(device)
            start = time.perf_counter()
            futures = []
            for r, at in zip(reqs, arrivals):
                delay = start + at - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futures.append(server.submit(r))
            for f in futures:
                f.result()
            torch.cuda.synchronize(device)
            served_runs.append((time.perf_counter() - start, server.stats(), _lib.launch_count() - launches0))
        server.close()
    served_all = sorted(x[0] for x in served_runs)
    served_s, stats, launches = sorted(served_runs, key=lambda x: x[0])[len(served_runs) // 2]
    del server
    gc.collect()
    torch.cuda.empty_cache()
    pct = lambda xs, q: 1e3 * sorted(xs)[min(len(xs) - 1, int(round(q / 100. * (len(xs) - 1))))]
    n = len(reqs)
    del reqs
    torch.cuda.empty_cache()
    if True:
        line = dict(metric=METRIC, value=n / served_s, unit='recons/s', n_gpus=world, steps=1, warmup=1,
                    ms_per_step=served_s * 1e3, higher_is_better=True, scaling='weak', vs_baseline=None,
                    dtype=w['dtype'], data='synthetic: seeded lognormal catalogues, one per nmesh, requests take prefixes',
                    config=dict(workload=w['name'], requests=n, slots=w['slots'], max_batch=w.get('max_batch', 1),
                                hbm_budget_gb=round(budget / 1e9, 1),
                                arrivals='poisson {:g}/s'.format(w['rate']) if w['kind'] == 'serving' else 'all at once',
                                nmesh=w['nmesh'], algorithms=w['algorithms'],
                                timing='wall clock, device synchronised; median of {} timed pass(es)'.format(passes)),
                    served=dict(recons_per_s=n / served_s, p50_ms=stats['p50_ms'], p99_ms=stats['p99_ms'],
                                peak_in_flight=stats['peak_active'],
                                passes_recons_per_s=[round(n / x, 1) for x in served_all]),
                    plain=dict(recons_per_s=n / plain_s, p50_ms=pct(lat_plain, 50), p99_ms=pct(lat_plain, 99),
                               fifo_p50_ms=pct(fifo, 50), fifo_p99_ms=pct(fifo, 99),
                               kernel_ms=plain_kernel_ms, wall_ms=plain_s * 1e3,
                               passes_recons_per_s=[round(n / x, 1) for x in plain_all],
                               top_kernels={k: round(v[1], 2) for k, v in top}),
                    served_vs_plain=(n / served_s) / (n / plain_s), gpu_launches=int(launches),
                    clocks=clocks.summary())
    return line


# Single-kernel timings through the C ABI (one launch per step, inputs above L2), for the per-kernel
# roofline and for ncu captures of one kernel: name -> (mesh dtype, nmesh).
KERNELS = {
    'mg_jacobi': ('f4', 512),          # damped-Jacobi sweeps (two per step), local line of sight, FP32
    'mg_jacobi_256': ('f4', 256),
    'mg_jacobi_f64': ('f8', 384),
    'mg_jacobi_axis': ('f4', 512),     # line of sight along z: the 7-point form of the operator
    'mg_jacobi_axis_256': ('f4', 256),
    'mg_residual': ('f4', 512),
    'mg_residual_axis': ('f4', 512),
    'smooth_real': ('f4', 256),        # truncated real-space Gaussian, radius 15 Mpc/h on 7.8 Mpc/h cells
    'iterative_fft': ('f4', 512),      # the FFT pipeline of IterativeFFTReconstruction.run on a mesh (3 iterations,
                                       # local line of sight), no particles: the FFT passes alone, ~6.5 GB on the device
}


def run_kernel_arm(args):
    import torch
    import numpy as np
    from pyrecon_b200 import _lib
    device = torch.device('cuda', 0)
    torch.cuda.set_device(device)
    dtype, n = KERNELS[args.kernel]
    tdt = torch.float32 if dtype == 'f4' else torch.float64
    item = 4 if dtype == 'f4' else 8
    g = torch.Generator(device=device).manual_seed(5)
    v = torch.rand((n, n, n), generator=g, device=device, dtype=tdt)
    f = torch.rand((n, n, n), generator=g, device=device, dtype=tdt)
    out = torch.empty_like(v)
    nm, bs, bc = _lib.i3((n, n, n)), _lib.d3([2000.] * 3), _lib.d3([2000.] * 3)
    st = _lib.stream_of(device)
    N = n ** 3
    los = _lib.d3([0., 0., 1.]) if 'axis' in args.kernel else None
    if args.kernel == 'iterative_fft':
        del f
        psi4 = torch.empty((n, n, n, 4), device=device, dtype=tdt)
        ws = torch.empty(_lib.load().prc_iterative_fft_workspace_bytes(nm, item, 1), dtype=torch.uint8, device=device)
        base = psi4.data_ptr()
        psis = [_lib.c_void_p(base + a * item) for a in range(3)]
        name, nbytes = 'prc_iterative_fft_' + _lib.suffix(dtype), None
        call = lambda: _lib.call(name, _lib.ptr(v), nm, bs, bc, 0.4, None, 3, *psis, 4, _lib.ptr(ws), ws.numel(), st)
    elif args.kernel.startswith('mg_jacobi'):
        # two sweeps per step (v -> out -> v), so the result lands back in v without a copy
        name, nbytes = 'prc_mg_jacobi_' + _lib.suffix(dtype), 2 * 3 * N * item
        call = lambda: _lib.call(name, _lib.ptr(v), _lib.ptr(f), _lib.ptr(out), nm, bs, bc, 0.4, 0.4, 2, los, st)
    elif args.kernel.startswith('mg_residual'):
        name, nbytes = 'prc_mg_residual_' + _lib.suffix(dtype), 3 * N * item
        call = lambda: _lib.call(name, _lib.ptr(v), _lib.ptr(f), _lib.ptr(out), nm, bs, bc, 0.4, los, st)
    else:
        box = np.array([15. / 2000.] * 3, dtype=dtype)
        ws = torch.empty(_lib.load().prc_smooth_gaussian_real_workspace_bytes(nm, _lib.d3(box), 2.5, item),
                         dtype=torch.uint8, device=device)
        name, nbytes = 'prc_smooth_gaussian_real_' + _lib.suffix(dtype), 2 * N * item
        call = lambda: _lib.call(name, _lib.ptr(v), _lib.ptr(out), nm, _lib.d3(box), 2.5, _lib.ptr(ws), ws.numel(), st)
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize(device)
    with ClockSampler(0) as clocks:
        time.sleep(1.0)
        _lib.profile_enable(True)
        total_ms, per = timed_loop(call, args.steps, device)
    prof = _lib.profile_collect()
    _lib.profile_enable(False)
    peak, peak_kind = load_peaks()
    ms = total_ms / args.steps
    line = dict(kernel=args.kernel, entry_point=name, nmesh=n, dtype=dtype, steps=args.steps, ms=ms,
                p50_ms=percentile(per, 50), peak=peak, peak_source=peak_kind, clocks=clocks.summary())
    if nbytes is not None:
        gbs = nbytes / 1e9 / (ms / 1e3)
        line.update(algorithmic_bytes=nbytes, gbs=gbs, frac=gbs / peak)
    # per launched kernel: launches, ms per step, algorithmic GB/s
    line['kernels'] = {k: dict(launches=v[0], ms_per_step=round(v[1] / args.steps, 4),
                               gbs=round((v[2] / 1e9) / (v[1] / 1e3), 1) if v[1] > 0 else None)
                       for k, v in sorted(prof.items())}
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS) + sorted(MULTI_WORKLOADS))
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-check', action='store_true', help='skip the FP64 comparison of the checked run')
    ap.add_argument('--no-multi', action='store_true', help='skip the batched and served comparison with the plain path')
    ap.add_argument('--kernel', default=None, choices=sorted(KERNELS),
                    help='time one kernel through the C ABI instead of a workload')
    ap.add_argument('--tune', action='append', default=[], metavar='NAME:KEY=VALUE',
                    help='set an entry of the run-time tuning table before running (repeatable)')
    args = ap.parse_args(argv)
    if args.tune:
        from pyrecon_b200 import _lib
        for item in args.tune:
            name, rest = item.split(':', 1)
            key, value = rest.split('=', 1)
            _lib.tune_set(name, int(key), int(value))
    if args.kernel is not None:
        return run_kernel_arm(args)
    if args.workload in MULTI_WORKLOADS:
        if args.impl == 'reference':
            print(json.dumps({'impl': 'reference', 'unavailable': 'multi-request workloads compare the request loop '
                              'with the plain GPU path; the CPU reference is timed on the single-request workloads'}))
            return 0
        return run_multi_arm(args, MULTI_WORKLOADS[args.workload])
    w = WORKLOADS[args.workload]
    if args.impl == 'reference':
        return run_reference_arm(args, w)
    return run_gpu_arm(args, w)


if __name__ == '__main__':
    sys.exit(main())
