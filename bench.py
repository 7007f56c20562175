"""Benchmark of the NNGP fit step (log-likelihood + gradient) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Default workload (the mixed-precision configuration the target is quoted on; synthetic data of
its shape, seed 0): n = 1,000,000 training points, d = 16, x from a 64-component Gaussian
mixture with means ~ U[-3, 3]^16 and std 0.5, y = 256 random Fourier features
(omega ~ N(0, 1/0.8^2), phases ~ U[0, 2 pi], weights N(0, 1) sqrt(2/256)) + N(0, 0.01^2),
m = 32, ConstantKernel(1) * RBF(0.8) + WhiteKernel(1e-4), alpha = 1e-10.  One step = one full
fit step over all n points: the prefix neighbour search (point i among points [0, i), FP32,
tensor-core screen, exact FP32 rescoring), the fused FP32 local systems with the adjoint
gradient (systems whose pivot falls below the threshold re-solved in FP64) and the FP64
reduction.  The line adds the log-likelihood error against FP64 local systems on the same
lists, the fraction of systems re-solved in FP64, the error against the reference's own FP64
NumpyNngpr on a 20,000-point subset, predict throughput at 100,000 test points and a short
served-predict stream.

--workload fit3d: the reference's FP32 GPU configuration (n = 434,874, d = 3,
x ~ U[-1, 1]^3 scaled per axis by (1, 0.7, 0.4), y = sum_k sin(3 x_k) + N(0, 0.05^2),
ConstantKernel(1) * RBF(0.2) + WhiteKernel(1e-3), FP64 local systems).  --workload
differentiation / serving: the other configurations (see WORKLOADS).

Our arm prints one JSON line (rank 0) with value = fit steps per second with the inputs
resident in HBM, e2e = the same through the public estimator API uploading X, y from pinned
host memory on every call, the roofline of the dominant kernel (the neighbour search for
d = 16 and d = 8, the FP64 local-systems kernel for d = 3), a cpu_baseline (the reference's
NumpyNngpr on the host cores: a row-sampled estimate of the full step, calibrated against a
full reference step on the first 20,000 points timed in the same run) and the SM clocks
sampled during the timed steps.

--impl reference runs the reference's own CPU implementation (NumpyNngpr from
baseline/_ref: its _log_likelihood_worker on a bounded sample of rows spread over the same
fit step, all host cores, with the same calibration) and prints the same metric.

With N > 1 GPUs (torchrun) the fit step is split into N row ranges; each rank searches and
solves its rows and the (1 + n_theta) partial sums are all-reduced over NCCL (strong scaling:
the total work is fixed).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_TRAIN = 434_874
D = 3
M = 32
LS = 0.2
NOISE = 1e-3
ALPHA = 1e-10
N_PRED = 100_000
METRIC = 'fit-step loglik+grad/s'
UNIT = 'fit-steps/s'
WORKLOAD = ('nngp fit step, n=434874 d=3 m=32, isotropic RBF l=0.2, noise 1e-3; '
            'fp32 exact neighbour search (tensor-core screen), fp64 local systems (allow_downcast_f32=only-nn)')
# precision of the local systems: at this nugget nearly every FP32 system has a pivot below the
# re-solve threshold, so FP64 systems are the faster exact choice (FP32 + re-solve: 51.9 ms/step)
LOCAL = 'f64'
# roofline kernel: 'local' (the FP64 local-systems kernel, the largest share of the d = 3 step once
# the search is pruned), 'fp32' (the search kernel's screen issue) or 'tensor' (its TF32 MMAs)
ROOF = 'local'
# FP32 local systems: re-solve in FP64 when a pivot falls below this fraction of the kernel
# diagonal (None: the library default, nngpr_b200.ops.DEFAULT_PIVOT_TOL)
PIVOT = None
DATA = 'synthetic (seeded stand-in for 3droad: shape 434874 x 3)'
DTYPE = 'f32 search (tf32-split tensor screen) + f64 local'

WORKLOADS = {
    'fit3d': {},
    'precision': dict(
        N_TRAIN=1_000_000, D=16, M=32, LS=0.8, NOISE=1e-4, ALPHA=1e-10, LOCAL='f32', ROOF='tensor', PIVOT=1e-6,
        WORKLOAD=('nngp fit step, n=1000000 d=16 m=32, 64-component Gaussian mixture, isotropic RBF l=0.8, '
                  'noise 1e-4; tensor-core fp32 exact neighbour search, fp32 local systems with fp64 re-solve of '
                  'small pivots, fp64 reductions'),
        DATA='synthetic (64-component GMM in 16-d, 256 random Fourier features; shape 1000000 x 16)',
        DTYPE='f32 search (bf16x3-split tensor screen) + f32 local (f64 re-solve) + f64 sums'),
}
WORKLOADS['differentiation'] = dict(
    N_TRAIN=434_874, D=8, M=32, NOISE=4e-4, ALPHA=1e-10, LOCAL='f32', ROOF='fp32',
    WORKLOAD=('nngp fit step, n=434874 d=8 m=32, x~U[0,1]^8, ARD RBF (8 length scales), noise 4e-4; '
              'fp32 exact neighbour search, fp32 local systems with fp64 re-solves, gradient w.r.t. 10 log '
              'hyperparameters; plus 50 device L-BFGS iterations through the autograd function'),
    DATA='synthetic (U[0,1]^8, 512 random Fourier features with log-uniform ARD length scales; shape 434874 x 8)',
    DTYPE='f32 search (tf32-split tensor screen) + f32 local (f64 re-solve) + f64 sums')
WORKLOADS['serving'] = dict(
    N_TRAIN=16_599, D=18, M=32, NOISE=1e-2, ALPHA=1e-10, LOCAL='f32',
    WORKLOAD=('served predict, fitted model n=16599 d=18 m=32 held in HBM, ARD RBF, noise 1e-2; Poisson stream '
              'of requests with log-uniform sizes in [1, 65536]; continuous batching, CUDA graphs per size bucket'),
    DATA='synthetic (N(0,1)^18, ARD length scales log-uniform in [0.5, 5], 256 random Fourier features)',
    DTYPE='f32 search (bf16x3-split tensor screen) + f32 local (f64 re-solve)')
_WL = 'fit3d'


def make_data(n=None, nq=N_PRED, seed=0):
    n = N_TRAIN if n is None else n
    rng = np.random.default_rng(seed)
    global LS
    if _WL == 'serving':
        x = rng.normal(size=(n, D))
        xq = rng.normal(size=(nq, D))
        LS = np.exp(rng.uniform(np.log(0.5), np.log(5.0), D))
        omega = rng.normal(size=(256, D)) / LS
        y = np.cos(x @ omega.T + rng.uniform(0, 2 * np.pi, 256)) @ (rng.normal(size=256) * np.sqrt(2.0 / 256))
        y += rng.normal(0, 0.1, n)
        return x, y, xq
    if _WL == 'differentiation':
        x = rng.uniform(0, 1, (n, D))
        xq = rng.uniform(0, 1, (nq, D))
        LS = np.exp(rng.uniform(np.log(0.1), np.log(1.0), D))
        omega = rng.normal(size=(512, D)) / LS
        phase = rng.uniform(0, 2 * np.pi, 512)
        w = rng.normal(size=512) * np.sqrt(2.0 / 512)
        y = np.empty(n)
        for i0 in range(0, n, 65536):
            y[i0:i0 + 65536] = np.cos(x[i0:i0 + 65536] @ omega.T + phase) @ w
        y += rng.normal(0, 0.02, n)
        return x, y, xq
    if _WL == 'precision':
        means = rng.uniform(-3, 3, (64, D))
        x = means[rng.integers(0, 64, n)] + 0.5 * rng.normal(size=(n, D))
        xq = means[rng.integers(0, 64, nq)] + 0.5 * rng.normal(size=(nq, D))
        omega = rng.normal(0, 1 / 0.8, (256, D))
        phase = rng.uniform(0, 2 * np.pi, 256)
        w = rng.normal(size=256) * np.sqrt(2.0 / 256)
        y = np.empty(n)
        for i0 in range(0, n, 65536):
            y[i0:i0 + 65536] = np.cos(x[i0:i0 + 65536] @ omega.T + phase) @ w
        y += rng.normal(0, 0.01, n)
        return x, y, xq
    scale = np.array([1.0, 0.7, 0.4])
    x = rng.uniform(-1, 1, (n, D)) * scale
    y = np.sin(3 * x).sum(1) + rng.normal(0, 0.05, n)
    xq = rng.uniform(-1, 1, (nq, D)) * scale
    return x, y, xq


def make_kernel():
    from sklearn.gaussian_process import kernels as skk
    return skk.ConstantKernel(1.0) * skk.RBF(LS) + skk.WhiteKernel(NOISE)


# ------------------------------------------------------------------------------------------
# CPU baseline: the reference's NumpyNngpr on a bounded sample of rows
# ------------------------------------------------------------------------------------------
_CPU = {}


def _ref_worker(tasks):
    from nngpr.base_nngpr import DummyQueue
    g = _CPU['gpr']
    t0 = time.perf_counter()
    lml, grad = g._log_likelihood_worker(0, DummyQueue(tasks), _CPU['n_theta'], _CPU['kernel'], _CPU['x'],
                                         _CPU['y'], True)
    return time.perf_counter() - t0, float(lml), np.asarray(grad)


def _import_reference():
    ref_dir = os.path.join(ROOT, 'baseline', '_ref')
    if os.path.isdir(os.path.join(ref_dir, 'nngpr')):
        sys.path.insert(0, ref_dir)
        try:
            from nngpr.numpy_nngpr import NumpyNngpr
            from nngpr import batched_kernels
            return NumpyNngpr, batched_kernels, 'reference'
        except Exception:
            sys.path.remove(ref_dir)
    return None, None, 'port'


def default_cpu_workers(gb_per_worker=4.0, cap=32):
    """Host processes for the CPU implementation: every core, but no more than the free RAM
    allows (one reference task at this n peaks at ~2-3 GB) and at most ``cap``."""
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail_gb = psutil.virtual_memory().available / 2 ** 30
    except Exception:
        avail_gb = 16.0
    return max(1, min(cores, cap, int(avail_gb / gb_per_worker)))


class CpuBaseline:
    """Times the reference's FP64 worker (``_log_likelihood_worker``, default ``only-nn``
    search) on ``cores`` processes, each processing one batch of ``rows`` points placed at
    stratified positions of the full fit step, and extrapolates to all n points.

    ``calibrate`` checks that model against a full step: the reference's own
    ``log_marginal_likelihood(theta, eval_gradient=True)`` on the first ``subset`` points (its
    multiprocessing pool over the same cores), beside the row-sampled estimate of that same
    subset step; the ratio scales the full-size estimate."""

    def __init__(self, x, y, rows_per_task=200, cores=None, seed=1):
        NumpyNngpr, bk, kind = _import_reference()
        self.kind = kind
        self.cores = int(cores or default_cpu_workers())
        self.rows = rows_per_task
        self.n = x.shape[0]
        self.rng = np.random.default_rng(seed)
        self.ratio = 1.0
        self.calibration = None
        self.x, self.y = x, y
        if kind == 'reference':
            self.NumpyNngpr, self.bk = NumpyNngpr, bk
            kernel = bk.ConstantKernel(1.0) * bk.RBF(LS) + bk.WhiteKernel(NOISE)
            gpr = NumpyNngpr(kernel=kernel, num_nn=M, alpha=ALPHA, optimizer=None, batch_size=rows_per_task,
                             num_workers=1, distribute_method='sequential')
            # fitted state set directly, as the reference's own tests do (nngpr_base_tester.py:182):
            # fit() would evaluate the whole n-point log-likelihood on the host first
            gpr.X_train_, gpr.y_train_, gpr.kernel_ = np.asarray(x, np.float64), np.asarray(y, np.float64), kernel
            self.kernel = gpr.kernel_
            _CPU.update(gpr=gpr, kernel=gpr.kernel_, n_theta=len(gpr.kernel_.theta), x=gpr.X_train_,
                        y=gpr.y_train_[:, None])
        self.n_tasks = (self.n + rows_per_task - 1) // rows_per_task

    def _reference_gpr(self, n, **kw):
        """The reference estimator in its fitted state on the first n points, its own pool over
        ``self.cores`` processes (``distribute_method`` left at the reference's default)."""
        kernel = self.bk.ConstantKernel(1.0) * self.bk.RBF(LS) + self.bk.WhiteKernel(NOISE)
        g = self.NumpyNngpr(kernel=kernel, num_nn=M, alpha=ALPHA, optimizer=None, num_workers=self.cores, **kw)
        g.X_train_, g.y_train_, g.kernel_ = (np.asarray(self.x[:n], np.float64), np.asarray(self.y[:n], np.float64),
                                             kernel)
        return g

    def full_subset_step(self, n, repeats=2, **kw):
        """Seconds of the reference's full log_marginal_likelihood(theta, eval_gradient=True) on
        the first n points (best of ``repeats``), with its lml and gradient."""
        g = self._reference_gpr(n, **kw)
        best, out = None, None
        for _ in range(repeats):
            t0 = time.perf_counter()
            lml, grad = g.log_marginal_likelihood(g.kernel_.theta, eval_gradient=True)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
            out = (float(lml), np.asarray(grad, np.float64))
        return best, out

    def calibrate(self, subset=20000, repeats=3):
        """Row-sampled estimate vs a full reference step on the first ``subset`` points (the
        estimator's task size, and the reference's default batch size beside it); sets
        ``self.ratio`` = full / estimate."""
        if self.kind != 'reference' or self.n < 2 * subset:
            return None
        full_s, _ = self.full_subset_step(subset, batch_size=self.rows)
        default_s, _ = self.full_subset_step(subset, repeats=1)
        sub_tasks = (subset + self.rows - 1) // self.rows
        est = []
        for _ in range(repeats):
            dt, rows = self.sample(n_tasks=sub_tasks)
            est.append(dt * subset / rows / self.cores)
        est_s = float(np.median(est))
        self.ratio = full_s / est_s
        self.calibration = {
            'subset_n': subset, 'subset_full_step_s': full_s, 'subset_sampled_estimate_s': est_s,
            'ratio_full_over_estimate': self.ratio, 'subset_full_step_default_batch_s': default_s,
            'note': (f'full reference log_marginal_likelihood(theta, eval_gradient=True) on the first {subset} points '
                     f'with its multiprocessing pool over {self.cores} processes (batch_size {self.rows}, the '
                     f'estimator\'s task size; with the reference\'s default batch size beside it), against the '
                     f'row-sampled estimate of the same subset step; the full-size estimate is multiplied by the '
                     f'ratio')}
        return self.calibration

    def reference_fp64(self, subset=20000):
        """The reference's own FP64 result (allow_downcast_f32='no': FP64 search and systems) of
        the fit step on the first ``subset`` points: (lml, gradient), or None without it."""
        if self.kind != 'reference':
            return None
        _, out = self.full_subset_step(min(subset, self.n), repeats=1, batch_size=self.rows,
                                       allow_downcast_f32='no')
        return out

    def sample(self, n_tasks=None):
        """One bounded sample: ``cores`` tasks at stratified positions of the first ``n_tasks``
        tasks (default: the whole step), run in parallel on the host cores.  Returns the summed
        per-task seconds (each task timed inside its worker process) and the rows processed."""
        n_tasks = self.n_tasks if n_tasks is None else n_tasks
        edges = np.linspace(0, n_tasks, self.cores + 1)
        tasks = [int(self.rng.integers(int(a), max(int(a) + 1, int(b)))) for a, b in zip(edges[:-1], edges[1:])]
        tasks = sorted(set(min(t, n_tasks - 1) for t in tasks))
        rows = sum(min(self.n, (t + 1) * self.rows) - t * self.rows for t in tasks)
        env_keys = ('OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS', 'OMP_NUM_THREADS')
        bak = {k: os.environ.get(k) for k in env_keys}
        for k in env_keys:
            os.environ[k] = '1'  # the reference's distribute_environ default (base_nngpr.py:173-178)
        t0 = time.perf_counter()
        task_s = None
        if self.kind == 'reference':
            import multiprocessing as mp
            with mp.get_context('fork').Pool(len(tasks)) as pool:
                res = pool.map(_ref_worker, [[t] for t in tasks])
            task_s = float(sum(r[0] for r in res))
        else:
            from oracle import nngp_oracle as O
            rows_idx = np.concatenate([np.arange(t * self.rows, min(self.n, (t + 1) * self.rows)) for t in tasks])
            x, y = _CPU_PORT['x'], _CPU_PORT['y']
            nbr = O.knn(x, x[rows_idx], M, 0, LS, query_index=rows_idx)
            full = np.full((self.n, M), -1, np.int32)
            full[rows_idx] = nbr
            O.loglik_terms(x, y, full, _CPU_PORT['params'], ALPHA, True, rows_idx)
        dt = time.perf_counter() - t0 if task_s is None else task_s
        for k, v in bak.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        return dt, rows


_CPU_PORT = {}


def cpu_steps_per_s(cb: CpuBaseline, steps: int):
    """Fit steps per second of the CPU implementation: core-seconds per row measured on the
    samples, times n rows, divided by the cores, times the calibration ratio (a full reference
    step against the same estimate on a subset, ``CpuBaseline.calibrate``; 1 without it).
    Returns (steps/s, calibrated step seconds, rows sampled, core-seconds, uncalibrated step s)."""
    tot_t, tot_rows = 0.0, 0
    for _ in range(steps):
        dt, rows = cb.sample()
        tot_t += dt
        tot_rows += rows
    raw_s = tot_t * cb.n / tot_rows / cb.cores
    full_step_s = raw_s * cb.ratio
    return 1.0 / full_step_s, full_step_s, tot_rows, tot_t, raw_s


L2_NOTE = 'GPU arm: 256 MB written before every timed step (L2 flushed); CPU arm: inputs larger than its caches'
SUBSET = 20000  # points of the full reference step that calibrates the CPU estimate (and the FP64 check)


def cpu_baseline_obj(cb, sps, full_s, rows, t, raw_s, steps):
    """The line's cpu_baseline object (what was timed, how it was scaled)."""
    o = {'value': sps, 'unit': UNIT, 'cores': cb.cores, 'kind': cb.kind,
         'sample': (f'{rows} rows in batches of {cb.rows} at stratified positions of the n={cb.n} fit step over '
                    f'{steps} samples ({t:.1f} core-s); full step = core-s per row x n / {cb.cores} cores = '
                    f'{raw_s:.1f} s, x {cb.ratio:.3f} (full {SUBSET}-point reference step / its row-sampled '
                    f'estimate) = {full_s:.1f} s'),
         'full_step_s': full_s, 'sampled_estimate_s': raw_s}
    if cb.calibration is not None:
        o['calibration'] = cb.calibration
        o['subset_full_step_s'] = cb.calibration['subset_full_step_s']
        o['subset_sampled_estimate_s'] = cb.calibration['subset_sampled_estimate_s']
    return o


def prepare_cpu_baseline(x, y):
    cb = CpuBaseline(x, y)
    if cb.kind != 'reference':
        from nngpr_b200.kernel_params import extract
        from oracle import nngp_oracle as O
        p = extract(make_kernel())
        _CPU_PORT.update(x=x, y=y[:, None], params=O.KernelParams(p.rbf_level, p.const_value, p.noise_level,
                                                                  p.length_scale, p.idx_rbf_level, p.idx_const,
                                                                  p.idx_noise, p.idx_ls, p.n_theta))
        cb.cores = 1
    return cb


# ------------------------------------------------------------------------------------------
# Clocks during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (host time, csv line)
        self.t_start = self.t_end = None

    def mark_start(self):
        self.t_start = time.time()

    def mark_end(self):
        self.t_end = time.time()

    def wait_first_sample(self, timeout=5.0):
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.05)

    def __enter__(self):
        if self.proc is not None:
            return self
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.gpu}', f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        """Median SM clock and the throttle reasons seen in the samples taken between
        mark_start and mark_end (the timed steps; the sample in flight at either end included)."""
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        lo = (self.t_start or 0) - 0.06
        hi = (self.t_end or time.time()) + 0.06
        for t, ln in self.lines:
            if not lo <= t <= hi:
                continue
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled'], 'samples': 0}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': float(max(mx)), 'reasons': sorted(reasons),
                'samples': len(sm)}


# ------------------------------------------------------------------------------------------
# Our arm
# ------------------------------------------------------------------------------------------
PROFILE = {'fit3d': 'local_warp_kernel_fit_fp64_n434874_d3_m32.md', 'precision': 'knn_tc_kernel_fit_n1000000_d16_m32.md',
           'differentiation': 'knn_tc_kernel_fit_n434874_d8_m32.md'}


def read_profile_traffic():
    """DRAM bytes per launch of the roofline kernel of this workload from the committed ncu
    summary (line 'traffic_bytes_per_launch: <int>'), or None."""
    if _WL not in PROFILE:
        return None
    path = os.path.join(ROOT, 'profiles', PROFILE[_WL])
    try:
        for ln in open(path):
            if ln.startswith('traffic_bytes_per_launch:'):
                return int(ln.split(':', 1)[1].strip())
    except OSError:
        pass
    return None


def tensor_peak_tflops(bf16_operands):
    """Dense tensor rate of the search's operand type: the BF16 dense rate measured on this
    pool's B200s (MEASURED_PEAKS.json, burst) for BF16 operands, half of it for TF32 (the ratio
    of NVIDIA's dense figures, 1.1 vs 2.25 PFLOP/s)."""
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            bf16 = float(json.load(f)['bf16_tflops'])
        src = 'MEASURED_PEAKS.json bf16_tflops (burst)'
    except Exception:
        bf16, src = 1590.0, 'fallback 1.59 PFLOP/s BF16 dense'
    if bf16_operands:
        return bf16, src + ': the BF16 dense rate'
    return bf16 / 2.0, src + ' / 2: the TF32 dense rate'


def fp32_peak_tflops(torch, L, stream_ptr):
    """FP32 FMA rate of this GPU measured with the library's probe kernel (TFLOP/s)."""
    import ctypes
    blocks = 148 * 8
    out = torch.empty(blocks * 256, dtype=torch.float32, device='cuda')
    iters = 4096
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        st = L.nngp_fma_probe(ctypes.c_void_p(out.data_ptr()), iters, blocks, stream_ptr)
        e.record()
        torch.cuda.synchronize()
        assert st == 0
        flops = blocks * 256 * iters * 128
        best = max(best, flops / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def fp64_peak_tflops(torch, L, stream_ptr):
    """FP64 FMA rate of this GPU measured with the library's probe kernel (TFLOP/s)."""
    import ctypes
    blocks = 148 * 8
    out = torch.empty(blocks * 256, dtype=torch.float64, device='cuda')
    iters = 1024
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        st = L.nngp_fma_probe_f64(ctypes.c_void_p(out.data_ptr()), iters, blocks, stream_ptr)
        e.record()
        torch.cuda.synchronize()
        assert st == 0
        flops = blocks * 256 * iters * 128
        best = max(best, flops / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def local_flops_per_point(m, d, n_theta):
    """FP64 flops of one local system of the fit step with its gradient: the Cholesky of the
    augmented (m + 1) x (m + 1) matrix (2 k^3 / 3), its fill (k (k + 1) / 2 entries of 3d + 4
    flops, the exponential counted once), the gradient terms (4 flops per entry and
    hyperparameter) and the triangular solves (4 k^2)."""
    k = m + 1
    entries = k * (k + 1) // 2
    return 2.0 * k ** 3 / 3.0 + entries * (3 * d + 4) + 4.0 * entries * n_theta + 4.0 * k * k


def our_launches_per_step(n, d, m):
    """Kernels of this library one fit step launches (CUB's sort and scan kernels not counted):
    scale, centre sums and tile build; per seed level (the prefixes n, n/8, ... of at least
    8,192 points) bounds, two x (Morton keys, inverse, coordinate gather), cross positions and
    the seed kernel; the pruned search's planning (21, the index-order fallback's two
    included), a second tile build, two search
    launches and two merges, or one search launch; the local systems and the final sum."""
    seeded = n >= 8192
    levels = 0
    p_ = n
    while seeded and p_ >= 8192:
        levels += 1
        p_ //= 8
    from nngpr_b200.sharding import search_is_pruned
    pruned = seeded and search_is_pruned(n, d)
    search = (21 + 1 + 2 + 2) if pruned else 1
    return 3 + 9 * levels + search + 2


def run_plain(args, torch, x32, y64, xq32, p, flags, flush, lml_ours):
    """Time the plain FP32 GPU form of the same fit step and predict (the comparator of the
    metric): returns the 'plain_gpu' object of the bench line."""
    from nngpr_b200 import ops, plain_ref
    from nngpr_b200.plain import plain_knn, plain_loglik, plain_predict

    y32 = y64.to(torch.float32)
    nbr_ours = ops.knn(x32, x32, M, 0, LS, flags=flags)
    # the reference's own calc_nn and fill_nn_kernel, compiled from the installed reference's
    # source, when it is there (else this library's restatement of calc_nn and a torch fill)
    ref_root = os.path.join(ROOT, 'baseline', '_ref')
    ref_root = ref_root if plain_ref.available(ref_root) else None

    def step(ev=None):
        nb = plain_knn(x32, x32, M, 0, LS, ref_root=ref_root)
        if ev is not None:
            ev.record()
        return nb, plain_loglik(x32, y32, nb, p, ALPHA, True, ref_root=ref_root)

    step()  # warm-up
    ms, knn_ms = [], []
    for _ in range(args.plain_steps):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        flush.zero_()
        a.record()
        nb, (lml, grad) = step(b)
        c.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(c))
        knn_ms.append(a.elapsed_time(b))
    same = bool(torch.equal(nb, nbr_ours))
    rows_differ = int((nb != nbr_ours).any(dim=1).sum().item())
    lml = float(lml.item())
    # predict at the benchmark's query count
    nq = plain_knn(x32, xq32, M, None, LS, ref_root=ref_root)
    plain_predict(x32, y32, xq32, nq, p, ALPHA, ref_root=ref_root)
    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    a.record()
    nq = plain_knn(x32, xq32, M, None, LS, ref_root=ref_root)
    plain_predict(x32, y32, xq32, nq, p, ALPHA, ref_root=ref_root)
    c.record()
    torch.cuda.synchronize()
    pred_ms = a.elapsed_time(c)
    step_ms = float(np.min(ms))  # the comparator's best step (its torch batched solvers vary run to run)
    return {'value': 1e3 / step_ms, 'unit': UNIT, 'ms_per_step': step_ms, 'knn_ms': float(np.min(knn_ms)),
            'ms_all_steps': [float(v) for v in ms],
            'steps': args.plain_steps, 'lists_identical': same, 'rows_with_different_lists': rows_differ,
            'lml': lml, 'lml_rel_diff_vs_ours': abs(lml - lml_ours) / abs(lml_ours),
            'predict': {'value': N_PRED / (pred_ms * 1e-3), 'unit': 'points/s', 'ms': pred_ms},
            'form': ('the reference\'s own calc_nn and fill_nn_kernel (cuda_kernel_accelerators.py:663-863), compiled '
                     'with NVRTC for sm_100a from the installed reference, + torch FP32 batched Cholesky and '
                     'cholesky_solve with the materialised dK (the reference worker), one launch per stage'
                     if ref_root else
                     'one thread per query FP32 search (calc_nn structure) + torch FP32 batched fill, '
                     'Cholesky and cholesky_solve with materialised dK (the reference worker), one launch per stage')}


def _pct(v, q):
    return float(np.percentile(np.asarray(v) * 1e3, q)) if len(v) else None


def run_serving(args):
    """Served predict: a Poisson stream of requests against PredictServer (continuous batching,
    CUDA graphs per size bucket), then the same stream one request per launch through the plain
    FP32 form.  Latency = completion on the host - scheduled arrival (host clock: it is what a
    client sees, H2D/D2H and queueing included)."""
    import torch
    from nngpr_b200 import B200Nngpr
    from nngpr_b200.plain import plain_knn, plain_predict
    from nngpr_b200.serving import PredictServer

    dev = torch.device('cuda', int(os.environ.get('LOCAL_RANK', '0')))
    torch.cuda.set_device(dev)
    x, y, _ = make_data()
    kernel = make_kernel()
    gpr = B200Nngpr(kernel=kernel, num_nn=M, alpha=ALPHA, optimizer=None, allow_downcast_f32='yes',
                    device=dev).fit(x, y)
    rng = np.random.default_rng(1)
    n_req = args.requests
    sizes = np.minimum(np.exp(rng.uniform(0, np.log(65536), n_req)).astype(int), 65536)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, n_req))
    reqs = [rng.normal(size=(int(s), D)) for s in sizes]
    clocks = ClockSampler(dev.index).__enter__()
    clocks.wait_first_sample()
    srv = PredictServer(gpr)
    for r in reqs[:8]:  # warm-up
        srv.predict(r)
    # 1k-point requests on an idle server
    one_k = []
    for _ in range(args.warmup + 50):
        q = rng.normal(size=(1000, D))
        t0 = time.perf_counter()
        srv.predict(q)
        one_k.append(time.perf_counter() - t0)
    one_k = one_k[args.warmup:]
    # the stream
    done_at = [0.0] * n_req
    futs = [None] * n_req
    with clocks:
        clocks.mark_start()
        t0 = time.perf_counter()
        for k in range(n_req):
            wait = t0 + arrivals[k] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            futs[k] = srv.submit(reqs[k])
            futs[k].add_done_callback(lambda f, k=k: done_at.__setitem__(k, time.perf_counter()))
        for f in futs:
            f.result()
        t_end = max(done_at)
        clocks.mark_end()
    # capacity: the same requests submitted at once
    ts = time.perf_counter()
    for f in [srv.submit(r) for r in reqs]:
        f.result()
    t_sat = time.perf_counter() - ts
    srv.close()
    lat = [done_at[k] - (t0 + arrivals[k]) for k in range(n_req)]
    small = [lat[k] for k in range(n_req) if sizes[k] <= 1024]
    points = int(sizes.sum())
    ours = {'points_per_s': points / (t_end - t0), 'p50_ms': _pct(lat, 50), 'p99_ms': _pct(lat, 99),
            'p50_ms_le_1k_points': _pct(small, 50), 'p99_ms_le_1k_points': _pct(small, 99)}
    # plain FP32 form, one request per launch, same arrival times
    p = gpr._params(gpr.kernel_)
    xt32 = torch.from_numpy(x).to(dev, torch.float32)
    yt32 = torch.from_numpy((y - gpr._y_train_mean) / gpr._y_train_std).to(dev, torch.float32)
    ls = gpr._search_ls(p)

    def plain_one(xq):
        q = torch.from_numpy(xq).to(dev, torch.float32)
        nb = plain_knn(xt32, q, M, None, ls)
        mean, std = plain_predict(xt32, yt32, q, nb, p, ALPHA)
        return mean.cpu().numpy(), std.cpu().numpy()

    for r in reqs[:4]:
        plain_one(r)
    n_plain = min(n_req, args.plain_requests)
    plain_lat = []
    t0p = time.perf_counter()
    for k in range(n_plain):
        arr = t0p + arrivals[k]
        now = time.perf_counter()
        if now < arr:
            time.sleep(arr - now)
        plain_one(reqs[k])
        plain_lat.append(time.perf_counter() - arr)
    t_plain = time.perf_counter() - t0p
    p_small = [plain_lat[k] for k in range(n_plain) if sizes[k] <= 1024]
    plain = {'points_per_s': float(sizes[:n_plain].sum()) / t_plain, 'p50_ms': _pct(plain_lat, 50),
             'p99_ms': _pct(plain_lat, 99), 'p99_ms_le_1k_points': _pct(p_small, 99), 'requests': n_plain,
             'form': 'one request per launch: H2D, one-thread-per-query FP32 search, torch FP32 local systems, D2H'}
    line = {'metric': 'served predict points/s', 'value': ours['points_per_s'], 'unit': 'points/s', 'n_gpus': 1,
            'steps': n_req, 'warmup': args.warmup, 'higher_is_better': True, 'vs_baseline': None, 'dtype': DTYPE,
            'data': DATA, 'config': {'workload': WORKLOAD, 'n': N_TRAIN, 'd': D, 'm': M, 'requests': n_req,
                                     'rate_per_s': args.rate, 'points': points, 'slots': srv.n_slots,
                                     'buckets': list(srv.buckets)},
            'latency': ours,
            'saturated': {'points_per_s': int(sizes.sum()) / t_sat, 'seconds': t_sat,
                          'note': 'all requests of the stream submitted at once'},
            'one_k_alone': {'p50_ms': _pct(one_k, 50), 'p99_ms': _pct(one_k, 99), 'n': len(one_k)},
            'plain_gpu': plain, 'speedup_points_per_s': ours['points_per_s'] / plain['points_per_s'],
            'clocks': clocks.summary()}
    print(json.dumps(line))


def serving_summary(args):
    """The served-predict configuration (n = 16,599, d = 18: PredictServer under a Poisson stream),
    run as a child process of this benchmark after its own timed steps, condensed for this line."""
    cmd = [sys.executable, os.path.abspath(__file__), '--workload', 'serving', '--requests', str(args.serve_requests),
           '--rate', str(args.rate), '--plain-requests', str(args.serve_plain_requests), '--warmup', '3']
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        line = next(ln for ln in reversed(r.stdout.splitlines()) if ln.startswith('{'))
        d = json.loads(line)
    except Exception as e:  # reported, never fatal to the fit-step line
        return {'error': f'{type(e).__name__}: {e}'[:300]}
    lat = d['latency']
    return {'metric': 'served predict', 'config': d['config'], 'points_per_s': d['value'],
            'p50_ms': lat['p50_ms'], 'p99_ms': lat['p99_ms'], 'p99_ms_le_1k_points': lat['p99_ms_le_1k_points'],
            'one_k_alone': d['one_k_alone'], 'saturated_points_per_s': d['saturated']['points_per_s'],
            'plain_gpu': {k: d['plain_gpu'][k] for k in ('points_per_s', 'p50_ms', 'p99_ms', 'requests')},
            'speedup_points_per_s': d['speedup_points_per_s'], 'clocks': d['clocks'],
            'note': 'latency = host completion - scheduled arrival (H2D, queueing and D2H included)'}


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    x, y, xq = make_data(n=args.n)
    n = x.shape[0]

    cpu = None
    ref_np64 = None  # the reference's own FP64 (lml, grad) on the first SUBSET points
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # before any CUDA call: the reference's worker pool forks
        cb = prepare_cpu_baseline(x, y)
        cb.calibrate(SUBSET)
        sps, full_s, rows, t, raw_s = cpu_steps_per_s(cb, args.cpu_samples)
        cpu = cpu_baseline_obj(cb, sps, full_s, rows, t, raw_s, args.cpu_samples)
        if not args.no_accuracy:
            ref_np64 = cb.reference_fp64(SUBSET)

    torch.cuda.set_device(local_rank)
    dev = torch.device('cuda', local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120), device_id=dev)

    from nngpr_b200 import B200Nngpr, _lib, ops
    from nngpr_b200.kernel_params import extract
    from nngpr_b200.sharding import fit_step_rows, row_partition, search_is_pruned

    L = _lib.lib()
    _lib.check(L.nngp_check_device(), 'nngp_check_device')
    kernel = make_kernel()
    p = extract(kernel)
    x64 = torch.from_numpy(x).to(dev, torch.float64)
    y64 = torch.from_numpy(y[:, None]).to(dev, torch.float64)
    x32 = x64.to(torch.float32)
    # the local systems' copies (FP64, or FP32 with FP64 re-solves for the precision workload)
    xl, yl = (x64, y64) if LOCAL == 'f64' else (x32, y64.to(torch.float32))
    bounds = row_partition(n, world, equal_rows=search_is_pruned(n, D))
    r0, r1 = bounds[rank], bounds[rank + 1]
    q_rows = x32[r0:r1]
    flags = ops.new_flags(dev)
    out = torch.empty(1 + p.n_theta, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream()

    def step(ev=None):
        if ev is None:
            fit_step_rows(x32, xl, yl, p, ALPHA, M, r0, r1, LS, pivot_tol=PIVOT, flags=flags, out=out)
        else:  # the same two calls, with an event between them to time the search alone
            nbr = ops.knn(x32, q_rows, M, r0, LS, flags=flags)  # rows [r0, r1) among points [0, i)
            ev.record()
            ops.loglik(xl, yl, nbr, p, ALPHA, True, pivot_tol=PIVOT, flags=flags, out=out, row_begin=r0)
        if world > 1:
            dist.all_reduce(out)
        return out

    clocks = ClockSampler(local_rank).__enter__()
    clocks.wait_first_sample()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if int(flags.item()) & ~_lib.NNGP_FLAG_FP64_FALLBACK:
        raise RuntimeError(f'kernel status flags {int(flags.item())}')
    partition = {'initial': list(bounds)}
    if world > 1:
        # one measured step per rank, then the rows are re-cut for equal predicted device time
        # (sharding.rebalance): what the static rule cannot see, e.g. shards whose tile lists fell
        # back to index order on the device
        from nngpr_b200.sharding import rebalance
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        t_me = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        t_all = [torch.zeros_like(t_me) for _ in range(world)]
        dist.all_gather(t_all, t_me)
        partition['measured_ms'] = [float(v.item()) for v in t_all]
        bounds = rebalance(bounds, partition['measured_ms'])
        r0, r1 = bounds[rank], bounds[rank + 1]
        q_rows = x32[r0:r1]
        for _ in range(2):
            step()
        torch.cuda.synchronize()
    partition['final'] = list(bounds)

    # ---- timed steps (device-resident inputs, L2 flushed before every step) -------------
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with clocks:
        clocks.mark_start()
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record()
            step(ev[i][1])
            ev[i][2].record()
        torch.cuda.synchronize()
        clocks.mark_end()
        if world > 1:
            dist.barrier()
    step_ms = [a.elapsed_time(c) for a, b, c in ev]
    knn_ms = [a.elapsed_time(b) for a, b, c in ev]
    tot_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([tot_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
    lml_val = float(out[0].item())
    lml_err = None
    accuracy = None
    if LOCAL != 'f64' and world == 1:
        # the mixed-precision result against FP64 local systems on the same lists, and how many
        # systems the FP32 pass handed to the FP64 re-solve
        nbr_all = ops.knn(x32, x32, M, 0, LS, flags=flags)
        g64 = ops.loglik(x64, y64, nbr_all, p, ALPHA, True, flags=flags).cpu().numpy()
        st = {}
        g32 = ops.loglik(xl, yl, nbr_all, p, ALPHA, True, pivot_tol=PIVOT, flags=flags, stats=st).cpu().numpy()
        n_fp64 = int(st['fp64_systems'].item())
        lml_err = abs(lml_val - g64[0]) / abs(g64[0])
        accuracy = {'lml_rel_err_vs_fp64_local': float(lml_err),
                    'grad_rel_err_vs_fp64_local': float(np.max(np.abs(g32[1:] - g64[1:])) / np.max(np.abs(g64[1:]))),
                    'fp64_resolved_systems': n_fp64, 'fp64_resolved_frac': n_fp64 / n, 'pivot_tol': PIVOT,
                    'note': 'FP64 local systems computed by the FP64 kernel on the same lists (that kernel equals '
                            'the reference FP64 worker to 1e-10 on the golden cases); pivot_tol is relative to the '
                            'kernel diagonal'}
    if ref_np64 is not None and world == 1:
        # the reference's own FP64 NumpyNngpr (FP64 search and systems) on the first SUBSET points,
        # against this library's fit step on the same points (FP32 search, mixed-precision systems)
        sub = min(SUBSET, n)
        nb_s = ops.knn(x32[:sub], x32[:sub], M, 0, LS, flags=flags)
        o_s = ops.loglik(xl[:sub].contiguous(), yl[:sub].contiguous(), nb_s, p, ALPHA, True, pivot_tol=PIVOT,
                         flags=flags).cpu().numpy()
        r_lml, r_grad = ref_np64
        accuracy = dict(accuracy or {})
        accuracy['vs_reference_numpy_fp64'] = {
            'n': sub, 'lml': float(o_s[0]), 'reference_lml': r_lml,
            'lml_rel_err': abs(float(o_s[0]) - r_lml) / abs(r_lml),
            'grad_rel_err': float(np.max(np.abs(o_s[1:] - r_grad)) / np.max(np.abs(r_grad))),
            'note': f'reference NumpyNngpr(allow_downcast_f32="no") log_marginal_likelihood on the first {sub} points '
                    f'(its own FP64 search), timed in the CPU-baseline phase of this run'}

    # ---- reused neighbour lists (isotropic length scale): what later L-BFGS steps cost -------
    reuse = None
    if world == 1 and not args.no_reuse and np.ndim(LS) == 0:
        c = min(M + 16, 64, n - 1)
        cand = ops.knn(x32, x32, c, 0, LS, flags=flags)
        max_norm = float(torch.linalg.vector_norm(x32.double(), dim=1).max())
        thr = ops.knn_reuse_prepare(x32, cand, LS, max_norm)
        ev_r = []
        failed_total = 0
        for k in range(args.warmup + args.steps):
            ls_k = LS * (1.0 + 0.02 * ((k % 5) - 2))  # length scales an L-BFGS run visits near LS
            p_k = p if ls_k == LS else extract(kernel.clone_with_theta(
                np.concatenate([kernel.theta[:p.idx_ls], [np.log(ls_k)], kernel.theta[p.idx_ls + 1:]])))
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            nbr_r, failed = ops.knn_reuse_rank(x32, cand, thr, ls_k, M)
            fails = int(failed.item())  # the estimator reads it to decide on a fresh search
            ops.loglik(xl, yl, nbr_r, p_k, ALPHA, True, flags=flags, out=out)
            b.record()
            torch.cuda.synchronize()
            if k >= args.warmup:
                ev_r.append(a.elapsed_time(b))
                failed_total += fails
        r_ms = float(np.mean(ev_r))
        reuse = {'value': 1e3 / r_ms, 'unit': UNIT, 'ms_per_step': r_ms, 'rows_not_proven': failed_total,
                 'note': 'fit steps at length scales within 4% of the candidate search (an L-BFGS run near its '
                         'optimum): rank 48 candidates per point with the rounding-bound check, then the local '
                         'systems; a refused row would trigger a fresh search'}

    # ---- differentiation workload: device L-BFGS through the autograd function ----------------
    lbfgs = None
    if _WL == 'differentiation' and world == 1:
        from nngpr_b200.autograd import LogLikProblem, fit_lbfgs
        prob = LogLikProblem(x32, xl, yl, p, M, ALPHA)
        theta0 = kernel.theta.copy()
        lml0 = float(prob.evaluate(theta0)[0].item())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        th, lml1, evals = fit_lbfgs(prob, theta0, kernel.bounds, max_iter=50)
        e1.record()
        torch.cuda.synchronize()
        lb_ms = e0.elapsed_time(e1)
        lbfgs = {'max_iter': 50, 'evaluations': evals, 'ms': lb_ms, 'ms_per_evaluation': lb_ms / max(evals, 1),
                 'lml_start': lml0, 'lml_end': lml1, 'theta_end': [float(v) for v in th]}

    # ---- predict throughput at 100,000 points ---------------------------------------------
    xq64 = torch.from_numpy(xq).to(dev, torch.float64)
    xq32 = xq64.to(torch.float32)
    pred_ms = None
    if world == 1 and not args.no_predict:
        pred_all = []
        for it in range(6):  # the first is a warm-up; the median of the other five is reported
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.zero_()
            s0.record()
            nq = ops.knn(x32, xq32, M, None, LS, flags=flags)
            mean, var = ops.predict(xl, yl, xq64 if LOCAL == 'f64' else xq32, nq, p, ALPHA, flags=flags)
            s1.record()
            torch.cuda.synchronize()
            pred_all.append(s0.elapsed_time(s1))
        pred_ms = float(np.median(pred_all[1:]))

    # ---- e2e through the public API, X and y uploaded from pinned host memory per call ----
    e2e = None
    if world == 1 and not args.no_e2e:
        gpr = B200Nngpr(kernel=kernel, num_nn=M, alpha=ALPHA, optimizer=None, keep_resident=False,
                        allow_downcast_f32='yes' if LOCAL == 'f32' else None, device=dev,
                        **({} if PIVOT is None else {'pivot_tol': PIVOT})).fit(x, y)
        theta = gpr.kernel_.theta.copy()
        for _ in range(max(1, args.warmup)):
            gpr.log_marginal_likelihood(theta, eval_gradient=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            lml_api, grad_api = gpr.log_marginal_likelihood(theta, eval_gradient=True)
        e2e_s = (time.perf_counter() - t0) / args.steps
        # X and y in the local systems' precision (the search copy is cast on the device)
        h2d = int(x.shape[0] * (D + 1) * (8 if LOCAL == 'f64' else 4))
        d2h = int((1 + p.n_theta + 1) * 8)  # [lml, grad..., status] in one float64 read
        e2e = {'value': 1.0 / e2e_s, 'unit': UNIT, 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
               'ms_per_step': e2e_s * 1e3}

    # ---- the plain FP32 GPU form (one thread per query search + batched torch FP32 systems) --
    plain = None
    if world == 1 and not args.no_plain:
        plain = run_plain(args, torch, x32, y64, xq32, p, flags, flush, lml_val)
        plain['lml_rel_err_vs_fp64_local'] = (None if lml_err is None else
                                              abs(plain['lml'] - lml_val) / abs(lml_val))
        plain['speedup'] = (1e3 / (tot_ms / args.steps)) / plain['value']

    serving = None
    if rank == 0 and world == 1 and not args.no_serving and _WL != 'serving':
        serving = serving_summary(args)

    if rank == 0:
        import ctypes
        peak = fp32_peak_tflops(torch, L, ctypes.c_void_p(stream.cuda_stream))
        pairs = (r1 * (r1 - 1) - r0 * (r0 - 1)) / 2.0  # prefix pairs of this rank's rows
        knn_avg_ms = float(np.mean(knn_ms))
        achieved = 2.0 * D * pairs / (knn_avg_ms * 1e-3) / 1e12
        ms_per_step = tot_ms / args.steps
        # the pipe that bounds the search: the FP32/ALU issue of the screen at small d (the distance
        # work is cheap), the tensor pipe at d = 16 (the survey's roofline for that configuration)
        bf16_ops = D >= 12  # the search's operand type: BF16 x3 split from d = 12, TF32 split below
        kmma = 16 if bf16_ops else 8
        kp = (3 * (D + 1) + kmma - 1) // kmma * kmma  # split width of the tensor-core operands
        issued = 2.0 * kp * pairs / (knn_avg_ms * 1e-3) / 1e12
        local_avg_ms = float(np.mean([a - b for a, b in zip(step_ms, knn_ms)]))
        screen = 'BF16x3-split (kind::f16)' if bf16_ops else 'TF32-split (kind::tf32)'
        search = {'kernel': f'knn_tc_kernel<{D}> (prefix search: tcgen05 {screen} screen, exact FP32 rescoring; '
                            f'seeded rows, pruned tile lists)',
                  'ms': knn_avg_ms,
                  'brute_force_equivalent_tflops': achieved,
                  'note': '2*d flops per (query, ref) pair over all n(n-1)/2 prefix pairs; the pruned search '
                          'screens a small fraction of them, so this is a rate of the problem, not of a pipe'}
        if ROOF == 'local':
            fpk = fp64_peak_tflops(torch, L, ctypes.c_void_p(stream.cuda_stream))
            lflops = local_flops_per_point(M, D, p.n_theta) * (r1 - r0)
            lach = lflops / (local_avg_ms * 1e-3) / 1e12
            roof = {'bound': 'fp64', 'achieved': lach, 'peak': fpk, 'unit': 'TFLOP/s', 'frac': lach / fpk,
                    'peak_source': 'FP64 FMA probe measured in this run (MEASURED_PEAKS.json has no FP64 figure)',
                    'kernel': 'local_warp_kernel<double, grad> (fused fill, Cholesky, solves, adjoint gradient)',
                    'work': 'per point: 2k^3/3 + k(k+1)/2 (3d + 4 + 4 n_theta) + 4k^2 FP64 flops, k = m + 1',
                    'local_ms': local_avg_ms, 'search': search}
        elif ROOF == 'tensor':
            tpk, tsrc = tensor_peak_tflops(bf16_ops)
            # the step's other kernel: the FP32 local systems (and the FP64 re-solve of marked points)
            lach = local_flops_per_point(M, D, p.n_theta) * (r1 - r0) / (local_avg_ms * 1e-3) / 1e12
            roof = {'bound': 'tensor', 'achieved': achieved, 'peak': tpk, 'unit': 'TFLOP/s', 'frac': achieved / tpk,
                    'peak_source': tsrc, 'issued_mma_tflops': issued, 'issued_frac': issued / tpk,
                    'fp32_fma_equivalent': {'peak': peak, 'frac': achieved / peak,
                                            'peak_source': 'FP32 FMA probe measured in this run'},
                    'local_systems': {'kernel': 'local_warp_kernel<float, grad> + local_redo_kernel',
                                      'ms': local_avg_ms, 'achieved': lach, 'peak': peak, 'unit': 'TFLOP/s',
                                      'frac': lach / peak,
                                      'peak_source': 'FP32 FMA probe measured in this run',
                                      'work': 'per point: 2k^3/3 + k(k+1)/2 (3d + 4 + 4 n_theta) + 4k^2 flops, '
                                              'k = m + 1'}}
        else:
            roof = {'bound': 'fp32', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s', 'frac': achieved / peak,
                    'peak_source': 'FP32 FMA probe measured in this run (MEASURED_PEAKS.json has no FP32 figure)',
                    'issued_mma_tflops': issued}
        line = {
            'metric': METRIC, 'value': 1e3 / ms_per_step, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms_per_step, 'higher_is_better': True,
            'scaling': 'strong' if world > 1 else 'weak', 'vs_baseline': None, 'dtype': DTYPE,
            'data': DATA,
            'config': {'workload': WORKLOAD, 'n': n, 'd': D, 'm': M, 'l2': L2_NOTE},
            'parallelism': f'rows{world}', 'partition': partition if world > 1 else None, 'lml': lml_val,
            'lml_rel_err_vs_fp64_local': lml_err,
            'e2e': e2e,
            'roofline': dict(roof, traffic=read_profile_traffic()) if ROOF == 'local' else dict(
                roof, traffic=read_profile_traffic(),
                kernel=f'knn_tc_kernel<{D}> (prefix search: tcgen05 {screen} screen, exact FP32 rescoring)',
                work='2*d flops per (query, ref) pair, n(n-1)/2 pairs, whichever pipe computes them; '
                     'issued_mma = 2*K\' per pair with the split width K\'',
                pruned=search_is_pruned(n, D),
                pruned_note='when pruned, the search screens only the pairs its tile lists keep, so achieved (and '
                            'frac) is the brute-force rate of the problem and can exceed the pipe\'s peak',
                knn_ms=knn_avg_ms),
            'cpu_baseline': cpu,
            'accuracy': accuracy,
            'plain_gpu': plain,
            'lbfgs': lbfgs,
            'reused_lists_step': reuse,
            'serving': serving,
            'predict': None if pred_ms is None else {'value': N_PRED / (pred_ms * 1e-3), 'unit': 'points/s',
                                                     'ms': pred_ms, 'n_query': N_PRED},
            'gpu_launches': args.steps * our_launches_per_step(n, D, M),  # row shards take the same path
            'gpu_launches_note': 'kernels of libnngp_b200.so per step (see our_launches_per_step); CUB sort and '
                                 'scan kernels the planning launches are not counted',
            'clocks': clocks.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------------------------------
# Reference arm
# ------------------------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    if rank != 0:
        return
    x, y, _ = make_data()
    cb = prepare_cpu_baseline(x, y)
    cb.calibrate(SUBSET)
    for _ in range(args.warmup):
        cb.sample()
    sps, full_s, rows, t, raw_s = cpu_steps_per_s(cb, args.steps)
    cpu = cpu_baseline_obj(cb, sps, full_s, rows, t, raw_s, args.steps)
    line = {
        'metric': METRIC, 'value': sps, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': full_s * 1e3, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64 systems (the reference default allow_downcast_f32=only-nn: f32 search)', 'data': DATA,
        'config': {'workload': WORKLOAD, 'n': N_TRAIN, 'd': D, 'm': M, 'l2': L2_NOTE},
        'parallelism': 'host processes', 'impl': 'reference',
        'cpu_baseline': cpu,
        'e2e': {'value': sps, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    ap.add_argument('--cpu-samples', type=int, default=2)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true', help='skip the end-to-end API timing')
    ap.add_argument('--no-predict', action='store_true', help='skip the predict timing')
    ap.add_argument('--no-plain', action='store_true', help='skip the plain FP32 GPU comparator')
    ap.add_argument('--no-reuse', action='store_true', help='skip the reused-neighbour-list step timing')
    ap.add_argument('--plain-steps', type=int, default=2, help='timed steps of the plain comparator (best reported)')
    ap.add_argument('--requests', type=int, default=400, help='serving workload: requests in the stream')
    ap.add_argument('--rate', type=float, default=200.0, help='serving workload: mean arrivals per second')
    ap.add_argument('--plain-requests', type=int, default=100, help='serving workload: requests the plain form runs')
    ap.add_argument('--serve-requests', type=int, default=300, help='requests of the served stream in the fit-step line')
    ap.add_argument('--serve-plain-requests', type=int, default=10,
                    help='requests the plain form runs for the served stream in the fit-step line')
    ap.add_argument('--no-accuracy', action='store_true',
                    help='skip the reference FP64 run on the first 20,000 points (the line\'s accuracy object)')
    ap.add_argument('--no-serving', action='store_true', help='skip the short served-predict stream')
    ap.add_argument('--workload', choices=sorted(WORKLOADS), default='precision',
                    help='precision: n=1,000,000 d=16 mixed precision (default); fit3d: n=434,874 d=3; '
                         'differentiation: n=434,874 d=8 ARD; serving: the served-predict stream alone')
    ap.add_argument('--n', type=int, default=None,
                    help='training points (smaller cases are for profiling; the metric is quoted at the '
                         'workload\'s own n)')
    ap.add_argument('--pivot-tol', type=float, default=None,
                    help='FP64 re-solve threshold of the FP32 local systems (relative to the kernel diagonal)')
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global _WL, PIVOT
    _WL = args.workload
    globals().update(WORKLOADS[args.workload])
    if args.pivot_tol is not None:
        PIVOT = args.pivot_tol
    if args.impl == 'reference':
        run_reference(args)
    elif args.workload == 'serving':
        run_serving(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
