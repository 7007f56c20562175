"""Continuous-batching predict server for a fitted model held in HBM.

The reference answers ``predict`` one call at a time: every call re-uploads the training set,
searches, fills and solves in worker batches (``nngpr/base_nngpr.py:763-894, 1032-1135``).
:class:`PredictServer` keeps the training set, its kernel parameters and the search copy
resident and serves a stream of predict requests of uneven sizes:

* requests are queued as they arrive (:meth:`PredictServer.submit` returns a future); a
  scheduler thread packs the queued points, oldest first, into one batch per free *slot* (a
  request larger than the biggest batch is split, a batch takes pieces of several requests).
  Small requests (at most ``small_points``) have their own queue and one slot of their own,
  so they never wait behind a batch of large ones;
* a batch is padded to the smallest size bucket that holds it and run as one CUDA graph
  captured for that bucket: cast, neighbour search, fused fill + Cholesky + solves, all on the
  slot's stream, between an H2D copy of the batch and a D2H copy of its results (pinned host
  buffers of the slot);
* several slots are in flight at once on their own streams, so requests that arrive while
  others run are admitted as soon as a slot is free and their work overlaps on the device.
  Slots are admitted by free device memory: the server starts with ``min_slots``; while requests
  wait and every slot is busy it adds a slot (its graphs captured on its own stream, all of its
  buckets sharing one memory pool, since a slot runs one batch at a time) whenever the free
  device memory, less ``reserve_bytes``, still holds one slot's footprint and the total stays
  within ``memory_budget``, up to ``max_slots``;
* a completion thread polls the batches' events, in any order, scatters the rows of each
  finished batch to their requests and completes a request's future when all its rows are back.

Every query row is computed independently (its own neighbour list and local system), so a
request's result does not depend on what it was batched with (tests/test_gpu_serving.py checks
it bit for bit).
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, ops

# batch sizes with a captured graph; the largest bounds one batch (a larger request is split), which
# also bounds how long a batch holds the SMs while small requests wait
DEFAULT_BUCKETS = (256, 1024, 4096, 16384)


@dataclass
class _Request:
    x: np.ndarray
    future: cf.Future
    t_submit: float
    mean: np.ndarray
    var: np.ndarray
    left: int
    t_done: float = 0.0


@dataclass
class _Batch:
    pieces: list  # (request, row offset in request, rows, row offset in batch)
    points: int
    bucket: int
    event: torch.cuda.Event = None


@dataclass
class _Slot:
    stream: torch.cuda.Stream
    x_in: torch.Tensor            # (max bucket, d) float64 device input
    x_pin: torch.Tensor           # pinned staging of the input
    mean_pin: torch.Tensor        # pinned results
    var_pin: torch.Tensor
    flags_pin: torch.Tensor
    graphs: dict = field(default_factory=dict)   # bucket -> (graph, mean_out, var_out, flags)
    busy: bool = False


class PredictServer:
    """Serve ``predict(X, return_std=True)`` of a fitted :class:`nngpr_b200.B200Nngpr`.

    ``buckets``: batch sizes (query points) with a captured CUDA graph each; the largest is the
    most points one batch takes.  ``slots``: batches in flight at most (``max_slots``);
    ``min_slots`` are created at start-up, the others when requests wait and the free device
    memory holds them (``memory_budget`` bytes at most for all slots; default ``memory_fraction``
    of the free memory at start-up; ``reserve_bytes`` always left free).  ``use_graphs=False``
    launches the kernels directly (same results; for comparison).
    """

    def __init__(self, gpr, buckets=DEFAULT_BUCKETS, slots: int = 4, use_graphs: bool = True,
                 memory_fraction: float = 0.5, small_points: int = 4096, min_slots: int | None = None,
                 memory_budget: int | None = None, reserve_bytes: int = 256 << 20):
        if not hasattr(gpr, 'X_train_'):
            raise ValueError('PredictServer needs a fitted model')
        self.gpr = gpr
        self.buckets = tuple(sorted(int(b) for b in buckets))
        self.max_batch = self.buckets[-1]
        self.use_graphs = use_graphs
        dev = torch.device(gpr._device)
        self.device = dev if dev.index is not None else torch.device('cuda', torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        kernel = gpr.kernel_
        self.p = gpr._params(kernel)
        self.search_dtype, self.local_dtype = gpr._dtypes()
        self.xt, self.yt = gpr._train_tensors(self.local_dtype)  # resident (keep_resident)
        self.xs_train = self.xt if self.search_dtype == self.local_dtype else self.xt.to(self.search_dtype)
        self.ls = gpr._search_ls(self.p)
        self.d = self.xt.shape[1]
        self.ydim = self.yt.shape[1] if self.yt.dim() == 2 else 1
        self.m = min(gpr._num_nn, self.xt.shape[0])
        self.alpha = float(gpr.alpha)
        self.pivot_tol = gpr.pivot_tol
        self.y_std = np.asarray(gpr._y_train_std, dtype=np.float64).reshape(1, -1)
        self.y_mean = np.asarray(gpr._y_train_mean, dtype=np.float64).reshape(1, -1)

        # slots are admitted by free device memory: one slot's footprint (inputs, outputs and the
        # shared pool of its graphs' workspaces) against the budget and the memory free right now
        self.slot_bytes = self._slot_bytes()
        free, _ = torch.cuda.mem_get_info(self.device)
        self.memory_budget = int(free * memory_fraction) if memory_budget is None else int(memory_budget)
        self.reserve_bytes = int(reserve_bytes)
        self.max_slots = max(1, int(slots))
        start = self.max_slots if min_slots is None else max(1, min(int(min_slots), self.max_slots))
        start = max(1, min(start, self.memory_budget // max(self.slot_bytes, 1)))
        # slot 0 (the small requests' lane when there are several slots) runs on a high-priority
        # stream: its blocks are scheduled ahead of queued blocks of the large batches
        self.slots = [self._make_slot(high_priority=(i == 0 and self.max_slots > 1)) for i in range(start)]
        self.slots_added = 0   # slots added after start-up (memory admission)
        self.slots_refused = 0  # times a slot was wanted but the free memory or the budget did not hold it

        self._queue = collections.deque()        # large requests: [request, next row offset]
        self._small = collections.deque()        # requests of at most small_points rows
        self.small_points = int(small_points)
        self._inflight = []                      # (slot, batch) launched, not yet completed
        self._cv = threading.Condition()
        self._stop = False
        self._error = None
        self.completed = []
        self._sched = threading.Thread(target=self._schedule_loop, name='nngp-sched', daemon=True)
        self._done = threading.Thread(target=self._complete_loop, name='nngp-done', daemon=True)
        self._sched.start()
        self._done.start()

    # ---- set-up ---------------------------------------------------------------------------
    @property
    def n_slots(self) -> int:
        return len(self.slots)

    def _slot_bytes(self) -> int:
        """Device bytes of one slot: its input and outputs for the largest bucket, plus the largest
        bucket's graph workspace (search workspace, lists, casts, predict outputs); the buckets'
        graphs share one pool."""
        b = self.max_batch
        io = b * self.d * 8 + b * (self.ydim + 1) * 8
        ws = int(_lib.lib().nngp_knn_workspace_size_f32(self.xt.shape[0], b, self.d, self.m)) + b * self.m * 4
        return 2 * io + ws + b * self.d * 8

    def _may_add_slot(self) -> bool:
        """Whether the free device memory (less the reserve) and the budget hold one more slot."""
        if len(self.slots) >= self.max_slots:
            return False
        free, _ = torch.cuda.mem_get_info(self.device)
        ok = (free - self.reserve_bytes >= self.slot_bytes and
              (len(self.slots) + 1) * self.slot_bytes <= self.memory_budget)
        if not ok:
            self.slots_refused += 1
        return ok

    def _run(self, slot: _Slot, b: int, flags: torch.Tensor):
        """Kernels of one batch of ``b`` points from ``slot.x_in`` (captured into the graphs)."""
        xq = slot.x_in[:b]
        xs = xq.to(self.search_dtype)
        xl = xs if self.local_dtype == self.search_dtype else xq.to(self.local_dtype)
        nbr = ops.knn(self.xs_train, xs, self.m, None, self.ls, flags=flags)
        return ops.predict(self.xt, self.yt, xl, nbr, self.p, self.alpha, self.pivot_tol, flags=flags)

    def _make_slot(self, high_priority: bool = False) -> _Slot:
        b = self.max_batch
        dev = self.device
        slot = _Slot(stream=torch.cuda.Stream(dev, priority=-1 if high_priority else 0),
                     x_in=torch.zeros((b, self.d), dtype=torch.float64, device=dev),
                     x_pin=torch.empty((b, self.d), dtype=torch.float64).pin_memory(),
                     mean_pin=torch.empty((b, self.ydim), dtype=torch.float64).pin_memory(),
                     var_pin=torch.empty((b,), dtype=torch.float64).pin_memory(),
                     flags_pin=torch.zeros(1, dtype=torch.int32).pin_memory())
        pool = torch.cuda.graph_pool_handle() if self.use_graphs else None  # one pool for the slot's graphs
        for bucket in self.buckets:
            flags = ops.new_flags(dev)
            mean_out = torch.zeros((bucket, self.ydim), dtype=torch.float64, device=dev)
            var_out = torch.zeros((bucket,), dtype=torch.float64, device=dev)
            graph = None
            if self.use_graphs:
                with torch.cuda.stream(slot.stream):
                    self._run(slot, bucket, flags)  # warm-up outside the capture
                slot.stream.synchronize()
                graph = torch.cuda.CUDAGraph()
                # thread-local capture: the completion thread keeps polling other slots' events
                with torch.cuda.graph(graph, pool=pool, stream=slot.stream, capture_error_mode='thread_local'):
                    flags.zero_()
                    mean, var = self._run(slot, bucket, flags)
                    mean_out.copy_(mean)
                    var_out.copy_(var)
            slot.graphs[bucket] = (graph, mean_out, var_out, flags)
        return slot

    # ---- client side ----------------------------------------------------------------------
    def submit(self, x) -> cf.Future:
        """Queue one predict request; the future resolves to ``(mean, std)`` in the estimator's
        output format (``B200Nngpr.predict(x, return_std=True)``)."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, self.d))
        fut = cf.Future()
        req = _Request(x=x, future=fut, t_submit=time.perf_counter(), mean=np.empty((x.shape[0], self.ydim)),
                       var=np.empty(x.shape[0]), left=x.shape[0])
        if x.shape[0] == 0:
            self._finish(req)
            return fut
        with self._cv:
            if self._error is not None:
                raise RuntimeError('predict server failed') from self._error
            (self._small if x.shape[0] <= self.small_points else self._queue).append([req, 0])
            self._cv.notify_all()
        return fut

    def predict(self, x):
        return self.submit(x).result()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._sched.join()
        self._done.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- scheduler ------------------------------------------------------------------------
    def _pick(self):
        """(slot, queue) to launch next, or None (under the lock).  Slot 0 serves the small
        queue only (when there are two or more slots); the others take large requests first."""
        for i, sl in enumerate(self.slots):
            if sl.busy:
                continue
            if i == 0 and len(self.slots) > 1:
                if self._small:
                    return sl, self._small
                continue
            if self._queue:
                return sl, self._queue
            if self._small:
                return sl, self._small
        return None

    def _pending(self) -> bool:
        return bool(self._queue or self._small)

    def _take_batch(self, queue) -> _Batch:
        """Pieces of the requests in ``queue``, oldest first, up to the largest bucket."""
        pieces, points = [], 0
        while queue and points < self.max_batch:
            entry = queue[0]
            req, off = entry
            rows = min(req.x.shape[0] - off, self.max_batch - points)
            pieces.append((req, off, rows, points))
            points += rows
            if off + rows == req.x.shape[0]:
                queue.popleft()
            else:
                entry[1] = off + rows
        bucket = next(b for b in self.buckets if b >= points)
        return _Batch(pieces=pieces, points=points, bucket=bucket)

    def _schedule_loop(self):
        torch.cuda.set_device(self.device)
        try:
            while True:
                grow = False
                with self._cv:
                    pick = self._pick()
                    while not self._stop and pick is None:
                        if self._pending() and self._may_add_slot():
                            grow = True
                            break
                        self._cv.wait()
                        pick = self._pick()
                if grow:  # every slot busy, requests waiting, memory for one more slot
                    slot = self._make_slot()
                    with self._cv:
                        self.slots.append(slot)
                        self.slots_added += 1
                    continue
                with self._cv:
                    pick = self._pick() if pick is None else pick
                    if pick is None:  # stopping and nothing left to launch
                        if not self._pending():
                            return
                        self._cv.wait(0.001)
                        continue
                    slot, queue = pick
                    batch = self._take_batch(queue)
                    slot.busy = True
                self._launch(slot, batch)
                with self._cv:
                    self._inflight.append((slot, batch))
                    self._cv.notify_all()
        except BaseException as e:  # surfaced to the clients
            self._fail(e)

    def _launch(self, slot: _Slot, batch: _Batch):
        for req, off, rows, at in batch.pieces:
            slot.x_pin[at:at + rows].numpy()[...] = req.x[off:off + rows]
        P = batch.points
        graph, mean_out, var_out, flags = slot.graphs[batch.bucket]
        with torch.cuda.stream(slot.stream):
            slot.x_in[:P].copy_(slot.x_pin[:P], non_blocking=True)
            if graph is not None:
                graph.replay()
            else:
                flags.zero_()
                mean, var = self._run(slot, batch.bucket, flags)
                mean_out.copy_(mean)
                var_out.copy_(var)
            slot.mean_pin[:P].copy_(mean_out[:P], non_blocking=True)
            slot.var_pin[:P].copy_(var_out[:P], non_blocking=True)
            slot.flags_pin.copy_(flags, non_blocking=True)
            batch.event = torch.cuda.Event()
            batch.event.record(slot.stream)

    # ---- completion -----------------------------------------------------------------------
    def _complete_loop(self):
        torch.cuda.set_device(self.device)
        try:
            while True:
                with self._cv:
                    while not self._inflight and not (self._stop and not self._pending() and self._idle()):
                        self._cv.wait()
                    if not self._inflight:
                        return
                    batches = list(self._inflight)
                done = [sb for sb in batches if sb[1].event.query()]
                if not done:  # nothing finished yet: poll again shortly (batches finish out of order)
                    time.sleep(2e-5)
                    continue
                for slot, batch in done:
                    fl = int(slot.flags_pin.item()) & ~(_lib.NNGP_FLAG_FP64_FALLBACK | _lib.NNGP_FLAG_NOT_PD)
                    mean = slot.mean_pin.numpy()
                    var = slot.var_pin.numpy()
                    finished = []
                    for req, off, rows, at in batch.pieces:
                        req.mean[off:off + rows] = mean[at:at + rows]
                        req.var[off:off + rows] = var[at:at + rows]
                        req.left -= rows
                        if req.left == 0:
                            finished.append(req)
                    with self._cv:
                        self._inflight.remove((slot, batch))
                        slot.busy = False
                        self._cv.notify_all()
                    for req in finished:
                        if fl:
                            req.future.set_exception(_lib.NngpError(f'predict server: kernel status flags {fl}'))
                        else:
                            self._finish(req)
        except BaseException as e:
            self._fail(e)

    def _idle(self) -> bool:
        return all(not s.busy for s in self.slots)

    def _finish(self, req: _Request):
        mean = self.y_std * req.mean + self.y_mean
        std = np.sqrt(req.var).reshape(-1, 1) * self.y_std
        if mean.shape[1] == 1:
            mean, std = mean[:, 0], std[:, 0]
        req.t_done = time.perf_counter()
        self.completed.append(req.t_done - req.t_submit)
        req.future.set_result((mean, std))

    def _fail(self, e):
        with self._cv:
            self._error = e
            pending = ([r for r, _ in self._queue] + [r for r, _ in self._small] +
                       [p[0] for _, b in self._inflight for p in b.pieces])
            self._queue.clear()
            self._small.clear()
            self._stop = True
            self._cv.notify_all()
        for r in pending:
            if not r.future.done():
                r.future.set_exception(e)
