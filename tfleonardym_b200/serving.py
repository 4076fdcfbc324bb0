"""Solve server: continuous batching of Wilson solve requests on one GPU.

Requests of different geometry, N, kappa, tolerance, precision and shift count
arrive at any time (``submit`` returns a future).  Each request is admitted by its HBM
footprint against a byte budget: a request that could never fit is rejected
(status REJECTED); one that fits but finds the budget in use waits in the
queue and is admitted as earlier requests finish and free their bytes.  Under
overload, a request is rejected at once when it finds ``max_queue`` requests
queued, or when its expected wait (the queue over the measured completion rate)
exceeds ``max_wait_s``.
Gauge fields stay resident in an LRU cache keyed by the caller's gauge key,
so repeated requests on the same configuration skip the upload.

Worker threads (one CUDA stream each) repeatedly take the oldest pending
request and batch every other pending request that shares its gauge, kappa,
tolerance, precision and operator form into one multi-right-hand-side solve
(``lym_wilson_solve``), up to ``max_batch`` right-hand sides.  Requests that
arrive while a batch runs join the next batch, and batches of different
gauges run concurrently on different streams.  A request with ``shifts``
solves (Q^2 + sigma_k) x_k = b for all its shifts in one multishift CG (by
default the even-odd lym_multishift_solve_eo in FP64) and is served on its own.  Every answer carries
the FP64 true residual (recomputed here for the shifted systems); a request
whose residual misses its tolerance completes with status NOT_CONVERGED.

Latency bookkeeping: ``submit`` time, admission time, start and end of the
batch that served the request.
"""
import collections
import concurrent.futures
import itertools
import queue
import threading
import time

import numpy as np
import torch

from . import _lib

OK, NOT_CONVERGED, REJECTED = "ok", "not_converged", "rejected"


class SolveRequest:
    """One solve of D x = b (or Q x = b when ``hermitian``) on a gauge field, or,
    with ``shifts``, of (Q^2 + sigma_k) x_k = b for every shift (Q = gamma_d D).

    ``gauge_key`` names the configuration for the resident cache; ``gauge``
    (complex128 (nd, N, N, V) CUDA tensor or a zero-argument callable
    producing it) is only used when the key is not cached.  ``b`` is one
    spinor (ns, N, V) or several (k, ns, N, V) on the device (one spinor for a
    shifted request; its solution is (nshift, ns, N, V)), or a zero-argument
    callable producing it when the request runs -- then ``nrhs`` gives the count
    (k >= 1: a (k, ns, N, V) source; a shifted request's callable gives one
    spinor) -- so that a queue of pending requests holds no source memory.
    """

    _ids = itertools.count()

    def __init__(self, gauge_key, geometry, nc, kappa, b, gauge=None, tol=1e-10, precision="f16",
                 hermitian=False, bc=-1.0, max_iter=5000, out=None, shifts=None, nrhs=None):
        self.id = next(self._ids)
        self.gauge_key = gauge_key
        self.geometry = tuple(int(g) for g in geometry)
        self.nc = int(nc)
        self.kappa = float(kappa)
        self.b = b
        self.gauge = gauge
        self.tol = float(tol)
        self.precision = precision
        self.hermitian = bool(hermitian)
        self.bc = complex(bc)
        self.max_iter = int(max_iter)
        self.out = out  # optional tensor (e.g. pinned host memory) the solution is copied into
        if callable(b):
            if nrhs is None:
                raise ValueError("a source given as a callable needs nrhs")
            self.nrhs = int(nrhs)
            self.batched = shifts is None
            self.on_device = True
        else:
            self.nrhs = 1 if b.dim() == 3 else int(b.shape[0])
            self.batched = b.dim() == 4
            self.on_device = b.is_cuda
        self.shifts = None if shifts is None else [float(s) for s in shifts]
        if self.shifts is not None:
            if self.nrhs != 1 or any(s < 0 for s in self.shifts):
                raise ValueError("a shifted request takes one source and shifts >= 0")
            self.hermitian = True
            self.precision = "f64"
        self.t_submit = self.t_admit = self.t_start = self.t_end = None
        self.future = concurrent.futures.Future()

    def source(self):
        """The source tensor (a callable source is produced here, once)."""
        if callable(self.b):
            self.b = self.b()
        return self.b

    def release_source(self):
        """Drop the source once the request ran (a produced one is freed)."""
        self.b = None

    @property
    def solves(self):
        """Linear systems the request solves (right-hand sides x shifts)."""
        return self.nrhs * (len(self.shifts) if self.shifts is not None else 1)

    def batch_key(self):
        if self.shifts is not None:
            return ("multishift", self.id)  # served on its own
        return (self.gauge_key, self.kappa, self.tol, self.precision, self.hermitian, self.bc)

    def class_key(self):
        """Requests of one class can share a multi-lattice solve (same D, N, inner
        precision and operator form; geometry, kappa, tolerance and field may differ)."""
        return (len(self.geometry), self.nc, self.precision, self.hermitian)


class SolveResult:
    def __init__(self, request, x, status, reports):
        self.request = request
        self.x = x
        self.status = status
        self.reports = reports

    @property
    def latency(self):
        r = self.request
        return r.t_end - r.t_submit


def footprint_bytes(geometry, nc, nrhs, precision="f16", with_gauge=True, nshift=0, shifted_precision=None):
    """Device bytes a request occupies: its sources and solutions, its share of
    the solver workspace and (when not resident yet) the gauge copies.  A
    shifted request holds nshift solutions and search vectors plus a few
    full-lattice FP64 work vectors (shifted_precision None: the full-lattice
    FP64 multishift), or with the even-odd multishift in shifted_precision its
    FP64 solutions, the FP64 (head) workspace, the inner precision's and up to
    nshift one-shift refinement groups."""
    vol = int(np.prod(geometry))
    nd = len(geometry)
    ns = 4 if nd == 4 else 2
    ncomp = ns * nc
    spin = vol * ncomp * 16
    if nshift:
        link = nd * nc * nc * vol * 16
        if shifted_precision is None:
            spins = 2 * nshift + 6
        else:
            spins = 9 + 3 * nshift  # FP64 store and FP64 (head) workspace
            if shifted_precision != "f64":
                ratio = {"f32": 0.5, "f16": 0.25 + 0.25 / ncomp, "bf16": 0.25 + 0.25 / ncomp}[shifted_precision]
                spins += 2 + (6 + nshift) * ratio + 0.5 * nshift + nshift * (2 + 8 * ratio)
        return int(spins * spin + (3 * link if with_gauge else 0))
    sloppy = {"f64": 16, "f32": 8, "f16": 4 + 4 / ncomp, "bf16": 4 + 4 / ncomp}[precision]
    per_rhs = 2 * spin + 7 * spin / 2 + 5 * (vol / 2) * ncomp * sloppy
    gauge = 0
    if with_gauge:
        link = nd * nc * nc * vol * 16
        gauge = 3 * link + (nd * vol * (nc - 1) * nc * 8 if precision != "f64" else 0)
    return int(nrhs * per_rhs + gauge)


class _Gauge:
    """A resident configuration.  Each worker solves through its own Dirac
    operator (and so its own lym_gauge and solver workspace), so batches on
    the same configuration can run concurrently on different streams."""

    def __init__(self, key, field, geometry, nc, bc, nbytes):
        self.key = key
        self.field = field
        self.geometry = geometry
        self.nc = nc
        self.bc = bc
        self.nbytes = nbytes
        self.ops = {}
        self.users = 0

    def op_for(self, widx, kappa, hermitian):
        from . import boundary_conditions, dirac
        from . import lattice as lt
        op = self.ops.get(widx)
        if op is None:
            cfg = lt.Configuration(self.field, self.geometry, self.nc, len(self.geometry))
            op = dirac.DiracWilsonOperator(cfg, kappa, hermitian, representation="fundamental",
                                           boundary_condition_provider=boundary_conditions.factor_provider(self.bc))
            self.ops[widx] = op
        op.kappa = kappa
        op.hermitian = hermitian
        return op

    def release(self):
        for op in self.ops.values():
            op.release()
        self.ops.clear()


class _Done:
    __slots__ = ("latency", "status")

    def __init__(self, res):
        self.latency, self.status = res.latency, res.status


class SolveServer:
    def __init__(self, hbm_budget_bytes, max_batch=16, workers=2, device=None, gauge_cache=8, solver_options=None,
                 shifted_precision="f64", multi_lattice=1, max_queue=None, max_wait_s=None, release="inline"):
        self.solver_options = dict(solver_options or {})  # delta, chunk, rhs_per_thread of the CG
        # shifted requests: a precision = the even-odd multishift (lym_multishift_solve_eo) with that inner
        # precision (FP64 by default: the fastest for the mixed request streams measured); None = the
        # full-lattice FP64 multishift (lym_multishift_solve)
        self.shifted_precision = shifted_precision
        # batches on up to this many different gauge fields of one class run as one
        # multi-lattice solve (lym_wilson_solve_multi); <= 1 (the default): each batch on
        # its own.  Opt-in: it helped the mixed stream at 100 req/s, but runs of the
        # 64-lattice batch through the server varied widely with it on: companions touch
        # more gauge fields per solve, so more fields leave the cache, and destroying a
        # field's lym_gauge synchronises the device (all workers' streams).
        self.multi_lattice = int(multi_lattice)
        self.budget = int(hbm_budget_bytes)
        # overload: a request that finds this many requests queued (admitted and waiting)
        # is rejected at once instead of joining an ever longer queue (None: no limit)
        self.max_queue = None if max_queue is None else int(max_queue)
        # overload, by latency: a request whose expected wait -- the requests queued ahead
        # of it over the server's service rate -- is above max_wait_s is rejected at once
        # (None: no limit).  The service rate is the larger of the requests completed per
        # second over the last RATE_WINDOW_S and the requests completed per second of
        # worker time spent on them (batch wall time over the worker count): a lightly
        # loaded server is credited with the rate it could sustain, not with the arrival
        # rate it happens to see.  Fewer than RATE_MIN_REQUESTS completions in the window
        # give no estimate (and no rejection).
        self.max_wait_s = None if max_wait_s is None else float(max_wait_s)
        self._done = collections.deque()  # (time, requests, busy seconds) of recent batches
        self._done_n = 0
        self._done_busy = 0.0
        self._nworkers = max(1, int(workers))
        self.max_batch = int(max_batch)
        self.device = device  # CUDA device index; None: the caller's current device
        self.cache_size = int(gauge_cache)
        self._lock = threading.Condition()
        self._pending = collections.deque()  # admitted, waiting for a worker
        self._waiting = collections.deque()  # fits the budget in principle, waiting for bytes
        self._in_use = 0
        self._gauges = collections.OrderedDict()
        self._closed = False
        # latency and status of finished requests (not the results: a result holds its
        # solution tensor, which the caller owns and frees); bounded
        self.completed = collections.deque(maxlen=1 << 18)
        if self.device is None and torch.cuda.is_available():
            self.device = torch.cuda.current_device()
        # evicted gauge fields: "inline" (the default), the evicting worker releases them
        # itself (releasing a lym_gauge synchronises the device); "async", a thread of
        # their own does.  Measured on the config-5 stream, neither is better at every
        # rate (986 against 792 solves/s at 100 req/s, 718 against 835 at 1000 req/s)
        if release not in ("async", "inline"):
            raise ValueError("release is 'async' or 'inline'")
        self.release = release
        self._reap_q = queue.SimpleQueue()
        self._reaper = threading.Thread(target=self._reap, daemon=True)
        self._reaper.start()
        self._workers = [threading.Thread(target=self._run, args=(i,), daemon=True) for i in range(workers)]
        for t in self._workers:
            t.start()

    # -- client side ----------------------------------------------------------
    def submit(self, req: SolveRequest):
        req.t_submit = time.perf_counter()
        need = self._request_bytes(req)
        if need > self.budget:
            req.t_end = req.t_submit
            req.future.set_result(SolveResult(req, None, REJECTED, []))
            return req.future
        with self._lock:
            if self._closed:
                raise RuntimeError("server closed")
            queued = len(self._pending) + len(self._waiting)
            if (self.max_queue is not None and queued >= self.max_queue) or self._wait_too_long(queued):
                req.t_end = time.perf_counter()
                req.future.set_result(SolveResult(req, None, REJECTED, []))
                return req.future
            req._bytes = need
            if self._in_use + need <= self.budget and not self._waiting:
                self._admit(req)
            else:
                self._waiting.append(req)
            self._lock.notify_all()
        return req.future

    def close(self, wait=True):
        with self._lock:
            self._closed = True
            self._lock.notify_all()
        if wait:
            for t in self._workers:
                t.join()
        self._reap_q.put(None)
        if wait:
            self._reaper.join()
        self._gauges.clear()

    def _reap(self):
        if self.device is not None and torch.cuda.is_available():
            torch.cuda.set_device(self.device)
        while True:
            item = self._reap_q.get()
            if item is None:
                return
            for g in item:
                g.release()

    def stats(self):
        lat = [r.latency for r in self.completed if r.status != REJECTED]
        if not lat:
            return {}
        return {"completed": len(lat), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99))}

    # -- internals ------------------------------------------------------------
    def _request_bytes(self, req):
        resident = req.gauge_key in self._gauges
        return footprint_bytes(req.geometry, req.nc, req.nrhs, req.precision, with_gauge=not resident,
                               nshift=len(req.shifts) if req.shifts is not None else 0,
                               shifted_precision=self.shifted_precision)

    def _admit(self, req):
        self._in_use += req._bytes
        req.t_admit = time.perf_counter()
        self._pending.append(req)

    RATE_WINDOW_S = 2.0
    RATE_MIN_REQUESTS = 8

    def drain_rate(self):
        """The service rate the expected wait is measured against (requests per second; None
        while fewer than RATE_MIN_REQUESTS requests finished in the last RATE_WINDOW_S)."""
        with self._lock:
            return self._drain_rate(time.perf_counter())

    def _drain_rate(self, now):
        while self._done and now - self._done[0][0] > self.RATE_WINDOW_S:
            _, n, busy = self._done.popleft()
            self._done_n -= n
            self._done_busy -= busy
        if self._done_n < self.RATE_MIN_REQUESTS or len(self._done) < 2:
            return None
        span = now - self._done[0][0]
        by_time = (self._done_n - self._done[0][1]) / span if span > 0.0 else 0.0
        by_work = self._done_n * self._nworkers / self._done_busy if self._done_busy > 0.0 else 0.0
        return max(by_time, by_work) or None

    def _wait_too_long(self, queued):
        if self.max_wait_s is None or not queued:
            return False
        rate = self._drain_rate(time.perf_counter())
        return rate is not None and (queued + 1) > rate * self.max_wait_s

    def _release(self, reqs, busy_s=None):
        """Frees the requests' bytes and admits waiting ones; busy_s: the worker time of
        the batch (default: from the requests' start and end times)."""
        if busy_s is None:
            ends = [r.t_end for r in reqs if getattr(r, "t_end", None) is not None]
            starts = [r.t_start for r in reqs if getattr(r, "t_start", None) is not None]
            busy_s = max(ends) - min(starts) if ends and starts else 0.0
        with self._lock:
            self._done.append((time.perf_counter(), len(reqs), max(0.0, float(busy_s))))
            self._done_n += len(reqs)
            self._done_busy += max(0.0, float(busy_s))
            for r in reqs:
                self._in_use -= r._bytes
            while self._waiting and self._in_use + self._waiting[0]._bytes <= self.budget:
                self._admit(self._waiting.popleft())
            self._lock.notify_all()

    # how far past the oldest pending request a worker looks for one whose gauge it
    # already serves (its operator, solver workspace and CUDA graphs exist)
    AFFINITY_LOOKAHEAD = 8

    def _take_batch(self, widx=None):
        """Oldest pending request -- or, within the next AFFINITY_LOOKAHEAD, the oldest
        whose gauge this worker already holds -- plus every compatible pending one,
        up to max_batch rhs."""
        with self._lock:
            while not self._pending and not (self._closed and not self._waiting):
                self._lock.wait(timeout=0.05)
            if not self._pending:
                return None
            pick = 0
            if widx is not None:
                for k, r in enumerate(itertools.islice(self._pending, self.AFFINITY_LOOKAHEAD)):
                    g = self._gauges.get(r.gauge_key)
                    if g is not None and widx in g.ops:
                        pick = k
                        break
            first = self._pending[pick]
            del self._pending[pick]
            key = first.batch_key()
            batch, rhs = [first], first.nrhs
            keep = collections.deque()
            while self._pending:
                r = self._pending.popleft()
                if r.batch_key() == key and rhs + r.nrhs <= self.max_batch:
                    batch.append(r)
                    rhs += r.nrhs
                else:
                    keep.append(r)
            self._pending = keep
            return batch

    def _take_companions(self, batch):
        """With multi_lattice > 1: pending unshifted batches of the same class on other
        gauge fields (one batch per field, at most multi_lattice - 1, each up to
        max_batch rhs) join `batch` in one multi-lattice solve."""
        first = batch[0]
        if self.multi_lattice <= 1 or first.shifts is not None:
            return [batch]
        with self._lock:
            cls = first.class_key()
            comp = collections.OrderedDict()  # gauge key -> [batch key, requests, rhs]
            keep = collections.deque()
            for r in self._pending:
                if r.shifts is None and r.gauge_key != first.gauge_key and r.class_key() == cls:
                    c = comp.get(r.gauge_key)
                    if c is None and len(comp) + 1 < self.multi_lattice:
                        c = comp[r.gauge_key] = [r.batch_key(), [], 0]
                    if c is not None and r.batch_key() == c[0] and c[2] + r.nrhs <= self.max_batch:
                        c[1].append(r)
                        c[2] += r.nrhs
                        continue
                keep.append(r)
            self._pending = keep
        return [batch] + [c[1] for c in comp.values()]

    def _gauge_for(self, req):
        with self._lock:
            g = self._gauges.get(req.gauge_key)
            if g is not None:
                self._gauges.move_to_end(req.gauge_key)
                g.users += 1
                return g
        u = req.gauge() if callable(req.gauge) else req.gauge
        if u is None:
            raise ValueError(f"gauge {req.gauge_key!r} is not resident and no field was given")
        if not u.is_cuda:
            u = u.to(torch.device("cuda", self.device))
        g = _Gauge(req.gauge_key, u, req.geometry, req.nc, req.bc,
                   footprint_bytes(req.geometry, req.nc, 0, req.precision, True))
        evicted = []
        with self._lock:
            old = self._gauges.get(req.gauge_key)
            if old is not None:  # another worker loaded it meanwhile
                old.users += 1
                return old
            self._gauges[req.gauge_key] = g
            g.users += 1
            while len(self._gauges) > self.cache_size:
                k = next(iter(self._gauges))
                if self._gauges[k].users:
                    break
                evicted.append(self._gauges.pop(k))
        if evicted:
            if self.release == "async":
                self._reap_q.put(evicted)  # destroyed on the reaper thread, not on this worker
            else:
                for e in evicted:
                    e.release()
        return g

    def _run(self, widx):
        from . import dirac_solver
        dirac_solver.VERBOSE = False
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(device=torch.device("cuda", self.device))
        while True:
            batch = self._take_batch(widx)
            if batch is None:
                return
            batches = self._take_companions(batch)
            reqs = [r for b in batches for r in b]
            t0 = time.perf_counter()
            for r in reqs:
                r.t_start = t0
            try:
                with torch.cuda.stream(stream):
                    if len(batches) == 1:
                        self._solve_batch(batch, widx)
                    else:
                        self._solve_multi(batches, widx)
            except Exception as exc:  # noqa: BLE001 - delivered to every waiter
                for r in reqs:
                    r.t_end = time.perf_counter()
                    if not r.future.done():
                        r.future.set_exception(exc)
            finally:
                for r in reqs:
                    r.release_source()
                self._release(reqs, time.perf_counter() - t0)

    def _solve_shifted(self, req, g, widx):
        """(Q^2 + sigma_k) x_k = b by multishift CG (the server's shifted_precision
        picks the solver), then each true residual in FP64 through the
        reference-layout operator."""
        from . import _dev, dirac, dirac_solver
        dev = torch.device("cuda", self.device)
        src = req.source()
        b = (src if src.dim() == 3 else src[0]).to(dev, non_blocking=True)
        op = g.op_for(widx, req.kappa, True)
        ms = dirac_solver.multishift_cg(req.max_iter, req.tol, precision=self.shifted_precision, delta=0.01)
        xs = ms.solve(dirac.SquareOperator(op), b, req.shifts)
        bn = float(np.sqrt(abs(_dev.cdot(b, b))))
        reports = []
        for k, (s, x) in enumerate(zip(req.shifts, xs)):
            r = _dev.axpby(1.0, b, -1.0, _dev.axpby(1.0, op.apply(op.apply(x)), s, x))
            res = float(np.sqrt(abs(_dev.cdot(r, r)))) / bn
            its = ms.reports[k]["iterations"] if ms.reports else ms.last_steps
            reports.append(dict(status=0, iterations=its, true_residual=res, shift=s))
        x = torch.stack(xs)
        if req.out is not None:
            req.out.copy_(x, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return x, reports

    def _solve_multi(self, batches, widx):
        """Batches on different gauge fields of one class in one multi-lattice solve
        (each batch one lattice: its field, kappa, tolerance and rhs)."""
        from . import dirac_solver
        dev = torch.device("cuda", self.device)
        gs = []
        try:
            for bt in batches:
                gs.append(self._gauge_for(bt[0]))
            ops = [g.op_for(widx, bt[0].kappa, bt[0].hermitian) for g, bt in zip(gs, batches)]
            bs = [torch.cat([(r.source() if r.batched else r.source()[None]).to(dev, non_blocking=True)
                             for r in bt]) for bt in batches]
            opts = {k: v for k, v in self.solver_options.items() if k in ("delta", "chunk")}
            xs, reps = dirac_solver.solve_lattices(ops, bs, precision=batches[0][0].precision,
                                                   max_steps=max(r.max_iter for bt in batches for r in bt),
                                                   tols=[bt[0].tol for bt in batches], **opts)
            outs = []
            for bt, x in zip(batches, xs):
                k = 0
                for r in bt:  # caller-provided outputs (pinned host buffers on the host path)
                    if r.out is not None:
                        r.out.copy_(x[k:k + r.nrhs] if r.batched else x[k], non_blocking=True)
                    k += r.nrhs
                if not bt[0].on_device and any(r.out is None for r in bt):
                    x = x.to("cpu", non_blocking=True)
                outs.append(x)
            torch.cuda.current_stream().synchronize()
        finally:
            with self._lock:
                for g in gs:
                    g.users -= 1
        t_end = time.perf_counter()
        total_rhs = sum(r.nrhs for bt in batches for r in bt)
        for bt, x, rp in zip(batches, outs, reps):
            k = 0
            for r in bt:
                mine = rp[k:k + r.nrhs]
                xr = r.out if r.out is not None else (x[k:k + r.nrhs] if r.batched else x[k])
                k += r.nrhs
                ok = all(m["status"] == 0 and m["true_residual"] <= r.tol for m in mine)
                r.t_end = t_end
                res = SolveResult(r, xr, OK if ok else NOT_CONVERGED, mine)
                res.batch_rhs = total_rhs
                self.completed.append(_Done(res))
                r.future.set_result(res)

    def _solve_batch(self, batch, widx=0):
        from . import dirac_solver
        first = batch[0]
        g = self._gauge_for(first)
        if first.shifts is not None:
            try:
                x, reps = self._solve_shifted(first, g, widx)
            finally:
                with self._lock:
                    g.users -= 1
            first.t_end = time.perf_counter()
            ok = all(m["true_residual"] <= first.tol for m in reps)
            res = SolveResult(first, first.out if first.out is not None else x, OK if ok else NOT_CONVERGED, reps)
            res.batch_rhs = 1
            self.completed.append(_Done(res))
            first.future.set_result(res)
            return
        dev = torch.device("cuda", self.device)
        host = not first.on_device
        try:
            # host sources (the reference-facing path) cross here, on this worker's stream,
            # straight into their slots of the batch's source tensor
            srcs = [r.source() if r.batched else r.source()[None] for r in batch]
            b = torch.empty((sum(t.shape[0] for t in srcs),) + tuple(srcs[0].shape[1:]), dtype=srcs[0].dtype,
                            device=dev)
            k = 0
            for t in srcs:
                b[k:k + t.shape[0]].copy_(t, non_blocking=True)
                k += t.shape[0]
            del srcs
            solver = dirac_solver.conjugate_gradient(max_steps=max(r.max_iter for r in batch), tol=first.tol,
                                                     precision=first.precision, **self.solver_options)
            op = g.op_for(widx, first.kappa, first.hermitian)
            x = solver.solve(op, b)
            k = 0
            for r in batch:  # caller-provided outputs (pinned host buffers on the host path)
                if r.out is not None:
                    r.out.copy_(x[k:k + r.nrhs] if r.batched else x[k], non_blocking=True)
                k += r.nrhs
            if host and any(r.out is None for r in batch):
                x = x.to("cpu", non_blocking=True)
            torch.cuda.current_stream().synchronize()
            reps = solver.reports
        finally:
            with self._lock:
                g.users -= 1
        t_end = time.perf_counter()
        batch_rhs = sum(r.nrhs for r in batch)
        k = 0
        for r in batch:
            mine = reps[k:k + r.nrhs]
            xr = r.out if r.out is not None else (x[k:k + r.nrhs] if r.batched else x[k])
            k += r.nrhs
            ok = all(m["status"] == 0 and m["true_residual"] <= r.tol for m in mine)
            r.t_end = t_end
            res = SolveResult(r, xr, OK if ok else NOT_CONVERGED, mine)
            res.batch_rhs = batch_rhs
            self.completed.append(_Done(res))
            r.future.set_result(res)
