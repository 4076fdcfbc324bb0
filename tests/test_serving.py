"""Solve server: admission by HBM budget and continuous batching (host logic on
CPU with a stand-in solve), and on the GPU: every answer is the same alone and
in a mixed stream of requests of different geometry, N, kappa and precision."""
import threading
import time

import numpy as np
import pytest
import torch

from tfleonardym_b200 import serving


class _FakeServer(serving.SolveServer):
    """Host logic only: the solve is replaced by a sleep and an identity answer."""

    def __init__(self, *a, **k):
        self.batches = []
        self.concurrent = 0
        self.max_concurrent = 0
        self._cl = threading.Lock()
        super().__init__(*a, **k)

    def _run(self, widx):
        while True:
            batch = self._take_batch()
            if batch is None:
                return
            with self._cl:
                self.concurrent += 1
                self.max_concurrent = max(self.max_concurrent, self.concurrent)
            self.batches.append([r.id for r in batch])
            t0 = time.perf_counter()
            time.sleep(0.02)
            for r in batch:
                r.t_start, r.t_end = t0, time.perf_counter()
                res = serving.SolveResult(r, r.b, serving.OK, [])
                self.completed.append(res)
                r.future.set_result(res)
            with self._cl:
                self.concurrent -= 1
            self._release(batch)


def _req(key, geom=(4, 4, 4, 4), nrhs=1, kappa=0.12, tol=1e-10):
    b = torch.zeros((nrhs, 4, 3, int(np.prod(geom))), dtype=torch.complex128)
    return serving.SolveRequest(key, geom, 3, kappa, b, gauge=None, tol=tol)


def test_shifted_footprint_follows_the_solver():
    """A shifted request's HBM estimate: the even-odd multishift keeps its FP64
    solutions, an FP64 (head) workspace and, for a reduced inner precision, that
    workspace and the refinement groups; the full-lattice FP64 multishift less."""
    geom, nc, nsh = (8, 8, 8, 16), 3, 12
    spin = int(np.prod(geom)) * 4 * nc * 16
    full = serving.footprint_bytes(geom, nc, 1, "f16", with_gauge=False, nshift=nsh, shifted_precision=None)
    eo64 = serving.footprint_bytes(geom, nc, 1, "f16", with_gauge=False, nshift=nsh, shifted_precision="f64")
    eo32 = serving.footprint_bytes(geom, nc, 1, "f16", with_gauge=False, nshift=nsh, shifted_precision="f32")
    assert full == (2 * nsh + 6) * spin
    assert eo64 == (9 + 3 * nsh) * spin
    assert full < eo64 < eo32
    link = 4 * nc * nc * int(np.prod(geom)) * 16
    with_gauge = serving.footprint_bytes(geom, nc, 1, "f16", with_gauge=True, nshift=nsh, shifted_precision="f64")
    assert with_gauge == eo64 + 3 * link


def test_overload_sheds_requests_beyond_the_queue_limit():
    """With max_queue, a request that finds that many queued is rejected at once;
    the queued ones are still served."""
    srv = _FakeServer(hbm_budget_bytes=1 << 40, workers=1, max_queue=3)
    futs = [srv.submit(_req("g", kappa=0.1 + 0.01 * k)) for k in range(12)]
    res = [f.result(timeout=10) for f in futs]
    srv.close()
    rejected = [r for r in res if r.status == serving.REJECTED]
    served = [r for r in res if r.status == serving.OK]
    assert rejected and served and len(rejected) + len(served) == 12
    assert all(r.latency < 1.0 for r in rejected)


def test_overload_sheds_requests_whose_expected_wait_is_too_long():
    """With max_wait_s, once the completion rate is known a request whose expected
    wait (queued requests over that rate) exceeds the limit is rejected at once, so
    the served requests' latency stays near the limit however fast requests arrive."""
    srv = _FakeServer(hbm_budget_bytes=1 << 40, workers=1, max_wait_s=0.2)  # ~50 requests/s served
    futs = []
    for k in range(120):  # ~200 requests/s offered
        futs.append(srv.submit(_req("g", kappa=0.1 + 0.001 * k)))
        time.sleep(0.005)
    res = [f.result(timeout=30) for f in futs]
    rate = srv.drain_rate()
    srv.close()
    rejected = [r for r in res if r.status == serving.REJECTED]
    served = [r for r in res if r.status == serving.OK]
    assert len(rejected) > 40 and len(served) > 20
    assert rate is None or 20 < rate < 80  # one worker, 20 ms per request
    assert all(r.latency < 0.05 for r in rejected)
    assert max(r.latency for r in served) < 1.0


def test_light_load_is_not_shed():
    """Below the service rate nothing is rejected: the rate the wait is measured against is
    requests per second of worker time, not the (low) arrival rate."""
    srv = _FakeServer(hbm_budget_bytes=1 << 40, workers=1, max_wait_s=0.1)  # ~50 requests/s served
    futs = []
    for k in range(30):  # bursts of 3 every 0.15 s: 20 requests/s offered
        futs.append(srv.submit(_req("g", kappa=0.1 + 0.001 * k)))
        if k % 3 == 2:
            time.sleep(0.15)
    res = [f.result(timeout=30) for f in futs]
    srv.close()
    assert all(r.status == serving.OK for r in res)


def test_callable_source_is_made_when_the_request_runs():
    """A source given as a callable is produced by the worker (a backlog holds no
    source memory) and released after the batch."""
    made = []

    def src():
        made.append(time.perf_counter())
        return torch.zeros((2, 4, 3, 256), dtype=torch.complex128)

    r = serving.SolveRequest("g", (4, 4, 4, 4), 3, 0.12, src, nrhs=2)
    assert r.nrhs == 2 and r.batched and not made
    with pytest.raises(ValueError):
        serving.SolveRequest("g", (4, 4, 4, 4), 3, 0.12, src)
    assert r.source().shape == (2, 4, 3, 256) and len(made) == 1
    r.source()
    assert len(made) == 1
    r.release_source()
    assert r.b is None


def test_rejects_requests_that_can_never_fit():
    srv = _FakeServer(hbm_budget_bytes=10_000, workers=1)
    f = srv.submit(_req("g", geom=(16, 16, 16, 16)))
    assert f.result(timeout=5).status == serving.REJECTED
    srv.close()


def test_batches_compatible_requests_and_keeps_order():
    srv = _FakeServer(hbm_budget_bytes=1 << 40, workers=1, max_batch=4)
    srv._lock.acquire()  # hold the queue so all requests are pending together
    futs = []
    try:
        for i in range(6):
            futs.append(srv.submit(_req("a")))
        futs.append(srv.submit(_req("b")))
        futs.append(srv.submit(_req("a", kappa=0.13)))
    finally:
        srv._lock.release()
    for f in futs:
        assert f.result(timeout=5).status == serving.OK
    srv.close()
    ids = [r for b in srv.batches for r in b]
    assert sorted(ids) == sorted(f.result().request.id for f in futs)
    first = srv.batches[0]
    assert len(first) == 4  # max_batch rhs of the same gauge / kappa
    # requests with another gauge or kappa never share a batch with "a"@0.12
    for b in srv.batches:
        keys = {next(f.result().request.batch_key() for f in futs if f.result().request.id == i) for i in b}
        assert len(keys) == 1


def test_waits_for_budget_and_admits_when_memory_frees():
    one = serving.footprint_bytes((4, 4, 4, 4), 3, 1, "f16", with_gauge=True)
    srv = _FakeServer(hbm_budget_bytes=int(1.5 * one), workers=2)
    futs = [srv.submit(_req(f"g{i}")) for i in range(5)]
    for f in futs:
        assert f.result(timeout=10).status == serving.OK
    srv.close()
    # only one request fits at a time, so no two batches ever ran together
    assert srv.max_concurrent == 1
    assert srv._in_use == 0


def test_workers_overlap_when_budget_allows():
    srv = _FakeServer(hbm_budget_bytes=1 << 40, workers=3)
    futs = [srv.submit(_req(f"g{i}")) for i in range(6)]
    for f in futs:
        f.result(timeout=10)
    srv.close()
    assert srv.max_concurrent >= 2


class _FakeSolveServer(serving.SolveServer):
    """The server's batch and companion selection with stand-in solves (no CUDA
    stream: the worker loop below mirrors SolveServer._run without the device)."""

    def __init__(self, *a, **k):
        self.calls = []
        super().__init__(*a, **k)

    def _run(self, widx):
        while True:
            batch = self._take_batch(widx)
            if batch is None:
                return
            batches = self._take_companions(batch)
            if len(batches) == 1:
                self._solve_batch(batch, widx)
            else:
                self._solve_multi(batches, widx)
            self._release([r for b in batches for r in b])

    def _finish(self, reqs):
        for r in reqs:
            r.t_end = time.perf_counter()
            res = serving.SolveResult(r, r.b, serving.OK, [])
            self.completed.append(res)
            r.future.set_result(res)

    def _solve_batch(self, batch, widx=0):
        self.calls.append([[r.id for r in batch]])
        self._finish(batch)

    def _solve_multi(self, batches, widx):
        self.calls.append([[r.id for r in b] for b in batches])
        self._finish([r for b in batches for r in b])


def _req3(key, geom=(4, 4, 4, 4), nc=3, kappa=0.12, tol=1e-10, precision="f16", shifts=None):
    nd = len(geom)
    ns = 2 if nd == 2 else 4
    b = torch.zeros((ns, nc, int(np.prod(geom))), dtype=torch.complex128)
    return serving.SolveRequest(key, geom, nc, kappa, b, gauge=None, tol=tol, precision=precision, shifts=shifts)


def test_batches_on_other_fields_of_one_class_join_a_multi_lattice_solve():
    srv = _FakeSolveServer(hbm_budget_bytes=1 << 40, workers=1, max_batch=2, multi_lattice=3)
    srv._lock.acquire()  # every request pending before the worker looks
    try:
        a1 = srv.submit(_req3("a"))
        a2 = srv.submit(_req3("a"))
        b1 = srv.submit(_req3("b", geom=(4, 4, 2, 6), kappa=0.13, tol=1e-9))  # other field, same class
        c1 = srv.submit(_req3("c", geom=(6, 4, 4, 4)))
        d1 = srv.submit(_req3("d"))                                           # beyond multi_lattice = 3
        e1 = srv.submit(_req3("e", nc=2))                                     # other class (N)
        f1 = srv.submit(_req3("f", precision="f32"))                          # other class (precision)
        s1 = srv.submit(_req3("g", shifts=[0.1]))                             # shifted: on its own
        b2 = srv.submit(_req3("b", geom=(4, 4, 2, 6), kappa=0.14, tol=1e-9))  # same field, other kappa
    finally:
        srv._lock.release()
    futs = [a1, a2, b1, c1, d1, e1, f1, s1, b2]
    for f in futs:
        assert f.result(timeout=5).status == serving.OK
    srv.close()
    ids = {f: f.result().request.id for f in futs}
    first = srv.calls[0]
    assert first == [[ids[a1], ids[a2]], [ids[b1]], [ids[c1]]]  # primary + two other fields
    singles = [c for c in srv.calls[1:]]
    flat = [i for c in singles for b in c for i in b]
    assert sorted(flat) == sorted(ids[f] for f in (d1, e1, f1, s1, b2))
    # the shifted request and the other classes never share a solve with anything
    for c in singles:
        members = [i for b in c for i in b]
        if ids[s1] in members or ids[e1] in members or ids[f1] in members:
            assert len(members) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("multi_lattice", [1, 8])
def test_same_answer_alone_and_in_the_mix(cuda_device, multi_lattice):
    """Each request's solution alone equals its solution inside a mixed stream
    (different geometry, N, kappa, precision, shifted and unshifted requests),
    within the solve tolerance, and every answer meets its FP64 true residual."""
    from oracle import lym_oracle as O
    from tfleonardym_b200 import boundary_conditions
    rng = np.random.default_rng(77)
    specs = [((8, 8, 8, 8), 3, 0.12), ((4, 4, 4, 8), 3, 0.13), ((16, 8), 2, 0.2), ((8, 4, 4, 4), 2, 0.11)]
    gauges, reqs = {}, []
    for gi, (geom, nc, kappa) in enumerate(specs):
        nd, vol = len(geom), int(np.prod(geom))
        u = O.unitary_sqrt_projection(rng.normal(size=(nd, nc, nc, vol)) + 1j * rng.normal(size=(nd, nc, nc, vol)))
        gauges[gi] = torch.from_numpy(u).cuda()
        ns = 2 if nd == 2 else 4
        for k in range(3):
            b = torch.from_numpy(rng.normal(size=(ns, nc, vol)) + 1j * rng.normal(size=(ns, nc, vol))).cuda()
            reqs.append((gi, geom, nc, kappa, b, "f16" if k % 2 == 0 else "f32", None))
        if gi in (0, 2):  # a shifted request: (Q^2 + sigma) x = b for three shifts
            reqs.append((gi, geom, nc, kappa, b, "f64", [0.0, 0.05, 0.5]))
    boundary_conditions.set_antiperiodic_field_in_t_direction((4, 4, 4, 8))

    def make(r):
        gi, geom, nc, kappa, b, prec, shifts = r
        return serving.SolveRequest(f"g{gi}", geom, nc, kappa, b, gauge=gauges[gi], tol=1e-10, precision=prec,
                                    shifts=shifts)

    alone = []
    srv = serving.SolveServer(hbm_budget_bytes=8 << 30, workers=1)
    for r in reqs:
        alone.append(srv.submit(make(r)).result(timeout=120))
    srv.close()
    srv = serving.SolveServer(hbm_budget_bytes=8 << 30, workers=3, max_batch=8, multi_lattice=multi_lattice)
    futs = [srv.submit(make(r)) for r in reqs]
    mixed = [f.result(timeout=300) for f in futs]
    srv.close()
    for r, a, m in zip(reqs, alone, mixed):
        assert a.status == serving.OK and m.status == serving.OK
        assert all(rep["true_residual"] <= 1e-10 for rep in m.reports)
        xa, xm = a.x.cpu().numpy(), m.x.cpu().numpy()
        assert np.linalg.norm(xa - xm) / np.linalg.norm(xa) < 1e-8
        if r[6] is not None:
            assert xm.shape[0] == len(r[6]) and m.request.solves == len(r[6])
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["p99_ms"] >= st["p50_ms"]


@pytest.mark.gpu
def test_concurrent_solves_on_two_threads_match_serial(cuda_device):
    """Two host threads solving at once -- on two gauge objects, and on one shared
    gauge object (calls on one object take turns under its lock) -- give the
    serial answers (both to true residual 1e-10, so within 1e-8 of each other)."""
    import threading

    from oracle import lym_oracle as O
    from tfleonardym_b200 import boundary_conditions as bcs
    from tfleonardym_b200 import dirac, dirac_solver
    from tfleonardym_b200 import lattice as lt
    geom, nc, kappa = (4, 4, 4, 8), 3, 0.12
    rng = np.random.default_rng(17)
    vol = int(np.prod(geom))
    u = O.unitary_sqrt_projection(rng.normal(size=(4, nc, nc, vol)) + 1j * rng.normal(size=(4, nc, nc, vol)))
    b = [torch.from_numpy(rng.normal(size=(4, 4, nc, vol)) + 1j * rng.normal(size=(4, 4, nc, vol))).cuda()
         for _ in range(2)]

    def op():
        cfg = lt.Configuration(torch.from_numpy(u).cuda(), geom, nc, 4)
        return dirac.DiracWilsonOperator(cfg, kappa, False, representation="fundamental",
                                         boundary_condition_provider=bcs.time_antiperiodic_provider(-1))

    def solve(o, src):
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            x = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", delta=0.01).solve(o, src)
        s.synchronize()
        return x

    ops = [op(), op()]
    serial = [solve(ops[k], b[k]).cpu() for k in range(2)]
    for shared in (False, True):
        targets = [ops[0], ops[0]] if shared else ops
        out = [None, None]
        errors = []

        def work(k):
            try:
                for _ in range(3):
                    out[k] = solve(targets[k], b[k]).cpu()
            except Exception as e:  # surfaced below
                errors.append(e)

        th = [threading.Thread(target=work, args=(k,)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errors, errors
        for k in range(2):
            diff = float(torch.linalg.vector_norm(out[k] - serial[k]) / torch.linalg.vector_norm(serial[k]))
            assert diff < 1e-8, (shared, k, diff)
