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
            time.sleep(0.02)
            for r in batch:
                r.t_start = r.t_end = time.perf_counter()
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


@pytest.mark.gpu
def test_same_answer_alone_and_in_the_mix(cuda_device):
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
    srv = serving.SolveServer(hbm_budget_bytes=8 << 30, workers=3, max_batch=8)
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
