#!/usr/bin/env python
"""Wilson-CG solves/s at 1e-10 true relative residual on one node.

Workload (the reference's GPU-method configuration): D=4 SU(3) 16^4,
kappa=0.13, links U = reunit(exp(i 0.25 H)) with H traceless Hermitian
(complex entries of unit variance), antiperiodic time boundary for the
fermions, sources unit complex Gaussian.  One step = one batched solve of
``--nrhs`` right-hand sides D x_i = b_i by the even-odd CG with norm-scaled
FP16 inner iterations and FP64 reliable updates, each answer verified by its
FP64 true residual.  The plain FP64 even-odd CG, one solve at a time, is
timed in the same run.  Inputs (nrhs x 12.6 MB of sources plus as much of
solutions) are larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lym|reference]

Multi-GPU: replicas only (independent solves per rank, no collective on the
data path); the value is the whole-job solves/s.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GEOMETRY = (16, 16, 16, 16)
NC = 3
KAPPA = 0.13
BETA = 5.6
EPS = 0.25
TOL = 1e-10
METRIC = "Wilson-CG solves/s at 1e-10 true relative residual"
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the solver hop
# (16^4, 16 rhs, L2 cold), keyed by (precision, nrhs, hop form, tile, compressed links);
# captured once per kernel change, the capture's summary is the file named here
STORED_TRAFFIC_FILE = "profiles/dslash_eo_f16_16x16x16x16_traffic.txt"
STORED_TRAFFIC = {("f16", 16, 1, 1, False): 40031488.0}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lym", choices=["lym", "reference"])
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--precision", default="f16", choices=["f64", "f32", "f16", "bf16"])
    ap.add_argument("--plain-solves", type=int, default=4)
    ap.add_argument("--cpu-sample", type=int, default=16,
                    help="MMMR steps of the CPU baseline's timed sample (GPU arm)")
    ap.add_argument("--ref-sample", type=int, default=4, help="MMMR steps per --impl reference step")
    ap.add_argument("--ref-max-steps", type=int, default=3000, help="MMMR step cap of the reference's whole solve")
    ap.add_argument("--step-requests", type=int, default=128,
                    help="single-rhs requests per timed step of the headline (served in batches of --nrhs)")
    ap.add_argument("--repeats", type=int, default=3, help="timed regions of the headline; value = their median")
    ap.add_argument("--delta", type=float, default=0.01, help="reliable-update trigger of the mixed solver")
    ap.add_argument("--chunk", type=int, default=8, help="CG iterations per CUDA graph launch")
    ap.add_argument("--workers", type=int, default=2, help="solve-server worker streams")
    ap.add_argument("--max-batch", type=int, default=0, help="solve-server batch limit in rhs (0: --nrhs)")
    ap.add_argument("--rhs-per-thread", type=int, default=0, help="hop-kernel tile (0: autotune)")
    ap.add_argument("--compressed-links", type=int, default=0, help="with a forced tile: 1 = N-1-row links")
    ap.add_argument("--mixed-fma", type=int, default=0,
                    help="with a forced tile and f16: 1 = the mixed-precision hop (f16 x f16 + f32 FMAs), "
                         "2 = the tensor-core hop (--rhs-per-thread 16), 3 = the packed-half hop, "
                         "4 = form 1 with arithmetic neighbours, 5 = form 4 with the t neighbours by warp shuffle")
    ap.add_argument("--dslash-sweep", action="store_true",
                    help="dslash throughput sweep at 16^4 and 32^4 (one JSON line per case), no solve timing")
    ap.add_argument("--hmc", action="store_true",
                    help="HMC trajectories/hour on 16^4 SU(3) (beta 5.6, kappa 0.13, Nf=2 Wilson, Omelyan "
                         "[10, 2], t = 1, even-odd CG at 1e-10): one JSON line, no solve timing")
    ap.add_argument("--trajectories", type=int, default=5)
    ap.add_argument("--hmc-inner", type=int, default=2, help="gauge steps per fermion step of the integrator")
    ap.add_argument("--hmc-outer", type=int, default=10, help="fermion steps per trajectory of the integrator")
    ap.add_argument("--batch-precision", default="f32", choices=["f32", "f16"],
                    help="inner precision of --batch-lattices (FP64 reliable updates either way)")
    ap.add_argument("--hmc-precision", default="f64", choices=["f64", "f32", "f16", "bf16"],
                    help="inner precision of the HMC's CG solves (f64: the plain FP64 method)")
    ap.add_argument("--serve-sweep", action="store_true",
                    help="serving under an open-loop Poisson stream of mixed requests (D, N, geometry, kappa, "
                         "rhs count, shifts, tolerance, gauge reuse), one JSON line per rate, then the same "
                         "requests as plain FP64 one-at-a-time solves")
    ap.add_argument("--batch-lattices", action="store_true",
                    help="64 independent lattices of uneven geometry, 4 rhs each, solved together through the "
                         "solve server (FP32 inner / FP64 outer, 1e-10), plus one gauge HMC step per lattice; "
                         "one JSON line")
    ap.add_argument("--precision-study", action="store_true",
                    help="24^3x48 SU(3), eps 0.3, kappa 0.12 and 0.13, 8 rhs: the even-odd CG with FP64 / FP32 / "
                         "FP16 / BF16 inner iterations against the FP64 solution, the full-lattice FP64 multishift CG "
                         "and the even-odd multishift CG in four inner precisions on Q^2 + sigma_k with the "
                         "reference's 17-pole rational approximation; one JSON line per case")
    ap.add_argument("--multishift", action="store_true",
                    help="24^3x48 SU(3), eps 0.3: the even-odd multishift CG on Q^2 + sigma_k with the reference's "
                         "17 metropolis shifts, --ms-rhs sources in one call, for every --ms-precisions x "
                         "--ms-switch; one JSON line per case")
    ap.add_argument("--kappa", type=float, default=0.13, help="hopping parameter of --multishift")
    ap.add_argument("--poles", default="zolotarev12", choices=["zolotarev12", "reference17"],
                    help="shifts of --multishift / --precision-study: the 12 poles of x^(-1/2) on [1e-4, 1] or the "
                         "reference's 17 metropolis shifts")
    ap.add_argument("--ms-rhs", type=int, default=8, help="sources of --multishift")
    ap.add_argument("--ms-precisions", default="f64,f32,f16,bf16", help="inner precisions of --multishift")
    ap.add_argument("--ms-switch", default="0",
                    help="FP64-head switch residuals of --multishift (0: the library default, <0: no head)")
    ap.add_argument("--serve-rates", default="20,100,400", help="request rates (per second) of --serve-sweep")
    ap.add_argument("--serve-max-queue", type=int, default=2000,
                    help="solve server: requests that find this many queued are rejected (overload shedding)")
    ap.add_argument("--serve-max-wait", type=float, default=1.0,
                    help="solve server: requests whose expected wait exceeds this many seconds are rejected "
                         "(overload shedding by latency; <= 0: no limit)")
    ap.add_argument("--serve-release", default="inline", choices=["async", "inline"],
                    help="solve server: evicted gauge fields released on a background thread or by the worker")
    ap.add_argument("--serve-plain", type=int, default=1,
                    help="--serve-sweep: 1 = end with the plain FP64 one-at-a-time pass at the lowest rate")
    ap.add_argument("--serve-multi", type=int, default=1,
                    help="solve server: batches on up to this many different gauge fields of one class run as one "
                         "multi-lattice solve (<= 1: each batch on its own)")
    ap.add_argument("--serve-shifted", default="f64", choices=["full", "f64", "f32", "f16"],
                    help="solver of --serve-sweep's shifted requests: the full-lattice FP64 multishift, or the "
                         "even-odd multishift with that inner precision")
    ap.add_argument("--serve-seconds", type=float, default=6.0, help="arrival window per rate")
    ap.add_argument("--serve-max-requests", type=int, default=600)
    ap.add_argument("--sweep-tiles", action="store_true",
                    help="with --dslash-sweep: also every forced hop tile at 16 right-hand sides")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: one short solve, then 3 solver dslash launches inside the NVTX "
                         "range 'dslash' (select them with ncu --nvtx --nvtx-include dslash/), no timing")
    return ap.parse_args()


def host_links(seed):
    """H per link (nd, V, N, N): traceless Hermitian, complex entries of unit variance."""
    rng = np.random.default_rng(seed)
    nd, vol = len(GEOMETRY), int(np.prod(GEOMETRY))
    a = rng.normal(size=(nd, vol, NC, NC)) + 1j * rng.normal(size=(nd, vol, NC, NC))
    h = (a + np.conj(np.swapaxes(a, -1, -2))) / 2
    tr = np.trace(h, axis1=-2, axis2=-1) / NC
    h = h - tr[..., None, None] * np.eye(NC)
    return h


def host_sources(seed, n):
    rng = np.random.default_rng(seed)
    vol = int(np.prod(GEOMETRY))
    return (rng.normal(size=(n, 4, NC, vol)) + 1j * rng.normal(size=(n, 4, NC, vol))) / np.sqrt(2)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own solve path, restated in the oracle, on the
# host's threads
# ---------------------------------------------------------------------------
def host_threads():
    return max(1, len(os.sched_getaffinity(0)))


def host_exp_links(seed):
    """The links of the GPU arm on the host: exp(i eps H) for the same H, by
    eigendecomposition (the GPU arm's Cayley-Hamilton exponential followed by
    reunitarisation gives the same SU(3) links up to rounding); (nd, N, N, V)."""
    h = host_links(seed)
    w, v = np.linalg.eigh(h)
    u = np.einsum("...ik,...k,...jk->...ij", v, np.exp(1j * EPS * w), np.conj(v))
    return np.ascontiguousarray(np.transpose(u, (0, 2, 3, 1)))


class HostWilson:
    """The oracle's restatement of the reference's Wilson operator (dirac.py:458-523,
    649-662) with every apply split over `threads` host threads by output sites
    (numpy releases the GIL inside its kernels), as TensorFlow's intra-op threads
    split the reference's einsums."""

    def __init__(self, seed, threads):
        from concurrent.futures import ThreadPoolExecutor

        from oracle import lym_oracle as O
        self.O = O
        self.tables = O.lookup_tables(GEOMETRY)
        self.gauge = O.apply_time_bc(host_exp_links(seed), O.antiperiodic_field(GEOMETRY))
        vol = int(np.prod(GEOMETRY))
        self.chunks = np.array_split(np.arange(vol), threads)
        self.pool = ThreadPoolExecutor(threads)
        self.threads = threads

    def apply(self, v, hermitian):
        O = self.O
        parts = self.pool.map(lambda s: O.wilson_apply_sites(self.gauge, v, KAPPA, hermitian, self.tables, s),
                              self.chunks)
        return np.concatenate(list(parts), axis=-1)

    def close(self):
        self.pool.shutdown()


def host_mmmr(op, b, max_steps):
    """D x = b the reference's way: multishift_solver.solve (dirac_solver.py:19-53,
    oracle.mmmr_multishift) on SquareOperator(Q) (dirac.py:27-37), Q = gamma_d D, with
    source gamma_d b and the single shift 0, stopping at |<r,r>| < 1e-20 |b|^2 (true
    relative residual 1e-10); then x = Q y.  Returns (x, MMMR steps, converged, seconds)."""
    O = op.O
    precision = 1e-20 * float(np.vdot(b, b).real)
    t0 = time.perf_counter()
    ys, steps, conv = O.mmmr_multishift(lambda v: op.apply(op.apply(v, True), True), O.gamma_d(b), [0.0],
                                        max_steps, precision)
    x = op.apply(ys[0], True)
    return x, steps, conv, time.perf_counter() - t0


def host_mmmr_seconds_per_step(op, b, steps):
    """Seconds per MMMR step of host_mmmr, timed over `steps` steps (a bounded sample)."""
    O = op.O
    t0 = time.perf_counter()
    O.mmmr_multishift(lambda v: op.apply(op.apply(v, True), True), O.gamma_d(b), [0.0], steps, 0.0)
    return (time.perf_counter() - t0) / steps


def max_over_ranks(ms, world, device):
    """The slowest rank's time (every rank takes the same collective step)."""
    if world == 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, units_per_rank, max_ms):
    """Whole-job rate of `world` independent replicas: all units over the slowest rank's time."""
    return world * units_per_rank / (max_ms / 1e3)


def workload_config(args, world):
    """The workload both arms report (the reference arm solves the same systems with
    the oracle port of the reference's algorithm on the host cores)."""
    return {"workload": "served wilson-eo-cg 16^4 SU(3) kappa=0.13 tol=1e-10", "geometry": list(GEOMETRY),
            "step": f"{args.step_requests} single-rhs requests", "max_batch_rhs": args.max_batch or args.nrhs,
            "server_workers": args.workers,
            "inner_precision": args.precision, "outer_precision": "f64",
            "reliable_update_delta": args.delta, "graph_chunk": args.chunk,
            "links": "reunit(exp(i 0.25 H)), H traceless Hermitian", "bc": "antiperiodic time",
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (the sources and solutions of the timed requests exceed 126 MB)"}


def run_reference(args, rank, world):
    """--impl reference: the reference's own algorithm for this solve (its MMMR
    multishift solver on Q^2 and its Wilson operator, restated in the oracle) on the
    host with all its threads, on the GPU arm's workload.  Each step times a bounded
    sample of --ref-sample MMMR steps; after the timed steps one whole solve runs to
    the 1e-10 true residual, which gives the MMMR step count per solve (and its
    wall time as a cross-check).  value = 1 / (seconds per MMMR step x steps per solve)."""
    if rank != 0:
        return 0
    threads = host_threads()
    op = HostWilson(1234, threads)
    b = host_sources(99, args.nrhs)[0]  # the GPU arm's first source
    per_step = []
    for step in range(args.warmup + args.steps):
        sec = host_mmmr_seconds_per_step(op, b, args.ref_sample)
        if step >= args.warmup:
            per_step.append(sec)
    x, steps, conv, full_s = host_mmmr(op, b, args.ref_max_steps)
    res = float(np.linalg.norm(b - op.apply(x, False)) / np.linalg.norm(b))
    op.close()
    executed = steps + 1
    sec_step = statistics.mean(per_step)
    value = 1.0 / (sec_step * executed)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec_step * args.ref_sample * 1e3,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic", "scaling": "weak", "vs_baseline": None,
        "config": workload_config(args, world),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"the reference's solve path (multishift_solver MMMR on SquareOperator(Q), shift "
                                   f"0, then x = Q y; dirac_solver.py:19-53, dirac.py:27-37,458-523) restated in "
                                   f"the oracle, each Wilson apply split over {threads} host threads; each step "
                                   f"times {args.ref_sample} MMMR steps ({sec_step:.3f} s per MMMR step), "
                                   f"extrapolated with the {executed} MMMR steps one whole solve took in this run "
                                   f"(true residual {res:.2e}, {full_s:.1f} s wall, converged={conv})"},
        "full_solve_s": full_s, "mmmr_steps_per_solve": executed, "true_residual": res,
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def _drop_solution(fut):
    if fut.exception() is None:
        fut.result().x = None


def run_lym(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from tfleonardym_b200 import _dev, _lib, boundary_conditions, dirac, dirac_solver, hmc
    from tfleonardym_b200 import lattice as lt

    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nd, vol = len(GEOMETRY), int(np.prod(GEOMETRY))
    # links: exp(i eps H) via the link-update kernel from unit links, reunitarised
    h = host_links(1234 + rank)
    p = torch.from_numpy(np.ascontiguousarray(np.transpose(1j * h, (0, 2, 3, 1)))).to(dev)
    ident = torch.zeros((nd, NC, NC, vol), dtype=torch.complex128, device=dev)
    for i in range(NC):
        ident[:, i, i] = 1
    links = hmc.update_link_field(ident, p, EPS, reunitarize=True)
    cfg = lt.Configuration(links, GEOMETRY, NC, nd)
    op = dirac.DiracWilsonOperator(cfg, KAPPA, False, representation="fundamental",
                                   boundary_condition_provider=boundary_conditions.time_antiperiodic_provider(-1))
    B = args.nrhs
    b_host = torch.from_numpy(host_sources(99 + rank, B)).pin_memory()
    b_dev = b_host.to(dev)
    mixed = dirac_solver.conjugate_gradient(max_steps=2000, tol=TOL, precision=args.precision, chunk=args.chunk,
                                            delta=args.delta, rhs_per_thread=args.rhs_per_thread,
                                            mixed_fma=args.mixed_fma,
                                            compressed_links=args.compressed_links)
    plain = dirac_solver.conjugate_gradient(max_steps=2000, tol=TOL, precision="f64", chunk=8)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    if args.profile:
        short = dirac_solver.conjugate_gradient(max_steps=16, tol=TOL, precision=args.precision, chunk=8,
                                                delta=args.delta, rhs_per_thread=max(1, args.rhs_per_thread),
                                                mixed_fma=args.mixed_fma,
                                                compressed_links=args.compressed_links)
        short.solve(op, b_dev)  # builds the workspace; stops early on purpose
        gauge = op.solver_gauge((args.precision,))
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("dslash")
        _lib.check(_lib.lib().lym_dslash_eo(gauge, _lib.PREC[args.precision], B, 3, _dev.stream()), "lym_dslash_eo")
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        if rank == 0:
            print(json.dumps({"profile": "dslash", "precision": args.precision, "nrhs": B,
                              "rhs_per_thread": short.reports[0]["rhs_per_thread"],
                              "mixed_fma": short.reports[0]["mixed_fma"],
                              "compressed_links": short.reports[0]["compressed_links"]}), flush=True)
        return 0

    def check(reports):
        bad = [r for r in reports if r["status"] != 0 or r["true_residual"] > TOL]
        if bad:
            raise RuntimeError(f"solve missed the tolerance: {bad[:2]}")

    # warm-up (also builds the graphs and workspaces)
    for _ in range(max(args.warmup, 3)):
        mixed.solve(op, b_dev)
        check(mixed.reports)
    plain.solve(op, b_dev[0])
    check(plain.reports)
    torch.cuda.synchronize()

    # ---- timed region: served mixed-precision solves ----
    # a burst of steps x nrhs single-right-hand-side requests through the solve
    # server (continuous batching, up to nrhs per batch); sources resident
    from tfleonardym_b200 import serving
    budget = int(0.8 * torch.cuda.get_device_properties(dev).total_memory)
    srv = serving.SolveServer(budget, max_batch=args.max_batch or B, workers=args.workers, device=local_rank,
                              solver_options=dict(delta=args.delta, chunk=args.chunk,
                                                  rhs_per_thread=args.rhs_per_thread,
                                                  mixed_fma=args.mixed_fma,
                                                  compressed_links=args.compressed_links))

    x_host = torch.empty_like(b_host).pin_memory()

    def served(nreq, src, rate=None):
        futs = []
        host = not src.is_cuda
        for i in range(nreq):
            if rate:
                # inter-arrival gaps capped at 50 ms: never binding at the measured
                # rates (hundreds per second), it bounds the phase under a profiler
                time.sleep(min(0.05, float(np.random.default_rng(i).exponential(1.0 / rate))))
            f = srv.submit(serving.SolveRequest("bench", GEOMETRY, NC, KAPPA, src[i % B], gauge=links,
                                                tol=TOL, precision=args.precision, bc=-1.0,
                                                max_iter=2000, out=x_host[i % B] if host else None))
            # a client that has taken its answer drops it: the solution's device memory
            # returns to the allocator as soon as its batch is done
            f.add_done_callback(_drop_solution)
            futs.append(f)
        res = [f.result() for f in futs]
        bad = [r for r in res if r.status != serving.OK]
        if bad:
            raise RuntimeError(f"served solve missed the tolerance: {bad[0].reports}")
        return res

    served(2 * B * args.workers, b_dev)  # warm the server: gauge copies, workspaces, graphs, autotuning
    torch.cuda.synchronize()
    nstep = args.step_requests

    # --repeats timed regions of exactly --steps steps each (a step = --step-requests
    # single-rhs requests); value = the median region's rate
    clocks = ClockSampler(local_rank)
    clocks.start()
    regions = []
    for rep in range(max(1, args.repeats)):
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_wall = time.perf_counter()
        ev0.record(stream)
        # process-wide NVTX start/end range (covers the server's worker threads):
        # ncu --nvtx --nvtx-include timed selects the timed region's launches
        nvtx_timed = torch.cuda.nvtx.range_start("timed")
        res = served(args.steps * nstep, b_dev)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_end(nvtx_timed)
        ev1.record(stream)
        ev1.synchronize()
        barrier()
        t_wall = time.perf_counter() - t_wall
        ms = max_over_ranks(ev0.elapsed_time(ev1), world, dev)
        regions.append((replica_throughput(world, args.steps * nstep, ms), ms, t_wall, res))
    clk = clocks.stop()
    ordered = sorted(regions, key=lambda t: t[0])
    value, total_ms, t_wall, res = ordered[len(ordered) // 2]
    launches = sum(r.reports[0]["kernel_launches"] / r.batch_rhs for r in res)
    iters = [m["iterations"] for r in res for m in r.reports]
    rupd = [m["reliable_updates"] for r in res for m in r.reports]
    batch_sizes = sorted({r.batch_rhs for r in res})
    tuned = {k: res[-1].reports[0].get(k) for k in ("rhs_per_thread", "compressed_links", "mixed_fma")}

    # ---- latency: Poisson arrivals at half the saturated rate ----
    rate = 0.5 * value / world
    lat_res = served(4 * B, b_dev, rate=rate)
    lat = sorted(1e3 * r.latency for r in lat_res)

    # ---- end to end through the serving API with host buffers ----
    torch.cuda.synchronize()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(2, args.steps // 4)
    ev2.record(stream)
    served(e2e_steps * nstep, b_host)
    torch.cuda.synchronize()
    ev3.record(stream)
    ev3.synchronize()
    e2e_total = max_over_ranks(ev2.elapsed_time(ev3), world, dev)
    e2e_value = replica_throughput(world, e2e_steps * nstep, e2e_total)
    srv.close()

    # ---- the same solves as direct batched calls (no server) ----
    for _ in range(2):
        mixed.solve(op, b_dev)
    torch.cuda.synchronize()
    direct_ms = []
    x_mixed = None
    for _ in range(max(2, args.steps // 2)):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        x_mixed = mixed.solve(op, b_dev)
        e.record(stream)
        torch.cuda.synchronize()
        check(mixed.reports)
        direct_ms.append(s.elapsed_time(e))
    direct_value = B / (statistics.mean(direct_ms) / 1e3)

    # ---- plain FP64 one solve at a time ----
    plain_ms, plain_iters, mixed_vs_fp64 = [], [], []
    for i in range(args.plain_solves):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        x_plain = plain.solve(op, b_dev[i % B])
        e.record(stream)
        torch.cuda.synchronize()
        check(plain.reports)
        plain_ms.append(s.elapsed_time(e))
        plain_iters.append(plain.reports[0]["iterations"])
        # the mixed-precision solution's distance from the FP64 one (same rhs)
        mixed_vs_fp64.append(float(torch.linalg.vector_norm(x_mixed[i % B] - x_plain) /
                                   torch.linalg.vector_norm(x_plain)))
    plain_value = 1e3 / statistics.mean(plain_ms)

    # ---- roofline: the solver's dslash timed alone, L2 flushed between launches ----
    gauge = op.solver_gauge((args.precision,))
    prec = _lib.PREC[args.precision]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    durs = []
    for i in range(20):
        flush.add_(1.0)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        _lib.check(_lib.lib().lym_dslash_eo(gauge, prec, B, 1, _dev.stream()), "lym_dslash_eo")
        e.record(stream)
        torch.cuda.synchronize()
        if i >= 3:
            durs.append(s.elapsed_time(e) / 1e3)
    hop_s = statistics.mean(durs)
    ns_, spin_reals = 4, 2 * 4 * NC
    bs = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}[args.precision]
    spinor_bytes = spin_reals * bs + (4 if args.precision in ("f16", "bf16") else 0)
    # links as the tuned kernel reads them: N-1 rows (12 reals for SU(3)) or the full 18
    rep0 = mixed.reports[0]
    comp = bool(rep0["compressed_links"])
    link_bytes = ((12 if NC == 3 else 4) if comp else 2 * NC * NC) * bs
    algo_bytes = B * (vol // 2) * 2 * spinor_bytes + nd * vol * link_bytes
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = algo_bytes / hop_s / 1e9
    kind = {0: "FP32-arithmetic", 1: "mixed-precision (f16 x f16 + f32 FMA)", 2: "tensor-core (mma.sync f16, f32 accum)",
            3: "packed-half (half2 FMA per direction, f32 accum)",
            4: "mixed-precision (f16 x f16 + f32 FMA), arithmetic neighbours",
            5: "mixed-precision (f16 x f16 + f32 FMA), arithmetic neighbours, t neighbours by warp shuffle"}
    traffic = STORED_TRAFFIC.get((args.precision, B, rep0["mixed_fma"], rep0["rhs_per_thread"], comp))

    # ---- CPU baseline (rank 0, N = 1 only): the reference's solve path on the host ----
    cpu = None
    if rank == 0 and world == 1:
        # MMMR steps per solve of this workload, from the reference's algorithm on the
        # device (lym_mmmr_solve: multishift_solver's arithmetic in its order)
        q_op = dirac.DiracWilsonOperator(cfg, KAPPA, True, representation="fundamental",
                                         boundary_condition_provider=boundary_conditions.time_antiperiodic_provider(-1))
        b0 = b_dev[0]
        mmmr = dirac_solver.multishift_solver(args.ref_max_steps, 1e-20 * float(torch.vdot(b0.flatten(),
                                                                                          b0.flatten()).real))
        g5b = b0.clone()
        g5b[2:] *= -1
        y = mmmr.solve(dirac.SquareOperator(q_op), g5b, [0.0])[0]
        mres = float(torch.linalg.vector_norm(b0 - op.apply(q_op.apply(y))) / torch.linalg.vector_norm(b0))
        executed = mmmr.last_steps + 1
        threads = host_threads()
        hop_cpu = HostWilson(1234 + rank, threads)
        sec_step = host_mmmr_seconds_per_step(hop_cpu, host_sources(99 + rank, B)[0], args.cpu_sample)
        hop_cpu.close()
        cpu = {"value": 1.0 / (sec_step * executed), "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"the reference's solve path (multishift_solver MMMR on SquareOperator(Q), shift 0, then "
                         f"x = Q y; dirac_solver.py:19-53, dirac.py:27-37,458-523) restated in the oracle, each "
                         f"Wilson apply split over {threads} host threads: {args.cpu_sample} MMMR steps timed "
                         f"({sec_step:.3f} s each), extrapolated with the {executed} MMMR steps the same algorithm "
                         f"took on this workload on the device in this run (true residual {mres:.2e})"}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": f"{args.precision}+f64",
        "data": "synthetic",
        "config": workload_config(args, world),
        "repeats": {"values": [r[0] for r in regions], "median": value,
                    "spread": (ordered[-1][0] - ordered[0][0]) / value,
                    "timed_s": [r[1] / 1e3 for r in regions],
                    "what": f"{len(regions)} timed regions of {args.steps} steps x {nstep} requests; value = median"},
        "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                       "what": f"request latency, Poisson arrivals at {rate:.0f} req/s (half the saturated rate)"},
        "batch_rhs_seen": batch_sizes,
        "direct_batched": {"value": world * direct_value, "unit": "solves/s",
                           "what": f"lym_wilson_solve on {B} rhs per call, no server"},
        "plain_fp64": {"value": world * plain_value, "unit": "solves/s", "ms_per_solve": statistics.mean(plain_ms),
                       "iterations": plain_iters},
        "speedup_vs_plain_fp64": value / (world * plain_value),
        "mixed_vs_fp64": {"max_rel_diff": max(mixed_vs_fp64), "rhs": len(mixed_vs_fp64),
                          "what": "|x_mixed - x_fp64| / |x_fp64| per rhs, both solved to true residual 1e-10"},
        "iterations_per_solve": {"mean": statistics.mean(iters), "max": max(iters),
                                 "reliable_updates_mean": statistics.mean(rupd)},
        "autotuned": tuned,
        "gpu_launches": int(launches),
        "e2e": {"value": e2e_value, "unit": "solves/s",
                "h2d_bytes_per_step": int(nstep * b_host[0].numel() * 16),
                "d2h_bytes_per_step": int(nstep * b_host[0].numel() * 16),
                "what": "the served path with pinned host sources; solutions come back to host memory"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "traffic_source": (f"stored: ncu dram__bytes of one launch of this kernel and tile "
                                        f"({STORED_TRAFFIC_FILE})") if traffic else None,
                     "kernel": f"solver hop 4D SU(3) {args.precision} s_o = H_oe p_e, {B} rhs, "
                               f"{kind.get(rep0['mixed_fma'], '')} "
                               f"{'rhs per CTA' if rep0['mixed_fma'] == 2 else 'rhs per thread'} "
                               f"{rep0['rhs_per_thread']}, {'compressed' if comp else 'full'} links, "
                               f"L2 flushed before each launch",
                     "algorithmic_bytes_per_launch": algo_bytes, "launch_us": hop_s * 1e6,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy), of measured" if peaks
                     else "fallback 6650 GB/s"},
        "clocks": clk,
        "wall_s_timed": t_wall,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_dslash_sweep(args, local_rank):
    """Dslash throughput against the HBM roofline at 16^4 and 32^4.

    Cases: the reference-layout FP64 Wilson operator (lym_wilson_apply_batch) and
    the solver's even-odd hop (lym_dslash_eo) in FP64 / FP32 / FP16 at 1 and 16
    right-hand sides.  Each is timed with CUDA events over 20 launches, once with
    a 256 MB write between launches (L2 flushed: DRAM-bound) and once back to back
    (L2-warm).  Achieved = algorithmic bytes per launch / mean duration (bytes as
    in the kernel table of the design notes: every field touched once per launch).
    """
    import torch

    from tfleonardym_b200 import _dev, _lib, boundary_conditions, dirac, dirac_solver, hmc
    from tfleonardym_b200 import lattice as lt
    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn, cold):
        durs = []
        for i in range(23):
            if cold:
                flush.add_(1.0)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            torch.cuda.synchronize()
            if i >= 3:
                durs.append(s.elapsed_time(e) / 1e3)
        return statistics.mean(durs)

    flops_site = 1320
    for geom in ((16, 16, 16, 16), (32, 32, 32, 32)):
        nd, vol = len(geom), int(np.prod(geom))
        rng = np.random.default_rng(7)
        a = rng.normal(size=(nd, vol, NC, NC)) + 1j * rng.normal(size=(nd, vol, NC, NC))
        h = (a + np.conj(np.swapaxes(a, -1, -2))) / 2
        h = h - (np.trace(h, axis1=-2, axis2=-1) / NC)[..., None, None] * np.eye(NC)
        p = torch.from_numpy(np.ascontiguousarray(np.transpose(1j * h, (0, 2, 3, 1)))).to(dev)
        del a, h
        ident = torch.zeros((nd, NC, NC, vol), dtype=torch.complex128, device=dev)
        for i in range(NC):
            ident[:, i, i] = 1
        links = hmc.update_link_field(ident, p, EPS, reunitarize=True)
        del p, ident
        op = dirac.DiracWilsonOperator(lt.Configuration(links, geom, NC, nd), KAPPA, False,
                                       representation="fundamental",
                                       boundary_condition_provider=boundary_conditions.time_antiperiodic_provider(-1))
        ns = 4
        spin = ns * NC * 16
        # full-lattice FP64 operator: in + out spinors, every link once, the int32 sup/sdn tables
        for nvec in (1, 4):
            x = torch.randn((nvec, ns, NC, vol), dtype=torch.complex128, device=dev)
            y = torch.empty_like(x)
            algo = nvec * vol * 2 * spin + vol * nd * NC * NC * 16 + vol * 2 * nd * 4
            for cold in (True, False):
                t = timed(lambda: _lib.check(_lib.lib().lym_wilson_apply_batch(
                    op.lattice.handle, NC, KAPPA, 0, -1.0, 0.0, _dev.ptr(op.fermion_gauge_field), nvec, _dev.ptr(x),
                    _dev.ptr(y), _dev.stream()), "apply"), cold)
                print(json.dumps({"dslash_sweep": "wilson_full_kernel f64 reference layout", "geometry": list(geom),
                                  "nrhs": nvec, "l2": "flushed" if cold else "warm", "us": t * 1e6,
                                  "algorithmic_bytes": algo, "gbs": algo / t / 1e9, "frac_hbm": algo / t / 1e9 / peak,
                                  "gflops": nvec * vol * (flops_site + 4 * ns * NC) / t / 1e9}), flush=True)
            del x, y
        # (rhs per thread, compressed links, mixed-precision FP16 hop); None: the autotuner's pick
        # (rhs per CTA, 0, 2): the tensor-core FP16 hop; (1, 0, 3): the packed-half FP16 hop;
        # (R, 0, 4): the mixed-precision hop with arithmetic neighbours
        forced = [None, (1, 0, 0), (1, 1, 0), (2, 0, 0), (4, 0, 0), (1, 0, 1), (2, 0, 1), (4, 0, 1),
                  (4, 0, 2), (8, 0, 2), (16, 0, 2), (1, 0, 3), (1, 0, 4), (2, 0, 4), (4, 0, 4), (1, 0, 5), (2, 0, 5)]
        for prec, nrhs in (("f64", 1), ("f32", 1), ("f16", 1), ("f32", 16), ("f16", 16)):
            b = torch.randn((nrhs, ns, NC, vol), dtype=torch.complex128, device=dev)
            tiles = [None]
            if nrhs == 16 and args.sweep_tiles:
                tiles = [t for t in forced if t is None or prec == "f16" or not t[2]]
            for tile in tiles:
                kw = {} if tile is None else dict(rhs_per_thread=tile[0], compressed_links=tile[1],
                                                  mixed_fma=tile[2])
                short = dirac_solver.conjugate_gradient(max_steps=4, tol=TOL, precision=prec, **kw)
                short.solve(op, b)
                rep = short.reports[0]
                gauge = op.solver_gauge((prec,) if prec != "f64" else ())
                bs = {"f64": 8, "f32": 4, "f16": 2}[prec]
                sbytes = 2 * ns * NC * bs + (4 if prec == "f16" else 0)
                if prec == "f64":
                    lbytes = 18 * 8
                else:
                    lbytes = (12 if rep["compressed_links"] else 18) * bs
                algo = nrhs * (vol // 2) * 2 * sbytes + nd * vol * lbytes
                for cold in (True, False):
                    t = timed(lambda: _lib.check(_lib.lib().lym_dslash_eo(gauge, _lib.PREC[prec], nrhs, 1,
                                                                          _dev.stream()), "dslash"), cold)
                    print(json.dumps({"dslash_sweep": f"cg_hop_kernel even-odd {prec}", "geometry": list(geom),
                                      "nrhs": nrhs, "tile": "autotuned" if tile is None else "forced",
                                      "rhs_per_thread": rep["rhs_per_thread"],
                                      "mixed_fma": rep["mixed_fma"],
                                      "tensor_core": rep["mixed_fma"] == 2,
                                      "compressed_links": rep["compressed_links"],
                                      "l2": "flushed" if cold else "warm",
                                      "us": t * 1e6, "algorithmic_bytes": algo, "gbs": algo / t / 1e9,
                                      "frac_hbm": algo / t / 1e9 / peak,
                                      "gflops": nrhs * (vol // 2) * flops_site / t / 1e9}), flush=True)
            del b
        del op, links
        torch.cuda.empty_cache()
    # on-disk gauge format: device decode of the XDR link section at 32^4 (read 48 B,
    # write 144 B per link), beside the oracle's numpy decode of an 8^4 sample on one core
    geom = (32, 32, 32, 32)
    nd, vol = 4, 32 ** 4
    rng = np.random.default_rng(5)
    words_h = rng.normal(size=vol * nd * 12).astype(">f4")
    words = torch.from_numpy(np.frombuffer(words_h.tobytes(), dtype=np.uint8).copy()).to(dev)
    gauge = torch.empty((nd, 3, 3, vol), dtype=torch.complex128, device=dev)
    algo = vol * nd * (48 + 144)
    t = timed(lambda: _lib.check(_lib.lib().lym_decode_xdr_gauge(nd, 3, vol, _dev.ptr(words), _dev.ptr(gauge),
                                                                 _dev.stream()), "xdr"), True)
    from oracle import lym_oracle as O
    small = 8 ** 4
    raw_small = np.frombuffer(words_h[:small * nd * 12].tobytes() + bytes(4 * nd + 24), dtype=np.uint8)
    t0 = time.perf_counter()
    O.read_config_xdr(raw_small, (8, 8, 8, 8))
    cpu_s = (time.perf_counter() - t0) * vol / small
    print(json.dumps({"dslash_sweep": "xdr_su3_decode (lattice.read_config)", "geometry": list(geom), "nrhs": 0,
                      "l2": "flushed", "us": t * 1e6, "algorithmic_bytes": algo, "gbs": algo / t / 1e9,
                      "frac_hbm": algo / t / 1e9 / peak,
                      "cpu_oracle_us_scaled": cpu_s * 1e6,
                      "cpu_sample": "oracle numpy decode of an 8^4 sample on one core, scaled by volume"}),
          flush=True)
    return 0


# ---------------------------------------------------------------------------
# serving under a mixed open-loop request stream
# ---------------------------------------------------------------------------
def _device_links(geometry, nc, eps, seed, dev):
    """reunit(exp(i eps H)) links with H traceless Hermitian from the request seed, on the device."""
    import torch

    from tfleonardym_b200 import hmc
    nd, vol = len(geometry), int(np.prod(geometry))
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    a = torch.complex(torch.randn((nd, nc, nc, vol), generator=g, device=dev, dtype=torch.float64),
                      torch.randn((nd, nc, nc, vol), generator=g, device=dev, dtype=torch.float64))
    h = (a + torch.conj(a.transpose(1, 2))) / 2
    tr = torch.diagonal(h, dim1=1, dim2=2).sum(-1) / nc  # (nd, vol)
    for i in range(nc):
        h[:, i, i] -= tr
    ident = torch.zeros_like(h)
    for i in range(nc):
        ident[:, i, i] = 1
    return hmc.update_link_field(ident, 1j * h, eps, reunitarize=True)


def _request_specs(rng, n, max_bytes=2 << 30):
    """Mixed requests: D in {2, 3, 4}, N in {2, 3}, extents log-uniform between 8 and 24
    (space) / 48 (time) in 4D, between 8 and 96 in 3D and between 8 and 816 in 2D (even),
    footprint <= 2 GB; kappa in [0.10, 0.14]; 1-16 rhs or (half of the 2D / 4D requests)
    one rhs with 12 shifts log-spaced in [1e-4, 1] (3D has no hermitian Q, so no Q^2
    shifts); tol log-uniform in [1e-12, 1e-8]; eps in [0.1, 0.4]; 30% reuse one of the
    last 8 gauge fields."""
    from tfleonardym_b200 import serving
    specs, recent = [], []
    for i in range(n):
        if recent and rng.uniform() < 0.3:
            key, geom, nc, eps, seed = recent[int(rng.integers(len(recent)))]
        else:
            while True:
                nd = int(rng.choice([2, 3, 4]))
                nc = int(rng.choice([2, 3]))
                if nd == 4:
                    geom = tuple(2 * int(round(np.exp(rng.uniform(np.log(8), np.log(hi))) / 2))
                                 for hi in (24, 24, 24, 48))
                elif nd == 3:
                    geom = tuple(2 * int(round(np.exp(rng.uniform(np.log(8), np.log(96))) / 2)) for _ in range(3))
                else:
                    geom = tuple(2 * int(round(np.exp(rng.uniform(np.log(8), np.log(816))) / 2)) for _ in range(2))
                if serving.footprint_bytes(geom, nc, 16, "f16") <= max_bytes:
                    break
            eps, seed = float(rng.uniform(0.1, 0.4)), int(rng.integers(1 << 30))
            key = f"cfg{seed}"
            recent = (recent + [(key, geom, nc, eps, seed)])[-8:]
        shifted = len(geom) != 3 and rng.uniform() < 0.5
        specs.append(dict(key=key, geometry=geom, nc=nc, eps=eps, seed=seed, kappa=float(rng.uniform(0.10, 0.14)),
                          nrhs=1 if shifted else int(rng.integers(1, 17)),
                          shifts=list(np.logspace(-4, 0, 12)) if shifted else None,
                          tol=float(10 ** rng.uniform(-12, -8)), src_seed=int(rng.integers(1 << 30))))
    return specs


def _serve(specs, times, precision, workers, max_batch, dev, budget, shifted_precision="f64", multi_lattice=1,
           max_queue=None, max_wait_s=None, release="inline"):
    import torch

    from tfleonardym_b200 import serving
    srv = serving.SolveServer(budget, max_batch=max_batch, workers=workers, device=dev.index,
                              shifted_precision=shifted_precision, multi_lattice=multi_lattice, max_queue=max_queue,
                              max_wait_s=max_wait_s, release=release)
    futs = []
    t0 = time.perf_counter()
    for sp, t in zip(specs, times):
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        nd, vol = len(sp["geometry"]), int(np.prod(sp["geometry"]))
        ns = 4 if nd == 4 else 2
        shape = (sp["nrhs"], ns, sp["nc"], vol) if sp["shifts"] is None else (ns, sp["nc"], vol)

        def source(shape=shape, seed=sp["src_seed"]):
            # produced when the request runs, so that a backlog holds no source memory
            g = torch.Generator(device=dev)
            g.manual_seed(seed)
            return torch.complex(torch.randn(shape, generator=g, device=dev, dtype=torch.float64),
                                 torch.randn(shape, generator=g, device=dev, dtype=torch.float64)) / np.sqrt(2)

        gauge = (lambda s=sp: _device_links(s["geometry"], s["nc"], s["eps"], s["seed"], dev))
        f = srv.submit(serving.SolveRequest(sp["key"], sp["geometry"], sp["nc"], sp["kappa"], source, gauge=gauge,
                                            tol=sp["tol"], precision=precision, bc=-1.0, max_iter=4000,
                                            shifts=sp["shifts"], nrhs=sp["nrhs"]))
        f.add_done_callback(_drop_solution)
        futs.append(f)
    res = [f.result() for f in futs]
    wall = time.perf_counter() - t0
    srv.close()
    ok = [r for r in res if r.status == serving.OK]
    lat = sorted(1e3 * r.latency for r in res if r.status != serving.REJECTED)
    return {"requests": len(res), "ok": len(ok), "not_converged": sum(r.status == serving.NOT_CONVERGED for r in res),
            "rejected": sum(r.status == serving.REJECTED for r in res),
            "solves": int(sum(r.request.solves for r in ok)), "wall_s": wall,
            "solves_per_s": sum(r.request.solves for r in ok) / wall,
            "p50_ms": lat[len(lat) // 2] if lat else None,
            "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))] if lat else None,
            "max_true_residual_over_tol": max((m["true_residual"] / r.request.tol for r in res
                                               if r.status != serving.REJECTED for m in r.reports), default=None)}


def run_serve_sweep(args, local_rank):
    """Open-loop Poisson streams of mixed solve requests through the solve server at
    each rate of --serve-rates (arrivals over --serve-seconds, at most
    --serve-max-requests), inner precision FP16 for unshifted requests (shifted ones
    run the even-odd multishift CG in --serve-shifted's precision, FP64 by default, or
    with --serve-shifted full the full-lattice FP64 multishift), every answer checked
    by its FP64 true residual.
    Then the lowest rate's requests again as plain FP64 one-at-a-time solves (one
    worker, batches of one)."""
    import torch

    from tfleonardym_b200 import dirac_solver
    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    budget = int(0.8 * torch.cuda.get_device_properties(dev).total_memory)
    rates = [float(r) for r in args.serve_rates.split(",")]
    shifted = None if args.serve_shifted == "full" else args.serve_shifted
    warm = _request_specs(np.random.default_rng(1), 24)
    _serve(warm, [0.0] * len(warm), "f16", args.workers, args.nrhs, dev, budget, shifted, args.serve_multi)  # warm-up
    first = None
    for rate in rates:
        rng = np.random.default_rng(int(rate) + 7)
        times = np.cumsum(rng.exponential(1.0 / rate, size=args.serve_max_requests))
        times = times[times < args.serve_seconds]
        specs = _request_specs(rng, len(times))
        if first is None:
            first = (specs, times)
        max_wait = args.serve_max_wait if args.serve_max_wait > 0 else None
        r = _serve(specs, times, "f16", args.workers, args.nrhs, dev, budget, shifted, args.serve_multi,
                   args.serve_max_queue, max_wait, args.serve_release)
        print(json.dumps({"serve_sweep": "mixed", "rate_per_s": rate, "workers": args.workers,
                          "window_s": args.serve_seconds, "max_queue": args.serve_max_queue,
                          "max_wait_s": max_wait, "release": args.serve_release,
                          "max_batch_rhs": args.nrhs, "shifted_solver": args.serve_shifted,
                          "multi_lattice": args.serve_multi, **r}), flush=True)
    if not args.serve_plain:
        return 0
    specs, times = first
    r = _serve(specs, times, "f64", 1, 1, dev, budget, None, 1)  # plain: one request at a time, full-lattice multishift
    print(json.dumps({"serve_sweep": "plain_fp64_one_at_a_time", "rate_per_s": rates[0], **r}), flush=True)
    return 0


def run_batch_lattices(args, local_rank):
    """64 independent lattices -- thirds of 2D SU(2) from 8^2 to 64^2, 3D SU(2) from 8^3
    to 16^3 and 4D SU(3) from 8^4 to 12^3 x 24, kappa in [0.10, 0.14], links
    reunit(exp(i eps H)) with eps in
    [0.1, 0.4] -- with 4 unit complex Gaussian rhs each (256 solves), submitted
    together to the solve server (4 workers, one CUDA stream each) with FP32 (or
    --batch-precision) inner
    and FP64 outer iterations to true relative residual 1e-10; the same 256 solves
    with all lattices of one (D, N) class in the same launches
    (dirac_solver.solve_lattices, two calls).  Then the same 256
    solves as plain FP64 one-at-a-time solves, and one gauge HMC step on every lattice
    (staples and force fused into the momentum update, then the link update): lattice
    by lattice (128 launches), and all lattices together (lym_gauge_hmc_step_multi,
    two launches).
    Device time of each phase by CUDA events around it (the server's streams are
    joined by a device synchronise)."""
    import torch

    from tfleonardym_b200 import dirac_solver, gauge_action, hmc, serving
    from tfleonardym_b200 import lattice as lt
    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    rng = np.random.default_rng(44)
    lattices = []
    for i in range(64):
        if i % 3 == 0:
            n = int(2 * round(np.exp(rng.uniform(np.log(8), np.log(64))) / 2))
            m = int(2 * round(np.exp(rng.uniform(np.log(8), np.log(64))) / 2))
            geom, nc = (n, m), 2
        elif i % 3 == 1:
            geom, nc = tuple(int(rng.choice([8, 10, 12, 14, 16])) for _ in range(3)), 2
        else:
            geom = tuple(int(rng.choice([8, 10, 12])) for _ in range(3)) + (int(rng.choice([8, 12, 16, 20, 24])),)
            nc = 3
        lattices.append(dict(geometry=geom, nc=nc, kappa=float(rng.uniform(0.10, 0.14)),
                             eps=float(rng.uniform(0.1, 0.4)), seed=int(rng.integers(1 << 30))))
    gauges = [_device_links(l["geometry"], l["nc"], l["eps"], l["seed"], dev) for l in lattices]
    sources = []
    for l in lattices:
        nd, vol = len(l["geometry"]), int(np.prod(l["geometry"]))
        ns = 4 if nd == 4 else 2
        g = torch.Generator(device=dev)
        g.manual_seed(l["seed"] + 1)
        sources.append(torch.complex(torch.randn((4, ns, l["nc"], vol), generator=g, device=dev, dtype=torch.float64),
                                     torch.randn((4, ns, l["nc"], vol), generator=g, device=dev, dtype=torch.float64))
                       / np.sqrt(2))
    budget = int(0.8 * torch.cuda.get_device_properties(dev).total_memory)

    def solve_all(precision, workers, max_batch, multi_lattice=1):
        srv = serving.SolveServer(budget, max_batch=max_batch, workers=workers, device=local_rank,
                                  multi_lattice=multi_lattice)
        futs = []
        for k, l in enumerate(lattices):
            reqs = [sources[k]] if max_batch >= 4 else [sources[k][j] for j in range(4)]
            for b in reqs:
                futs.append(srv.submit(serving.SolveRequest(f"lat{k}", l["geometry"], l["nc"], l["kappa"], b,
                                                            gauge=gauges[k], tol=1e-10, precision=precision,
                                                            bc=-1.0, max_iter=4000)))
        res = [f.result() for f in futs]
        srv.close()
        return res

    bp = args.batch_precision
    solve_all(bp, 4, 16, args.serve_multi)  # warm-up: workspaces, autotuning, graphs
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = solve_all(bp, 4, 16, args.serve_multi)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ok = sum(r.status == serving.OK for r in res)
    worst = max(m["true_residual"] for r in res for m in r.reports)
    # the same 256 solves with every lattice of one (D, N) class in the same launches
    from tfleonardym_b200 import boundary_conditions, dirac
    prov = boundary_conditions.time_antiperiodic_provider(-1)
    ops = [dirac.DiracWilsonOperator(lt.Configuration(g, l["geometry"], l["nc"], len(l["geometry"])), l["kappa"],
                                     False, representation="fundamental", boundary_condition_provider=prov)
           for g, l in zip(gauges, lattices)]
    classes = {}
    for k, l in enumerate(lattices):
        classes.setdefault((len(l["geometry"]), l["nc"]), []).append(k)

    def solve_together():
        worst_m, launches = 0.0, 0
        for ks in classes.values():
            _, reps = dirac_solver.solve_lattices([ops[k] for k in ks], [sources[k] for k in ks], tol=1e-10,
                                                  precision=bp, delta=0.01)
            worst_m = max([worst_m] + [m["true_residual"] for r in reps for m in r])
            launches += reps[0][0]["kernel_launches"]
            ok_m = all(m["status"] == 0 for r in reps for m in r)
            if not ok_m:
                return worst_m, launches, False
        return worst_m, launches, True

    solve_together()  # warm-up: workspaces
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    worst_multi, multi_launches, multi_ok = solve_together()
    torch.cuda.synchronize()
    multi_wall = time.perf_counter() - t0
    solve_all("f64", 1, 1, 1)  # warm-up of the plain path
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = solve_all("f64", 1, 1, 1)
    torch.cuda.synchronize()
    plain_wall = time.perf_counter() - t0
    # one gauge HMC step per lattice: P += eps F (fused), U <- exp(eps P) U
    stream = torch.cuda.current_stream()
    cfgs = [lt.Configuration(g, l["geometry"], l["nc"], len(l["geometry"])) for g, l in zip(gauges, lattices)]
    moms = [hmc.random_momenta(l["nc"], len(l["geometry"]), int(np.prod(l["geometry"]))) for l in lattices]
    acts = [gauge_action.yang_mills(c, 5.6 if l["nc"] == 3 else 2.3) for c, l in zip(cfgs, lattices)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for rep in range(2):
        e0.record(stream)
        for c, p, a in zip(cfgs, moms, acts):
            p2 = hmc._kick(a, p, -0.05)
            hmc.update_link_field(c.gauge_field, p2, 0.05)
        e1.record(stream)
        torch.cuda.synchronize()
    per_lattice_ms = e0.elapsed_time(e1)
    betas = [5.6 if l["nc"] == 3 else 2.3 for l in lattices]
    for rep in range(3):
        e0.record(stream)
        hmc.gauge_step_lattices(cfgs, moms, betas, -0.05, 0.05)
        e1.record(stream)
        torch.cuda.synchronize()
    two_launch_ms = e0.elapsed_time(e1)
    print(json.dumps({"batch_lattices": "64 uneven lattices x 4 rhs", "solves": 256, "ok": ok,
                      "worst_true_residual": worst, "wall_s": wall, "solves_per_s": 256 / wall,
                      "one_launch_per_class": {"what": "lym_wilson_solve_multi: the lattices of each (D, N) class "
                                                       "(2D SU(2), 3D SU(2), 4D SU(3)) in one set of launches",
                                               "all_ok": multi_ok, "worst_true_residual": worst_multi,
                                               "wall_s": multi_wall, "solves_per_s": 256 / multi_wall,
                                               "kernel_launches": multi_launches},
                      "plain_fp64_one_at_a_time": {"ok": sum(r.status == serving.OK for r in plain),
                                                   "wall_s": plain_wall, "solves_per_s": 256 / plain_wall},
                      "gauge_hmc_step_all_lattices_ms": {"per_lattice_two_launches_each": per_lattice_ms,
                                                         "all_lattices_two_launches":
                                                         two_launch_ms},
                      "config": {"lattices": "22 x 2D SU(2) 8^2..64^2 + 21 x 3D SU(2) 8^3..16^3 + "
                                                 "21 x 4D SU(3) 8^4..12^3x24",
                                 "inner_precision": bp, "outer_precision": "f64", "tol": 1e-10,
                                 "server_workers": 4, "max_batch_rhs": 16,
                                 "server_multi_lattice": args.serve_multi}}), flush=True)
    return 0


# shifts of the reference's metropolis rational approximation: the second half of
# metropolis_rational_approximation_coefficients (approximations.py:127-139), which the
# reference's driver passes as the betas of RationalApproximation (TfLeonardYMNDim.py:326-332)
REFERENCE_17_POLES = [708.456969133708774250236839, 20.5545836704482543092111935, 5.16460586130848066092696251,
                      1.77335742461795338089518681, 0.663483773139054161068555408, 0.251260388600611110026798526,
                      0.0933210176761593454438480966, 0.0334329670158591978976640839,
                      0.0114225244703120473204264627, 0.00368309198965533868820332893,
                      0.00110757598877812519195949185, 0.000305911192767903423411472490,
                      0.0000759625965715284538520399041, 0.0000164241384694373051997536552,
                      0.00000293320679744054879906466158, 0.000000390128040236098295575734048,
                      0.0000000269253347571438797470449799]


def study_shifts(name):
    """(label, shifts) of the multishift studies: "zolotarev12" = the 12 poles of
    x^(-1/2) on [1e-4, 1] (approximations.inverse_sqrt_rational_approximation_coefficients),
    "reference17" = the reference's 17 metropolis shifts."""
    if name == "reference17":
        return "17 reference shifts", list(REFERENCE_17_POLES)
    from tfleonardym_b200 import approximations
    _, betas = approximations.split(approximations.inverse_sqrt_rational_approximation_coefficients)
    return "12 poles of x^(-1/2) on [1e-4, 1]", [float(x) for x in betas]


def _multishift_case(sq, q, b, prec, switch, ref, stream, shifts):
    """One timed even-odd multishift solve of all sources in b (after a warm-up
    solve) on `shifts`; returns (JSON-ready dict, solutions (rhs, shift, ...)).
    ref: FP64 solutions to compare with, or None."""
    import torch

    from tfleonardym_b200 import dirac_solver
    nrhs, nsh = b.shape[0], len(shifts)
    ms = dirac_solver.multishift_cg(20000, 1e-10, precision=prec, delta=0.01, switch_residual=switch)
    ms.solve(sq, b, shifts)  # warm-up: workspaces, graphs
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    xs = ms.solve(sq, b, shifts)
    e.record(stream)
    torch.cuda.synchronize()
    xs = torch.stack(xs, 1)  # (rhs, shift, ...)
    reps = ms.reports
    out = {"inner_precision": prec, "switch_residual": switch, "rhs": nrhs, "ms": s.elapsed_time(e),
           "ms_per_rhs": s.elapsed_time(e) / nrhs,
           "iterations_per_shift_max": [max(reps[i * nsh + k]["iterations"] for i in range(nrhs))
                                        for k in range(nsh)],
           "reliable_updates_max": max(r["reliable_updates"] for r in reps),
           "true_residual_per_shift_max": [max(reps[i * nsh + k]["true_residual"] for i in range(nrhs))
                                           for k in range(nsh)],
           "kernel_launches": reps[0]["kernel_launches"],
           "status_ok": all(r["status"] == 0 for r in reps)}
    # independent FP64 check of source 0 through the reference-layout operator
    bn = float(torch.linalg.vector_norm(b[0]))
    out["rhs0_reference_layout_residual_max"] = max(
        float(torch.linalg.vector_norm(b[0] - (q.apply(q.apply(xs[0, k])) + sg * xs[0, k]))) / bn
        for k, sg in enumerate(shifts))
    out["shifts"] = shifts
    if ref is not None:
        out["rel_diff_to_fp64_per_shift_max"] = [
            max(float(torch.linalg.vector_norm(xs[i, k] - ref[i, k]) / torch.linalg.vector_norm(ref[i, k]))
                for i in range(nrhs)) for k in range(nsh)]
    return out, xs


def _study_setup(dev, nrhs):
    """24^3 x 48 SU(3) links reunit(exp(i 0.3 H)) (seed 2026) and nrhs unit complex Gaussian sources (seed 7)."""
    import torch

    from tfleonardym_b200 import lattice as lt
    geom = (24, 24, 24, 48)
    vol = int(np.prod(geom))
    links = _device_links(geom, NC, 0.3, 2026, dev)
    cfg = lt.Configuration(links, geom, NC, 4)
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    b = torch.complex(torch.randn((nrhs, 4, NC, vol), generator=g, device=dev, dtype=torch.float64),
                      torch.randn((nrhs, 4, NC, vol), generator=g, device=dev, dtype=torch.float64)) / np.sqrt(2)
    return geom, cfg, b


def run_multishift(args, local_rank):
    """The even-odd multishift CG (lym_multishift_solve_eo) on 24^3 x 48 SU(3)
    (links reunit(exp(i 0.3 H)), antiperiodic time) at --kappa, the reference's
    17 metropolis shifts, --ms-rhs unit complex Gaussian sources in one call,
    for each inner precision and FP64-head switch residual: time (CUDA events,
    after a warm-up solve), iterations, the FP64 true residual of every (rhs,
    shift) and, after an FP64 case, each shift's largest relative difference
    to the FP64 solutions."""
    import torch

    from tfleonardym_b200 import boundary_conditions, dirac, dirac_solver
    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    geom, cfg, b = _study_setup(dev, args.ms_rhs)
    stream = torch.cuda.current_stream()
    prov = boundary_conditions.time_antiperiodic_provider(-1)
    q = dirac.DiracWilsonOperator(cfg, args.kappa, True, representation="fundamental",
                                  boundary_condition_provider=prov)
    sq = dirac.SquareOperator(q)
    label, shifts = study_shifts(args.poles)
    ref = None
    for prec in args.ms_precisions.split(","):
        for sw in (float(x) for x in args.ms_switch.split(",")):
            if prec == "f64" and sw != float(args.ms_switch.split(",")[0]):
                continue  # no head to switch from
            out, xs = _multishift_case(sq, q, b, prec, sw, ref, stream, shifts)
            if prec == "f64" and ref is None:
                ref = xs.clone()
            print(json.dumps({"multishift": f"even-odd multishift CG, {label}", "geometry": list(geom),
                              "kappa": args.kappa, **out}), flush=True)
    return 0


def run_precision_study(args, local_rank):
    """The precision study on 24^3 x 48 SU(3) (links
    reunit(exp(i 0.3 H)), antiperiodic time) at kappa 0.12 and 0.13, 8 unit complex
    Gaussian rhs: (a) the even-odd CG to true relative residual 1e-10 with FP64, FP32,
    FP16 and BF16 inner iterations (FP64 reliable updates), each solution's relative
    difference to the FP64 one; (b) the FP64 multishift CG on Q^2 + sigma_k (Q = gamma_d D)
    for the shifts of --poles (default: the 12 poles of x^(-1/2) on [1e-4, 1]), per-shift
    FP64 true residual; (c) the even-odd multishift CG on the same shifts, all 8 rhs in
    one call, inner iterations in FP64, FP32, FP16 and BF16 with FP64 reliable updates,
    each (rhs, shift) verified by its FP64 true residual, and each shift's largest
    relative difference to the FP64 solutions."""
    import torch

    from tfleonardym_b200 import boundary_conditions, dirac, dirac_solver
    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    geom, cfg, b = _study_setup(dev, 8)
    stream = torch.cuda.current_stream()
    prov = boundary_conditions.time_antiperiodic_provider(-1)
    for kappa in (0.12, 0.13):
        op = dirac.DiracWilsonOperator(cfg, kappa, False, representation="fundamental",
                                       boundary_condition_provider=prov)
        ref = None
        for prec in ("f64", "f32", "f16", "bf16"):
            solver = dirac_solver.conjugate_gradient(max_steps=20000, tol=1e-10, precision=prec, delta=0.01)
            solver.solve(op, b)  # warm-up: workspace, autotuning, graphs
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            x = solver.solve(op, b)
            e.record(stream)
            torch.cuda.synchronize()
            if ref is None:
                ref = x.clone()
            diff = [float(torch.linalg.vector_norm(x[i] - ref[i]) / torch.linalg.vector_norm(ref[i]))
                    for i in range(8)]
            print(json.dumps({"precision_study": "even-odd CG", "geometry": list(geom), "kappa": kappa,
                              "inner_precision": prec, "rhs": 8, "ms": s.elapsed_time(e),
                              "iterations": [r["iterations"] for r in solver.reports],
                              "reliable_updates": [r["reliable_updates"] for r in solver.reports],
                              "true_residual_max": max(r["true_residual"] for r in solver.reports),
                              "rel_diff_to_fp64_max": max(diff)}), flush=True)
        q = dirac.DiracWilsonOperator(cfg, kappa, True, representation="fundamental", boundary_condition_provider=prov)
        ms_cg = dirac_solver.multishift_cg(20000, 1e-10)
        sq = dirac.SquareOperator(q)
        label, shifts = study_shifts(args.poles)
        ms_cg.solve(sq, b[0], shifts)  # warm-up
        res, times, iters = [], [], []
        for i in range(2):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            xs = ms_cg.solve(sq, b[i], shifts)
            e.record(stream)
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
            iters.append(ms_cg.last_steps)
            bn = float(torch.linalg.vector_norm(b[i]))
            res.append([float(torch.linalg.vector_norm(b[i] - (q.apply(q.apply(x)) + sg * x))) / bn
                        for sg, x in zip(shifts, xs)])
        print(json.dumps({"precision_study": f"multishift CG FP64 (full lattice), {label}", "geometry": list(geom),
                          "kappa": kappa, "rhs": 2, "ms_per_rhs": statistics.mean(times), "iterations": iters,
                          "true_residual_per_shift_max": [max(r[k] for r in res) for k in range(len(shifts))]}),
              flush=True)
        # the even-odd multishift, all 8 sources in one call, inner precision swept;
        # errors per shift against its FP64 solutions
        ref_ms = None
        for prec in ("f64", "f32", "f16", "bf16"):
            out, xs = _multishift_case(sq, q, b, prec, 0.0, ref_ms, stream, shifts)
            if ref_ms is None:
                ref_ms = xs.clone()
            print(json.dumps({"precision_study": f"even-odd multishift CG, {label}", "geometry": list(geom),
                              "kappa": kappa, **out}), flush=True)
    return 0


def run_hmc(args, rank, world, local_rank):
    """HMC on 4D SU(3) 16^4: beta = 5.6, Nf = 2 Wilson fermions at kappa = 0.13
    (pseudofermion phi = Q eta, Q = gamma_d D, antiperiodic time), links
    reunit(exp(i 0.25 H)) to start, Gaussian su(3) momenta, Omelyan nested
    integrator with ``--hmc-outer`` (default 10) outer (fermion) steps and ``--hmc-inner`` (default 2)
    inner (gauge) steps per outer step, trajectory length 1, force and energy solves (Q^2)^-1 phi by two
    even-odd CG solves of Q at 1e-10 true relative residual.  One warm-up
    trajectory, then ``--trajectories`` timed with CUDA events; the value is
    trajectories per hour.  A reversibility check (forward then backward
    trajectory) follows the timed ones."""
    import torch

    from tfleonardym_b200 import (boundary_conditions, dirac, dirac_solver, fermion_action, gauge_action, hmc,
                                  measurements)
    from tfleonardym_b200 import lattice as lt
    dirac_solver.VERBOSE = False
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nd, vol = len(GEOMETRY), int(np.prod(GEOMETRY))
    h = host_links(1234 + rank)
    p = torch.from_numpy(np.ascontiguousarray(np.transpose(1j * h, (0, 2, 3, 1)))).to(dev)
    ident = torch.zeros((nd, NC, NC, vol), dtype=torch.complex128, device=dev)
    for i in range(NC):
        ident[:, i, i] = 1
    cfg = lt.Configuration(hmc.update_link_field(ident, p, EPS, reunitarize=True), GEOMETRY, NC, nd)
    del p, ident
    q = dirac.DiracWilsonOperator(cfg, KAPPA, True, representation="fundamental",
                                  boundary_condition_provider=boundary_conditions.time_antiperiodic_provider(-1))
    solver = dirac_solver.eo_square_solver(tol=TOL, precision=args.hmc_precision, delta=args.delta, chunk=args.chunk)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    ym = gauge_action.yang_mills(cfg, BETA)
    gen = torch.Generator(device=dev)
    gen.manual_seed(2026 + rank)
    rng = np.random.default_rng(2026 + rank)
    steps = [args.hmc_outer, args.hmc_inner]
    stream = torch.cuda.current_stream()
    records = []
    clocks = None
    for k in range(1 + args.trajectories):
        if k == 1:
            clocks = ClockSampler(local_rank)
            clocks.start()
        eta = hmc.generate_random_vector(NC, 4, stddev=1 / np.sqrt(2), volume=vol, generator=gen)
        momenta = hmc.random_momenta(NC, nd, vol, generator=gen)
        it0 = solver.total_iterations
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        nf.set_gauge_configuration(cfg)
        nf.initialize_pseudofermions([eta])
        cfg, minus_dh, acc = hmc.hybrid_mc(cfg, [nf, ym], steps, 1.0, momenta=momenta, uniform=float(rng.uniform()))
        e.record(stream)
        torch.cuda.synchronize()
        plaq = measurements.plaquette(cfg).value
        records.append({"seconds": s.elapsed_time(e) / 1e3, "dH": -minus_dh, "accepted": bool(acc),
                        "plaquette": plaq, "cg_iterations": solver.total_iterations - it0})
    clk = clocks.stop()
    timed = records[1:]
    sec = statistics.mean(r["seconds"] for r in timed)
    eta = hmc.generate_random_vector(NC, 4, stddev=1 / np.sqrt(2), volume=vol, generator=gen)
    nf.set_gauge_configuration(cfg)
    nf.initialize_pseudofermions([eta])
    rev = hmc.reversibility_check(cfg, [nf, ym], steps, 1.0, momenta=hmc.random_momenta(NC, nd, vol, generator=gen))
    line = {"metric": "HMC trajectories/hour", "value": world * 3600.0 / sec, "unit": "trajectories/hour",
            "n_gpus": world, "trajectories": args.trajectories, "warmup": 1, "higher_is_better": True,
            "seconds_per_trajectory": sec, "dtype": f"{args.hmc_precision}+f64" if args.hmc_precision != "f64"
            else "f64", "data": "synthetic",
            "config": {"workload": "hmc nf2 wilson 16^4 SU(3) beta=5.6 kappa=0.13", "geometry": list(GEOMETRY),
                       "integrator": f"omelyan nested {steps}, t = 1", "solver": "even-odd CG on Q twice, tol 1e-10",
                       "inner_precision": args.hmc_precision, "start": "reunit(exp(i 0.25 H))"},
            "acceptance": statistics.mean(1.0 if r["accepted"] else 0.0 for r in timed),
            "reversibility_dH": rev, "per_trajectory": records, "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.dslash_sweep:
        return run_dslash_sweep(args, local_rank)
    if args.hmc:
        return run_hmc(args, rank, world, local_rank)
    if args.serve_sweep:
        return run_serve_sweep(args, local_rank)
    if args.batch_lattices:
        return run_batch_lattices(args, local_rank)
    if args.precision_study:
        return run_precision_study(args, local_rank)
    if args.multishift:
        return run_multishift(args, local_rank)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_lym(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
