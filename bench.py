"""Benchmark of the SmallStrainFFT solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload serve|plain128|...] [--mode bench|kernels|request|accuracy|sweep]

Default workload: the RVE serving stream -- 512 homogenisation requests arriving as
a Poisson process at 50 req/s, N ~ U{32,48,64,96}, 20-400 periodic Voronoi grains,
elastic or FCC crystal plasticity, uniaxial or biaxial strain rate, 10-50 load steps --
served on one warm server.  The K timed steps are K consecutive slices of that stream (by
arrival), run as one continuous stream; beside the headline the line carries the served
throughput and latency at 1-20 req/s, the plain single-request FP64 GPU solve of a prefix
of the stream, and CPU numbers measured on complete solves of the stream's requests.

Multi-GPU runs are replicas: the stream is partitioned across ranks (no exchange step),
so ``scaling`` is "strong".  Prints one JSON line (rank 0).
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "served RVE solves/s + p50/p99 latency vs plain GPU solve at <=1e-5 stress err"

WORKLOADS = {
    # Plain method on GPU at scale: cubic elastic 250/150/120, 128^3, 500 periodic
    # Voronoi grains with uniform SO(3) orientations, uniaxial x strain rate 1e-3 for
    # 20 steps, float fields/FFT with double residuals and norms, tolerance 1e-6.
    "plain128": dict(n=128, grains=500, steps=20, dt=1.0, rate=1e-3, gtol=1e-6,
                     ltol=1e-5, precision="mixed", seed=0),
    "plain64": dict(n=64, grains=200, steps=20, dt=1.0, rate=1e-3, gtol=1e-6,
                    ltol=1e-5, precision="mixed", seed=0),
    # kernel-profiling cases of the crystal-plasticity requests (per-voxel tangents)
    "evp64": dict(n=64, grains=200, steps=5, dt=0.2, rate=1e-3, gtol=1e-6, ltol=1e-5,
                  precision="mixed", seed=0, model="evp"),
    "evp96": dict(n=96, grains=200, steps=5, dt=0.2, rate=1e-3, gtol=1e-6, ltol=1e-5,
                  precision="mixed", seed=0, model="evp"),
    # Crystal EVP plain GPU solve: FCC, Voce 0.1/0.3/1.0, latent ratio 1.4, 64^3, 200
    # grains, uniaxial x 1e-3 to 2% strain in 100 steps.
    "evp64_latent": dict(n=64, grains=200, steps=100, dt=0.2, rate=1e-3, gtol=1e-6,
                         ltol=1e-5, precision="mixed", seed=0, model="evp", latent=1.4),
    # Two-phase large RVE: 256^3, 2000 grains, each grain EVP (as above, latent 1) or cubic
    # elastic x10 with probability 1/2, uniaxial x 1e-3 to 1% strain in 50 steps.
    "twophase256": dict(n=256, grains=2000, steps=50, dt=0.2, rate=1e-3, gtol=1e-6,
                        ltol=1e-5, precision="mixed", seed=0, model="twophase"),
    # its 128^3 analog: the same physics and grain size (250 grains), eight times cheaper
    "twophase128": dict(n=128, grains=250, steps=50, dt=0.2, rate=1e-3, gtol=1e-6,
                        ltol=1e-5, precision="mixed", seed=0, model="twophase"),
    # Serving stream: requests with N ~ U{32,48,64,96}, 20-400 periodic Voronoi grains,
    # elastic or FCC EVP (p = 1/2), uniaxial or biaxial strain rate 1e-3, 10-50 steps,
    # Poisson arrivals at 50 req/s; the first `count` requests of the seeded stream.
    # Beside it: the sweep rates (each over the prefix that arrives in `sweep_seconds`),
    # the plain FP64 single-request solve of the first `plain_count` requests, and the
    # stream's 32^3 elastic requests among the first `cpu_count` (the CPU-feasible class,
    # solved in full by the CPU baselines).
    "serve": dict(count=512, rate=50.0, slots=16, seed=1000, sweep_rates=(1, 2, 5, 10, 20),
                  sweep_seconds=20.0, plain_count=128, e2e_count=128, cpu_count=512),
}

def plane_path(n):
    """True when the z and y passes of an n^3 float solve run plane-fused: in one block (a
    padded yz plane pair of complex floats fits the 200 KB shared-memory budget) or split
    over a thread-block cluster of 2, 4 or 8 blocks, each holding two buffers of its rows'
    padded z lines (or of its columns' y lines) within the same budget."""
    padded = lambda m: m + (m >> 4) + 1
    if (2 * padded(n * (n + 2)) + 2 * n) * 8 <= 200 * 1024:
        return True
    hs = n // 2 if n % 2 == 0 else n // 2 + 1
    for c in (2, 4, 8):
        if n % c or (2 * hs) % c:
            continue
        cap = max(padded(n // c * n), 2 * (n // c) * hs, n * (2 * hs // c))
        if (2 * cap + 2 * n) * 8 <= 200 * 1024:
            return True
    return False


# Algorithmic HBM bytes per voxel of each Krylov-iteration kernel with float fields:
# planar vectors are 24 B/voxel (6 x 4 B); the stored half spectrum is 6 x hs/n x 8 B with
# hs = n/2 columns on even grids (the zeroed Nyquist column is not stored), (n+1)/2 on odd.
# The update kernel applies the previous iteration's vector update (reads y', u, w1, w2, x;
# writes u', w, x) and writes tau = K v over y'; the forward z pass reads tau and writes the
# spectrum; the inverse z pass writes P tau over y', which the epilogue kernel turns into
# y' (with the MINRES dot products).  With the plane-fused passes the y transforms happen in
# shared memory inside the z kernels and move no bytes of their own.
def kernel_bytes_per_voxel(n, table_mode=True):
    spec = 6 * (n // 2 if n % 2 == 0 else n // 2 + 1) / n * 8.0
    kin = 4.0 if table_mode else 84.0
    ypass = 0.0 if plane_path(n) else 2 * spec
    return {
        "zfwd": 24.0 + spec,                # read tau; write spectrum
        "yfwd": ypass,
        "xpass": 2 * spec,                  # read + write spectrum
        "yinv": ypass,
        "zinv": spec + 24.0,                # read spectrum; write P tau
        "update": 8 * 24.0 + kin + 24.0,    # update vectors, tangent; write tau
        "epilogue": 4 * 24.0,               # read P tau, u_{j-1}, u_j; write y'
    }


KERNEL_NAMES = ["zfwd", "yfwd", "xpass", "yinv", "zinv", "update", "epilogue"]


def cubic_mandel(C11, C12, C44):
    s = np.array([1, 1, 1, np.sqrt(2), np.sqrt(2), np.sqrt(2)])
    V = np.zeros((6, 6))
    V[:3, :3] = C12
    V[[0, 1, 2], [0, 1, 2]] = C11
    V[[3, 4, 5], [3, 4, 5]] = C44
    return V * np.outer(s, s)


def build_microstructure(w):
    from materialite_b200.microstructure import (periodic_voronoi, periodic_voronoi_device,
                                                 quaternion_random_rotations)
    n = w["n"]
    rng = np.random.default_rng(w["seed"])
    # the device search returns the tree query's regions; it saves seconds from 128^3 up
    gen = periodic_voronoi_device if n >= 128 else periodic_voronoi
    ids = gen((n, n, n), w["grains"], rng)
    rot = quaternion_random_rotations(w["grains"], rng)
    return rot, ids.astype(np.int32)


def phase_of_points(w, ids):
    """Two-phase workloads: phase 0 (EVP) or 1 (elastic x10) per grain with probability
    1/2, drawn from the workload's seed after the microstructure."""
    if w.get("model") != "twophase":
        return None
    rng = np.random.default_rng(w["seed"] + 1)
    return (rng.random(w["grains"]) < 0.5).astype(np.int32)[ids]


def uniaxial_x(rate):
    mask = np.array([0, 1, 1, 1, 1, 1], dtype=float)
    er = np.array([rate, 0, 0, 0, 0, 0], dtype=float)
    zero = np.zeros(6)
    return mask, (lambda t, dt: er * dt), (lambda t, dt: zero), (lambda t, dt: zero)


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_handle(w, rot, ids, device, precision=None):
    from materialite_b200.engine import PhaseSpec, SolverHandle
    from materialite_b200.serving import evp_phase
    mask, *_ = uniaxial_x(w["rate"])
    n = w["n"]
    h = SolverHandle((n, n, n), mask, precision or w["precision"], global_tolerance=w["gtol"],
                     linear_solver_tolerance=w["ltol"], device=device)
    elastic = PhaseSpec("elastic", cubic_mandel(250.0, 150.0, 120.0))
    if w.get("model") == "evp":
        h.set_phases([evp_phase(w.get("latent", 1.0))])
    elif w.get("model") == "twophase":
        h.set_phases([evp_phase(), PhaseSpec("elastic", cubic_mandel(250.0, 150.0, 120.0) * 10)])
    else:
        h.set_phases([elastic])
    h.set_microstructure(rot, ids, phase_of_points(w, ids))
    return h


def run_solve(h, w, stats=None):
    from materialite_b200.engine import solve
    _, de, ds, s = uniaxial_x(w["rate"])
    return solve(h, de, ds, s, end_time=w["steps"] * w["dt"], initial_time_increment=w["dt"],
                 stats=stats)


def cpu_sample(w, max_seconds=40.0):
    """Time the numpy oracle (single process) on the first load increment of the
    workload, plus its one-off Gamma-hat build, and extrapolate to a full solve."""
    from oracle import ssfft_oracle as O
    from materialite_b200.engine import unique_rotations  # noqa: F401
    rot, ids = build_microstructure(w)
    n = w["n"]
    R = rot[ids]
    mask, de, ds, s = uniaxial_x(w["rate"])
    t0 = time.perf_counter()
    G = O.projection_operator((n, n, n), mask)
    t_build = time.perf_counter() - t0
    del G
    load = O.LoadOracle(de, ds, s, mask)
    t0 = time.perf_counter()
    O.solve((n, n, n), R, O.ElasticOracle(cubic_mandel(250.0, 150.0, 120.0)), load,
            end_time=w["dt"], initial_time_increment=w["dt"], global_tolerance=w["gtol"],
            linear_solver_tolerance=w["ltol"])
    t_first = time.perf_counter() - t0 - t_build  # solve() rebuilds Gamma-hat once
    per_solve = t_build + w["steps"] * t_first
    return per_solve, t_build, t_first


CPU_CLASS = "elastic32"


def cpu_subset_tags(w, count=None):
    """Tags of the stream's 32^3 elastic requests (stream order): the class that a CPU solves
    in full within seconds (a 96^3 crystal-plasticity request takes hours on one core)."""
    from materialite_b200.serving import request_kind
    n = count or w["cpu_count"]
    return [t for t in range(n) if request_kind(t, w["seed"])[0] == CPU_CLASS]


def oracle_solve_request(r):
    """The numpy oracle (the reference's numpy path restated) on one request of the stream,
    in full; returns seconds and the final stress (V, 6)."""
    from oracle import ssfft_oracle as O
    from materialite_b200.serving import cubic
    t0 = time.perf_counter()
    p = r.phases[0]
    if p.kind == "evp":
        model = O.EVPOracle(p.stiffness, p.schmid, p.reference_slip_rate, p.rate_exponent,
                            p.slip_resistance, "voce", p.hardening_props)
    else:
        model = O.ElasticOracle(cubic(250.0, 150.0, 120.0))
    load = O.LoadOracle.constant_rates(r.strain_rate, np.zeros(6), r.stress_mask)
    out = O.solve(r.dims, r.rotations[r.grain], model, load, end_time=r.steps * r.dt,
                  initial_time_increment=r.dt, global_tolerance=r.global_tolerance,
                  linear_solver_tolerance=r.linear_solver_tolerance)
    return time.perf_counter() - t0, out["stress"]


def _ref_solve_tag(args):
    """Worker of the CPU pools: build request `tag` of the stream and solve it in full with
    the oracle (one thread)."""
    tag, seed = args
    from materialite_b200.serving import make_request
    r = make_request(tag, np.random.default_rng(seed + tag))
    secs, _ = oracle_solve_request(r)
    return tag, secs


SINGLE_THREAD_ENV = {"OMP_NUM_THREADS": "1", "OPENBLAS_NUM_THREADS": "1",
                     "MKL_NUM_THREADS": "1", "NUMEXPR_NUM_THREADS": "1"}


def single_thread_pool(workers):
    """Spawned worker processes whose BLAS/OpenMP run one thread each (the environment is
    set before they start, so numpy picks it up)."""
    import multiprocessing as mp
    os.environ.update(SINGLE_THREAD_ENV)
    return mp.get_context("spawn").Pool(workers)


def host_workers():
    cores = os.cpu_count() or 1
    try:
        import psutil
        mem_workers = max(1, int(psutil.virtual_memory().available / (2 * 2**30)))
    except Exception:
        mem_workers = 4
    return max(1, min(cores, mem_workers))


def _ref_worker(w):
    return cpu_sample(w)


def reference_arm_single(args, w):
    """--impl reference for a single-solve workload (plain128, ...): every host core runs the
    oracle on the workload's Gamma-hat build and first load increment, extrapolated to the
    workload's increments (a full 128^3 CPU solve takes tens of minutes); the sample says
    so."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    workers = max(1, min(host_workers(), 8))
    times = []
    with single_thread_pool(workers) as pool:
        for i in range(args.warmup + args.steps):
            res = pool.map(_ref_worker, [w] * workers)
            if i >= args.warmup:
                times.append(max(r[0] for r in res))
    per_solve = statistics.mean(times)
    value = workers / per_solve
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_solve * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded periodic Voronoi, uniform SO(3))", "impl": "reference",
            "config": {"workload": args.workload, **{k: w[k] for k in ("n", "grains", "steps")}},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": "port",
                             "sample": "per worker: Gamma-hat build + first load increment, "
                                       "extrapolated to all load increments"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_config(w, count):
    return {"workload": f"serve: {count} requests of the seeded RVE serving stream, Poisson "
                        f"arrivals at {w['rate']} req/s, N in {{32,48,64,96}}, 20-400 "
                        "periodic Voronoi grains, elastic or FCC EVP, uniaxial/biaxial strain "
                        "rate 1e-3, 10-50 load steps; one step = one slice of the stream by "
                        "arrival, the stream run once continuously",
            "count": count, "rate_per_s": w["rate"],
            "sweep_rates_per_s": list(w["sweep_rates"]) + [w["rate"]]}


def reference_arm(args, w):
    """--impl reference: the reference's numpy path (the oracle restatement; the reference is
    pure Python and the oracle matches it to 1e-15) on every host core.  A CPU solves the
    stream's 32^3 elastic requests in seconds but its 96^3 crystal-plasticity requests in
    hours, so the arm measures complete solves of the 32^3 elastic requests of the stream:
    one worker process per core works through them continuously; a step is one completed
    request; after W warm-up completions, value = K completions / the time they took."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    tags = cpu_subset_tags(w)
    workers = host_workers()
    need = args.warmup + args.steps + workers
    todo = [(tags[i % len(tags)], w["seed"]) for i in range(need)]
    done_t = []
    pool = single_thread_pool(workers)
    try:
        t_start = time.perf_counter()
        for _tag, _secs in pool.imap_unordered(_ref_solve_tag, todo):
            done_t.append(time.perf_counter())
            if len(done_t) >= args.warmup + args.steps:
                break
    finally:
        pool.terminate()
        pool.join()
    t0 = done_t[args.warmup - 1] if args.warmup > 0 else t_start
    t1 = done_t[args.warmup + args.steps - 1]
    value = args.steps / (t1 - t0)
    sample = (f"numpy oracle, complete solves of the stream's {CPU_CLASS} requests "
              f"({len(tags)} of the first {w['cpu_count']}, cycled in stream order), "
              f"{workers} single-threaded worker processes working continuously; one step = "
              "one completed request, timed after the warm-up completions")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (t1 - t0) / args.steps * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded request stream: periodic Voronoi, "
                                    "uniform SO(3))",
            "impl": "reference", "config": serve_config(w, args.count or w["count"]),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_mode(args, w):
    """Serving benchmark of the RVE request stream on one warm server (mixed precision): the
    W warm-up steps serve one request of every class of the stream at once; the K timed
    steps are the whole stream at its Poisson arrivals (one continuous run).  Then: the same
    stream's prefix end to end with every stress field read back, the sweep of arrival
    rates, the plain single-request FP64 GPU solve of a prefix against the served solve of
    the same requests (throughput and stress error), the 32^3 elastic requests the CPU
    baselines solve, the 128^3 roofline, and the one-core CPU baseline.  Under torchrun the
    stream is partitioned across the ranks (replicas)."""
    from materialite_b200 import replicas
    from materialite_b200.serving import (RVEServer, arrival_times, latency_stats,
                                          request_stream, run_stream, solve_plain)
    count = args.count or w["count"]
    # every request is built before the first GPU call (spawned pool)
    reqs_all = request_stream(count, w["rate"], seed=w["seed"], workers=host_workers())
    world, rank, local = replicas.init("nccl")
    reqs = replicas.partition(reqs_all, world, rank) if world > 1 else reqs_all
    per_step = -(-len(reqs) // args.steps)
    voxels = sum(int(np.prod(r.dims)) for r in reqs)
    classes = {}
    for r in reqs:
        classes.setdefault(r.kind, r)

    failures = {}

    def one_pass(srv, rs, keep, rate=None, saturate=False):
        saved = [r.arrival for r in rs]
        if rate is not None:
            for r, t in zip(rs, arrival_times(len(rs), rate, w["seed"])):
                r.arrival = float(t)
        if saturate:
            for r in rs:
                r.arrival = 0.0
        t0 = min(r.arrival for r in rs)
        for r in rs:
            r.keep_stress = keep
            r.arrival -= t0
        try:
            comps, span = run_stream(srv, rs, timeout=3600)
        finally:
            for r, a in zip(rs, saved):
                r.arrival = a
        # a failed request is reported in the line (and not counted as a solve) rather than
        # ending the run
        for c in comps:
            if c.status != 0:
                failures.setdefault(int(c.tag), (int(c.status),
                                                 c.message.decode(errors="replace")))
        return comps, span

    def n_ok(comps):
        return sum(1 for c in comps if c.status == 0)

    import torch
    srv = RVEServer(device=local, max_slots=w["slots"], precision="mixed",
                    krylov_floor=args.krylov_floor,
                    krylov_forcing=args.krylov_forcing)
    warm = list(classes.values())
    for _ in range(args.warmup):
        one_pass(srv, warm, False, saturate=True)
    torch.cuda.synchronize(local)
    replicas.barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    l0 = srv.kernel_launches()
    comps, span = one_pass(srv, reqs, False)
    l1 = srv.kernel_launches()
    torch.cuda.synchronize(local)
    clocks = sampler.stop()
    t_max = replicas.max_over_ranks(span, world, local)
    total = replicas.sum_over_ranks(n_ok(comps), world, local)
    value = total / t_max
    lat = latency_stats(comps)
    kinds = {}
    for r, c in zip(reqs, comps):
        kinds.setdefault(r.kind, []).append(c.end_time - c.submit_time)
    per_class = {k: {"count": len(v), "p50_s": float(np.percentile(v, 50)),
                     "p99_s": float(np.percentile(v, 99))} for k, v in sorted(kinds.items())}
    # end to end: a prefix of the stream with every stress field copied to the host
    e2e_reqs = reqs[:min(len(reqs), w["e2e_count"])]
    comps_e2e, span_e2e = one_pass(srv, e2e_reqs, True)
    e2e_value = replicas.sum_over_ranks(n_ok(comps_e2e), world, local) / \
        replicas.max_over_ranks(span_e2e, world, local)
    h2d = sum(r.grain.nbytes + r.rotations.nbytes for r in e2e_reqs) / max(1, len(e2e_reqs))
    d2h = sum(int(np.prod(r.dims)) * 48 for r in e2e_reqs) / max(1, len(e2e_reqs))
    # arrival-rate sweep: each rate over the prefix that arrives in sweep_seconds
    sweep = []
    for rate in w["sweep_rates"]:
        n = max(8, min(len(reqs), int(w["sweep_seconds"] * rate)))
        cs, sp = one_pass(srv, reqs[:n], False, rate=rate)
        sweep.append({"rate_per_s": rate, "count": n, "solves_per_s": n_ok(cs) / sp,
                      **latency_stats(cs)})
    sweep.append({"rate_per_s": w["rate"], "count": len(reqs), "solves_per_s": n_ok(comps) / span,
                  **lat})
    # plain single-request FP64 GPU solve of a prefix, against the served mixed solve of the
    # same requests (all submitted at once)
    sub = reqs[:min(len(reqs), w["plain_count"])]
    comps_sub, span_sub = one_pass(srv, sub, True, saturate=True)
    stress_mixed = [r.stress.copy() for r in sub]
    krylov_floor, krylov_forcing = srv.krylov_floor, srv.krylov_forcing
    srv.close()
    secs_plain, pouts = solve_plain(sub, "fp64", device=local)
    stress_fp64 = [r.stress.copy() for r in sub]
    errs = [float(np.linalg.norm(a - b) / np.linalg.norm(b))
            for a, b, c in zip(stress_mixed, stress_fp64, comps_sub) if c.status == 0]
    plain_value = len(sub) / sum(secs_plain)
    served_sub = n_ok(comps_sub) / span_sub
    # the CPU class (32^3 elastic requests of the stream), on the GPU: served and plain
    cpu_tags = set(cpu_subset_tags(w, count))
    cpu_reqs = [r for r in reqs if r.tag in cpu_tags]
    cpu_gpu = None
    if cpu_reqs:
        srv2 = RVEServer(device=local, max_slots=w["slots"], precision="mixed",
                         krylov_floor=args.krylov_floor,
                         krylov_forcing=args.krylov_forcing)
        _, span_c = one_pass(srv2, cpu_reqs, False, saturate=True)
        srv2.close()
        secs_c, _ = solve_plain(cpu_reqs, "fp64", device=local, keep_stress=False)
        cpu_gpu = {"workload": f"the stream's {len(cpu_reqs)} {CPU_CLASS} requests among the "
                               f"first {count}",
                   "served_solves_per_s": len(cpu_reqs) / span_c,
                   "plain_fp64_solves_per_s": len(cpu_reqs) / sum(secs_c)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded request stream: periodic Voronoi, uniform SO(3))",
            "config": {**serve_config(w, count),
                       "requests_per_step": per_step,
                       "parallelism": f"replicas x{world} (stream partitioned by cost)",
                       "slots_per_class": w["slots"], "voxels": voxels,
                       "precision": "float Krylov vectors, tangents and matvec FFTs; double "
                                    "strain/stress fields, residuals, norms, Krylov scalars "
                                    "and crystal-plasticity Newton",
                       "krylov_floor": krylov_floor,
                       "krylov_forcing": krylov_forcing,
                       "l2": "inputs larger than L2: the stream's fields stream through HBM"},
            "served": {"solves_per_s": value, **lat, "makespan_s": t_max,
                       "per_class_latency": per_class},
            "sweep": sweep,
            "plain_fp64_single_request": {"workload": f"first {len(sub)} requests of the "
                                                      "stream, one at a time",
                                          "solves_per_s": plain_value,
                                          "served_solves_per_s_same_requests": served_sub,
                                          "newton": int(sum(o.newton_iterations for o in pouts)),
                                          "krylov": int(sum(o.krylov_iterations for o in pouts)),
                                          "served_newton": int(sum(c.result.newton_iterations
                                                                   for c in comps_sub)),
                                          "served_krylov": int(sum(c.result.krylov_iterations
                                                                   for c in comps_sub))},
            # the same requests both ways; the served side is all of them at once, so its
            # makespan ends with the longest request (a tail the one-at-a-time sum has not)
            "served_over_plain": served_sub / plain_value,
            # the stream's steady served rate over the plain rate of the same prefix's mix
            "served_stream_over_plain": value / plain_value,
            "stress_rel_l2_mixed_vs_fp64": {"max": max(errs) if errs else None,
                                            "median": float(np.median(errs)) if errs else None,
                                            "requests": len(errs)},
            "cpu_class_on_gpu": cpu_gpu,
            "failed_requests": {"count": len(failures),
                                "first": [[t, st, m] for t, (st, m) in
                                          sorted(failures.items())[:10]]},
            "clocks": clocks,
            "gpu_launches": int(l1 - l0),
            "e2e": {"value": e2e_value, "unit": "solves/s",
                    "h2d_bytes_per_step": int(h2d * per_step),
                    "d2h_bytes_per_step": int(d2h * per_step),
                    "workload": f"first {len(e2e_reqs)} requests of the stream at "
                                f"{w['rate']} req/s, submitted from host numpy arrays, every "
                                "stress field copied back to a host numpy array"},
        }
        if not args.no_roofline:
            line["roofline"] = plain128_roofline(local)
        if world == 1 and not args.no_cpu_baseline and cpu_reqs:
            secs, _ = oracle_solve_request(cpu_reqs[0])
            line["cpu_baseline"] = {
                "value": 1.0 / secs, "unit": "solves/s", "cores": 1, "kind": "port",
                "sample": f"numpy oracle (the reference's numpy path), one complete solve of "
                          f"request {cpu_reqs[0].tag} of the stream ({cpu_reqs[0].kind}, "
                          f"{cpu_reqs[0].steps} load steps) on one core: {secs:.1f} s"}
        print(json.dumps(line), flush=True)
    replicas.destroy(world)


def sweep_mode(args, w):
    """Arrival-rate sweep of the serving stream on one warm server: the first ``--count``
    requests submitted as Poisson arrivals at each rate of ``--rates``; per rate the served
    solves/s (count / makespan from first arrival to last completion) and the p50/p99/mean
    latency from submission to completion."""
    from materialite_b200.serving import RVEServer, latency_stats, request_stream, run_stream
    count = args.count or 64
    rates = [float(x) for x in args.rates.split(",")]
    srv = RVEServer(device=0, max_slots=w["slots"], precision="mixed",
                    krylov_floor=args.krylov_floor,
                    krylov_forcing=args.krylov_forcing)
    run_stream(srv, request_stream(min(count, 8), 0.0, seed=w["seed"]), timeout=1800)
    out = {"workload": f"serve sweep: {count} requests of the serving stream, "
                       f"{w['slots']} slots per class, mixed precision", "rates": []}
    for rate in rates:
        reqs = request_stream(count, rate, seed=w["seed"], workers=host_workers())
        comps, span = run_stream(srv, reqs, timeout=3600)
        bad = [c.tag for c in comps if c.status != 0]
        if bad:
            raise RuntimeError(f"requests failed: {bad}")
        lat = latency_stats(comps)
        out["rates"].append({"rate_per_s": rate, "solves_per_s": count / span,
                             "makespan_s": span, **lat})
        print(json.dumps(out["rates"][-1]), flush=True)
    srv.close()
    print(json.dumps(out), flush=True)


def classes_mode(args, w):
    """Per class of the serving stream's first ``--count`` requests (default 64): the plain
    single-request FP64 solve (one request at a time) against the served mixed solve of the
    same requests (all submitted at once, the class alone on the GPU): solves/s of each,
    their ratio, iteration totals and the stress error between them.  Both arms are warmed
    with one-step copies of the class's requests first."""
    from materialite_b200.serving import RVEServer, request_stream, run_stream, solve_plain
    count = args.count or 64
    reqs = request_stream(count, w["rate"], seed=w["seed"], workers=host_workers())
    by = {}
    for r in reqs:
        by.setdefault(r.kind, []).append(r)
    out = {"workload": f"first {count} requests of the serving stream, by class", "classes": {}}
    import dataclasses
    for kind in sorted(by):
        rs = by[kind]
        # one-step copies of the class's requests warm both arms first: the plain handle of
        # the grid size, and the server's group with every slot allocated and its graphs
        # built; neither is timed
        warm = [dataclasses.replace(r, tag=r.tag + 1000000, steps=1, keep_stress=False,
                                    stress=None, arrival=0.0) for r in rs]
        secs, pouts = solve_plain(warm[:1] + rs, precision="fp64", device=0, keep_stress=True)
        secs, pouts = secs[1:], pouts[1:]
        ref = [r.stress.copy() for r in rs]
        srv = RVEServer(device=0, max_slots=w["slots"], precision="mixed",
                        krylov_floor=args.krylov_floor,
                        krylov_forcing=args.krylov_forcing)
        run_stream(srv, warm, timeout=3600)
        for r in rs:
            r.keep_stress = True
            r.arrival = 0.0
        comps, span = run_stream(srv, rs, timeout=3600)
        srv.close()
        err = max(float(np.linalg.norm(r.stress - a) / np.linalg.norm(a)) for r, a in zip(rs, ref))
        plain = len(rs) / float(sum(secs))
        served = len(rs) / span
        out["classes"][kind] = {
            "count": len(rs), "plain_fp64_solves_per_s": plain, "served_solves_per_s": served,
            "served_over_plain": served / plain,
            "newton": int(sum(c.result.newton_iterations for c in comps)),
            "krylov": int(sum(c.result.krylov_iterations for c in comps)),
            "plain_newton": int(sum(o.newton_iterations for o in pouts)),
            "plain_krylov": int(sum(o.krylov_iterations for o in pouts)),
            "stress_rel_l2_max": err}
        print(json.dumps({kind: out["classes"][kind]}), flush=True)
    print(json.dumps(out), flush=True)


def group_mode(args, w):
    """The first ``--count`` requests of one class (``--kind``, e.g. evp64) of the serving
    stream, all submitted at once to a fresh server: the class alone on the GPU, every
    Krylov launch batching all of its slots (the case the batched kernels are profiled
    on)."""
    from materialite_b200.serving import RVEServer, request_kind, request_stream, run_stream
    count = args.count or 16
    tags, t = [], 0
    while len(tags) < count and t < 100000:
        if request_kind(t, seed=w["seed"])[0] == args.kind:
            tags.append(t)
        t += 1
    reqs = request_stream(len(tags), w["rate"], seed=w["seed"], workers=host_workers(), tags=tags)
    srv = RVEServer(device=0, max_slots=w["slots"], precision=args.precision,
                    krylov_floor=args.krylov_floor,
                    krylov_forcing=args.krylov_forcing)
    for r in reqs:
        r.arrival = 0.0
    comps, span = run_stream(srv, reqs, timeout=3600)
    launches = srv.kernel_launches()
    srv.close()
    print(json.dumps({"kind": args.kind, "count": len(reqs), "precision": args.precision,
                      "solves_per_s": len(reqs) / span, "seconds": span,
                      "newton": int(sum(c.result.newton_iterations for c in comps)),
                      "krylov": int(sum(c.result.krylov_iterations for c in comps)),
                      "kernel_launches": launches,
                      "failed": sum(1 for c in comps if c.status != 0)}), flush=True)


def request_mode(args, w):
    """One request of the serving stream (``--tag``), alone, in the chosen precision:
    the target of per-request kernel profiles."""
    from materialite_b200.serving import RVEServer, request_stream, run_stream
    reqs = request_stream(args.tag + 1, 0.0, seed=w["seed"])
    r = reqs[args.tag]
    srv = RVEServer(max_slots=1, precision=args.precision)
    comps, span = run_stream(srv, [r])
    srv.close()
    c = comps[0]
    print(json.dumps({"tag": args.tag, "kind": r.kind, "steps": r.steps, "status": c.status,
                      "newton": c.result.newton_iterations, "krylov": c.result.krylov_iterations,
                      "device_s": c.result.device_seconds, "wall_s": c.end_time - c.start_time}),
          flush=True)


def kernels_mode(args, w):
    """One load increment of the workload, then the Krylov-iteration kernels timed with
    CUDA events on the handle's stream (``--reps`` iterations); prints microseconds and
    algorithmic GB/s per kernel slot."""
    rot, ids = build_microstructure(w)
    h = make_handle(w, rot, ids, 0)
    run_solve(h, dict(w, steps=1))
    prof = h.profile_krylov(reps=args.reps)
    h.close()
    n = w["n"]
    V = n ** 3
    bpv = kernel_bytes_per_voxel(n, table_mode=w.get("model") != "evp")
    out = {"workload": args.workload, "plane_path": plane_path(n), "reps": args.reps,
           "iteration_us": prof[7] * 1e6,
           "iteration_gbs": sum(bpv.values()) * V / prof[7] / 1e9, "kernels": {}}
    for i, k in enumerate(KERNEL_NAMES):
        out["kernels"][k] = {"us": prof[i] * 1e6,
                             "gbs": bpv[k] * V / prof[i] / 1e9 if prof[i] > 1e-7 else None}
    print(json.dumps(out), flush=True)


def accuracy_mode(args, w):
    """One full solve of the workload in mixed precision and in FP64 on the same inputs:
    device seconds, iteration counts and the mixed stress field's relative L2 error
    against FP64 (the size-independent check at sizes the oracle cannot reach; the FP64
    path itself is pinned to the oracle at small sizes)."""
    from materialite_b200.engine import SolveStats
    if args.load_steps:
        w = dict(w, steps=args.load_steps)
    rot, ids = build_microstructure(w)
    out = {"workload": args.workload, "n": w["n"], "steps": w["steps"]}
    stress = {}
    for prec in ("mixed", "fp64"):
        h = make_handle(w, rot, ids, 0, precision=prec)
        st = SolveStats()
        h.timer_start()
        failure = None
        try:
            res, _ = run_solve(h, w, st)
        except ValueError as e:  # the reference's own failure: min time increment reached
            failure, res = str(e), None
        t = h.timer_stop()
        reached = sum(a[1] for a in st.attempts if a[2])
        out[prec] = {"device_s": t, "steps": st.steps, "cutbacks": getattr(st, "cutbacks", None),
                     "newton": int(sum(st.newton_iterations)),
                     "krylov": int(sum(st.krylov_iterations)), "time_reached": reached,
                     "end_time": w["steps"] * w["dt"], "failure": failure}
        if res is not None:
            stress[prec] = res["stress"]
            out[prec]["mean_stress_xx"] = float(res["stress"][:, 0].mean())
        h.close()
        print(json.dumps({prec: out[prec]}), flush=True)
        # per attempted increment: t, dt, converged, Newton, Krylov, eq. error, max
        # constitutive iterations (where the two precisions part ways)
        print(json.dumps({prec + "_attempts": st.attempts}), flush=True)
    if "mixed" in stress and "fp64" in stress:
        a, b = stress["mixed"], stress["fp64"]
        out["stress_rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    print(json.dumps(out), flush=True)


# DRAM read + write bytes of one steady-state launch of each Krylov kernel on plain128
# (128^3, mixed precision, three-pass cluster path), from one-launch ncu captures of
# `--mode kernels --workload plain128` (profiles/krylov_kernels_plain128.md).  The update
# kernel reads 260.1 MB and writes 154.2 MB against 461 MB algorithmic: part of its writes
# are still in L2 when it ends.
PLAIN128_TRAFFIC_BYTES = {"update": 414.4e6, "epilogue": 171.7e6, "zfwd": 57.1e6,
                          "xpass": 52.6e6, "zinv": 58.7e6}


def plain128_roofline(device):
    """Roofline of the dominant Krylov kernel on the 128^3 plain solve (the HBM-bound
    regime), timed live with CUDA events on the handle's stream."""
    w = WORKLOADS["plain128"]
    rot, ids = build_microstructure(w)
    h = make_handle(w, rot, ids, device)
    run_solve(h, dict(w, steps=1))
    prof = h.profile_krylov(reps=10)
    h.close()
    n = w["n"]
    V = n ** 3
    bpv = kernel_bytes_per_voxel(n)
    per_kernel = {k: prof[i] for i, k in enumerate(KERNEL_NAMES)}
    dom = max(per_kernel, key=per_kernel.get)
    peak, kind = read_peaks()
    achieved = bpv[dom] * V / per_kernel[dom] / 1e9
    return {"bound": "hbm", "workload": "plain128 Krylov iteration", "kernel": dom,
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": PLAIN128_TRAFFIC_BYTES.get(dom),
            "traffic_unit": "bytes per launch (ncu capture)",
            "algorithmic_bytes": bpv[dom] * V, "peak_kind": kind,
            "per_kernel_us": {k: v * 1e6 for k, v in per_kernel.items()},
            "krylov_iteration_us": prof[7] * 1e6,
            "krylov_iteration_gbs": sum(bpv.values()) * V / prof[7] / 1e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="serve", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--mode", default="bench",
                    choices=["bench", "kernels", "request", "accuracy", "sweep", "classes",
                             "group"],
                    help="kernels: one load increment, then the Krylov kernels timed in "
                         "isolation (the target of the ncu captures under profiles/); "
                         "request: one request of the serving stream alone; accuracy: one "
                         "solve of the workload in mixed and in FP64, stress error between")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--rates", default="1,2,4,8,50",
                    help="sweep: Poisson arrival rates (requests/s)")
    ap.add_argument("--load-steps", type=int, default=0,
                    help="accuracy: solve only the first N load increments of the workload")
    ap.add_argument("--count", type=int, default=0, help="serve: number of requests")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--tag", type=int, default=0, help="request mode: index in the stream")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--kind", default="evp64", help="group mode: request class (e.g. evp64)")
    ap.add_argument("--krylov-forcing", type=float, default=None,
                    help="served requests' MINRES relative forcing; default: the server's")
    ap.add_argument("--krylov-floor", type=float, default=None,
                    help="served requests' MINRES floor (fraction of the tolerance); "
                         "default: the server's (0.1 mixed, 0 FP64)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.mode == "kernels":
        kernels_mode(args, w)
        return
    if args.mode == "classes":
        classes_mode(args, WORKLOADS["serve"])
        return
    if args.mode == "group":
        group_mode(args, WORKLOADS["serve"])
        return
    if args.mode == "accuracy":
        accuracy_mode(args, w)
        return
    if args.mode == "request":
        request_mode(args, WORKLOADS["serve"])
        return
    if args.mode == "sweep":
        sweep_mode(args, WORKLOADS["serve"])
        return
    if args.workload == "serve" and args.impl == "ours":
        serve_mode(args, w)
        return
    if args.impl == "reference":
        if args.workload == "serve":
            reference_arm(args, w)
        else:
            reference_arm_single(args, w)
        return
    from materialite_b200 import replicas
    world, rank, local = replicas.init("nccl")
    from materialite_b200.engine import SolveStats
    rot, ids = build_microstructure(w)
    h = make_handle(w, rot, ids, local)
    for _ in range(args.warmup):
        run_solve(h, w)
    _, launches0 = h.stats()
    replicas.barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    st = SolveStats()
    h.timer_start()
    for _ in range(args.steps):
        run_solve(h, w, st)
    t = h.timer_stop()
    clocks = sampler.stop()
    _, launches1 = h.stats()
    t_max = replicas.max_over_ranks(t, world, local)
    total_solves = replicas.sum_over_ranks(args.steps, world, local)
    value = total_solves / t_max
    # accuracy self-check of the timed solve is covered by the parity tests; record the
    # solver work for context
    krylov_per_solve = sum(st.krylov_iterations) / args.steps
    newton_per_solve = sum(st.newton_iterations) / args.steps

    # roofline of the dominant Krylov kernel, timed live with CUDA events on the
    # handle's stream
    prof = h.profile_krylov(reps=20)
    n = w["n"]
    V = n ** 3
    bpv = kernel_bytes_per_voxel(n)
    per_kernel = {k: prof[i] for i, k in enumerate(KERNEL_NAMES)}
    dom = max(per_kernel, key=per_kernel.get)
    peak, peak_kind = read_peaks()
    achieved = bpv[dom] * V / per_kernel[dom] / 1e9
    iter_bytes = sum(bpv.values()) * V
    iter_gbs = iter_bytes / prof[7] / 1e9

    # end to end through the host API: upload the microstructure, solve, read back
    # stress and strain
    e2e_times = []
    from materialite_b200.engine import SolverHandle  # noqa: F401
    h.close()
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        he = make_handle(w, rot, ids, local)
        out, _ = run_solve(he, w)
        he.close()
        e2e_times.append(time.perf_counter() - t0)
    e2e_max = replicas.max_over_ranks(statistics.mean(e2e_times), world, local)
    e2e_value = replicas.sum_over_ranks(1.0, world, local) / e2e_max
    h2d = ids.nbytes + rot.nbytes
    d2h = 2 * V * 6 * 8

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        per_solve, t_build, t_first = cpu_sample(w)
        cpu = {"value": 1.0 / per_solve, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"numpy oracle: Gamma-hat build ({t_build:.1f} s) + first load "
                         f"increment ({t_first:.1f} s) of this workload, extrapolated to "
                         f"{w['steps']} increments"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded periodic Voronoi, uniform SO(3) quaternions)",
            "config": {"workload": f"{args.workload}: plain SmallStrainFFT solve, cubic elastic "
                                   f"250/150/120, {n}^3, {w['grains']} periodic Voronoi grains, "
                                   f"uniaxial x 1e-3, {w['steps']} steps, float fields/FFT with "
                                   f"double residuals and norms, tolerance {w['gtol']}",
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2",
                       "krylov_iterations_per_solve": krylov_per_solve,
                       "newton_iterations_per_solve": newton_per_solve},
            "clocks": clocks,
            "gpu_launches": int(launches1 - launches0),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": (PLAIN128_TRAFFIC_BYTES.get(dom)
                                     if args.workload == "plain128" else None),
                         "peak_kind": peak_kind,
                         "per_kernel_us": {k: v * 1e6 for k, v in per_kernel.items()},
                         "krylov_iteration_us": prof[7] * 1e6,
                         "krylov_iteration_gbs": iter_gbs},
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
