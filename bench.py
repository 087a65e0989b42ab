"""Benchmark of the SmallStrainFFT solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plain128]

One "step" is one complete RVE solve of the workload (every load increment, Newton
iterations and device MINRES), with the microstructure already resident in HBM.
Multi-GPU runs are independent replicas (one RVE solve stream per GPU; the path has no
exchange step), so ``scaling`` is "weak".

Prints one JSON line (rank 0).
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
    # Serving stream: requests with N ~ U{32,48,64,96}, 20-400 periodic Voronoi grains,
    # elastic or FCC EVP (p = 1/2), uniaxial or biaxial strain rate 1e-3, 10-50 steps,
    # Poisson arrivals; the first `count` requests of the seeded stream.
    "serve": dict(count=24, rate=50.0, slots=16, seed=1000),
}

def plane_path(n):
    """True when the z and y passes of an n^3 float solve run plane-fused (a padded yz
    plane pair of complex floats fits the 200 KB shared-memory budget)."""
    padded = lambda m: m + (m >> 4) + 1
    return (2 * padded(n * (n + 2)) + 2 * n) * 8 <= 200 * 1024


# Algorithmic HBM bytes per voxel of each Krylov-iteration kernel with float fields:
# planar vectors are 24 B/voxel (6 x 4 B); the half spectrum is 6 x (n/2+1)/n x 8 B.  The
# forward z pass also applies the previous iteration's vector update (reads y', u, w1,
# w2, x; writes u', w, x).  With the plane-fused passes the y transforms happen in shared
# memory inside the z kernels and move no bytes of their own.
def kernel_bytes_per_voxel(n, table_mode=True):
    spec = 6 * (n // 2 + 1) / n * 8.0
    kin = 4.0 if table_mode else 84.0
    ypass = 0.0 if plane_path(n) else 2 * spec
    return {
        "zfwd": 8 * 24.0 + kin + spec,      # update vectors, tangent; write spectrum
        "yfwd": ypass,
        "xpass": 2 * spec,                  # read + write spectrum
        "yinv": ypass,
        "zinv": spec + 3 * 24.0,            # read spectrum, u_{j-1}, u_j; write y'
        "update": 0.0,                      # fused into the forward z pass
    }


KERNEL_NAMES = ["zfwd", "yfwd", "xpass", "yinv", "zinv", "update"]


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


SERVE_SAMPLE_STEPS = 3


def cpu_serve_sample(seed=1000):
    """Time the numpy oracle (this process, one core) on the first SERVE_SAMPLE_STEPS
    load increments of a 32^3 elastic request and a 32^3 EVP request of the serving mix,
    plus the 32^3 Gamma-hat build.  Returns seconds per increment per kind and the build
    time."""
    from oracle import ssfft_oracle as O
    from materialite_b200.serving import cubic, elastic_phase, evp_phase, make_request
    out = {}
    t0 = time.perf_counter()
    O.projection_operator((32, 32, 32), [0, 1, 1, 1, 1, 1])
    out["build32"] = time.perf_counter() - t0
    for kind in ("elastic", "evp"):
        r = make_request(0, np.random.default_rng(seed), sizes=(32,), grains=(100, 100),
                         steps=(10, 10))
        if kind == "evp":
            p = evp_phase()
            model = O.EVPOracle(p.stiffness, p.schmid, p.reference_slip_rate, p.rate_exponent,
                                p.slip_resistance, "voce", p.hardening_props)
            dt = 0.2
        else:
            model = O.ElasticOracle(cubic(250.0, 150.0, 120.0))
            dt = 1.0
        load = O.LoadOracle.constant_rates(r.strain_rate, np.zeros(6), r.stress_mask)
        t0 = time.perf_counter()
        O.solve(r.dims, r.rotations[r.grain], model, load, end_time=SERVE_SAMPLE_STEPS * dt,
                initial_time_increment=dt, global_tolerance=r.global_tolerance,
                linear_solver_tolerance=r.linear_solver_tolerance)
        out[kind] = (time.perf_counter() - t0 - out["build32"]) / SERVE_SAMPLE_STEPS
    return out


def cpu_serve_seconds(reqs, sample):
    """Extrapolated oracle seconds per request: (Gamma-hat build + steps x seconds per
    increment of its kind) x (N/32)^3."""
    per = []
    for r in reqs:
        scale = (r.dims[0] / 32.0) ** 3
        kind = "evp" if r.kind.startswith("evp") else "elastic"
        per.append((sample["build32"] + r.steps * sample[kind]) * scale)
    return float(np.mean(per))


SERVE_SAMPLE_TEXT = (f"numpy oracle on the first {SERVE_SAMPLE_STEPS} load increments of a 32^3 "
                     "elastic and a 32^3 FCC EVP request plus the 32^3 Gamma-hat build, "
                     "extrapolated to every request of the stream by its step count and "
                     "(N/32)^3; EVP increments after the onset of slip need more Newton "
                     "iterations than the sampled ones, so this underestimates the CPU time")


SINGLE_THREAD_ENV = {"OMP_NUM_THREADS": "1", "OPENBLAS_NUM_THREADS": "1",
                     "MKL_NUM_THREADS": "1", "NUMEXPR_NUM_THREADS": "1"}


def single_thread_pool(workers):
    """Spawned worker processes whose BLAS/OpenMP run one thread each (the environment is
    set before they start, so numpy picks it up)."""
    import multiprocessing as mp
    os.environ.update(SINGLE_THREAD_ENV)
    return mp.get_context("spawn").Pool(workers)


def reference_arm(args, w):
    """--impl reference: the oracle restatement of the reference's numpy path on the host
    cores (the reference is pure Python; the oracle matches it to 1e-15).  Each step runs a
    bounded sample in every worker process at once; value = workers / extrapolated seconds
    per solve."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    try:
        import psutil
        mem_workers = max(1, int(psutil.virtual_memory().available / (12 * 2**30)))
    except Exception:
        mem_workers = 4
    serve = args.workload == "serve"
    workers = max(1, min(cores, mem_workers, 16))
    times = []
    reqs = None
    if serve:
        from materialite_b200.serving import request_stream
        reqs = request_stream(args.count or w["count"], w["rate"], seed=w["seed"])
    with single_thread_pool(workers) as pool:
        for i in range(args.warmup + args.steps):
            if serve:
                res = pool.map(_ref_serve_worker, [w["seed"]] * workers)
                worst = {k: max(r[k] for r in res) for k in res[0]}
                t = cpu_serve_seconds(reqs, worst)
            else:
                res = pool.map(_ref_worker, [w] * workers)
                t = max(r[0] for r in res)
            if i >= args.warmup:
                times.append(t)
    per_solve = statistics.mean(times)
    value = workers / per_solve
    if serve:
        cfg = {"workload": f"serve: {len(reqs)} requests of the serving stream (see the ours line)"}
        sample = SERVE_SAMPLE_TEXT
    else:
        cfg = {"workload": args.workload, **{k: w[k] for k in ("n", "grains", "steps")}}
        sample = ("per worker: Gamma-hat build + first load increment, extrapolated to all "
                  "load increments")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_solve * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded periodic Voronoi, uniform SO(3))",
            "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _ref_worker(w):
    return cpu_sample(w)


def _ref_serve_worker(seed):
    return cpu_serve_sample(seed)


def serve_mode(args, w):
    """Serving benchmark on one warm server: W untimed and K timed passes of the seeded
    request stream (Poisson arrivals, up to `slots` requests resident, mixed precision);
    then the same stream end to end with every request's stress field read back to the
    host, the saturated stream (all arrivals at 0), and the plain single-request FP64 GPU
    solve (one slot, requests one after another) with the stress error of mixed against
    it.  Under torchrun every rank serves its own stream (replicas)."""
    from materialite_b200 import replicas
    from materialite_b200.serving import RVEServer, latency_stats, request_stream, run_stream
    world, rank, local = replicas.init("nccl")
    count = args.count or w["count"]
    reqs = request_stream(count, w["rate"], seed=w["seed"] + 1000 * rank)
    voxels = sum(int(np.prod(r.dims)) for r in reqs)
    h2d = sum(r.grain.nbytes + r.rotations.nbytes for r in reqs)

    def one_pass(srv, keep, saturate=False):
        arrivals = [r.arrival for r in reqs]
        for r in reqs:
            r.keep_stress = keep
            if saturate:
                r.arrival = 0.0
        comps, span = run_stream(srv, reqs, timeout=1800)
        for r, a in zip(reqs, arrivals):
            r.arrival = a
        bad = [(c.tag, c.status, c.message.decode(errors="replace")) for c in comps
               if c.status != 0]
        if bad:
            raise RuntimeError(f"requests failed: {bad}")
        return comps, span

    srv = RVEServer(device=local, max_slots=w["slots"], precision="mixed")
    for _ in range(args.warmup):
        one_pass(srv, False)
    replicas.barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    spans, comps_all = [], []
    for _ in range(args.steps):
        comps, span = one_pass(srv, False)
        spans.append(span)
        comps_all += comps
    clocks = sampler.stop()
    launches = sum(int(c.result.kernel_launches) for c in comps_all)
    t_served = replicas.max_over_ranks(sum(spans), world, local)
    total = replicas.sum_over_ranks(count * args.steps, world, local)
    value = total / t_served
    lat = latency_stats(comps_all)
    # end to end: the same stream with each request's stress field copied to the host
    e2e_spans = []
    for _ in range(max(1, args.e2e_steps)):
        _, span = one_pass(srv, True)
        e2e_spans.append(span)
    stress_mixed = [r.stress.copy() for r in reqs]
    t_e2e = replicas.max_over_ranks(sum(e2e_spans), world, local)
    e2e_value = replicas.sum_over_ranks(count * len(e2e_spans), world, local) / t_e2e
    _, span_sat = one_pass(srv, False, saturate=True)
    srv.close()
    plain_srv = RVEServer(device=local, max_slots=1, precision="fp64")
    plain, span_plain = one_pass(plain_srv, True, saturate=True)
    plain_srv.close()
    stress_fp64 = [r.stress.copy() for r in reqs]
    errs = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(stress_mixed, stress_fp64)]
    span_sat = replicas.max_over_ranks(span_sat, world, local)
    span_plain = replicas.max_over_ranks(span_plain, world, local)
    count_all = replicas.sum_over_ranks(count, world, local)
    lat_plain = latency_stats(plain)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_served / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded request stream: periodic Voronoi, uniform SO(3))",
            "config": {"workload": f"serve: one step = one pass of {count} requests of the "
                                   f"serving stream at {w['rate']} req/s Poisson, N in "
                                   "{32,48,64,96}, 20-400 grains, elastic or FCC EVP, "
                                   "uniaxial/biaxial, 10-50 steps; "
                                   f"{w['slots']} resident slots, float fields with double "
                                   "residuals/norms/EVP Newton",
                       "parallelism": f"replicas x{world}", "voxels_per_step": voxels,
                       "l2": "inputs larger than L2: one pass streams every request's "
                             "fields through HBM; each request's own solve runs L2-resident "
                             "as it does in service"},
            "served": {"solves_per_s": value, **lat, "makespan_s_per_step": t_served / args.steps},
            "saturation": {"solves_per_s": count_all / span_sat, "makespan_s": span_sat},
            "plain_fp64_single_request": {"solves_per_s": count_all / span_plain,
                                          **{k: v for k, v in lat_plain.items()},
                                          "makespan_s": span_plain},
            "served_over_plain": value / (count_all / span_plain),
            "stress_rel_l2_mixed_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
            "clocks": clocks,
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": "solves/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(voxels * 48),
                    "note": "requests submitted from host numpy arrays (grain ids, "
                            "rotations), stress fields copied back to host numpy arrays"},
        }
        if not args.no_roofline:
            line["roofline"] = plain128_roofline(local)
        if world == 1 and not args.no_cpu_baseline:
            with single_thread_pool(1) as pool:
                sample = pool.map(_ref_serve_worker, [w["seed"]])[0]
            per = cpu_serve_seconds(reqs, sample)
            line["cpu_baseline"] = {"value": 1.0 / per, "unit": "solves/s", "cores": 1,
                                    "kind": "port", "sample": SERVE_SAMPLE_TEXT}
        print(json.dumps(line), flush=True)
    replicas.destroy(world)


def sweep_mode(args, w):
    """Arrival-rate sweep of the serving stream on one warm server: the same seeded
    requests submitted as Poisson arrivals at each rate of ``--rates``; per rate the served
    solves/s (count / makespan from first arrival to last completion) and the p50/p99/mean
    latency from submission to completion."""
    from materialite_b200.serving import RVEServer, latency_stats, request_stream, run_stream
    count = args.count or 32
    rates = [float(x) for x in args.rates.split(",")]
    srv = RVEServer(device=0, max_slots=w["slots"], precision="mixed")
    run_stream(srv, request_stream(min(count, 8), 0.0, seed=w["seed"]), timeout=1800)
    out = {"workload": f"serve sweep: {count} requests of the serving stream, "
                       f"{w['slots']} slots, mixed precision", "rates": []}
    for rate in rates:
        reqs = request_stream(count, rate, seed=w["seed"])
        comps, span = run_stream(srv, reqs, timeout=1800)
        bad = [c.tag for c in comps if c.status != 0]
        if bad:
            raise RuntimeError(f"requests failed: {bad}")
        lat = latency_stats(comps)
        out["rates"].append({"rate_per_s": rate, "solves_per_s": count / span,
                             "makespan_s": span, **lat})
        print(json.dumps(out["rates"][-1]), flush=True)
    srv.close()
    print(json.dumps(out), flush=True)


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
        res, _ = run_solve(h, w, st)
        t = h.timer_stop()
        stress[prec] = res["stress"]
        out[prec] = {"device_s": t, "steps": st.steps, "cutbacks": getattr(st, "cutbacks", None),
                     "newton": int(sum(st.newton_iterations)),
                     "krylov": int(sum(st.krylov_iterations)),
                     "mean_stress_xx": float(res["stress"][:, 0].mean())}
        h.close()
        print(json.dumps({prec: out[prec]}), flush=True)
    a, b = stress["mixed"], stress["fp64"]
    out["stress_rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    print(json.dumps(out), flush=True)


# DRAM read + write bytes of one steady-state zfwd launch on plain128, from an ncu
# --set full capture of `--mode kernels --workload plain128`: 260.4 MB read + 168.9 MB
# written (algorithmic 462 MB).
ZFWD_PLAIN128_TRAFFIC_BYTES = 429.4e6


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
            "traffic": ZFWD_PLAIN128_TRAFFIC_BYTES if dom == "zfwd" else None,
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
                    choices=["bench", "kernels", "request", "accuracy", "sweep"],
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
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.mode == "kernels":
        kernels_mode(args, w)
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
        reference_arm(args, w)
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
                         "traffic": (ZFWD_PLAIN128_TRAFFIC_BYTES
                                     if args.workload == "plain128" and dom == "zfwd" else None),
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
