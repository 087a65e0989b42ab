"""Serving many RVE homogenisation solves on one GPU (libssfft's ssfft_server_*).

``RVEServer`` wraps the C server: requests (grid, phases, microstructure, constant-rate
load schedule) are copied at submission, join the batched group of their class (grid,
precision, tangent kind) when a slot and device memory are free, advance together with the
other requests of the group -- every kernel launch covers all of them -- and come back as
completions carrying queue/start/end times.  ``request_stream`` generates the seeded request mix of the serving
benchmark.
"""

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _native as nat
from .engine import hardening_props_vector
from .microstructure import periodic_voronoi, quaternion_random_rotations

# MINRES absolute floor of served mixed-precision requests, as a fraction of the global
# tolerance: a linear solve stops once its residual could move the next equilibrium error
# by at most a tenth of the tolerance.  An elastic request's later increments then start
# at equilibrium to round-off and need no Krylov iterations, where the reference's relative
# test spends 30-45 iterations resolving that round-off.
SERVED_KRYLOV_FLOOR = 0.1

# Relative forcing of served mixed-precision requests' linear solves (inexact Newton): a
# solve also stops once its residual is 1% of its right-hand side.  The Newton iterations
# converge at a rate set by the constitutive nonlinearity, not by the last digits of each
# linear solve: a batched group of 16 crystal-plasticity 64^3 requests took the same Newton
# iterations (4417 against 4425) and 40% fewer Krylov iterations, 35% faster.
SERVED_KRYLOV_FORCING = 0.01


class SsfftPhase(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("n_slip", ctypes.c_int32), ("hardening", ctypes.c_int32),
        ("n_props", ctypes.c_int32), ("stiffness", ctypes.c_double * 36),
        ("schmid", ctypes.c_double * 72), ("reference_slip_rate", ctypes.c_double),
        ("rate_exponent", ctypes.c_double), ("slip_resistance", ctypes.c_double),
        ("latent_ratio", ctypes.c_double), ("hardening_props", ctypes.c_double * 4),
    ]


class SsfftRequest(ctypes.Structure):
    _fields_ = [
        ("config", nat.SsfftConfig), ("n_phases", ctypes.c_int32), ("n_orient", ctypes.c_int32),
        ("phases", SsfftPhase * 8), ("rotations", ctypes.POINTER(ctypes.c_double)),
        ("orient_of_point", ctypes.POINTER(ctypes.c_int32)),
        ("phase_of_point", ctypes.POINTER(ctypes.c_int32)),
        ("schedule", nat.SsfftRateSchedule), ("tag", ctypes.c_int64),
        ("stress_out", ctypes.POINTER(ctypes.c_double)),
    ]


class SsfftCompletion(ctypes.Structure):
    _fields_ = [
        ("tag", ctypes.c_int64), ("status", ctypes.c_int32), ("slot", ctypes.c_int32),
        ("submit_time", ctypes.c_double), ("start_time", ctypes.c_double),
        ("end_time", ctypes.c_double), ("device_bytes", ctypes.c_size_t),
        ("result", nat.SsfftSolveOut), ("message", ctypes.c_char * 160),
    ]


def _bind(lib):
    if getattr(lib, "_server_bound", False):
        return lib
    P = ctypes.c_void_p
    lib.ssfft_server_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                        ctypes.POINTER(P)]
    lib.ssfft_server_submit.argtypes = [P, ctypes.POINTER(SsfftRequest)]
    lib.ssfft_server_poll.argtypes = [P, ctypes.POINTER(SsfftCompletion), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int)]
    lib.ssfft_server_pending.argtypes = [P]
    lib.ssfft_server_clock.argtypes = [P]
    lib.ssfft_server_clock.restype = ctypes.c_double
    lib.ssfft_server_destroy.argtypes = [P]
    lib.ssfft_server_launches.argtypes = [P, ctypes.POINTER(ctypes.c_int64)]
    for n in ("ssfft_server_create", "ssfft_server_submit", "ssfft_server_poll",
              "ssfft_server_pending", "ssfft_server_destroy", "ssfft_server_launches"):
        getattr(lib, n).restype = ctypes.c_int
    lib._server_bound = True
    return lib


@dataclass
class RVERequest:
    """One homogenisation solve.  ``phases`` are engine.PhaseSpec objects; ``grain`` maps
    points to rows of ``rotations``; the load is LoadSchedule.from_constant_rates with
    ``stress_mask``."""
    tag: int
    dims: tuple
    phases: list
    rotations: np.ndarray
    grain: np.ndarray
    stress_mask: np.ndarray
    strain_rate: np.ndarray
    stress_rate: np.ndarray
    dt: float
    steps: int
    phase_of_point: Optional[np.ndarray] = None
    global_tolerance: float = 1e-6
    linear_solver_tolerance: float = 1e-5
    arrival: float = 0.0
    kind: str = ""
    keep_stress: bool = False
    stress: Optional[np.ndarray] = field(default=None, repr=False)


def _phase_struct(p):
    if p.kind not in ("elastic", "evp"):
        raise ValueError(f"serving requests take elastic and evp phases, not {p.kind!r}; "
                         "solve J2 phases through SmallStrainFFT or SolverHandle")
    s = SsfftPhase()
    s.kind = 0 if p.kind == "elastic" else 1
    C = np.asarray(p.stiffness, dtype=np.float64).ravel()
    for i in range(36):
        s.stiffness[i] = C[i]
    s.latent_ratio = float(p.latent_ratio)
    if p.kind == "evp":
        P = np.asarray(p.schmid, dtype=np.float64).reshape(-1, 6)
        s.n_slip = P.shape[0]
        for i, v in enumerate(P.ravel()):
            s.schmid[i] = v
        s.reference_slip_rate = float(p.reference_slip_rate)
        s.rate_exponent = float(p.rate_exponent)
        s.slip_resistance = float(p.slip_resistance)
        s.hardening = nat.HARDENING_IDS[p.hardening]
        props = hardening_props_vector(p.hardening, p.hardening_props)
        s.n_props = len(props)
        for i, v in enumerate(props):
            s.hardening_props[i] = v
    return s


class RVEServer:
    def __init__(self, device=0, max_slots=16, hbm_budget_bytes=0, precision="mixed",
                 krylov_floor=None, krylov_forcing=None):
        """``krylov_floor`` / ``krylov_forcing``: the MINRES absolute floor and relative
        forcing of every request (ssfft_config.krylov_floor, .krylov_forcing); None gives
        SERVED_KRYLOV_FLOOR / SERVED_KRYLOV_FORCING in mixed precision and 0 (the reference's
        stopping test alone) in FP64."""
        self.lib = _bind(nat.load_library())
        h = ctypes.c_void_p()
        nat.check(self.lib.ssfft_server_create(int(device), int(max_slots),
                                                int(hbm_budget_bytes), ctypes.byref(h)))
        self.h = h
        self.precision = precision
        if krylov_floor is None:
            krylov_floor = SERVED_KRYLOV_FLOOR if precision != "fp64" else 0.0
        self.krylov_floor = float(krylov_floor)
        if krylov_forcing is None:
            krylov_forcing = SERVED_KRYLOV_FORCING if precision != "fp64" else 0.0
        self.krylov_forcing = float(krylov_forcing)
        self._keep = {}

    def clock(self):
        return self.lib.ssfft_server_clock(self.h)

    def submit(self, r: RVERequest):
        req = SsfftRequest()
        cfg = req.config
        for d in range(3):
            cfg.n[d] = int(r.dims[d])
        cfg.precision = nat.SSFFT_FP64 if self.precision == "fp64" else nat.SSFFT_MIXED
        cfg.max_newton_iterations = 100
        cfg.global_tolerance = r.global_tolerance
        cfg.strain_correction_tolerance = 1e-2
        cfg.linear_solver_tolerance = r.linear_solver_tolerance
        cfg.krylov_floor = self.krylov_floor
        cfg.krylov_forcing = self.krylov_forcing
        for c in range(6):
            cfg.stress_mask[c] = float(r.stress_mask[c])
        req.n_phases = len(r.phases)
        for i, p in enumerate(r.phases):
            req.phases[i] = _phase_struct(p)
        rot = np.ascontiguousarray(r.rotations, dtype=np.float64).reshape(-1, 9)
        grain = np.ascontiguousarray(r.grain, dtype=np.int32)
        req.n_orient = rot.shape[0]
        req.rotations = nat.as_double_ptr(rot)
        req.orient_of_point = nat.as_int_ptr(grain)
        ph = None
        if r.phase_of_point is not None:
            ph = np.ascontiguousarray(r.phase_of_point, dtype=np.int32)
            req.phase_of_point = nat.as_int_ptr(ph)
        sc = req.schedule
        for c in range(6):
            sc.strain_rate[c] = float(r.strain_rate[c])
            sc.stress_rate[c] = float(r.stress_rate[c])
        sc.start_time = 0.0
        sc.end_time = r.dt * r.steps
        sc.initial_time_increment = r.dt
        req.tag = int(r.tag)
        if r.keep_stress:
            r.stress = np.empty((int(np.prod(r.dims)), 6))
            req.stress_out = nat.as_double_ptr(r.stress)
            self._keep[r.tag] = r.stress
        nat.check(self.lib.ssfft_server_submit(self.h, ctypes.byref(req)))

    def poll(self, max_items=256):
        buf = (SsfftCompletion * max_items)()
        n = ctypes.c_int()
        nat.check(self.lib.ssfft_server_poll(self.h, buf, max_items, ctypes.byref(n)))
        out = [buf[i] for i in range(n.value)]
        for c in out:
            self._keep.pop(c.tag, None)
        return out

    def pending(self):
        return self.lib.ssfft_server_pending(self.h)

    def kernel_launches(self):
        """Kernels the server's groups have launched so far."""
        n = ctypes.c_int64()
        nat.check(self.lib.ssfft_server_launches(self.h, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.ssfft_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cubic(C11, C12, C44, scale=1.0):
    s = np.array([1, 1, 1, np.sqrt(2), np.sqrt(2), np.sqrt(2)])
    V = np.zeros((6, 6))
    V[:3, :3] = C12
    V[[0, 1, 2], [0, 1, 2]] = C11
    V[[3, 4, 5], [3, 4, 5]] = C44
    return V * np.outer(s, s) * scale


def fcc_schmid():
    from .slip_system import SlipSystem
    return SlipSystem.octahedral().schmid_mandel()


def elastic_phase():
    from .engine import PhaseSpec
    return PhaseSpec("elastic", cubic(250.0, 150.0, 120.0))


def evp_phase(latent=1.0):
    """FCC {111}<110>, cubic 250/150/120, reference slip rate 1e-3, n = 20, Voce with
    tau0 = 0.1, tau_sat = 0.3 (tau_1 = 0.2), h0 = 1 (theta_1 = 0)."""
    from .engine import PhaseSpec
    return PhaseSpec("evp", cubic(250.0, 150.0, 120.0), fcc_schmid(), 1e-3, 20.0, 0.1, "voce",
                     {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0}, latent)


def request_draws(rng, sizes=(32, 48, 64, 96), grains=(20, 400), steps=(10, 50)):
    """The scalar draws of one request of the serving mix, in order: grid N ~ U{sizes},
    G ~ U[20, 400] grains, crystal plasticity with probability 1/2, biaxial with probability
    1/2, 10-50 load steps.  The microstructure is drawn after these from the same rng."""
    n = int(rng.choice(sizes))
    G = int(rng.integers(grains[0], grains[1] + 1))
    is_evp = bool(rng.random() < 0.5)
    biaxial = bool(rng.random() < 0.5)
    nsteps = int(rng.integers(steps[0], steps[1] + 1))
    return n, G, is_evp, biaxial, nsteps


def request_kind(tag, seed=1000, **kw):
    """Class of request `tag` of the seeded stream ("evp64", "elastic32", ...) and its step
    count, without building its microstructure."""
    n, G, is_evp, biaxial, nsteps = request_draws(np.random.default_rng(seed + tag), **kw)
    return ("evp" if is_evp else "elastic") + f"{n}", nsteps


def make_request(tag, rng, sizes=(32, 48, 64, 96), grains=(20, 400), steps=(10, 50)):
    """One request of the serving mix: grid N ~ U{sizes}, G ~ U[20, 400] periodic Voronoi
    grains with uniform SO(3) orientations, elastic or FCC EVP with probability 1/2,
    uniaxial or biaxial constant strain rate 1e-3, 10-50 steps (dt 1 for elastic, 0.2
    for EVP)."""
    n, G, is_evp, biaxial, nsteps = request_draws(rng, sizes, grains, steps)
    ids = periodic_voronoi((n, n, n), G, rng)
    rot = quaternion_random_rotations(G, rng)
    rate = np.zeros(6)
    mask = np.ones(6)
    rate[0] = 1e-3
    mask[0] = 0.0
    if biaxial:
        rate[1] = 1e-3
        mask[1] = 0.0
    return RVERequest(tag=tag, dims=(n, n, n), phases=[evp_phase() if is_evp else elastic_phase()],
                      rotations=rot, grain=ids.astype(np.int32), stress_mask=mask,
                      strain_rate=rate, stress_rate=np.zeros(6), dt=0.2 if is_evp else 1.0,
                      steps=nsteps, kind=("evp" if is_evp else "elastic") + f"{n}")


def _make_tagged(args):
    tag, seed, kw = args
    return make_request(tag, np.random.default_rng(seed + tag), **kw)


def arrival_times(count, rate, seed=1000):
    """Poisson arrival times of a stream of `count` requests at `rate` per second (rate <=
    0: all at t = 0), drawn from np.random.default_rng(seed - 1)."""
    if rate <= 0:
        return np.zeros(count)
    return np.cumsum(np.random.default_rng(seed - 1).exponential(1.0 / rate, size=count))


def request_stream(count, rate, seed=1000, workers=1, tags=None, **kw):
    """``count`` requests with Poisson arrival times at ``rate`` per second (rate <= 0:
    all at t = 0).  Request i draws from np.random.default_rng(seed + i).  ``workers`` > 1
    builds the microstructures in that many spawned processes; ``tags`` selects requests of
    the stream (they keep their arrival times)."""
    tags = list(range(count)) if tags is None else list(tags)
    arrivals = arrival_times(max(tags) + 1 if tags else 0, rate, seed)
    jobs = [(t, seed, kw) for t in tags]
    if workers > 1 and len(jobs) > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            reqs = pool.map(_make_tagged, jobs, chunksize=4)
    else:
        reqs = [_make_tagged(j) for j in jobs]
    for r in reqs:
        r.arrival = float(arrivals[r.tag]) if rate > 0 else 0.0
    return reqs


def run_stream(server, requests, timeout=600.0, sleep=0.002):
    """Submit each request at its arrival time (server clock) and collect completions.
    Returns the completions in tag order and the makespan (first arrival to last end)."""
    import time
    t_start = server.clock()
    pending = sorted(requests, key=lambda r: r.arrival)
    done = {}
    i = 0
    deadline = time.time() + timeout
    while len(done) < len(requests):
        now = server.clock() - t_start
        while i < len(pending) and pending[i].arrival <= now:
            server.submit(pending[i])
            i += 1
        for c in server.poll():
            done[c.tag] = c
        if time.time() > deadline:
            raise TimeoutError(f"{len(done)}/{len(requests)} requests finished in {timeout} s")
        if i < len(pending):
            time.sleep(min(sleep, max(0.0, pending[i].arrival - now)))
        else:
            time.sleep(sleep)
    comps = [done[r.tag] for r in requests]
    makespan = max(c.end_time for c in comps) - t_start
    return comps, makespan


def latency_stats(completions, requests=None):
    lat = np.array([c.end_time - c.submit_time for c in completions])
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}


def solve_plain(requests, precision="fp64", device=0, keep_stress=True):
    """The plain single-request GPU solve: each request alone, one after another, through a
    solver handle running the native time loop (ssfft_solve_constant_rates); one handle per
    grid size is reused.  Stores each request's final stress in ``r.stress`` (keep_stress)
    and returns (per-request seconds, solve records)."""
    import time
    from .engine import SolverHandle
    handles = {}
    secs, outs = [], []
    try:
        for r in requests:
            t0 = time.perf_counter()
            h = handles.get(tuple(r.dims))
            if h is None:
                h = SolverHandle(r.dims, r.stress_mask, precision, device=device)
                handles[tuple(r.dims)] = h
            h.set_options(r.stress_mask, r.global_tolerance, 1e-2, r.linear_solver_tolerance)
            h.set_phases(r.phases)
            h.set_microstructure(r.rotations, r.grain, r.phase_of_point)
            out = h.solve_constant_rates(r.strain_rate, r.stress_rate, r.dt * r.steps, r.dt)
            if keep_stress:
                r.stress = h.field("stress")
            secs.append(time.perf_counter() - t0)
            outs.append(out)
    finally:
        for h in handles.values():
            h.close()
    return secs, outs
