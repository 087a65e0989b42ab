"""Array-level driver of libssfft: one solver handle per RVE and the time loop of
materialite's SmallStrainFFT.run (materialite/models/small_strain_fft/small_strain_fft.py:
60-279).

``SmallStrainFFT`` (the drop-in class) and the serving loop both call ``solve``; the
per-step Newton/Krylov work runs on the GPU inside ``ssfft_step``.
"""

import ctypes
import logging
import math
from collections import defaultdict
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _native as nat


@dataclass
class PhaseSpec:
    """One constitutive phase: ``kind`` is "elastic", "evp" or "j2"; stiffness is a 6x6
    Mandel matrix.  EVP phases carry Mandel Schmid tensors (S,6) and the parameters of
    ElasticViscoplastic (elastic_viscoplastic.py:21-50); J2 phases the parameters of
    IsotropicElasticPlastic (isotropic_elastic_plastic.py:18-53): ``modulus``,
    ``shear_modulus`` and the initial yield stress in ``slip_resistance``."""
    kind: str
    stiffness: np.ndarray
    schmid: Optional[np.ndarray] = None
    reference_slip_rate: float = 1.0
    rate_exponent: float = 1.0
    slip_resistance: float = 1.0
    hardening: str = "perfect_plasticity"
    hardening_props: tuple = ()
    latent_ratio: float = 1.0
    modulus: float = 0.0
    shear_modulus: float = 0.0


def hardening_props_vector(kind, props):
    """Order the hardening-property dict as libssfft expects (hardening_laws.py:18-90)."""
    props = props or {}
    if kind == "perfect_plasticity":
        return ()
    if kind == "linear":
        return (float(props["hardening_rate"]),)
    if kind == "voce":
        return (float(props["tau_1"]), float(props["theta_0"]), float(props["theta_1"]))
    if kind == "armstrong_frederick":
        return (float(props["direct_hardening"]), float(props["dynamic_recovery"]))
    raise ValueError(f"unknown hardening law {kind}")


def unique_rotations(R):
    """Deduplicate per-point rotation matrices: returns (table (n,3,3), index (V,))."""
    R = np.ascontiguousarray(np.asarray(R, dtype=np.float64).reshape(-1, 9))
    table, index = np.unique(R, axis=0, return_inverse=True)
    return table.reshape(-1, 3, 3), index.reshape(-1).astype(np.int32)


class SolverHandle:
    """Owns one libssfft handle (device buffers of one RVE grid)."""

    def __init__(self, dims, stress_mask, precision="mixed", global_tolerance=1.0e-3,
                 strain_correction_tolerance=1.0e-2, linear_solver_tolerance=1.0e-5,
                 max_newton_iterations=100, max_krylov_iterations=0, device=0,
                 krylov_floor=0.0, krylov_forcing=0.0):
        """``krylov_floor`` > 0 adds an absolute floor and ``krylov_forcing`` > 0 a relative
        forcing term to the MINRES stopping test (ssfft_config.krylov_floor,
        .krylov_forcing); 0 keeps the reference's test alone."""
        self.lib = nat.load_library()
        cfg = nat.SsfftConfig()
        for d in range(3):
            cfg.n[d] = int(dims[d])
        cfg.precision = nat.SSFFT_FP64 if precision == "fp64" else nat.SSFFT_MIXED
        cfg.device = int(device)
        cfg.max_newton_iterations = int(max_newton_iterations)
        cfg.max_krylov_iterations = int(max_krylov_iterations)
        cfg.global_tolerance = float(global_tolerance)
        cfg.strain_correction_tolerance = float(strain_correction_tolerance)
        cfg.linear_solver_tolerance = float(linear_solver_tolerance)
        cfg.krylov_floor = float(krylov_floor)
        cfg.krylov_forcing = float(krylov_forcing)
        for c in range(6):
            cfg.stress_mask[c] = float(stress_mask[c])
        self.cfg = cfg
        self.dims = tuple(int(d) for d in dims)
        self.V = int(np.prod(self.dims))
        self.precision = precision
        h = ctypes.c_void_p()
        nat.check(self.lib.ssfft_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.nslip = 0
        self.has_j2 = False
        self.phases = []

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.ssfft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_phases(self, phases):
        self.phases = list(phases)
        for i, p in enumerate(self.phases):
            C = np.ascontiguousarray(p.stiffness, dtype=np.float64).reshape(36)
            if p.kind == "elastic":
                nat.check(self.lib.ssfft_set_phase_elastic(self.h, i, nat.as_double_ptr(C)))
            elif p.kind == "evp":
                P = np.ascontiguousarray(p.schmid, dtype=np.float64).reshape(-1, 6)
                props = np.ascontiguousarray(
                    list(hardening_props_vector(p.hardening, p.hardening_props)) + [0.0],
                    dtype=np.float64)
                nprops = len(hardening_props_vector(p.hardening, p.hardening_props))
                nat.check(self.lib.ssfft_set_phase_evp(
                    self.h, i, nat.as_double_ptr(C), P.shape[0], nat.as_double_ptr(P),
                    float(p.reference_slip_rate), float(p.rate_exponent),
                    float(p.slip_resistance), nat.HARDENING_IDS[p.hardening],
                    nat.as_double_ptr(props), nprops, float(p.latent_ratio)))
                self.nslip = max(self.nslip, P.shape[0])
            elif p.kind == "j2":
                pv = list(hardening_props_vector(p.hardening, p.hardening_props))
                props = np.ascontiguousarray(pv + [0.0], dtype=np.float64)
                nat.check(self.lib.ssfft_set_phase_j2(
                    self.h, i, float(p.modulus), float(p.shear_modulus),
                    float(p.slip_resistance), nat.HARDENING_IDS[p.hardening],
                    nat.as_double_ptr(props), len(pv)))
                self.nslip = max(self.nslip, 1)
                self.has_j2 = True
            else:
                raise ValueError(f"unknown phase kind {p.kind}")

    def set_microstructure(self, rotations, orient_of_point, phase_of_point=None):
        R = np.ascontiguousarray(rotations, dtype=np.float64).reshape(-1, 9)
        o = np.ascontiguousarray(orient_of_point, dtype=np.int32).reshape(-1)
        if o.size != self.V:
            raise ValueError("orientation index must have one entry per point")
        ph = None
        if phase_of_point is not None:
            ph = np.ascontiguousarray(phase_of_point, dtype=np.int32).reshape(-1)
            if ph.size != self.V:
                raise ValueError("phase index must have one entry per point")
        nat.check(self.lib.ssfft_set_microstructure(
            self.h, R.shape[0], nat.as_double_ptr(R), nat.as_int_ptr(o),
            nat.as_int_ptr(ph) if ph is not None else None))

    def reset(self):
        nat.check(self.lib.ssfft_reset(self.h))

    def set_options(self, stress_mask=None, global_tolerance=None,
                    strain_correction_tolerance=None, linear_solver_tolerance=None,
                    krylov_floor=None, krylov_forcing=None):
        """Change the stress mask and tolerances of the handle (same grid and precision)."""
        cfg = self.cfg
        if stress_mask is not None:
            for c in range(6):
                cfg.stress_mask[c] = float(stress_mask[c])
        if global_tolerance is not None:
            cfg.global_tolerance = float(global_tolerance)
        if strain_correction_tolerance is not None:
            cfg.strain_correction_tolerance = float(strain_correction_tolerance)
        if linear_solver_tolerance is not None:
            cfg.linear_solver_tolerance = float(linear_solver_tolerance)
        if krylov_floor is not None:
            cfg.krylov_floor = float(krylov_floor)
        if krylov_forcing is not None:
            cfg.krylov_forcing = float(krylov_forcing)
        nat.check(self.lib.ssfft_set_options(self.h, ctypes.byref(cfg)))

    def solve_constant_rates(self, strain_rate, stress_rate, end_time, initial_time_increment,
                             start_time=0.0, max_time_increment=0.0, min_time_increment=0.0):
        """The whole time loop natively for LoadSchedule.from_constant_rates with the handle's
        stress mask (ssfft_solve_constant_rates); returns the SsfftSolveOut record."""
        sc = nat.SsfftRateSchedule()
        for c in range(6):
            sc.strain_rate[c] = float(strain_rate[c])
            sc.stress_rate[c] = float(stress_rate[c])
        sc.start_time = float(start_time)
        sc.end_time = float(end_time)
        sc.initial_time_increment = float(initial_time_increment)
        sc.max_time_increment = float(max_time_increment)
        sc.min_time_increment = float(min_time_increment)
        out = nat.SsfftSolveOut()
        nat.check(self.lib.ssfft_solve_constant_rates(self.h, ctypes.byref(sc), ctypes.byref(out)))
        return out

    def step(self, dE, dS, Sbar, dt, summed_vm, step_id, reset):
        si = nat.SsfftStepIn()
        for c in range(6):
            si.strain_increment[c] = float(dE[c])
            si.stress_increment[c] = float(dS[c])
            si.mean_applied_stress[c] = float(Sbar[c])
        si.dt = float(dt)
        si.summed_von_mises_stress = float(summed_vm)
        si.time_step_id = int(step_id)
        si.reset_fluctuation = int(bool(reset))
        so = nat.SsfftStepOut()
        nat.check(self.lib.ssfft_step(self.h, ctypes.byref(si), ctypes.byref(so)))
        if so.status != 0:
            raise nat.SsfftError(so.status, "non-finite equilibrium error")
        return so

    def commit(self, scale):
        nat.check(self.lib.ssfft_commit(self.h, float(scale)))

    def scale_fluctuation(self, f):
        nat.check(self.lib.ssfft_scale_fluctuation(self.h, float(f)))

    def field(self, name):
        if name in ("slip_resistances", "slip_system_shear_strains"):
            width = self.nslip
        elif name in ("yield_stresses", "eq_plastic_strains"):
            width = 1
        else:
            width = 6
        out = np.empty((self.V, width), dtype=np.float64)
        nat.check(self.lib.ssfft_get_field(self.h, nat.FIELD_IDS[name], nat.as_double_ptr(out), 1))
        return out

    def apply_projection(self, tau):
        tau = np.ascontiguousarray(tau, dtype=np.float64).reshape(self.V, 6)
        out = np.empty_like(tau)
        nat.check(self.lib.ssfft_apply_projection(self.h, nat.as_double_ptr(tau),
                                                  nat.as_double_ptr(out)))
        return out.ravel()

    def timer_start(self):
        nat.check(self.lib.ssfft_timer(self.h, 1, None))

    def timer_stop(self):
        s = ctypes.c_double()
        nat.check(self.lib.ssfft_timer(self.h, 0, ctypes.byref(s)))
        return s.value

    def profile_krylov(self, reps=20):
        out = np.zeros(8)
        nat.check(self.lib.ssfft_profile_krylov(self.h, int(reps), nat.as_double_ptr(out)))
        return out

    def stats(self):
        s = ctypes.c_double()
        n = ctypes.c_int64()
        nat.check(self.lib.ssfft_stats(self.h, ctypes.byref(s), ctypes.byref(n)))
        return s.value, n.value


@dataclass
class SolveStats:
    steps: int = 0
    cutbacks: int = 0
    newton_iterations: list = field(default_factory=list)
    krylov_iterations: list = field(default_factory=list)
    device_seconds: float = 0.0
    # one record per attempted increment: time, dt, converged, Newton and Krylov
    # iterations, final equilibrium error, most constitutive iterations
    attempts: list = field(default_factory=list)


# the reference's logger name (small_strain_fft.py:53)
_log = logging.getLogger("SmallStrainFFT")


def solve(handle, dstrain, dstress, stress, end_time=1.0, initial_time_increment=None,
          max_time_increment=None, min_time_increment=1.0e-9, start_time=0.0,
          output_times=None, output_variables=None, stats=None, outputs_hook=None):
    """The time loop of SmallStrainFFT.run (small_strain_fft.py:73-246) over a prepared
    handle.  ``dstrain``, ``dstress`` and ``stress`` are the LoadSchedule closures
    returning Mandel 6-vectors.  Returns (final_outputs, history) where history maps each
    output name to the list of values at ``output_times``."""
    dt = end_time if initial_time_increment is None else initial_time_increment
    dt_max = dt if max_time_increment is None else max_time_increment
    t = start_time
    t_tol = min_time_increment / 2.0
    if output_times is not None:
        out_idx = 0
        output_times = np.append(output_times, np.inf)
        next_out = output_times[0]
    else:
        next_out = np.inf
    history = defaultdict(list)
    old_max_inc = 0.0
    summed_vm = 0.0
    step_id = 0
    handle.reset()
    while t < end_time - t_tol:
        dE = np.asarray(dstrain(t, dt), dtype=np.float64).reshape(6)
        dS = np.asarray(dstress(t, dt), dtype=np.float64).reshape(6)
        Sbar = np.asarray(stress(t, dt), dtype=np.float64).reshape(6)
        max_inc = dE[np.argmax(np.abs(dE))]
        reset = max_inc * old_max_inc < 0.0
        _log.info(f"New increment: time {t} + {dt}")
        out = handle.step(dE, dS, Sbar, dt, summed_vm, step_id, reset)
        # the Newton loop runs on the device; its outcome is logged once per increment
        _log.debug(f"global iterations {out.newton_iterations}")
        _log.debug(f"linear solver iterations: {out.krylov_iterations}")
        _log.debug(f"equilibrium error: {out.equilibrium_error}")
        _log.debug(f"scaled strain error: {out.scaled_strain_error}")
        if not out.converged and not out.constitutive_failed:
            _log.info("Too many iterations in macroloading loop")
        if stats is not None:
            stats.newton_iterations.append(out.newton_iterations)
            stats.krylov_iterations.append(out.krylov_iterations)
            stats.device_seconds += handle.stats()[0]
            stats.attempts.append((t, dt, bool(out.converged), int(out.newton_iterations),
                                   int(out.krylov_iterations), float(out.equilibrium_error),
                                   int(out.max_constitutive_iterations)))
        if out.converged:
            handle.commit(1.0)
            summed_vm += out.mean_von_mises_stress
            old_max_inc = max_inc
            step_id += 1
            t += dt
            if t >= next_out - t_tol:
                if outputs_hook is not None:
                    outputs_hook(history, handle, output_variables)
                else:
                    _collect(history, handle, output_variables)
                out_idx += 1
                next_out = output_times[out_idx]
            # _get_new_time_increment (small_strain_fft.py:266-279)
            fixed = min(next_out - t, end_time - t)
            new_dt = min(dt_max, fixed,
                         dt * 2.0 if out.max_constitutive_iterations < 11 else dt)
            handle.scale_fluctuation(new_dt / dt)
            if stats is not None:
                stats.steps += 1
            dt = new_dt
        else:
            dt = dt / 2.0
            handle.scale_fluctuation(0.5)
            if stats is not None:
                stats.cutbacks += 1
            if dt < min_time_increment:
                raise ValueError("min time increment reached")
    final = {"stress": handle.field("stress"), "strain": handle.field("strain")}
    for v in (output_variables or []):
        final[v] = handle.field(v)
    return final, history


def _collect(history, handle, output_variables):
    for v in (output_variables or []):
        history[v].append(handle.field(v))
    history["stress"].append(handle.field("stress"))
    history["strain"].append(handle.field("strain"))
