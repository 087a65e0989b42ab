"""GPU parity of the libssfft path against the CPU oracle (numpy restatement of
materialite's SmallStrainFFT), through the C ABI."""

import numpy as np
import pytest

from oracle import ssfft_oracle as O
from materialite_b200.engine import PhaseSpec, SolverHandle, SolveStats, solve, unique_rotations
from materialite_b200.microstructure import (bunge_random_rotations, first_appearance_order,
                                             periodic_voronoi)

pytestmark = pytest.mark.gpu

UNIAXIAL_X_MASK = [0, 1, 1, 1, 1, 1]
# The two projector pipelines of a Krylov iteration: plane-fused z+y passes (grids whose yz
# plane fits in shared memory) and the five-pass fallback of larger grids, forced here on
# small grids with SSFFT_NO_PLANE=1 (read when a handle is created).
PATHS = ["plane", "five_pass"]


def use_path(monkeypatch, path):
    if path == "five_pass":
        monkeypatch.setenv("SSFFT_NO_PLANE", "1")
    else:
        monkeypatch.delenv("SSFFT_NO_PLANE", raising=False)


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def voronoi_micro(dims, grains, seed, spacing=(1, 1, 1), periodic=True):
    rng = np.random.default_rng(seed)
    ids = periodic_voronoi(dims, grains, rng, spacing=spacing, periodic=periodic)
    order = first_appearance_order(ids)
    R = bunge_random_rotations(len(order), rng)
    lut = np.zeros(grains, dtype=int)
    lut[order] = np.arange(len(order))
    return R[lut[ids]]


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("dims", [(4, 4, 4), (3, 4, 5), (6, 5, 8), (16, 16, 16), (12, 9, 7),
                                  (32, 16, 8), (1, 4, 6)])
@pytest.mark.parametrize("mask", [[0, 0, 0, 0, 0, 0], UNIAXIAL_X_MASK, [1] * 6])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 3e-6)])
def test_projection_matches_oracle(dims, mask, precision, tol, path, monkeypatch):
    use_path(monkeypatch, path)
    V = int(np.prod(dims))
    tau = np.random.default_rng(7).standard_normal((V, 6))
    h = SolverHandle(dims, mask, precision)
    out = h.apply_projection(tau)
    ref = O.apply_projection(O.projection_operator(dims, mask), tau)
    assert rel_l2(out, ref) < tol
    h.close()


def elastic_case(dims, grains, seed):
    R = voronoi_micro(dims, grains, seed)
    C = O.cubic_stiffness(250.0, 150.0, 120.0)
    return R, C


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_elastic_voronoi_solve(precision, tol, path, monkeypatch):
    """Config-1 physics at 16^3 (20 periodic Voronoi grains, cubic 250/150/120,
    uniaxial x strain rate 1e-3), 4 steps."""
    use_path(monkeypatch, path)
    dims = (16, 16, 16)
    R, C = elastic_case(dims, 20, 0)
    load = O.LoadOracle.uniaxial(1e-3, "x")
    kw = dict(end_time=4.0, initial_time_increment=1.0, global_tolerance=1e-6,
              linear_solver_tolerance=1e-8)
    ref = O.solve(dims, R, O.ElasticOracle(C), load, **kw)
    table, idx = unique_rotations(R)
    h = SolverHandle(dims, load.mask, precision, global_tolerance=1e-6,
                     linear_solver_tolerance=1e-8)
    h.set_phases([PhaseSpec("elastic", C)])
    h.set_microstructure(table, idx)
    st = SolveStats()
    out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=4.0,
                   initial_time_increment=1.0, stats=st)
    assert st.steps == 4
    assert rel_l2(out["stress"], ref["stress"]) < tol
    assert rel_l2(out["strain"], ref["strain"]) < tol
    h.close()


def evp_voce_phase(C):
    n, d = O.octahedral_slip_systems()
    return O.schmid_mandel(n, d)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-7), ("mixed", 1e-5)])
def test_evp_voce_reference_case(precision, tol, path, monkeypatch):
    """tests/test_elastic_viscoplastic_model.py:147-161 of the reference: 8^3 grid on a
    3x3x3 box, 10 Voronoi grains (seed 0), Voce hardening; mean stress norm 541.043871."""
    use_path(monkeypatch, path)
    dims = (8, 8, 8)
    R = voronoi_micro(dims, 10, 0, spacing=(3 / 7,) * 3, periodic=False)
    Cv = np.array([[160e3, 90e3, 66e3, 0, 0, 0], [90e3, 160e3, 66e3, 0, 0, 0],
                   [66e3, 66e3, 181.7e3, 0, 0, 0], [0, 0, 0, 46.5e3, 0, 0],
                   [0, 0, 0, 0, 46.5e3, 0], [0, 0, 0, 0, 0, 35e3]])
    C = O.voigt_to_mandel_stiffness(Cv)
    P = evp_voce_phase(C)
    props = {"tau_1": 100.0, "theta_0": 20000.0, "theta_1": 10.0}
    load = O.LoadOracle.uniaxial(1.0, "z")
    ref = O.solve(dims, R, O.EVPOracle(C, P, 1.0, 10.0, 300.0, "voce", props), load,
                  end_time=5e-3, initial_time_increment=1e-3, global_tolerance=1e-7)
    table, idx = unique_rotations(R)
    h = SolverHandle(dims, load.mask, precision, global_tolerance=1e-7)
    h.set_phases([PhaseSpec("evp", C, P, 1.0, 10.0, 300.0, "voce", props)])
    h.set_microstructure(table, idx)
    out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=5e-3,
                   initial_time_increment=1e-3)
    mean_norm = np.linalg.norm(out["stress"].mean(axis=0))
    assert abs(mean_norm - 541.043871) / 541.043871 < max(tol, 1e-7)
    assert rel_l2(out["stress"], ref["stress"]) < tol
    h.close()


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("device_loop", [True, False])
def test_krylov_iteration_limit_matches_oracle(device_loop, path, monkeypatch):
    """max_krylov_iterations = 4 (scipy's maxiter): every MINRES solve stops at the limit
    (istop 6) with its last update applied, through the device-side Krylov loop and through
    the host-polled one; the inexact-Newton solve and its iteration counts match the
    oracle's."""
    use_path(monkeypatch, path)
    if not device_loop:
        monkeypatch.setenv("SSFFT_NO_DEVICE_LOOP", "1")
    dims = (16, 16, 16)
    R, C = elastic_case(dims, 20, 0)
    load = O.LoadOracle.uniaxial(1e-3, "x")
    ost = {}
    ref = O.solve(dims, R, O.ElasticOracle(C), load, end_time=3.0, initial_time_increment=1.0,
                  global_tolerance=1e-6, linear_solver_tolerance=1e-8, stats=ost,
                  krylov_maxiter=4)
    table, idx = unique_rotations(R)
    h = SolverHandle(dims, load.mask, "fp64", global_tolerance=1e-6,
                     linear_solver_tolerance=1e-8, max_krylov_iterations=4)
    h.set_phases([PhaseSpec("elastic", C)])
    h.set_microstructure(table, idx)
    st = SolveStats()
    out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=3.0,
                   initial_time_increment=1.0, stats=st)
    h.close()
    assert max(ost["krylov"]) == 4
    assert sum(st.newton_iterations) == len(ost["krylov"])
    assert sum(st.krylov_iterations) == sum(ost["krylov"])
    assert rel_l2(out["stress"], ref["stress"]) < 1e-9


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("dims", [(10, 6, 9), (12, 9, 7)])
@pytest.mark.parametrize("precision,tol_elastic,tol_evp", [("fp64", 1e-12, 1e-6),
                                                           ("mixed", 1e-6, 1e-5)])
def test_solves_on_odd_non_cubic_grids(dims, precision, tol_elastic, tol_evp, path,
                                       monkeypatch):
    """Grids with odd and mixed-radix axes (radix 3, 5, 7 stages, partial tiles).  The
    elastic solve isolates the transforms and the fused MINRES path: FP64 to round-off.
    Crystal plasticity (rate exponent 20, two load steps past the onset of slip) differs from
    the oracle by the per-point stopping of the inner Newton against the reference's
    half-converged subset rule (elastic_viscoplastic.py:116-158), up to ~6e-7 here."""
    use_path(monkeypatch, path)
    R = voronoi_micro(dims, max(2, int(np.prod(dims)) // 40), 5)
    C = O.cubic_stiffness(250.0, 150.0, 120.0)
    n, d = O.octahedral_slip_systems()
    P = O.schmid_mandel(n, d)
    props = {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0}
    load = O.LoadOracle.uniaxial(1e-3, "x")
    table, idx = unique_rotations(R)

    refe = O.solve(dims, R, O.ElasticOracle(C), load, end_time=2.0, initial_time_increment=1.0,
                   global_tolerance=1e-6, linear_solver_tolerance=1e-8)
    h = SolverHandle(dims, load.mask, precision, global_tolerance=1e-6,
                     linear_solver_tolerance=1e-8)
    h.set_phases([PhaseSpec("elastic", C)])
    h.set_microstructure(table, idx)
    oute, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=2.0,
                    initial_time_increment=1.0)
    h.close()
    assert rel_l2(oute["stress"], refe["stress"]) < tol_elastic

    ref = O.solve(dims, R, O.EVPOracle(C, P, 1e-3, 20.0, 0.1, "voce", props), load,
                  end_time=1.2, initial_time_increment=0.6, global_tolerance=1e-6)
    h = SolverHandle(dims, load.mask, precision, global_tolerance=1e-6)
    h.set_phases([PhaseSpec("evp", C, P, 1e-3, 20.0, 0.1, "voce", props)])
    h.set_microstructure(table, idx)
    out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=1.2,
                   initial_time_increment=0.6)
    h.close()
    assert rel_l2(out["stress"], ref["stress"]) < tol_evp
