"""GPU parity at the grid sizes the benchmark workloads run, against the CPU oracle, through
the C ABI.

* 48^3 and 96^3 carry radix-3 stages (the serving stream's sizes).
* 96^3 in FP64 runs the five-pass projector because its yz plane does not fit in shared
  memory; 96^3 in float runs plane-fused.
* 128-point yz planes (the plane of the 128^3 workload) and other planes too large for one
  block run plane-fused on thread-block clusters (2 blocks in float, 4 in FP64 at 128x128;
  SSFFT_CLUSTER asks for larger clusters), and on the five-pass projector.
* Crystal plasticity at 32^3 (the smallest serving size) on both projector paths.
* One case with CUDA graphs off (SSFFT_NO_GRAPHS=1): every Krylov kernel launched from the
  host.

Tolerances: elastic FP64 <= 1e-9, crystal plasticity FP64 <= 1e-6 (the per-point inner
Newton stopping against the reference's half-converged subset rule,
elastic_viscoplastic.py:116-158), mixed precision <= 1e-5 (relative L2 of stress and
strain fields).
"""

import functools

import numpy as np
import pytest

from oracle import ssfft_oracle as O
from materialite_b200.engine import PhaseSpec, SolverHandle, SolveStats, solve, unique_rotations
from materialite_b200.microstructure import (bunge_random_rotations, first_appearance_order,
                                             periodic_voronoi)

pytestmark = pytest.mark.gpu

C_CUBIC = O.cubic_stiffness(250.0, 150.0, 120.0)
VOCE = {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0}


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def micro(dims, grains, seed):
    rng = np.random.default_rng(seed)
    ids = periodic_voronoi(dims, grains, rng)
    order = first_appearance_order(ids)
    R = bunge_random_rotations(len(order), rng)
    lut = np.zeros(grains, dtype=int)
    lut[order] = np.arange(len(order))
    return R[lut[ids]]


def schmid():
    n, d = O.octahedral_slip_systems()
    return O.schmid_mandel(n, d)


def assert_counts_close(st, ost):
    """FP64 Krylov iteration counts follow the oracle's: one Newton iteration per linear
    solve, and each solve's count within one iteration (a stopping test that lands within
    round-off of the tolerance may go either way)."""
    assert sum(st.newton_iterations) == len(ost["krylov"])
    assert abs(sum(st.krylov_iterations) - sum(ost["krylov"])) <= len(ost["krylov"])


def use_path(monkeypatch, path):
    if path == "five_pass":
        monkeypatch.setenv("SSFFT_NO_PLANE", "1")
    else:
        monkeypatch.delenv("SSFFT_NO_PLANE", raising=False)


def use_cluster(monkeypatch, path):
    """plane: the default plane-fused path (clusters where one block cannot hold the
    plane); clusterN: clusters of at least N blocks; five_pass: no plane fusion."""
    monkeypatch.delenv("SSFFT_CLUSTER", raising=False)
    use_path(monkeypatch, "five_pass" if path == "five_pass" else "plane")
    if path.startswith("cluster"):
        monkeypatch.setenv("SSFFT_CLUSTER", path[len("cluster"):])


@functools.lru_cache(maxsize=None)
def elastic_reference(dims, steps, grains=40, seed=3):
    R = micro(dims, grains, seed)
    load = O.LoadOracle.uniaxial(1e-3, "x")
    st = {}
    ref = O.solve(dims, R, O.ElasticOracle(C_CUBIC), load, end_time=float(steps),
                  initial_time_increment=1.0, global_tolerance=1e-6,
                  linear_solver_tolerance=1e-8, stats=st)
    return R, ref, st


@functools.lru_cache(maxsize=None)
def evp_reference(dims, steps, grains=40, seed=3):
    R = micro(dims, grains, seed)
    load = O.LoadOracle.uniaxial(1e-3, "x")
    ref = O.solve(dims, R, O.EVPOracle(C_CUBIC, schmid(), 1e-3, 20.0, 0.1, "voce", VOCE), load,
                  end_time=0.6 * steps, initial_time_increment=0.6, global_tolerance=1e-6)
    return R, ref


def run_elastic(dims, R, steps, precision):
    load = O.LoadOracle.uniaxial(1e-3, "x")
    table, idx = unique_rotations(R)
    h = SolverHandle(dims, load.mask, precision, global_tolerance=1e-6,
                     linear_solver_tolerance=1e-8)
    try:
        h.set_phases([PhaseSpec("elastic", C_CUBIC)])
        h.set_microstructure(table, idx)
        st = SolveStats()
        out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=float(steps),
                       initial_time_increment=1.0, stats=st)
    finally:
        h.close()
    return out, st


def run_evp(dims, R, steps, precision):
    load = O.LoadOracle.uniaxial(1e-3, "x")
    table, idx = unique_rotations(R)
    h = SolverHandle(dims, load.mask, precision, global_tolerance=1e-6)
    try:
        h.set_phases([PhaseSpec("evp", C_CUBIC, schmid(), 1e-3, 20.0, 0.1, "voce", VOCE)])
        h.set_microstructure(table, idx)
        out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=0.6 * steps,
                       initial_time_increment=0.6)
    finally:
        h.close()
    return out


@pytest.mark.parametrize("path", ["plane", "cluster2", "five_pass"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_elastic_48(precision, tol, path, monkeypatch):
    """48^3 (radix 3 x 16), 40 periodic Voronoi grains, two load steps; cluster2 runs the
    plane passes on 2-block clusters although one block would hold the plane."""
    use_cluster(monkeypatch, path)
    dims = (48, 48, 48)
    R, ref, ost = elastic_reference(dims, 2)
    out, st = run_elastic(dims, R, 2, precision)
    assert st.steps == 2
    assert rel_l2(out["stress"], ref["stress"]) < tol
    assert rel_l2(out["strain"], ref["strain"]) < tol
    if precision == "fp64":
        assert_counts_close(st, ost)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_elastic_96(precision, tol):
    """96^3: five-pass in FP64 (the double yz plane exceeds shared memory), plane-fused in
    float; one load step."""
    dims = (96, 96, 96)
    R, ref, ost = elastic_reference(dims, 1)
    out, st = run_elastic(dims, R, 1, precision)
    assert rel_l2(out["stress"], ref["stress"]) < tol
    assert rel_l2(out["strain"], ref["strain"]) < tol
    if precision == "fp64":
        assert_counts_close(st, ost)


@pytest.mark.parametrize("path", ["plane", "cluster8", "five_pass"])
@pytest.mark.parametrize("dims", [(4, 128, 128), (3, 128, 135), (2, 144, 120)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 3e-6)])
def test_cluster_projection(dims, precision, tol, path, monkeypatch):
    """The projection on planes too large for one block: 128x128 (the 128^3 workload's
    plane), an odd z length (135 = 3^3 5, 68 stored columns) and 144x120 (radix 3 along y,
    radix 3 and 5 along z), against the oracle's Gamma-hat."""
    use_cluster(monkeypatch, path)
    V = int(np.prod(dims))
    mask = [0, 1, 1, 1, 1, 1]
    tau = np.random.default_rng(11).standard_normal((V, 6))
    h = SolverHandle(dims, mask, precision)
    try:
        out = h.apply_projection(tau)
    finally:
        h.close()
    ref = O.apply_projection(O.projection_operator(dims, mask), tau)
    assert rel_l2(out, ref) < tol


@pytest.mark.parametrize("path", ["plane", "cluster4", "five_pass"])
@pytest.mark.parametrize("dims", [(16, 128, 128), (128, 32, 32)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_elastic_128_axes(dims, precision, tol, path, monkeypatch):
    """128-point axes: 16x128x128 has the 128x128 yz plane of the 128^3 workload (cluster
    passes, or five passes); 128x32x32 has the 128-point x pass of that workload."""
    use_cluster(monkeypatch, path)
    R, ref, ost = elastic_reference(dims, 2)
    out, st = run_elastic(dims, R, 2, precision)
    assert rel_l2(out["stress"], ref["stress"]) < tol
    assert rel_l2(out["strain"], ref["strain"]) < tol
    if precision == "fp64":
        assert_counts_close(st, ost)


@pytest.mark.parametrize("path", ["plane", "five_pass"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_evp_cluster(precision, tol, path, monkeypatch):
    """Crystal plasticity (per-point tangents) on a 4x128x128 grid: the Krylov passes with
    the per-voxel tangent on the cluster path, two load steps past the onset of slip."""
    use_cluster(monkeypatch, path)
    dims = (4, 128, 128)
    R, ref = evp_reference(dims, 2)
    out = run_evp(dims, R, 2, precision)
    assert rel_l2(out["stress"], ref["stress"]) < tol
    assert rel_l2(out["strain"], ref["strain"]) < tol


@pytest.mark.parametrize("path", ["plane", "cluster4", "five_pass"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_evp_32(precision, tol, path, monkeypatch):
    """Serving-size crystal plasticity: 32^3, 40 grains, FCC Voce (config-3 parameters at
    latent ratio 1), two load steps of dt 0.6 past the onset of slip; cluster4 on 4-block
    clusters of 512 threads."""
    use_cluster(monkeypatch, path)
    dims = (32, 32, 32)
    R, ref = evp_reference(dims, 2)
    out = run_evp(dims, R, 2, precision)
    assert rel_l2(out["stress"], ref["stress"]) < tol
    assert rel_l2(out["strain"], ref["strain"]) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_without_graphs(precision, tol, monkeypatch):
    """SSFFT_NO_GRAPHS=1: the Krylov chunk launched kernel by kernel from the host."""
    monkeypatch.setenv("SSFFT_NO_GRAPHS", "1")
    dims = (48, 48, 48)
    R, ref, ost = elastic_reference(dims, 2)
    out, st = run_elastic(dims, R, 2, precision)
    assert rel_l2(out["stress"], ref["stress"]) < tol
    if precision == "fp64":
        assert_counts_close(st, ost)
