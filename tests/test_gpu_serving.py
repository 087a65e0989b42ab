"""Serving: requests solved concurrently on one GPU give the same result as alone, the
native time loop equals the Python one, and admission respects the device-memory
budget."""

import numpy as np
import pytest

from materialite_b200.engine import SolverHandle, solve, unique_rotations
from materialite_b200.serving import (SERVED_KRYLOV_FLOOR, SERVED_KRYLOV_FORCING, RVEServer,
                                      elastic_phase, evp_phase, make_request, run_stream,
                                      solve_plain)

pytestmark = pytest.mark.gpu


def small_requests():
    rs = []
    for tag, seed in enumerate([11, 12, 13, 14]):
        r = make_request(tag, np.random.default_rng(seed), sizes=(32,), grains=(20, 60),
                         steps=(4, 6))
        r.keep_stress = True
        rs.append(r)
    rs[1].phases = [evp_phase()]  # one crystal-plasticity request in the mix
    rs[1].dt = 0.2
    return rs


def test_result_identical_alone_and_in_the_mix():
    reqs = small_requests()
    alone = RVEServer(max_slots=1)
    comps, _ = run_stream(alone, [reqs[1]])
    alone.close()
    assert comps[0].status == 0
    ref = reqs[1].stress.copy()
    reqs2 = small_requests()
    server = RVEServer(max_slots=4)
    comps, _ = run_stream(server, reqs2)
    server.close()
    assert all(c.status == 0 for c in comps)
    # overlapping on the device did not change a single bit of the result
    assert np.array_equal(reqs2[1].stress, ref)
    starts = sorted(c.start_time for c in comps)
    ends = sorted(c.end_time for c in comps)
    assert starts[-1] < ends[0]  # all four were resident at the same time


def test_native_time_loop_matches_python_loop():
    r = make_request(0, np.random.default_rng(21), sizes=(32,), grains=(30, 30), steps=(5, 5))
    r.keep_stress = True
    server = RVEServer(max_slots=1)
    comps, _ = run_stream(server, [r])
    server.close()
    assert comps[0].status == 0
    h = SolverHandle(r.dims, r.stress_mask, "mixed", global_tolerance=r.global_tolerance,
                     linear_solver_tolerance=r.linear_solver_tolerance,
                     krylov_floor=SERVED_KRYLOV_FLOOR, krylov_forcing=SERVED_KRYLOV_FORCING)
    h.set_phases(r.phases)
    table, idx = unique_rotations(r.rotations[r.grain])
    h.set_microstructure(table, idx)
    er = r.strain_rate * (1 - r.stress_mask)
    z = np.zeros(6)
    out, _ = solve(h, lambda t, dt: er * dt, lambda t, dt: z, lambda t, dt: z,
                   end_time=r.dt * r.steps, initial_time_increment=r.dt)
    h.close()
    # same kernels, same order of every reduction: bitwise equal
    assert np.array_equal(out["stress"], r.stress)


def test_admission_by_memory_budget():
    reqs = [r for r in small_requests() if r.tag != 1][:2]
    for r in reqs:  # two elastic requests of the same size: the same device footprint
        r.keep_stress = False
        r.phases = [elastic_phase()]
        r.dt = 1.0
    # a budget below one request's footprint: rejected, not hung
    tiny = RVEServer(max_slots=2, hbm_budget_bytes=1 << 20)
    comps, _ = run_stream(tiny, reqs[:1], timeout=60)
    tiny.close()
    assert comps[0].status == -3
    # a budget for one request at a time: both finish, one after the other
    one = RVEServer(max_slots=2, hbm_budget_bytes=int(1.5 * comps[0].device_bytes))
    comps, _ = run_stream(one, reqs, timeout=120)
    one.close()
    assert all(c.status == 0 for c in comps)
    a, b = sorted(comps, key=lambda c: c.start_time)
    assert b.start_time >= a.end_time


def evp_requests(seeds, steps=(3, 5)):
    rs = []
    for tag, seed in enumerate(seeds):
        r = make_request(tag, np.random.default_rng(seed), sizes=(32,), grains=(20, 60),
                         steps=steps)
        r.phases = [evp_phase()]
        r.dt = 0.2
        r.keep_stress = True
        rs.append(r)
    return rs


def test_batched_requests_identical_alone_and_in_the_group():
    """Four crystal-plasticity requests of one class share a group: every kernel launch
    covers all four (each at its own Newton iteration), and each result is
    still bitwise the one it gets alone (every reduction is private to its slot)."""
    seeds = [31, 32, 33, 34]
    alone = []
    for r in evp_requests(seeds):
        srv = RVEServer(max_slots=1)
        comps, _ = run_stream(srv, [r])
        srv.close()
        assert comps[0].status == 0
        alone.append(r.stress.copy())
    mix = evp_requests(seeds)
    srv = RVEServer(max_slots=4)
    comps, _ = run_stream(srv, mix)
    launches = srv.kernel_launches()
    srv.close()
    assert all(c.status == 0 for c in comps)
    for r, a in zip(mix, alone):
        assert np.array_equal(r.stress, a)
    starts = sorted(c.start_time for c in comps)
    ends = sorted(c.end_time for c in comps)
    assert starts[-1] < ends[0]  # all four were resident at the same time
    assert launches > 0


def test_group_time_loop_matches_python_loop_crystal_plasticity():
    """The device-side Newton decisions, commits and dt updates of a group reproduce the
    host-driven time loop (engine.solve through a handle) bitwise for a crystal-plasticity
    request."""
    r = evp_requests([41], steps=(4, 4))[0]
    server = RVEServer(max_slots=2)
    comps, _ = run_stream(server, [r])
    server.close()
    assert comps[0].status == 0
    h = SolverHandle(r.dims, r.stress_mask, "mixed", global_tolerance=r.global_tolerance,
                     linear_solver_tolerance=r.linear_solver_tolerance,
                     krylov_floor=SERVED_KRYLOV_FLOOR, krylov_forcing=SERVED_KRYLOV_FORCING)
    h.set_phases(r.phases)
    table, idx = unique_rotations(r.rotations[r.grain])
    h.set_microstructure(table, idx)
    er = r.strain_rate * (1 - r.stress_mask)
    z = np.zeros(6)
    out, _ = solve(h, lambda t, dt: er * dt, lambda t, dt: z, lambda t, dt: z,
                   end_time=r.dt * r.steps, initial_time_increment=r.dt)
    h.close()
    assert np.array_equal(out["stress"], r.stress)


def test_late_request_joins_a_running_group():
    """A request that arrives while a long request of its class is running takes a free
    slot at once (the running graph returns at its next pass boundary to load it) instead of
    waiting for the long request to finish, and its result is still bitwise the one it gets
    alone."""
    long_r, short_r = evp_requests([51, 52], steps=(4, 4))
    long_r.steps = 60
    short_r.steps = 2
    short_r.arrival = 0.05
    alone = evp_requests([52], steps=(4, 4))[0]
    alone.steps = 2
    srv = RVEServer(max_slots=1)
    comps, _ = run_stream(srv, [alone])
    srv.close()
    assert comps[0].status == 0
    srv = RVEServer(max_slots=4)
    comps, _ = run_stream(srv, [long_r, short_r])
    srv.close()
    a, b = comps
    assert a.status == 0 and b.status == 0
    assert b.submit_time > a.start_time          # the long request was running
    assert b.end_time < a.end_time               # and the short one did not wait for it
    assert np.array_equal(short_r.stress, alone.stress)


def test_krylov_floor_keeps_the_fp64_result():
    """The served mixed form's MINRES floor (a linear solve stops once its residual could
    move the next equilibrium error by a tenth of the tolerance) takes fewer Krylov
    iterations than the plain FP64 solve, which keeps the reference's stopping test alone,
    with the same increments and cutbacks and stresses within 1e-6 of it, for an elastic
    and a crystal-plasticity request."""
    reqs = small_requests()[:2]  # one elastic, one crystal-plasticity request
    plain = small_requests()[:2]
    _, pouts = solve_plain(plain, precision="fp64")
    server = RVEServer(max_slots=2, krylov_forcing=0.0)  # the floor alone
    comps, _ = run_stream(server, reqs)
    server.close()
    comps = sorted(comps, key=lambda c: c.tag)
    for r, p, c, po in zip(reqs, plain, comps, pouts):
        assert c.status == 0
        assert c.result.steps == po.steps and c.result.cutbacks == po.cutbacks
        err = np.linalg.norm(r.stress - p.stress) / np.linalg.norm(p.stress)
        assert err <= 1e-6, (r.tag, err)
        assert c.result.krylov_iterations < po.krylov_iterations
    assert comps[0].result.newton_iterations == pouts[0].newton_iterations  # elastic


def test_krylov_forcing_stays_within_tolerance():
    """The relative forcing (inexact Newton: each linear solve also ends once its residual is
    1% of its right-hand side) on top of the floor: the same increments and cutbacks as the
    plain FP64 solve, stresses within 2e-6 of it, and fewer Krylov iterations than the floor
    alone for the crystal-plasticity request."""
    plain = small_requests()[:2]
    _, pouts = solve_plain(plain, precision="fp64")
    runs = []
    for forcing in (0.0, 0.01):
        reqs = small_requests()[:2]
        server = RVEServer(max_slots=2, krylov_forcing=forcing)
        comps, _ = run_stream(server, reqs)
        server.close()
        runs.append((reqs, sorted(comps, key=lambda c: c.tag)))
    reqs, comps = runs[1]
    for r, p, c, po in zip(reqs, plain, comps, pouts):
        assert c.status == 0
        assert c.result.steps == po.steps and c.result.cutbacks == po.cutbacks
        err = np.linalg.norm(r.stress - p.stress) / np.linalg.norm(p.stress)
        assert err <= 2e-6, (r.tag, err)
    assert comps[1].result.krylov_iterations < runs[0][1][1].result.krylov_iterations
