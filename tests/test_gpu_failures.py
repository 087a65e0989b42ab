"""Failure paths, made on the host (no GPU fault): a solve that cannot converge cuts its
time increment down to min_time_increment and raises as the reference does
(small_strain_fft.py:242-246); in the server such a request completes with an error status
and message while the requests beside it finish exactly as they do alone."""

import logging

import numpy as np
import pytest

from oracle import ssfft_oracle as O
from materialite_b200.engine import PhaseSpec, SolverHandle, SolveStats, solve, unique_rotations
from materialite_b200.serving import RVEServer, make_request, run_stream

pytestmark = pytest.mark.gpu


def test_unconverged_steps_cut_back_to_min_time_increment(caplog):
    dims = (8, 8, 8)
    R = np.tile(np.eye(3), (512, 1, 1))
    load = O.LoadOracle.uniaxial(1e-3, "x")
    table, idx = unique_rotations(R)
    # one Newton iteration per attempt against an unreachable tolerance: every attempt fails
    h = SolverHandle(dims, load.mask, "fp64", global_tolerance=1e-30, max_newton_iterations=1)
    h.set_phases([PhaseSpec("elastic", O.cubic_stiffness(250.0, 150.0, 120.0))])
    h.set_microstructure(table, idx)
    st = SolveStats()
    with caplog.at_level(logging.DEBUG, logger="SmallStrainFFT"):
        with pytest.raises(ValueError, match="min time increment"):
            solve(h, load.dstrain, load.dstress, load.stress, end_time=1.0,
                  initial_time_increment=1.0, min_time_increment=0.2, stats=st)
    h.close()
    assert st.cutbacks == 3 and st.steps == 0           # dt 1 -> 0.5 -> 0.25 -> 0.125
    assert "New increment: time 0.0 + 0.25" in caplog.text
    assert "Too many iterations in macroloading loop" in caplog.text


def small_requests():
    rs = [make_request(t, np.random.default_rng(40 + t), sizes=(32,), grains=(30, 30),
                       steps=(4, 4)) for t in range(3)]
    for r in rs:
        r.keep_stress = True
    return rs


def test_failing_request_leaves_its_neighbours_untouched():
    alone = []
    for r in small_requests():
        if r.tag == 1:
            continue
        srv = RVEServer(max_slots=1)
        comps, _ = run_stream(srv, [r])
        srv.close()
        assert comps[0].status == 0
        alone.append(r.stress.copy())
    mix = small_requests()
    mix[1].global_tolerance = 1e-30        # never converges: cut back to the minimum dt
    srv = RVEServer(max_slots=3)
    comps, _ = run_stream(srv, mix, timeout=300)
    srv.close()
    bad = comps[1]
    assert bad.status == -1 and b"min time increment" in bad.message
    assert comps[0].status == 0 and comps[2].status == 0
    assert np.array_equal(mix[0].stress, alone[0])
    assert np.array_equal(mix[2].stress, alone[1])
