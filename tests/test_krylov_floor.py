"""The served requests' MINRES floor and relative forcing, checked on the CPU through the
oracle: against the reference-written golden fields of the 16^3 cubic-elastic case (10
increments) and the 8^3 FCC crystal-plasticity case (20 increments), a solve whose linear
solves also stop at the floor (residual <= 0.1 x tolerance x mean von Mises stress) takes the
same Newton iterations and fewer Krylov iterations, and its stress stays within 1e-7 of the
reference's; with a relative forcing of 0.01 on top (residual <= 0.01 |b|) fewer still,
within 1e-6.  The GPU side of the same claims is in test_gpu_serving.py."""

import pytest

from oracle import ssfft_oracle as O
from test_oracle import config3_model, golden, per_point_rotations, rel

FLOOR = 0.1  # materialite_b200.serving.SERVED_KRYLOV_FLOOR


def run(case, floor, forcing=0.0):
    stats = {}
    if case == "elastic":
        g = golden("config1_elastic16")
        out = O.solve((16, 16, 16), per_point_rotations(g),
                      O.ElasticOracle(O.cubic_stiffness(250.0, 150.0, 120.0)),
                      O.LoadOracle.uniaxial(1e-3, "x"), end_time=10.0,
                      initial_time_increment=1.0, global_tolerance=1e-6, stats=stats,
                      krylov_floor=floor, krylov_forcing=forcing)
    else:
        g = golden("config3_evp8")
        out = O.solve((8, 8, 8), per_point_rotations(g), config3_model(),
                      O.LoadOracle.uniaxial(1e-3, "x"), end_time=4.0,
                      initial_time_increment=0.2, global_tolerance=1e-6, stats=stats,
                      krylov_floor=floor, krylov_forcing=forcing)
    return out, stats, g


@pytest.mark.parametrize("case", ["elastic", "evp"])
def test_floor_keeps_the_reference_result(case):
    out0, st0, g = run(case, 0.0)
    out1, st1, _ = run(case, FLOOR)
    assert rel(out0["stress"], g["stress"]) < 1e-10  # the oracle without the floor
    assert rel(out1["stress"], g["stress"]) < 1e-7
    assert st1["newton"] == st0["newton"]
    assert sum(st1["krylov"]) < sum(st0["krylov"])
    if case == "elastic":
        # a linear material under a constant strain rate: after the first increments every
        # right-hand side is under the floor
        assert sum(st1["krylov"]) * 10 < sum(st0["krylov"])
        assert all(k == 0 for k in st1["krylov"][3:])


def test_forcing_keeps_the_reference_result():
    """Inexact Newton on the 8^3 crystal-plasticity case: the relative forcing ends each
    linear solve at 1% of its right-hand side; the Newton iterations stay within 5% and the
    stress within 1e-6."""
    out0, st0, g = run("evp", FLOOR)
    out1, st1, _ = run("evp", FLOOR, 0.01)
    assert rel(out1["stress"], g["stress"]) < 1e-6
    assert sum(st1["newton"]) <= 1.05 * sum(st0["newton"])
    assert sum(st1["krylov"]) < 0.8 * sum(st0["krylov"])


def test_floor_on_the_minres_restatement():
    """With the floor above beta1 no iteration runs; below it the solve stops no later than
    without it, with a residual under the floor or the relative test met."""
    import numpy as np

    from oracle.minres import minres
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((60, 60)))
    A = Q @ np.diag(np.linspace(1.0, 50.0, 60)) @ Q.T
    b = rng.standard_normal(60)
    x, its = minres(lambda v: A @ v, b, 1e-12, atol=2.0 * np.linalg.norm(b))
    assert its == 0 and not x.any()
    x0, its0 = minres(lambda v: A @ v, b, 1e-12)
    atol = 1e-3 * np.linalg.norm(b)
    x1, its1 = minres(lambda v: A @ v, b, 1e-12, atol=atol)
    assert its1 < its0
    assert np.linalg.norm(b - A @ x1) <= 1.01 * atol
