"""The CPU oracle pinned against the reference: its own known-answer tests
(tests/test_elastic_model.py, tests/test_elastic_viscoplastic_model.py of materialite
0.1.3) and golden fields produced by running the reference (tests/golden/*.npz)."""

import os

import numpy as np
import pytest
from numpy.testing import assert_allclose

from oracle import ssfft_oracle as O
from oracle.minres import minres

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
VOIGT_TEST = np.array([[160e3, 90e3, 66e3, 0, 0, 0], [90e3, 160e3, 66e3, 0, 0, 0],
                       [66e3, 66e3, 181.7e3, 0, 0, 0], [0, 0, 0, 46.5e3, 0, 0],
                       [0, 0, 0, 0, 46.5e3, 0], [0, 0, 0, 0, 0, 35e3]])


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("seed,indefinite", [(0, False), (1, True), (2, False)])
def test_minres_restatement_matches_scipy(seed, indefinite):
    from scipy.sparse.linalg import minres as sp_minres
    rng = np.random.default_rng(seed)
    n = 60
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = rng.uniform(1, 10, n) * (np.where(rng.random(n) < 0.3, -1, 1) if indefinite else 1)
    A = Q @ np.diag(ev) @ Q.T
    b = rng.standard_normal(n)
    its = []
    x_ref, _ = sp_minres(A, b, rtol=1e-10, callback=lambda xk: its.append(1))
    x, it = minres(lambda v: A @ v, b, 1e-10)
    assert it == len(its)
    assert_allclose(x, x_ref, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("tag", ["4x4x4", "3x4x5", "6x5x8"])
def test_projection_matches_reference(tag):
    g = golden(f"projection_{tag}")
    G = O.projection_operator(tuple(g["dims"]), g["mask"])
    out = O.apply_projection(G, g["tau"])
    assert rel(out, g["out"]) < 1e-13


def test_projection_operator_properties():
    G = O.projection_operator((6, 5, 4), [0, 1, 1, 1, 1, 1])
    assert_allclose(G, np.swapaxes(G, -1, -2), atol=1e-15)          # symmetric
    GG = np.einsum("xyzij,xyzjk->xyzik", G, G)
    assert_allclose(GG, G, atol=1e-13)                               # idempotent
    assert_allclose(G[0, 0, 0], np.diag([0, 1, 1, 1, 1, 1]))         # Gamma(0) = diag(mask)
    assert np.all(G[:, :, 2] == 0)                                   # Nyquist plane (even nz)


def test_elastic_known_answer_evpfft_comparison():
    """test_elastic_model.py:130-145: mean stress norm 6.5890252."""
    from materialite_b200.microstructure import euler_to_rotation
    dims = (4, 4, 4)
    R = np.tile(euler_to_rotation(np.array([0.0, np.pi / 4, 0.0])), (64, 1, 1))
    z = np.arange(64) % 4
    R[z <= 1.5] = np.eye(3)  # Box(max_corner=[., ., sizes[2]/2]) with sizes = 3
    load = O.LoadOracle.constant_rates([0, 0, 1.0, 0, 0, 0], np.zeros(6), [1, 1, 0, 0, 0, 0])
    out = O.solve(dims, R, O.ElasticOracle(O.voigt_to_mandel_stiffness(VOIGT_TEST)), load,
                  end_time=5e-5, linear_solver_tolerance=1e-7)
    assert_allclose(np.linalg.norm(out["stress"].mean(axis=0)), 6.5890252)


def evp(kind, props):
    C = O.voigt_to_mandel_stiffness(VOIGT_TEST)
    n, d = O.octahedral_slip_systems()
    return O.EVPOracle(C, O.schmid_mandel(n, d), 1.0, 10.0, 300.0, kind, props)


@pytest.mark.parametrize("tag,kind,props,end,expected", [
    ("voce", "voce", {"tau_1": 100.0, "theta_0": 20000.0, "theta_1": 10.0}, 5e-3, 541.043871),
    ("af", "armstrong_frederick", {"direct_hardening": 10000.0, "dynamic_recovery": 15.0},
     5e-3, 539.345343),
    ("pp", "perfect_plasticity", None, 4e-3, 442.608112),
])
def test_evp_known_answers_and_fields(tag, kind, props, end, expected):
    """test_elastic_viscoplastic_model.py:147-194 (mean stress norms), plus the full
    reference stress and state fields."""
    g = golden(f"evp_{tag}8")
    load = O.LoadOracle.uniaxial(1.0, "z")
    out = O.solve((8, 8, 8), g["rotations"], evp(kind, props), load, end_time=end,
                  initial_time_increment=1e-3, global_tolerance=1e-7,
                  output_variables=["slip_resistances"])
    assert_allclose(np.linalg.norm(out["stress"].mean(axis=0)), expected)
    assert_allclose(out["strain"].mean(axis=0)[2], end)
    assert rel(out["stress"], g["stress"]) < 1e-10
    assert rel(out["slip_resistances"], g["slip_resistances"]) < 1e-10
    assert rel(out["plastic_strains"], g["plastic_strains"]) < 1e-8
    assert rel(out["slip_system_shear_strains"], g["slip_system_shear_strains"]) < 1e-8


def test_evp_linear_hardening_with_pore():
    """test_elastic_viscoplastic_model.py:128-144: 361.276725, multiphase with a
    zero-stiffness pore."""
    g = golden("evp_linear_pore8")
    phase = g["phase"]
    idx = [np.nonzero(phase == 1)[0], np.nonzero(phase == 2)[0]]
    C = O.voigt_to_mandel_stiffness(VOIGT_TEST)
    models = [evp("linear", {"hardening_rate": 10}), O.ElasticOracle(C * 0.0)]
    load = O.LoadOracle.uniaxial(1.0, "z")
    out = O.solve((8, 8, 8), g["rotations"], O.MultiphaseOracle(models, idx, 512), load,
                  end_time=4e-3, initial_time_increment=1e-3, global_tolerance=1e-7)
    assert_allclose(np.linalg.norm(out["stress"].mean(axis=0)), 361.276725)
    assert rel(out["stress"], g["stress"]) < 1e-10


def test_evp_full_strain_control():
    """test_elastic_viscoplastic_model.py:197-224: S33 426.923816, norm 428.328875."""
    g = golden("evp_strainbc8")
    rate = np.array([-0.35, -0.35, 1.0, 0, 0, 0])
    load = O.LoadOracle.constant_rates(rate, np.zeros(6), np.zeros(6))
    out = O.solve((8, 8, 8), g["rotations"], evp("perfect_plasticity", None), load,
                  end_time=4e-3, initial_time_increment=1e-3, global_tolerance=1e-7)
    m = out["stress"].mean(axis=0)
    assert_allclose(np.linalg.norm(m), 428.328875)
    assert_allclose(m[2], 426.923816)
    assert rel(out["stress"], g["stress"]) < 1e-10


def per_point_rotations(g):
    return g["rotations"][np.searchsorted(np.unique(g["grain"]), g["grain"])]


def test_config1_elastic_matches_reference():
    g = golden("config1_elastic16")
    load = O.LoadOracle.uniaxial(1e-3, "x")
    out = O.solve((16, 16, 16), per_point_rotations(g),
                  O.ElasticOracle(O.cubic_stiffness(250.0, 150.0, 120.0)), load, end_time=10.0,
                  initial_time_increment=1.0, global_tolerance=1e-6)
    assert rel(out["stress"], g["stress"]) < 1e-10
    assert rel(out["strain"], g["strain"]) < 1e-10


def config3_model():
    n, d = O.octahedral_slip_systems()
    return O.EVPOracle(O.cubic_stiffness(250.0, 150.0, 120.0), O.schmid_mandel(n, d), 1e-3, 20.0,
                       0.1, "voce", {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0})


def test_config3_evp_matches_reference():
    g = golden("config3_evp8")
    load = O.LoadOracle.uniaxial(1e-3, "x")
    out = O.solve((8, 8, 8), per_point_rotations(g), config3_model(), load, end_time=4.0,
                  initial_time_increment=0.2, global_tolerance=1e-6)
    assert rel(out["stress"], g["stress"]) < 1e-9
    assert rel(out["slip_resistances"], g["slip_resistances"]) < 1e-9


def test_config5_two_phase_matches_reference():
    g = golden("config5_twophase8")
    phase = g["phase"]
    idx = [np.nonzero(phase == 0)[0], np.nonzero(phase == 1)[0]]
    models = [config3_model(), O.ElasticOracle(O.cubic_stiffness(250.0, 150.0, 120.0) * 10.0)]
    load = O.LoadOracle.uniaxial(1e-3, "x")
    out = O.solve((8, 8, 8), per_point_rotations(g), O.MultiphaseOracle(models, idx, 512), load,
                  end_time=3.0, initial_time_increment=0.2, global_tolerance=1e-6)
    assert rel(out["stress"], g["stress"]) < 1e-9


def test_hardening_laws_closed_forms():
    """hardening_laws.py:18-90 against direct evaluation (q = 1)."""
    rng = np.random.default_rng(0)
    g_old = rng.uniform(100, 200, (5, 12))
    Gam = rng.uniform(0, 0.01, 5)
    gdot = rng.standard_normal((5, 12)) * 1e-2
    dt = 0.5
    dg = dt * np.abs(gdot).sum(-1)
    assert_allclose(O.hardening("linear", {"hardening_rate": 7.0}, Gam, g_old, gdot, dt),
                    g_old + 7.0 * dg[:, None])
    af = O.hardening("armstrong_frederick", {"direct_hardening": 100.0, "dynamic_recovery": 2.0},
                     Gam, g_old, gdot, dt)
    assert_allclose(af, g_old + (100.0 - 2.0 * g_old) * (dg / (1 + 2.0 * dg))[:, None])
    # Voce with theta_1 = 0 integrates to g0 + tau1 (1 - exp(-theta0/tau1 Gamma))
    tau1, th0 = 30.0, 1000.0
    g0 = 150.0 + tau1 * (1 - np.exp(-th0 / tau1 * Gam))
    v = O.hardening("voce", {"tau_1": tau1, "theta_0": th0, "theta_1": 0.0}, Gam,
                    np.repeat(g0[:, None], 12, 1), gdot, dt)
    assert_allclose(v[:, 0], 150.0 + tau1 * (1 - np.exp(-th0 / tau1 * (Gam + dg))))


J2_E, J2_G = 150000.0, 60000.0


def j2_model(kind, props, y=150.0):
    return O.J2Oracle(J2_E, J2_G, y, kind, props)


@pytest.mark.parametrize("kind,props,end,expected", [
    ("perfect_plasticity", None, 15e-4, 150.0),
    ("linear", {"hardening_rate": 1000.0}, 15e-4, 150.3980086),
    ("voce", {"tau_1": 30.0, "theta_0": 10000.0, "theta_1": 100.0}, 50e-4, 171.694205),
])
def test_j2_known_answers(kind, props, end, expected):
    """test_isotropic_plasticity.py:30-128: mean stress norms of a uniform 8^3 material."""
    R = np.tile(np.eye(3), (512, 1, 1))
    out = O.solve((8, 8, 8), R, j2_model(kind, props), O.LoadOracle.uniaxial(1.0, "z"),
                  end_time=end, initial_time_increment=1e-4)
    assert_allclose(np.linalg.norm(out["stress"].mean(axis=0)), expected)


def test_j2_multiphase_known_answer():
    """test_multiphase.py:42-73: two identical J2 phases (a box of phase 1 in phase 0)
    give the uniform answer 150.3980086 and uniform plastic strains."""
    R = np.tile(np.eye(3), (512, 1, 1))
    # points in C order (x, y, z) with z fastest; Box(max_corner=[2,2,2]) on a 3x3x3 box
    xs, ys, zs = [a.ravel() * 3.0 / 7.0 for a in np.meshgrid(np.arange(8), np.arange(8),
                                                             np.arange(8), indexing="ij")]
    in_box = (xs <= 2) & (ys <= 2) & (zs <= 2)
    idx = [np.nonzero(~in_box)[0], np.nonzero(in_box)[0]]
    lin = {"hardening_rate": 1000.0}
    model = O.MultiphaseOracle([j2_model("linear", lin), j2_model("linear", lin)], idx, 512)
    out = O.solve((8, 8, 8), R, model, O.LoadOracle.uniaxial(1.0, "z"), end_time=15e-4,
                  initial_time_increment=1e-4)
    assert_allclose(np.linalg.norm(out["stress"].mean(axis=0)), 150.3980086)
    eq = out["eq_plastic_strains"]
    assert_allclose(eq, np.full_like(eq, eq.mean()))


def j2_golden_model(g, second):
    phase = g["phase"]
    idx = [np.nonzero(phase == 0)[0], np.nonzero(phase == 1)[0]]
    lin = j2_model("linear", {"hardening_rate": 1000.0})
    if second == "voce":
        other = j2_model("voce", {"tau_1": 30.0, "theta_0": 10000.0, "theta_1": 100.0}, 120.0)
    else:
        other = O.ElasticOracle(O.cubic_stiffness(250e3, 150e3, 120e3))
    return O.MultiphaseOracle([lin, other], idx, 512)


@pytest.mark.parametrize("tag,second", [("j2two8", "voce"), ("j2incl8", "elastic")])
def test_j2_golden_fields(tag, second):
    """Heterogeneous J2 solves against fields written by the reference itself."""
    g = golden(tag)
    out = O.solve((8, 8, 8), g["rotations"], j2_golden_model(g, second),
                  O.LoadOracle.uniaxial(1.0, "z"), end_time=15e-4,
                  initial_time_increment=1e-4, global_tolerance=1e-7)
    assert rel(out["stress"], g["stress"]) < 1e-10
    assert rel(out["strain"], g["strain"]) < 1e-10
    j2 = g["phase"] == 0
    assert rel(out["eq_plastic_strains"][j2], g["eq_plastic_strains"][j2]) < 1e-9
    assert rel(out["plastic_strains"][j2], g["plastic_strains"][j2]) < 1e-9
    assert rel(out["yield_stresses"][j2], g["yield_stresses"][j2]) < 1e-12
