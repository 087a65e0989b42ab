"""The reference's own SmallStrainFFT tests, restated against the drop-in API
(materialite_b200 in place of materialite), running on the GPU in FP64.

Sources: tests/test_elastic_model.py:130-270, tests/test_elastic_viscoplastic_model.py:
128-224 and tests/test_hardening_laws.py:74-170 of materialite 0.1.3."""

from functools import partial

import numpy as np
import pandas as pd
import pytest
from numpy.testing import assert_allclose

from materialite_b200 import (Box, Material, Order2SymmetricTensor, Order4SymmetricTensor,
                              Orientation, SlipSystem, Sphere, Vector)
from materialite_b200.small_strain_fft import (Elastic, ElasticViscoplastic, LoadSchedule,
                                               SmallStrainFFT, armstrong_frederick, linear,
                                               perfect_plasticity, voce)

pytestmark = pytest.mark.gpu
assert_allclose_with_atol = partial(assert_allclose, atol=1e-14)

VOIGT = np.array([[160e3, 90e3, 66e3, 0, 0, 0], [90e3, 160e3, 66e3, 0, 0, 0],
                  [66e3, 66e3, 181.7e3, 0, 0, 0], [0, 0, 0, 46.5e3, 0, 0],
                  [0, 0, 0, 0, 46.5e3, 0], [0, 0, 0, 0, 0, 35e3]])


@pytest.fixture
def elastic_model():
    return Elastic(Order4SymmetricTensor.from_voigt(VOIGT))


@pytest.fixture
def material():
    m = Material(dimensions=[4, 4, 4])
    return m.create_uniform_field(
        "orientation", Orientation.from_euler_angles([0, np.pi / 4, 0])).insert_feature(
        Box(max_corner=[None, None, m.sizes[2] / 2]),
        fields={"orientation": Orientation.identity()})


@pytest.fixture
def material_with_defect(elastic_model):
    rng = np.random.default_rng(0)
    sizes = [3, 3, 3]
    mid = sizes[2] / 2
    regional = pd.DataFrame({"phase": [1, 2],
                             "constitutive_model": [elastic_model,
                                                    Elastic(elastic_model.stiffness * 0.0)]})
    return (Material(dimensions=[8, 8, 8], sizes=sizes)
            .create_voronoi(num_regions=10, rng=rng).assign_random_orientations(rng=rng)
            .create_uniform_field("phase", 1)
            .insert_feature(Sphere(radius=1, centroid=[mid, mid, mid]), fields={"phase": 2})
            .create_regional_fields("phase", regional))


def test_compare_elasticity_with_evpfft(material, elastic_model):
    ls = LoadSchedule.from_constant_rates(Order2SymmetricTensor([0, 0, 1.0, 0, 0, 0]),
                                          Order2SymmetricTensor.zero(), np.array([1, 1, 0, 0, 0, 0]))
    model = SmallStrainFFT(load_schedule=ls, end_time=5.0e-5, constitutive_model=elastic_model)
    out = model(material, linear_solver_tolerance=1.0e-7)
    assert_allclose(out.extract("stress").mean().norm.components, 6.5890252)


def test_stress_bc(material_with_defect):
    end_time = 1.0e-4
    ls = LoadSchedule.from_constant_rates(
        Order2SymmetricTensor.zero(), Order2SymmetricTensor(np.array([0, 0, 6, 0, 0, 0])) / end_time,
        np.ones(6))
    out = SmallStrainFFT(load_schedule=ls, end_time=end_time)(
        material_with_defect, phase_label="phase", linear_solver_tolerance=1.0e-7)
    assert_allclose(out.extract("stress").mean().norm.components, 6.0)


def test_elasticity_with_defect(material_with_defect):
    ls = LoadSchedule.from_constant_uniaxial_strain_rate(direction="z")
    out = SmallStrainFFT(load_schedule=ls, end_time=5.0e-5, initial_time_increment=5.0e-5)(
        material_with_defect, phase_label="phase", linear_solver_tolerance=1.0e-7)
    assert_allclose(out.extract("stress").mean().norm.components, 4.547568053)


@pytest.mark.parametrize("rate", [Order2SymmetricTensor([-0.35, -0.35, 1.0, 0, 0, 0]),
                                  Order2SymmetricTensor.from_cartesian(
                                      np.array([[0, 1, 0], [1, 0, 0], [0, 0, 0]]))])
def test_single_crystal_isostrain(elastic_model, rate):
    """test_elastic_model.py:183-222 (tension and shear of a single crystal)."""
    simple = Material(dimensions=[3, 4, 5]).create_uniform_field("orientation",
                                                                  Orientation.identity())
    end_time = 0.001
    expected = (elastic_model.stiffness @ rate * end_time).components
    ls = LoadSchedule.from_constant_rates(rate, Order2SymmetricTensor.zero(), np.zeros(6))
    out = SmallStrainFFT(load_schedule=ls, end_time=end_time, constitutive_model=elastic_model)(
        simple, linear_solver_tolerance=1.0e-7)
    for s in out.extract("stress").components:
        assert_allclose_with_atol(s, expected)


def test_periodicity(elastic_model):
    """test_elastic_model.py:225-270: per-grain stress sets are invariant under periodic
    shifts of the origin."""
    gps = 4
    grains = np.arange(gps ** 3) + 1
    orient = Orientation.random(gps ** 3, rng=np.random.default_rng(12345))
    regional = {"grain": grains, "orientation": orient}
    model = SmallStrainFFT(load_schedule=LoadSchedule.from_constant_uniaxial_strain_rate(direction="z"),
                           end_time=1.0e-4, constitutive_model=elastic_model)
    n = 16
    x, y, z = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    size = 15.0 / gps  # sizes = 15 on a 16^3 unit-spaced grid

    def grain_field(shift):
        ids = lambda c: np.clip(((c + shift) % 16) // (16 / gps), 0, gps - 1).astype(int)
        g = ids(x) * gps * gps + ids(y) * gps + ids(z) + 1
        return g.ravel()

    results = []
    for shift in (0, 2, 8):
        m = Material(dimensions=[n, n, n]).create_fields({"grain": grain_field(shift)})
        m = m.create_regional_fields("grain", regional)
        out = model(m, linear_solver_tolerance=1.0e-7)
        results.append((out.extract("stress").norm.components, m.get_region_indices("grain")))
    base, idx0 = results[0]
    for other, idx in results[1:]:
        for gr in grains:
            assert_allclose(np.sort(other[idx[gr]]), np.sort(base[idx0[gr]]))


@pytest.fixture
def stiffness_tensor():
    return Order4SymmetricTensor.from_voigt(VOIGT)


@pytest.fixture
def material_no_defect():
    rng = np.random.default_rng(0)
    return (Material(dimensions=[8, 8, 8], sizes=[3, 3, 3]).create_voronoi(num_regions=10, rng=rng)
            .assign_random_orientations(rng=rng).create_uniform_field("phase", 1))


def evp(stiffness, law, props):
    return ElasticViscoplastic(stiffness=stiffness, slip_systems=SlipSystem.octahedral(),
                               reference_slip_rate=1.0, rate_exponent=10.0, slip_resistance=300.0,
                               hardening_function=law, hardening_properties=props)


def test_evp_with_linear_hardening_defect(material_no_defect, stiffness_tensor):
    mid = material_no_defect.sizes[2] / 2
    m = material_no_defect.insert_feature(Sphere(radius=1, centroid=[mid, mid, mid]),
                                          fields={"phase": 2})
    e = evp(stiffness_tensor, linear, {"hardening_rate": 10})
    m = m.create_regional_fields("phase", pd.DataFrame(
        {"phase": [1, 2], "constitutive_model": [e, Elastic(e.stiffness * 0.0)]}))
    model = SmallStrainFFT(load_schedule=LoadSchedule.from_constant_uniaxial_strain_rate(direction="z"),
                           end_time=4.0e-3, initial_time_increment=1.0e-3)
    out = model(m, phase_label="phase", global_tolerance=1.0e-7)
    assert_allclose(out.extract("stress").mean().norm.components, 361.276725)
    assert_allclose(out.extract("strain").mean().components[2], 0.004)


@pytest.mark.parametrize("law,props,end,expected", [
    (voce, {"tau_1": 100.0, "theta_0": 20000.0, "theta_1": 10.0}, 5.0e-3, 541.043871),
    (armstrong_frederick, {"direct_hardening": 10000.0, "dynamic_recovery": 15.0}, 5.0e-3,
     539.345343),
    (perfect_plasticity, None, 4.0e-3, 442.608112),
])
def test_evp_hardening_cases(material_no_defect, stiffness_tensor, law, props, end, expected):
    model = SmallStrainFFT(load_schedule=LoadSchedule.from_constant_uniaxial_strain_rate(direction="z"),
                           end_time=end, initial_time_increment=1.0e-3,
                           constitutive_model=evp(stiffness_tensor, law, props))
    out = model(material_no_defect, global_tolerance=1.0e-7)
    assert_allclose(out.extract("stress").mean().norm.components, expected)
    assert_allclose(out.extract("strain").mean().components[2], end)


def test_strain_bcs(material_no_defect, stiffness_tensor):
    rate = Order2SymmetricTensor.from_strain_voigt(np.array([-0.35, -0.35, 1.0, 0, 0, 0]))
    ls = LoadSchedule.from_constant_rates(strain_rate=rate, stress_rate=Order2SymmetricTensor.zero(),
                                          stress_mask=np.zeros(6))
    model = SmallStrainFFT(load_schedule=ls, end_time=4.0e-3, initial_time_increment=1.0e-3,
                           constitutive_model=evp(stiffness_tensor, perfect_plasticity, None))
    out = model(material_no_defect, global_tolerance=1.0e-7)
    s = out.extract("stress").mean()
    assert_allclose(s.norm.components, 428.328875)
    assert_allclose(s.components[2], 426.923816)
    assert_allclose(out.extract("strain").mean().components, rate.components * 0.004, atol=1e-14)


# ---- test_hardening_laws.py: 4^3 single crystal, one slip system, 50 output times ----

@pytest.fixture
def hl_material():
    return Material(dimensions=[4, 4, 4]).create_uniform_field("orientation", Orientation(np.eye(3)))


@pytest.fixture
def hl_setup():
    dt = 1.0e-4
    return {"load_schedule": LoadSchedule.from_constant_uniaxial_strain_rate(direction="x"),
            "initial_time_increment": dt, "end_time": 50 * dt}


@pytest.fixture
def hl_params():
    return {"stiffness": Order4SymmetricTensor.from_isotropic_constants(modulus=150000.0,
                                                                        shear_modulus=60000.0),
            "reference_slip_rate": 1.0, "rate_exponent": 50.0, "slip_resistance": 150.0,
            "slip_systems": SlipSystem(Vector([[1.0, 1.0, 0.0]], "s"), Vector([[1.0, -1.0, 0.0]], "s"))}


HL_TIMES = np.arange(1.0e-4, 50.1e-4, 1.0e-4)
HL_VARS = ["slip_system_shear_strains", "plastic_strains", "slip_resistances"]


def hl_outputs(m):
    g = m.extract("slip_resistances").mean("p").mean("s").components
    gam = m.extract("slip_system_shear_strains").mean("p").mean("s").components
    ep = m.extract("plastic_strains").mean("p").components
    return g, gam, ep


def hl_run(hl_material, hl_setup, hl_params, law, props):
    model = SmallStrainFFT(**hl_setup, constitutive_model=ElasticViscoplastic(
        **hl_params, hardening_function=law, hardening_properties=props))
    return hl_outputs(model(hl_material, output_times=HL_TIMES, output_variables=HL_VARS))


def test_perfect_plasticity(hl_material, hl_setup, hl_params):
    g, _, ep = hl_run(hl_material, hl_setup, hl_params, perfect_plasticity, None)
    assert_allclose(g, hl_params["slip_resistance"])
    assert_allclose(np.sum(ep[:, :3], axis=1), 0, atol=1e-14)


def test_linear_hardening(hl_material, hl_setup, hl_params):
    g, gam, ep = hl_run(hl_material, hl_setup, hl_params, linear, {"hardening_rate": 1000.0})
    assert_allclose((g[-1] - g[0]) / gam[-1], 1000.0)
    assert_allclose(np.sum(ep[:, :3], axis=1), 0, atol=1e-14)


def test_voce_hardening(hl_material, hl_setup, hl_params):
    tau1, th0, th1 = 30.0, 10000.0, 100.0
    g, gam, ep = hl_run(hl_material, hl_setup, hl_params, voce,
                        {"tau_1": tau1, "theta_0": th0, "theta_1": th1})
    integrated = lambda x: hl_params["slip_resistance"] + (tau1 + th1 * x) * (1 - np.exp(-x * abs(th0 / tau1)))
    idx = gam > 1.0e-10
    assert idx.any()
    assert_allclose(integrated(gam[idx]), g[idx])
    assert_allclose(np.sum(ep[:, :3], axis=1), 0, atol=1e-14)


def test_af_hardening(hl_material, hl_setup, hl_params):
    h, r = 10000.0, 20.0
    g, gam, ep = hl_run(hl_material, hl_setup, hl_params, armstrong_frederick,
                        {"direct_hardening": h, "dynamic_recovery": r})
    idx = gam > 1.0e-10
    slips, crss = gam[idx], g[idx]
    assert_allclose((crss[1:] - crss[:-1]) / (h - r * crss[1:]), slips[1:] - slips[:-1])
    assert_allclose(np.sum(ep[:, :3], axis=1), 0, atol=1e-14)
