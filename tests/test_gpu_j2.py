"""J2 plasticity (IsotropicElasticPlastic) on the GPU.

* The reference's own tests, restated against the drop-in API: tests/
  test_isotropic_plasticity.py:30-128 and tests/test_multiphase.py:42-73 of materialite
  0.1.3.
* Heterogeneous solves against fields written by the reference itself
  (tests/golden/j2two8.npz, j2incl8.npz; tests/golden/make_golden.py::j2_cases), through
  the C ABI, in FP64 and in mixed precision.
"""

import os

import numpy as np
import pandas as pd
import pytest
from numpy.testing import assert_allclose

from oracle import ssfft_oracle as O
from materialite_b200 import Box, Material, Orientation
from materialite_b200.engine import PhaseSpec, SolverHandle, solve, unique_rotations
from materialite_b200.small_strain_fft import (IsotropicElasticPlastic, LoadSchedule,
                                               SmallStrainFFT, linear, perfect_plasticity,
                                               voce)

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
E, G, Y = 150000.0, 60000.0, 150.0
PRECISIONS = [("fp64", 1e-9), ("mixed", 1e-5)]


def uniform_material():
    return (Material(dimensions=[8, 8, 8], sizes=[3, 3, 3])
            .create_uniform_field("orientation", Orientation(np.eye(3)))
            .create_uniform_field("phase", 1))


def run_dropin(model, end_time, precision, output_variables=None):
    ls = LoadSchedule.from_constant_uniaxial_strain_rate(direction="z")
    n = int(round(end_time / 1.0e-4))
    sm = SmallStrainFFT(load_schedule=ls, end_time=end_time, initial_time_increment=1.0e-4,
                        constitutive_model=model, precision=precision)
    times = np.round((np.arange(n) + 1) * 1.0e-4, 10)
    return sm(uniform_material(), output_times=times, output_variables=output_variables)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-7), ("mixed", 1e-5)])
def test_perfect_plasticity(precision, tol):
    """test_isotropic_plasticity.py:30-53: 150.0, axial stress at yield from step 10."""
    m = run_dropin(IsotropicElasticPlastic(E, G, Y, perfect_plasticity, None), 15.0e-4,
                   precision)
    stress = m.extract("stress")
    assert_allclose(stress[:, -1].mean().norm.components, 150.0, rtol=tol)
    assert_allclose(stress.mean("p").components[9:, 2], 150.0, rtol=tol)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-7), ("mixed", 1e-5)])
def test_linear_hardening(precision, tol):
    """test_isotropic_plasticity.py:56-89: 150.3980086; axial stress = yield + H eps_p."""
    m = run_dropin(IsotropicElasticPlastic(E, G, Y, linear, {"hardening_rate": 1000.0}),
                   15.0e-4, precision, ["eq_plastic_strains"])
    stress = m.extract("stress")
    axial = stress.mean("p").components[:, 2]
    eq = m.extract("eq_plastic_strains").mean("p").components
    assert_allclose(stress[:, -1].mean().norm.components, 150.3980086, rtol=tol)
    assert_allclose(stress[:, -1].components[:, 2], axial[-1], rtol=tol)
    assert_allclose(axial[12:], 1000.0 * eq[11:-1] + Y, rtol=tol)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-7), ("mixed", 1e-5)])
def test_voce_hardening(precision, tol):
    """test_isotropic_plasticity.py:92-128: 171.694205; axial stress follows the
    integrated Voce law of the equivalent plastic strain."""
    props = {"tau_1": 30.0, "theta_0": 10000.0, "theta_1": 100.0}
    m = run_dropin(IsotropicElasticPlastic(E, G, Y, voce, props), 50.0e-4, precision,
                   ["eq_plastic_strains"])
    stress = m.extract("stress")
    axial = stress.mean("p").components[:, 2]
    eq = m.extract("eq_plastic_strains").mean("p").components
    integrated = lambda x: Y + (30.0 + 100.0 * x) * (1 - np.exp(-x * np.abs(10000.0 / 30.0)))
    assert_allclose(stress[:, -1].mean().norm.components, 171.694205, rtol=tol)
    assert_allclose(stress[:, -1].components[:, 2], axial[-1], rtol=tol)
    assert_allclose(axial[11:], integrated(eq[10:-1]), rtol=tol)


def test_multiphase_linear_hardening():
    """test_multiphase.py:42-73: two identical J2 phases give the uniform answer and
    uniform plastic strains."""
    lin = {"hardening_rate": 1000.0}
    regional = {"phase": [0, 1],
                "constitutive_model": [IsotropicElasticPlastic(E, G, Y, linear, lin),
                                       IsotropicElasticPlastic(E, G, Y, linear, lin)]}
    mat = (Material(dimensions=[8, 8, 8], sizes=[3, 3, 3])
           .create_uniform_field("orientation", Orientation(np.eye(3)))
           .create_uniform_field("phase", 0)
           .insert_feature(Box(max_corner=[2, 2, 2]), fields={"phase": 1})
           .create_regional_fields(region_label="phase", regional_fields=regional))
    ls = LoadSchedule.from_constant_uniaxial_strain_rate(direction="z")
    times = np.round((np.arange(15) + 1) * 1.0e-4, 10)
    m = SmallStrainFFT(load_schedule=ls, end_time=15.0e-4, initial_time_increment=1.0e-4,
                       precision="fp64")(mat, output_times=times,
                                         output_variables=["eq_plastic_strains"],
                                         phase_label="phase")
    stress = m.extract("stress")
    axial = stress.mean("p").components[:, 2]
    eq = m.extract("eq_plastic_strains")
    mean_eq = eq.mean("p").components
    assert_allclose(stress[:, -1].mean().norm.components, 150.3980086)
    assert_allclose(axial[12:], 1000.0 * mean_eq[11:-1] + Y)
    assert_allclose(eq.components, np.tile(mean_eq, (len(eq), 1)))


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def j2_spec(kind, props, y):
    return PhaseSpec("j2", O.isotropic_stiffness(E, G), slip_resistance=y, hardening=kind,
                     hardening_props=props, modulus=E, shear_modulus=G)


@pytest.mark.parametrize("tag", ["j2two8", "j2incl8"])
@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_heterogeneous_j2_matches_reference_fields(tag, precision, tol):
    g = golden(tag)
    lin = j2_spec("linear", {"hardening_rate": 1000.0}, 150.0)
    if tag == "j2two8":
        other = j2_spec("voce", {"tau_1": 30.0, "theta_0": 10000.0, "theta_1": 100.0}, 120.0)
    else:
        other = PhaseSpec("elastic", O.cubic_stiffness(250e3, 150e3, 120e3))
    load = O.LoadOracle.uniaxial(1.0, "z")
    table, idx = unique_rotations(g["rotations"])
    h = SolverHandle((8, 8, 8), load.mask, precision, global_tolerance=1e-7)
    try:
        h.set_phases([lin, other])
        h.set_microstructure(table, idx, g["phase"].astype(np.int32))
        out, _ = solve(h, load.dstrain, load.dstress, load.stress, end_time=15e-4,
                       initial_time_increment=1e-4,
                       output_variables=["yield_stresses", "plastic_strains",
                                         "eq_plastic_strains"])
    finally:
        h.close()
    assert rel(out["stress"], g["stress"]) < tol
    assert rel(out["strain"], g["strain"]) < tol
    j2 = g["phase"] == 0
    assert rel(out["eq_plastic_strains"][j2, 0], g["eq_plastic_strains"][j2]) < 100 * tol
    assert rel(out["plastic_strains"][j2], g["plastic_strains"][j2]) < 100 * tol
    assert rel(out["yield_stresses"][j2, 0], g["yield_stresses"][j2]) < tol
