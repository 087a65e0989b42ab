"""Host-side mirror of the reference API (no GPU): tensors, Material generators,
LoadSchedule closures and SmallStrainFFT argument handling, against the reference's own
known answers (tests/test_material.py, test_orientation.py, test_load_schedule.py)."""

import numpy as np
import pandas as pd
import pytest
from numpy.testing import assert_allclose, assert_array_equal

from oracle import ssfft_oracle as O
from materialite_b200 import (Box, Material, Order2SymmetricTensor, Order4SymmetricTensor,
                              Orientation, SlipSystem, Sphere, Vector)
from materialite_b200.microstructure import euler_to_rotation
from materialite_b200.small_strain_fft import (Elastic, ElasticViscoplastic,
                                               IsotropicElasticPlastic, LoadSchedule,
                                               SmallStrainFFT, linear, voce)


def test_create_voronoi_known_answers():
    """test_material.py:801-821 (seed 12345, non-periodic and periodic)."""
    m = Material(dimensions=[2, 3, 4], origin=[1, 1, 1]).create_voronoi(
        num_regions=3, rng=np.random.default_rng(12345))
    assert_array_equal(m.extract("region"),
                       [1, 1, 2, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 2, 2, 1, 1, 2, 0, 1, 1, 1, 0])
    m = Material(dimensions=[2, 3, 4], origin=[1, 1, 1]).create_voronoi(
        num_regions=3, rng=np.random.default_rng(12345), periodic=True)
    assert_array_equal(m.extract("region"),
                       [0, 1, 2, 0, 0, 1, 0, 0, 0, 1, 2, 0, 0, 1, 2, 0, 0, 1, 0, 0, 0, 1, 2, 0])


def test_assign_random_orientations_known_answer():
    """test_material.py:823-841: regions by first appearance get Orientation.random
    draws in order."""
    m = Material(dimensions=[2, 3, 4]).assign_random_orientations(
        region_label="z_id", rng=np.random.default_rng(12345))
    z1 = 2 * np.pi * np.array([0.22733602, 0.31675834, 0.79736546 - 1, 0.67625467 - 1])
    x2 = np.arccos(2 * np.array([0.39110955, 0.33281393, 0.59830875, 0.18673419]) - 1)
    z3 = 2 * np.pi * np.array([0.67275604 - 1, 0.94180287 - 1, 0.24824571, 0.94888115 - 1])
    expected = euler_to_rotation(np.tile(np.c_[z1, x2, z3], (6, 1)))
    assert_allclose(m.extract("orientation").rotation_matrix, expected, atol=1e-7)


def test_orientation_random_known_answer():
    """test_orientation.py:107-110."""
    o = Orientation.random(1, rng=np.random.default_rng(12345))
    expected = euler_to_rotation(np.array([1.42839436, 1.94602287, 5.00999493 - 2 * np.pi]))
    assert_allclose(o.rotation_matrix, expected, atol=1e-7)  # squeezed, as in the reference


def check_outputs(ls, t, dt, e_dstrain, e_dstress, e_stress):
    assert_allclose(ls.strain_increment(t, dt).components, e_dstrain, atol=1e-14)
    assert_allclose(ls.stress_increment(t, dt).components, e_dstress, atol=1e-14)
    assert_allclose(ls.stress(t, dt).components, e_stress, atol=1e-14)


def test_load_schedule_constant_rates():
    """test_load_schedule.py:19-33."""
    ls = LoadSchedule.from_constant_rates(Order2SymmetricTensor([1.0, 0, 2.0, 0, 0, 0]),
                                          Order2SymmetricTensor([0, 3.0, 1.0, 0, 0, 0]),
                                          np.array([1, 1, 0, 1, 1, 1]))
    check_outputs(ls, 3.0, 2.0, [0, 0, 4.0, 0, 0, 0], [0, 6.0, 0, 0, 0, 0], [0, 15.0, 0, 0, 0, 0])


def test_load_schedule_uniaxial():
    """test_load_schedule.py:36-55."""
    for d, k in (("x", 0), ("y", 1), ("z", 2)):
        e = np.zeros(6)
        e[k] = 2.0
        check_outputs(LoadSchedule.from_constant_uniaxial_strain_rate(direction=d), 1.0, 2.0, e,
                      np.zeros(6), np.zeros(6))


def test_load_schedule_rejects_non_binary_mask():
    with pytest.raises(ValueError):
        LoadSchedule(None, None, None, np.array([0, 0.5, 1, 1, 1, 1]))


def test_cyclic_strain_schedule():
    amp = Order2SymmetricTensor([1.0, 0, 0, 0, 0, 0])
    ls = LoadSchedule.from_cyclic_strain(amp, 0.25, np.array([0, 1, 1, 1, 1, 1]))
    assert_allclose(ls.strain_increment(0.0, 1.0).components, [1.0, 0, 0, 0, 0, 0], atol=1e-14)


def test_stiffness_conversions_match_oracle():
    C = Order4SymmetricTensor.from_cubic_constants(250.0, 150.0, 120.0)
    assert_allclose(C.components, O.cubic_stiffness(250.0, 150.0, 120.0))
    E = Order4SymmetricTensor.from_isotropic_constants(150000.0, 60000.0)
    assert_allclose(E.components, O.isotropic_stiffness(150000.0, 60000.0))
    assert_allclose(C.voigt[3, 3], 120.0)
    # directional modulus of a cubic crystal along <100>
    s11 = np.linalg.inv(C.voigt)[0, 0]
    assert_allclose(float(C.directional_modulus([1, 0, 0]).components), 1 / s11)


def test_rotations_match_cartesian_definition():
    rng = np.random.default_rng(3)
    R = euler_to_rotation(rng.uniform(0, np.pi, (5, 3)))
    o = Orientation(R)
    assert_allclose(o.rotation_matrix_mandel, O.rotation_matrix_mandel(R))
    eps = Order2SymmetricTensor(rng.standard_normal((5, 6)), "p")
    crys = eps.to_crystal_frame(o)
    expected = np.einsum("pmi,pnj,pij->pmn", R, R, eps.cartesian)
    assert_allclose(crys.cartesian, expected, atol=1e-14)
    assert_allclose(crys.to_specimen_frame(o).components, eps.components, atol=1e-14)


def test_schmid_tensors_match_oracle():
    n, d = O.octahedral_slip_systems()
    assert_allclose(SlipSystem.octahedral().schmid_mandel(), O.schmid_mandel(n, d))


def test_tensor_dims_reductions():
    s = Order2SymmetricTensor(np.arange(2 * 3 * 6, dtype=float).reshape(2, 3, 6), "pt")
    assert s.mean("p").dims_str == "t"
    assert s[:, -1].dims_str == "p"
    assert_allclose(s.mean().components, s.components.reshape(-1, 6).mean(0))
    assert_allclose(s.dev.trace.components, 0.0, atol=1e-12)


def test_material_regional_fields_and_indices():
    m = (Material(dimensions=[4, 4, 4]).create_uniform_field("phase", 1)
         .insert_feature(Box(max_corner=[None, None, 1.5]), fields={"phase": 2}))
    idx = m.get_region_indices("phase")
    assert sorted(idx) == [1, 2]
    assert len(idx[2]) == 32 and len(idx[1]) == 32
    m = m.create_regional_fields("phase", pd.DataFrame({"phase": [1, 2], "E": [10.0, 20.0]}))
    e = m.extract("E")
    assert_allclose(e[idx[1]], 10.0)
    assert_allclose(e[idx[2]], 20.0)
    with pytest.raises(ValueError):
        m.create_regional_fields("phase", {"phase": [1], "F": [1.0]})


def test_sphere_feature():
    m = Material(dimensions=[8, 8, 8], sizes=[3, 3, 3]).create_uniform_field("phase", 1)
    m = m.insert_feature(Sphere(radius=1, centroid=[1.5, 1.5, 1.5]), fields={"phase": 2})
    pts = np.column_stack([m.extract("x"), m.extract("y"), m.extract("z")])
    inside = np.linalg.norm(pts - 1.5, axis=1) <= 1
    assert_array_equal(m.extract("phase") == 2, inside)


def test_smallstrainfft_argument_errors():
    ls = LoadSchedule.from_constant_uniaxial_strain_rate(direction="z")
    mat = Material(dimensions=[4, 4, 4]).create_uniform_field("orientation", Orientation.identity())
    el = Elastic(Order4SymmetricTensor.from_cubic_constants(250.0, 150.0, 120.0))
    with pytest.raises(ValueError, match="cannot specify phase and constitutive model"):
        SmallStrainFFT(load_schedule=ls, constitutive_model=el)(mat, phase_label="phase")
    with pytest.raises(ValueError, match="must specify phase label"):
        SmallStrainFFT(load_schedule=ls)(mat)
    with pytest.raises(ValueError):
        SmallStrainFFT(load_schedule=ls, constitutive_model=el, precision="fp16")


def test_evp_phase_spec_maps_config3_parameters():
    C = Order4SymmetricTensor.from_cubic_constants(250.0, 150.0, 120.0)
    evp = ElasticViscoplastic(C, SlipSystem.octahedral(), 1e-3, 20.0, 0.1, voce,
                              {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0}, latent_ratio=1.4)
    spec = evp.phase_spec()
    assert spec.kind == "evp" and spec.schmid.shape == (12, 6)
    assert spec.hardening == "voce" and spec.latent_ratio == 1.4

    def custom(props, a, b, c, d):
        return b
    with pytest.raises(NotImplementedError):
        ElasticViscoplastic(C, SlipSystem.octahedral(), 1e-3, 20.0, 0.1, custom, {}).phase_spec()


def test_vector_outer_and_norm():
    v = Vector([[3.0, 4.0, 0.0]], "s")
    assert_allclose(v.norm.components, [5.0])
    assert v.outer(v).sym.components.shape == (1, 6)


def test_j2_phase_spec_maps_reference_parameters():
    """IsotropicElasticPlastic(modulus, shear_modulus, yield_stress, law, props)
    (isotropic_elastic_plastic.py:18-53) becomes a "j2" phase."""
    j2 = IsotropicElasticPlastic(150000.0, 60000.0, 150.0, voce,
                                 {"tau_1": 30.0, "theta_0": 10000.0, "theta_1": 100.0})
    spec = j2.phase_spec()
    assert spec.kind == "j2" and spec.hardening == "voce"
    assert spec.modulus == 150000.0 and spec.shear_modulus == 60000.0
    assert spec.slip_resistance == 150.0
    assert abs(j2.bulk_modulus - 60000.0 * 150000.0 / (3 * (180000.0 - 150000.0))) < 1e-9
    assert "eq_plastic_strains" in j2.available_state_variables

    def custom(props, a, b, c, d):
        return b
    with pytest.raises(NotImplementedError):
        IsotropicElasticPlastic(150000.0, 60000.0, 150.0, custom, None).phase_spec()
