"""Generate golden fixtures by running the reference materialite (0.1.3) itself.

    MATERIALITE_REFERENCE=/path/to/materialite python tests/golden/make_golden.py

Needs the reference checkout (imported through oracle/refshim.py); the fixtures it writes
(tests/golden/*.npz) are committed so that tests run without it.  Every case stores its
inputs (grid, per-point rotation matrices and phases, model parameters) together with the
reference's outputs.
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.refshim import import_reference  # noqa: E402

import_reference()
import pandas as pd  # noqa: E402
from materialite import (Material, Order2SymmetricTensor, Order4SymmetricTensor,  # noqa: E402
                         Orientation, SlipSystem, Sphere)
from materialite.models.small_strain_fft import (Elastic, ElasticViscoplastic,  # noqa: E402
                                                 IsotropicElasticPlastic, LoadSchedule,
                                                 SmallStrainFFT, armstrong_frederick, linear,
                                                 perfect_plasticity, voce)

from materialite_b200.microstructure import quaternion_random_rotations  # noqa: E402

VOIGT_TEST_STIFFNESS = np.array([[160e3, 90e3, 66e3, 0, 0, 0], [90e3, 160e3, 66e3, 0, 0, 0],
                                 [66e3, 66e3, 181.7e3, 0, 0, 0], [0, 0, 0, 46.5e3, 0, 0],
                                 [0, 0, 0, 0, 46.5e3, 0], [0, 0, 0, 0, 0, 35e3]])


def save(name, **arrays):
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


def projection_cases():
    rng = np.random.default_rng(2024)
    for dims, mask in [((4, 4, 4), [1, 1, 0, 1, 1, 1]), ((3, 4, 5), [0, 0, 0, 0, 0, 0]),
                       ((6, 5, 8), [1, 1, 1, 1, 1, 1])]:
        V = int(np.prod(dims))
        tau = rng.standard_normal((V, 6))
        ls = LoadSchedule(None, None, None, np.array(mask, dtype=float))
        m = SmallStrainFFT(load_schedule=ls)
        m._dimensions = np.array(dims)
        m._num_points = V
        m._projection = m._get_projection_operator()
        out = m._apply_projection_tensor(Order2SymmetricTensor(tau, "p"))
        tag = "x".join(str(d) for d in dims)
        save(f"projection_{tag}", dims=np.array(dims), mask=np.array(mask, float), tau=tau,
             out=out)


def config1_elastic():
    """Config-1 physics: 16^3, 20 periodic Voronoi grains, normalised Gaussian
    quaternion orientations, cubic 250/150/120, uniaxial x 1e-3, 10 steps, tol 1e-6."""
    rng = np.random.default_rng(0)
    mat = Material(dimensions=[16, 16, 16]).create_voronoi(num_regions=20, label="grain",
                                                           rng=rng, periodic=True)
    grains = np.unique(mat.extract("grain"))
    rot = quaternion_random_rotations(len(grains), rng)
    mat = mat.create_regional_fields("grain", {"grain": grains, "orientation": Orientation(rot)})
    C = Order4SymmetricTensor.from_cubic_constants(250.0, 150.0, 120.0)
    model = SmallStrainFFT(load_schedule=LoadSchedule.from_constant_uniaxial_strain_rate(1e-3, "x"),
                           end_time=10.0, initial_time_increment=1.0,
                           constitutive_model=Elastic(C))
    t0 = time.time()
    out = model(mat, global_tolerance=1e-6)
    print(f"config 1 reference solve {time.time() - t0:.2f} s")
    save("config1_elastic16", grain=mat.extract("grain"), rotations=rot,
         stress=out.extract("stress").components, strain=out.extract("strain").components)


def evp_material(defect):
    rng = np.random.default_rng(0)
    m = (Material(dimensions=[8, 8, 8], sizes=[3, 3, 3])
         .create_voronoi(num_regions=10, rng=rng).assign_random_orientations(rng=rng)
         .create_uniform_field("phase", 1))
    if defect:
        mid = m.sizes[2] / 2
        m = m.insert_feature(Sphere(radius=1, centroid=[mid, mid, mid]), fields={"phase": 2})
    return m


def reference_evp_cases():
    """The reference's own EVP tests (tests/test_elastic_viscoplastic_model.py:128-224)
    with their full stress fields."""
    C = Order4SymmetricTensor.from_voigt(VOIGT_TEST_STIFFNESS)
    common = dict(stiffness=C, slip_systems=SlipSystem.octahedral(), reference_slip_rate=1.0,
                  rate_exponent=10.0, slip_resistance=300.0)
    laws = {
        "voce": (voce, {"tau_1": 100.0, "theta_0": 20000.0, "theta_1": 10.0}, 5e-3),
        "af": (armstrong_frederick, {"direct_hardening": 10000.0, "dynamic_recovery": 15.0}, 5e-3),
        "pp": (perfect_plasticity, None, 4e-3),
    }
    ls = LoadSchedule.from_constant_uniaxial_strain_rate(direction="z")
    mat = evp_material(False)
    R = mat.extract("orientation").rotation_matrix
    for tag, (law, props, end) in laws.items():
        model = SmallStrainFFT(load_schedule=ls, end_time=end, initial_time_increment=1e-3,
                               constitutive_model=ElasticViscoplastic(
                                   **common, hardening_function=law, hardening_properties=props))
        out = model(mat, global_tolerance=1e-7,
                    output_variables=["slip_resistances", "plastic_strains",
                                      "slip_system_shear_strains"])
        save(f"evp_{tag}8", rotations=R, stress=out.extract("stress").components,
             strain=out.extract("strain").components,
             slip_resistances=out.extract("slip_resistances").components,
             plastic_strains=out.extract("plastic_strains").components,
             slip_system_shear_strains=out.extract("slip_system_shear_strains").components)
    # linear hardening with a zero-stiffness pore (multiphase)
    matd = evp_material(True)
    evp = ElasticViscoplastic(**common, hardening_function=linear,
                              hardening_properties={"hardening_rate": 10})
    pore = Elastic(C * 0.0)
    matd = matd.create_regional_fields("phase", pd.DataFrame({"phase": [1, 2],
                                                              "constitutive_model": [evp, pore]}))
    model = SmallStrainFFT(load_schedule=ls, end_time=4e-3, initial_time_increment=1e-3)
    out = model(matd, phase_label="phase", global_tolerance=1e-7)
    save("evp_linear_pore8", rotations=matd.extract("orientation").rotation_matrix,
         phase=matd.extract("phase"), stress=out.extract("stress").components,
         strain=out.extract("strain").components)
    # full strain control, perfect plasticity
    lsb = LoadSchedule.from_constant_rates(
        strain_rate=Order2SymmetricTensor.from_strain_voigt(np.array([-0.35, -0.35, 1.0, 0, 0, 0])),
        stress_rate=Order2SymmetricTensor.zero(), stress_mask=np.zeros(6))
    model = SmallStrainFFT(load_schedule=lsb, end_time=4e-3, initial_time_increment=1e-3,
                           constitutive_model=ElasticViscoplastic(
                               **common, hardening_function=perfect_plasticity,
                               hardening_properties=None))
    out = model(mat, global_tolerance=1e-7)
    save("evp_strainbc8", rotations=R, stress=out.extract("stress").components,
         strain=out.extract("strain").components)


def config3_evp_small():
    """Config-3 physics (FCC, cubic 250/150/120, reference rate 1e-3, n = 20, Voce
    tau0 = 0.1, tau1 = tau_sat - tau0 = 0.2, theta0 = 1, theta1 = 0) on a small grid:
    8^3, 12 periodic Voronoi grains, uniaxial x 1e-3, 20 steps of dt = 0.2 (0.4% strain,
    past the onset of slip)."""
    rng = np.random.default_rng(3)
    mat = Material(dimensions=[8, 8, 8]).create_voronoi(num_regions=12, label="grain", rng=rng,
                                                        periodic=True)
    grains = np.unique(mat.extract("grain"))
    rot = quaternion_random_rotations(len(grains), rng)
    mat = mat.create_regional_fields("grain", {"grain": grains, "orientation": Orientation(rot)})
    C = Order4SymmetricTensor.from_cubic_constants(250.0, 150.0, 120.0)
    evp = ElasticViscoplastic(C, SlipSystem.octahedral(), 1e-3, 20.0, 0.1, voce,
                              {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0})
    model = SmallStrainFFT(load_schedule=LoadSchedule.from_constant_uniaxial_strain_rate(1e-3, "x"),
                           end_time=4.0, initial_time_increment=0.2, constitutive_model=evp)
    t0 = time.time()
    out = model(mat, global_tolerance=1e-6, output_variables=["slip_resistances"])
    print(f"config 3 (8^3) reference solve {time.time() - t0:.2f} s")
    save("config3_evp8", grain=mat.extract("grain"), rotations=rot,
         stress=out.extract("stress").components, strain=out.extract("strain").components,
         slip_resistances=out.extract("slip_resistances").components)


def config5_two_phase_small():
    """Config-5 physics on a small grid: 8^3, 16 periodic Voronoi grains, each grain
    phase A (config-3 EVP) or B (cubic elastic x10) with probability 1/2, uniaxial x
    1e-3, 15 steps of dt = 0.2."""
    rng = np.random.default_rng(5)
    mat = Material(dimensions=[8, 8, 8]).create_voronoi(num_regions=16, label="grain", rng=rng,
                                                        periodic=True)
    grains = np.unique(mat.extract("grain"))
    rot = quaternion_random_rotations(len(grains), rng)
    phase_of_grain = (rng.random(len(grains)) < 0.5).astype(int)
    mat = mat.create_regional_fields("grain", {"grain": grains, "orientation": Orientation(rot)})
    lut = dict(zip(grains.tolist(), phase_of_grain.tolist()))
    phase = np.array([lut[g] for g in mat.extract("grain")])
    mat = mat.create_fields({"phase": phase})
    C = Order4SymmetricTensor.from_cubic_constants(250.0, 150.0, 120.0)
    evp = ElasticViscoplastic(C, SlipSystem.octahedral(), 1e-3, 20.0, 0.1, voce,
                              {"tau_1": 0.2, "theta_0": 1.0, "theta_1": 0.0})
    stiff = Elastic(C * 10.0)
    mat = mat.create_regional_fields("phase", pd.DataFrame({"phase": [0, 1],
                                                            "constitutive_model": [evp, stiff]}))
    model = SmallStrainFFT(load_schedule=LoadSchedule.from_constant_uniaxial_strain_rate(1e-3, "x"),
                           end_time=3.0, initial_time_increment=0.2)
    t0 = time.time()
    out = model(mat, phase_label="phase", global_tolerance=1e-6)
    print(f"config 5 (8^3) reference solve {time.time() - t0:.2f} s")
    save("config5_twophase8", grain=mat.extract("grain"), rotations=rot, phase=phase,
         stress=out.extract("stress").components, strain=out.extract("strain").components)


def j2_cases():
    """IsotropicElasticPlastic on heterogeneous microstructures: 8^3 on a 3x3x3 box, 10
    Voronoi grains (seed 1), each grain phase 0 or 1.  'j2two': phase 0 linear hardening
    (yield 150, rate 1000), phase 1 Voce (yield 120, 30/10000/100); 'j2incl': phase 0 J2
    linear, phase 1 cubic elastic inclusions (C11/C12/C44 = 250e3/150e3/120e3).  Uniaxial
    z at rate 1, dt 1e-4, 15 steps, with the J2 state fields."""
    rng = np.random.default_rng(1)
    m = (Material(dimensions=[8, 8, 8], sizes=[3, 3, 3])
         .create_voronoi(num_regions=10, label="grain", rng=rng)
         .assign_random_orientations(region_label="grain", rng=rng))
    grains = m.extract("grain")
    phase_of_grain = np.array([0, 1, 0, 0, 1, 0, 1, 0, 0, 1])
    phase = phase_of_grain[grains]
    m = m.create_fields({"phase": phase})
    R = m.extract("orientation").rotation_matrix
    ls = LoadSchedule.from_constant_uniaxial_strain_rate(direction="z")
    j2lin = IsotropicElasticPlastic(150000.0, 60000.0, 150.0, linear, {"hardening_rate": 1000.0})
    j2voce = IsotropicElasticPlastic(150000.0, 60000.0, 120.0, voce,
                                     {"tau_1": 30.0, "theta_0": 10000.0, "theta_1": 100.0})
    incl = Elastic(Order4SymmetricTensor.from_cubic_constants(250e3, 150e3, 120e3))
    for tag, models in [("j2two8", [j2lin, j2voce]), ("j2incl8", [j2lin, incl])]:
        mm = m.create_regional_fields("phase", pd.DataFrame({"phase": [0, 1],
                                                             "constitutive_model": models}))
        model = SmallStrainFFT(load_schedule=ls, end_time=15e-4, initial_time_increment=1e-4)
        out = model(mm, phase_label="phase", global_tolerance=1e-7,
                    output_variables=["yield_stresses", "plastic_strains", "eq_plastic_strains"])
        save(tag, rotations=R, phase=phase, stress=out.extract("stress").components,
             strain=out.extract("strain").components,
             yield_stresses=np.asarray(out.extract("yield_stresses").components, dtype=float),
             plastic_strains=out.extract("plastic_strains").components,
             eq_plastic_strains=out.extract("eq_plastic_strains").components)


def wire_formats():
    """Files written by the reference's own writers (material.py:1035-1091 export_to_evpfft,
    json_operations.py:102-122 write_to_json), with the inputs that built them: a 4x4x2
    material (5 Voronoi grains, random orientations, a spherical phase-2 feature) exported
    for EVP-FFT in degrees and in radians, and a 6x5x4 material with scalar, tensor,
    vector-valued, orientation and regional fields and a state, written as JSON."""
    import json

    from materialite import Scalar, write_to_json
    rng = np.random.default_rng(7)
    m = (Material(dimensions=[4, 4, 2])
         .create_voronoi(num_regions=5, label="grain", rng=rng, periodic=True)
         .assign_random_orientations(region_label="grain", rng=rng)
         .create_uniform_field("phase", 1)
         .insert_feature(Sphere(radius=1.2, centroid=[1, 1, 0]), fields={"phase": 2}))
    for tag, deg in (("degrees", True), ("radians", False)):
        out = os.path.join(HERE, f"evpfft_4x4x2_{tag}.txt")
        m.export_to_evpfft(output=out, euler_angles_to_degrees=deg)
        print(f"wrote {out}")
    save("evpfft_4x4x2_inputs", grain=m.extract("grain"), phase=m.extract("phase"),
         rotations=m.extract("orientation").rotation_matrix)
    rng = np.random.default_rng(12345)
    V = 6 * 5 * 4
    test = rng.random(V)
    arr = rng.random((V, 3))
    mj = (Material(dimensions=[6, 5, 4], origin=[1, 2, 3], spacing=[3, 2, 1])
          .create_voronoi(num_regions=6, label="grain", rng=rng)
          .assign_random_orientations(region_label="grain", rng=rng)
          .create_fields({"test": test, "scalar_test": Scalar(test * 100),
                          "array_test": list(arr)})
          .create_regional_fields("grain", pd.DataFrame({"grain": np.arange(6),
                                                         "grain_data": np.arange(6) * 0.1})))
    mj.state = {"1.0": {"stress": 1}, "2.0": {"strain": [1, 2, 3]}}
    out = os.path.join(HERE, "material_6x5x4.json")
    write_to_json(mj, out)
    print(f"wrote {out} ({os.path.getsize(out) / 1024:.0f} KiB)")
    save("material_6x5x4_inputs", grain=mj.extract("grain"), test=test, array_test=arr,
         rotations=mj.extract("orientation").rotation_matrix,
         regional_rotations=mj.extract_regional_field("grain", "orientation").rotation_matrix)
    json.loads(open(out).read())


if __name__ == "__main__":
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            globals()[name]()
        sys.exit(0)
    projection_cases()
    config1_elastic()
    reference_evp_cases()
    config3_evp_small()
    config5_two_phase_small()
    j2_cases()
    wire_formats()
