"""EVP-FFT and JSON files, against files written by the reference itself
(tests/golden/make_golden.py::wire_formats) and the reference's own tests of these formats
(tests/test_material.py:611-630, tests/test_importers.py:248-276,
tests/test_json_operations.py:44-80 of materialite 0.1.3)."""

import json
import os

import numpy as np
import pandas as pd
import pytest
from numpy.testing import assert_allclose, assert_array_equal

from materialite_b200 import (Material, Orientation, Scalar, Sphere, import_evpfft,
                              read_from_json, write_to_json)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden_path(name):
    return os.path.join(GOLDEN, name)


def evpfft_material():
    g = np.load(golden_path("evpfft_4x4x2_inputs.npz"))
    return (Material(dimensions=[4, 4, 2])
            .create_fields({"grain": g["grain"], "phase": g["phase"],
                            "orientation": Orientation(g["rotations"], "p")}))


@pytest.mark.parametrize("tag,degrees", [("degrees", True), ("radians", False)])
def test_export_to_evpfft_matches_reference_file(tmp_path, tag, degrees):
    out = tmp_path / "fields.txt"
    evpfft_material().export_to_evpfft(output=out, euler_angles_to_degrees=degrees)
    assert out.read_text() == open(golden_path(f"evpfft_4x4x2_{tag}.txt")).read()


def test_export_to_evpfft_first_line():
    """test_material.py:611-630."""
    sphere = Sphere(radius=1, centroid=[0, 0, 0])
    material = (Material(dimensions=[2, 2, 2])
                .create_uniform_field("orientation", Orientation.from_euler_angles([0, 0, 0]))
                .create_uniform_field("grain", 1)
                .create_uniform_field("phase", 1)
                .insert_feature(sphere, fields={
                    "grain": 2,
                    "orientation": Orientation.from_euler_angles([30, 45, 60], in_degrees=True)}))
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "small_model_fields.txt")
        material.export_to_evpfft(output=out, euler_angles_to_degrees=True)
        with open(out) as f:
            assert f.readline() == "30.00000 45.00000 60.00000 1 1 1 2 1\n"


def test_export_warns_on_non_power_of_two(tmp_path):
    m = Material(dimensions=[3, 2, 2]).create_uniform_field(
        "orientation", Orientation.identity()).create_uniform_field(
        "grain", 1).create_uniform_field("phase", 1)
    with pytest.warns(UserWarning, match="powers of 2"):
        m.export_to_evpfft(output=tmp_path / "f.txt")


def test_import_evpfft_reads_reference_file():
    """test_importers.py:248-276 on the reference-written file: angles, 0-based ids and
    grain / phase per point."""
    path = golden_path("evpfft_4x4x2_degrees.txt")
    rows = np.loadtxt(path)
    material = import_evpfft(path)
    assert_array_equal(material.dimensions, [4, 4, 2])
    expected = pd.DataFrame(rows, columns=["e1", "e2", "e3", "x_id", "y_id", "z_id", "grain",
                                           "phase"]).sort_values(by=["x_id", "y_id", "z_id"])
    assert_allclose(material.extract("orientation").euler_angles_in_degrees,
                    expected[["e1", "e2", "e3"]].to_numpy(), atol=1e-9)
    assert_array_equal(material.extract(["x_id", "y_id", "z_id"]) + 1,
                       expected[["x_id", "y_id", "z_id"]].to_numpy().astype(int))
    assert_array_equal(material.extract(["grain", "phase"]),
                       expected[["grain", "phase"]].to_numpy().astype(int))
    # the rotations are those of the exported material to the file's five decimals
    R = evpfft_material().extract("orientation").rotation_matrix
    assert_allclose(material.extract("orientation").rotation_matrix, R, atol=1e-6)


def test_euler_angles_round_trip():
    rng = np.random.default_rng(3)
    o = Orientation.random(50, rng=rng)
    back = Orientation.from_euler_angles(o.euler_angles)
    assert_allclose(back.rotation_matrix, o.rotation_matrix, atol=1e-12)
    z = Orientation.from_euler_angles([0.3, 0.0, 0.0])     # R22 = 1: rotation about z only
    assert_allclose(z.euler_angles, [0.3, 0.0, 0.0], atol=1e-15)


def json_material():
    g = np.load(golden_path("material_6x5x4_inputs.npz"))
    m = (Material(dimensions=[6, 5, 4], origin=[1, 2, 3], spacing=[3, 2, 1])
         .create_fields({"grain": g["grain"]})
         .create_regional_fields("grain", pd.DataFrame({
             "grain": np.arange(6),
             "orientation": list(Orientation(g["regional_rotations"], "p"))}))
         .create_fields({"test": g["test"], "scalar_test": Scalar(g["test"] * 100),
                         "array_test": list(g["array_test"])})
         .create_regional_fields("grain", pd.DataFrame({"grain": np.arange(6),
                                                        "grain_data": np.arange(6) * 0.1})))
    m.state = {"1.0": {"stress": 1}, "2.0": {"strain": [1, 2, 3]}}
    return m


def test_read_reference_json():
    m = read_from_json(golden_path("material_6x5x4.json"))
    ref = json_material()
    assert_array_equal(m.dimensions, [6, 5, 4])
    assert_array_equal(m.origin, [1, 2, 3])
    assert_array_equal(m.spacing, [3, 2, 1])
    assert_array_equal(m.extract("grain"), ref.extract("grain"))
    assert_array_equal(m.extract("test"), ref.extract("test"))
    assert_array_equal(m.extract("array_test"), ref.extract("array_test"))
    assert isinstance(m.extract("scalar_test"), Scalar)
    assert_array_equal(m.extract("scalar_test").components, ref.extract("scalar_test").components)
    assert_array_equal(m.extract("orientation").rotation_matrix,
                       ref.extract("orientation").rotation_matrix)
    assert_allclose(m.extract_regional_field("grain", "grain_data"), np.arange(6) * 0.1)
    assert m.state == ref.state


def test_written_json_equals_reference_json(tmp_path):
    out = tmp_path / "m.json"
    write_to_json(json_material(), out)
    ours = json.loads(out.read_text())
    theirs = json.loads(open(golden_path("material_6x5x4.json")).read())
    assert ours == theirs


@pytest.mark.parametrize("compress", [False, True])
def test_write_and_read_yields_same_material(tmp_path, compress):
    """test_json_operations.py:44-80, plain and gzip-compressed."""
    m = json_material()
    out = tmp_path / "m.json"
    write_to_json(m, out, compress=compress)
    back = read_from_json(out, decompress=compress)
    assert_array_equal(back.sizes, m.sizes)
    for label in ("x", "y", "z", "x_id", "y_id", "z_id", "grain", "test", "array_test"):
        assert_array_equal(back.extract(label), m.extract(label))
    assert_allclose(back.extract("orientation").rotation_matrix,
                    m.extract("orientation").rotation_matrix)
    assert_allclose(back.extract("scalar_test").components, m.extract("scalar_test").components)
    assert back.state == m.state
