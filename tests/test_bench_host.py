"""Host-side pieces of bench.py and the device-only entry points, on CPU: the byte model
behind the roofline, the plane-path rule, the two-phase assignment, the seeded request
stream, and a device path that fails loudly where there is no GPU."""

import numpy as np
import pytest

import bench
from materialite_b200 import _native as nat
from materialite_b200.microstructure import nearest_region_device
from materialite_b200.serving import request_stream


def test_plane_path_rule():
    # one block up to 96^3; clusters of 2 (128^3) and 8 (256^3) blocks; nothing at 512^3
    assert [bench.plane_path(n) for n in (32, 48, 64, 96, 128, 256, 512)] == [True] * 6 + [False]


def test_byte_model():
    b128 = bench.kernel_bytes_per_voxel(128)
    spec = 6 * 64 / 128 * 8.0  # the Nyquist column of an even grid is not stored
    assert b128["zfwd"] == pytest.approx(24 + spec)
    assert b128["update"] == pytest.approx(8 * 24 + 4 + 24) and b128["yfwd"] == 0.0
    assert sum(b128.values()) == pytest.approx(460.0)  # three-pass iteration, elastic tables
    assert bench.kernel_bytes_per_voxel(512)["yfwd"] == pytest.approx(2 * 6 * 256 / 512 * 8.0)
    b64 = bench.kernel_bytes_per_voxel(64, table_mode=False)
    assert b64["yfwd"] == 0.0 and b64["update"] == pytest.approx(8 * 24 + 84 + 24)


def test_two_phase_assignment_is_per_grain_and_seeded():
    w = bench.WORKLOADS["twophase256"]
    ids = np.random.default_rng(0).integers(0, w["grains"], 5000)
    p = bench.phase_of_points(w, ids)
    assert set(np.unique(p)) <= {0, 1}
    for g in np.unique(ids)[:50]:
        assert len(set(p[ids == g])) == 1
    assert np.array_equal(p, bench.phase_of_points(w, ids))
    assert bench.phase_of_points(bench.WORKLOADS["plain64"], ids) is None


def test_request_stream_is_deterministic_and_rate_independent():
    a = request_stream(6, 10.0, seed=1000)
    b = request_stream(6, 50.0, seed=1000)
    for x, y in zip(a, b):
        assert x.dims == y.dims and x.steps == y.steps and x.kind == y.kind
        assert np.array_equal(x.grain, y.grain) and np.array_equal(x.rotations, y.rotations)
    assert all(x.arrival < y.arrival for x, y in zip(a[1:], a[2:]))


def test_device_voronoi_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    seeds = np.random.default_rng(0).random((4, 3)) * 7
    with pytest.raises(nat.SsfftError):
        nearest_region_device((8, 8, 8), seeds, (7.0, 7.0, 7.0), periodic=True)
