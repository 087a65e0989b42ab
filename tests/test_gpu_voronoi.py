"""The device Voronoi generator (ssfft_voronoi) against the tree query of the host path,
which restates Material.create_voronoi (materialite/material.py:337-383) and is pinned to
the reference's grain-index known answers: every point gets the same region."""

import numpy as np
import pytest

from materialite_b200 import Material
from materialite_b200.microstructure import (grid_coordinates, nearest_region,
                                             nearest_region_device, periodic_voronoi,
                                             periodic_voronoi_device, voronoi_seeds)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,grains,periodic,spacing", [
    ((16, 16, 16), 20, True, (1, 1, 1)),
    ((32, 24, 40), 100, True, (1, 1, 1)),
    ((17, 9, 30), 57, False, (0.5, 1.25, 1.0)),
    ((64, 64, 64), 200, True, (1, 1, 1)),
    ((24, 24, 24), 1500, True, (1, 1, 1)),      # more seeds than one shared-memory tile
])
def test_device_regions_equal_tree_query(dims, grains, periodic, spacing):
    a = periodic_voronoi(dims, grains, np.random.default_rng(11), spacing=spacing,
                         periodic=periodic)
    b = periodic_voronoi_device(dims, grains, np.random.default_rng(11), spacing=spacing,
                                periodic=periodic)
    assert b.dtype == a.dtype and np.array_equal(a, b)


def test_material_create_voronoi_on_device_matches_host():
    """A material defined by its sizes (spacing = sizes / (N - 1), images shifted by the
    sizes themselves), as the reference's EVP tests build it."""
    host = Material(dimensions=[8, 8, 8], sizes=[3, 3, 3]).create_voronoi(
        num_regions=10, label="grain", rng=np.random.default_rng(0), periodic=True)
    dev = Material(dimensions=[8, 8, 8], sizes=[3, 3, 3]).create_voronoi(
        num_regions=10, label="grain", rng=np.random.default_rng(0), periodic=True, device=0)
    assert np.array_equal(host.extract("grain"), dev.extract("grain"))


def test_origin_offset_points():
    dims, sizes, origin = (12, 10, 14), np.array([11.0, 9.0, 13.0]), (-2.5, 1.0, 0.25)
    seeds = voronoi_seeds(30, sizes, origin, np.random.default_rng(3))
    points, _ = grid_coordinates(dims, origin)
    a = nearest_region(points, seeds, sizes, True)
    b = nearest_region_device(dims, seeds, sizes, origin, (1, 1, 1), True)
    assert np.array_equal(a, b)
