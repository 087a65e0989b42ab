"""Seeded microstructure generators with the reference's conventions.

* ``periodic_voronoi`` restates Material.create_voronoi (materialite/material.py:337-383):
  seeds ``rng.random((G,3)) * sizes + origin``; with ``periodic=True`` the seeds are
  tiled over the 27 images shifted by ``sizes`` (= spacing * (N - 1), not N * spacing,
  material.py:103-115) and each point takes the nearest image's region.  The reference
  also tiles the material points (util.repeat_data, util.py:57-88) but keeps only the
  first V answers, which are the untiled points; querying the V points directly gives the
  same regions.
* ``bunge_random_rotations`` restates Orientation.random + from_euler_angles
  (materialite/tensor.py:1855-1912), consuming the generator in the same order.
* ``quaternion_random_rotations`` draws normalised Gaussian quaternions (uniform on
  SO(3)), the sampler named for the large benchmark microstructures.
"""

import numpy as np
from scipy.spatial import cKDTree


def grid_coordinates(dimensions, origin=(0, 0, 0), spacing=(1, 1, 1)):
    """Point coordinates in C order of (x, y, z), z fastest (util.py:40-42)."""
    dims = np.asarray(dimensions, dtype=int)
    x, y, z = np.mgrid[0:dims[0], 0:dims[1], 0:dims[2]]
    ids = np.c_[x.ravel(), y.ravel(), z.ravel()]
    return ids * np.asarray(spacing, float) + np.asarray(origin, float), ids


def periodic_image_shifts(sizes):
    """The 27 shift vectors in util.repeat_data order (util.py:57-88)."""
    sx, sy, sz = (float(s) for s in sizes)
    shifts = [(0, 0, 0)]
    for dz in (-sz, 0.0, sz):
        for dy in (-sy, 0.0, sy):
            for dx in (-sx, 0.0, sx):
                if dx == 0.0 and dy == 0.0 and dz == 0.0:
                    continue
                shifts.append((dx, dy, dz))
    return np.array(shifts)


def voronoi_seeds(num_regions, sizes, origin, rng):
    return rng.random((num_regions, 3)) * np.asarray(sizes, float) + np.asarray(origin, float)


def nearest_region(points, seeds, sizes=None, periodic=False, chunk=1 << 20):
    """Index of the nearest seed (over periodic images when ``periodic``)."""
    G = seeds.shape[0]
    if periodic:
        tiled = (seeds[None, :, :] + periodic_image_shifts(sizes)[:, None, :]).reshape(-1, 3)
    else:
        tiled = seeds
    tree = cKDTree(tiled)
    out = np.empty(points.shape[0], dtype=np.int64)
    for s in range(0, points.shape[0], chunk):
        _, idx = tree.query(points[s:s + chunk], k=1)
        out[s:s + chunk] = idx % G
    return out


def periodic_voronoi(dimensions, num_regions, rng, origin=(0, 0, 0), spacing=(1, 1, 1),
                     periodic=True):
    dims = np.asarray(dimensions, dtype=int)
    sizes = np.asarray(spacing, float) * (dims - 1)
    seeds = voronoi_seeds(num_regions, sizes, origin, rng)
    points, _ = grid_coordinates(dims, origin, spacing)
    return nearest_region(points, seeds, sizes, periodic)


def nearest_region_device(dimensions, seeds, sizes, origin=(0, 0, 0), spacing=(1, 1, 1),
                          periodic=False, device=0):
    """nearest_region for the points of a regular grid, on the GPU (ssfft_voronoi): the
    same regions as the tree query, except for exact distance ties between two seeds."""
    import ctypes

    from . import _native as nat
    dims = np.asarray(dimensions, dtype=np.int32)
    seeds = np.ascontiguousarray(seeds, dtype=np.float64).reshape(-1, 3)
    out = np.empty(int(np.prod(dims.astype(np.int64))), dtype=np.int32)
    vec = lambda a: (ctypes.c_double * 3)(*[float(x) for x in a])
    lib = nat.load_library()
    nat.check(lib.ssfft_voronoi((ctypes.c_int32 * 3)(*[int(d) for d in dims]), vec(origin),
                                vec(spacing), vec(sizes), nat.as_double_ptr(seeds),
                                seeds.shape[0], 1 if periodic else 0, int(device),
                                nat.as_int_ptr(out)))
    return out.astype(np.int64)


def periodic_voronoi_device(dimensions, num_regions, rng, origin=(0, 0, 0), spacing=(1, 1, 1),
                            periodic=True, device=0):
    """periodic_voronoi with the nearest-seed search on the GPU: same seeds from ``rng``,
    same regions."""
    dims = np.asarray(dimensions, dtype=int)
    sizes = np.asarray(spacing, float) * (dims - 1)
    seeds = voronoi_seeds(num_regions, sizes, origin, rng)
    return nearest_region_device(dims, seeds, sizes, origin, spacing, periodic, device)


def euler_to_rotation(euler):
    """Bunge (z1, x2, z3) -> rotation taking specimen to crystal components
    (tensor.py:1855-1896)."""
    e = np.asarray(euler, dtype=np.float64)
    c1, c2, c3 = np.cos(e[..., 0]), np.cos(e[..., 1]), np.cos(e[..., 2])
    s1, s2, s3 = np.sin(e[..., 0]), np.sin(e[..., 1]), np.sin(e[..., 2])
    R = np.zeros(e.shape[:-1] + (3, 3))
    R[..., 0, 0] = c1 * c3 - c2 * s1 * s3
    R[..., 0, 1] = c3 * s1 + c1 * c2 * s3
    R[..., 0, 2] = s2 * s3
    R[..., 1, 0] = -c1 * s3 - c2 * c3 * s1
    R[..., 1, 1] = c1 * c2 * c3 - s1 * s3
    R[..., 1, 2] = c3 * s2
    R[..., 2, 0] = s1 * s2
    R[..., 2, 1] = -c1 * s2
    R[..., 2, 2] = c2
    return R


def bunge_random_rotations(n, rng):
    """Orientation.random(n, rng) (tensor.py:1899-1912)."""
    z1 = rng.random(n) * 2.0 * np.pi
    x2 = np.arccos(rng.random(n) * 2.0 - 1.0)
    z3 = rng.random(n) * 2.0 * np.pi
    return euler_to_rotation(np.stack([z1, x2, z3], axis=-1))


def quaternion_random_rotations(n, rng):
    """Uniform SO(3) rotations from normalised Gaussian quaternions (w, x, y, z); the
    returned matrices are the passive (specimen -> crystal) rotations."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y + w * z)
    R[:, 0, 2] = 2 * (x * z - w * y)
    R[:, 1, 0] = 2 * (x * y - w * z)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z + w * x)
    R[:, 2, 0] = 2 * (x * z + w * y)
    R[:, 2, 1] = 2 * (y * z - w * x)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def first_appearance_order(region_ids):
    """Regions in order of first appearance in point order (pandas unique semantics,
    material.py:408-410)."""
    _, first = np.unique(region_ids, return_index=True)
    return np.asarray(region_ids)[np.sort(first)]
