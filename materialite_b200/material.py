"""Material: a regular grid of points with per-point and per-region fields, the input
and output container of SmallStrainFFT (materialite/material.py:28-1093).

Point fields are stored column-wise as numpy arrays or tensor objects whose first dim is
the point dim "p" (the reference keeps one Python object per point in a pandas column;
the column form keeps fields contiguous for transfer to and from the device).  Regional
fields are pandas DataFrames keyed by a region field, as in the reference.
"""

import copy

import numpy as np
import pandas as pd

from . import microstructure as ms
from .tensor import Orientation, Scalar, Tensor, Vector


def _is_tensorlike(v):
    return isinstance(v, (Tensor, Orientation))


class Material:
    def __init__(self, dimensions=(16, 16, 16), origin=(0, 0, 0), spacing=(1, 1, 1),
                 sizes=None, fields=None):
        self._dimensions = np.array(dimensions, dtype=int)
        self._origin = np.array(origin, dtype=float)
        spacing = np.array(spacing, dtype=float)
        sizes = np.array(sizes, dtype=float) if sizes is not None else None
        self._spacing, self._sizes = self._get_spacing_and_sizes(spacing, sizes, self._dimensions)
        coords, ids = ms.grid_coordinates(self._dimensions, self._origin, self._spacing)
        self._fields = {"x": coords[:, 0], "y": coords[:, 1], "z": coords[:, 2],
                        "x_id": ids[:, 0], "y_id": ids[:, 1], "z_id": ids[:, 2]}
        if fields is not None:
            self._set_user_fields(fields)
        self.state = dict()
        self._regional_fields = dict()

    @staticmethod
    def _get_spacing_and_sizes(spacing, sizes, dimensions):
        """material.py:103-115: spacing = sizes / (N - 1), sizes = spacing * (N - 1)."""
        if sizes is not None:
            spacing = np.divide(sizes, dimensions - 1, out=np.zeros_like(sizes, dtype=float),
                                where=dimensions != 1)
            sizes = sizes.copy()
            sizes[np.where(dimensions == 1)[0]] = 0
        else:
            sizes = spacing * (dimensions - 1)
        return spacing, sizes

    def _set_user_fields(self, fields):
        df = pd.DataFrame(fields)
        if {"x", "y", "z"}.issubset(df.columns):
            df = df.sort_values(by=["x", "y", "z"]).reset_index(drop=True)
        if len(df) != self.num_points:
            raise ValueError("fields must have one row per grid point")
        for c in df.columns:
            if c in ("x", "y", "z"):
                continue
            self._fields[c] = self._column(df[c].to_list())

    def _column(self, values):
        if _is_tensorlike(values):
            if values.shape[:1] != (self.num_points,):
                raise ValueError("tensor field must have one entry per point")
            return values
        if isinstance(values, (list, tuple)) and values and _is_tensorlike(values[0]):
            return type(values[0]).from_list(list(values))
        arr = np.asarray(values)
        if arr.shape[:1] != (self.num_points,):
            raise ValueError("field must have one value per point")
        return arr

    # ---- geometry -----------------------------------------------------------------------
    @property
    def origin(self):
        return self._origin.copy()

    @property
    def dimensions(self):
        return self._dimensions.copy()

    @property
    def spacing(self):
        return self._spacing.copy()

    @property
    def sizes(self):
        return self._sizes.copy()

    @property
    def center(self):
        return self.origin + self.sizes / 2

    @property
    def far_corner(self):
        return self.origin + self.sizes

    @property
    def num_points(self):
        return int(np.prod(self._dimensions))

    def run(self, model, **kwargs):
        return model(self, **kwargs)

    def copy(self):
        new = copy.copy(self)
        new._fields = dict(self._fields)
        new._regional_fields = {k: v.copy() for k, v in self._regional_fields.items()}
        new.state = dict(self.state)
        return new

    # ---- fields ---------------------------------------------------------------------------
    @property
    def fields(self):
        return self.get_fields(include_regional=False)

    def get_fields(self, include_regional=True):
        data = {}
        for k, v in self._fields.items():
            data[k] = list(v) if _is_tensorlike(v) else v
        df = pd.DataFrame(data)
        if include_regional:
            for k, v in self._regional_fields.items():
                df = df.merge(v, on=k, how="left", suffixes=(False, False),
                              validate="many_to_one")
        return df

    def _regional_lookup(self, label):
        for region_label, df in self._regional_fields.items():
            if label in df.columns and label != region_label:
                keys = np.asarray(df[region_label].to_list())
                point_regions = np.asarray(self._fields[region_label])
                order = np.argsort(keys, kind="stable")
                pos = np.searchsorted(keys[order], point_regions)
                rows = order[np.clip(pos, 0, len(keys) - 1)]
                vals = df[label].to_list()
                if _is_tensorlike(vals[0]):
                    return type(vals[0]).from_list(vals)[rows]
                return np.asarray(vals)[rows]
        raise KeyError(label)

    def extract(self, labels):
        if isinstance(labels, str):
            if labels in self._fields:
                return self._fields[labels]
            return self._regional_lookup(labels)
        return np.column_stack([np.asarray(self.extract(l)) for l in labels])

    def create_fields(self, fields):
        material = self.copy()
        for k, v in fields.items():
            material._fields[k] = material._column(v)
        return material

    def create_uniform_field(self, label, value):
        if _is_tensorlike(value):
            if isinstance(value, Orientation):
                R = np.broadcast_to(value.rotation_matrix, (self.num_points, 3, 3)).copy()
                return self.create_fields({label: Orientation(R, "p")})
            return self.create_fields({label: value.repeat(self.num_points)})
        return self.create_fields({label: np.full(self.num_points, value)})

    def create_random_integer_field(self, label, low, high=None, rng=None):
        rng = np.random.default_rng() if rng is None else rng
        return self.create_fields({label: rng.integers(low=low, high=high, size=self.num_points)})

    def remove_field(self, field_label, in_regional_field=None):
        material = self.copy()
        if in_regional_field is not None:
            material._regional_fields[in_regional_field] = \
                material._regional_fields[in_regional_field].drop(field_label, axis=1)
        else:
            material._fields.pop(field_label, None)
            material._regional_fields.pop(field_label, None)
        return material

    # ---- generators -------------------------------------------------------------------
    def create_voronoi(self, num_regions=10, label="region", rng=None, periodic=False,
                       device=None):
        """material.py:337-383 (seeds, 27 periodic images shifted by ``sizes``).  With
        ``device`` (a CUDA ordinal) the nearest-seed search runs on that GPU."""
        rng = np.random.default_rng() if rng is None else rng
        seeds = ms.voronoi_seeds(num_regions, self.sizes, self.origin, rng)
        if device is not None:
            regions = ms.nearest_region_device(self.dimensions, seeds, self.sizes, self.origin,
                                               self.spacing, periodic, device)
        else:
            points = np.column_stack([self._fields["x"], self._fields["y"], self._fields["z"]])
            regions = ms.nearest_region(points, seeds, self.sizes, periodic)
        return self.create_fields({label: regions})

    def assign_random_orientations(self, region_label="region", orientation_label="orientation",
                                   rng=None):
        """material.py:385-419: Orientation.random over regions in order of first
        appearance, stored as a regional field sorted by region."""
        rng = np.random.default_rng() if rng is None else rng
        unique_regions = ms.first_appearance_order(self._fields[region_label])
        orientations = Orientation.random(len(unique_regions), rng=rng)
        if len(unique_regions) == 1:
            orientations = Orientation(orientations.rotation_matrix[None], "p")
        df = pd.DataFrame({region_label: unique_regions, orientation_label: list(orientations)})
        return self.create_regional_fields(
            region_label, df.sort_values(by=region_label, ignore_index=True))

    def insert_feature(self, feature, fields):
        """material.py:421-482."""
        points = Vector(np.column_stack([self._fields["x"], self._fields["y"], self._fields["z"]]),
                        "p")
        inside = np.asarray(feature.check_inside(points))
        new_fields = {}
        for label, values in fields.items():
            if label in self._fields:
                current = self._fields[label]
                new_values = current.copy()
            elif isinstance(values, Orientation):
                new_values = Orientation(np.broadcast_to(np.eye(3), (self.num_points, 3, 3)).copy(), "p")
            elif _is_tensorlike(values):
                new_values = type(values).zero().repeat(self.num_points)
            else:
                new_values = np.zeros(self.num_points)
            if inside.ndim == 1:
                rows = np.nonzero(inside)[0]
                cols = None
            else:
                idx = np.nonzero(inside)
                rows = idx[0]
                cols = np.ravel_multi_index(idx[1:], inside.shape[1:])
            uniform = np.isscalar(values) or (_is_tensorlike(values) and not values.dims_str)
            if isinstance(new_values, Orientation):
                R = new_values.rotation_matrix
                R[rows] = values.rotation_matrix if uniform else values.rotation_matrix[cols]
            elif _is_tensorlike(new_values):
                new_values.components[rows] = values.components if uniform else values.components[cols]
            else:
                new_values[rows] = values if uniform else np.asarray(values)[cols]
            new_fields[label] = new_values
        return self.create_fields(new_fields)

    # ---- regional fields --------------------------------------------------------------
    def create_regional_fields(self, region_label, regional_fields):
        """material.py:510-573."""
        if isinstance(regional_fields, dict):
            regional_fields = {k: (list(v) if _is_tensorlike(v) else v)
                               for k, v in regional_fields.items()}
        regional_fields = pd.DataFrame(regional_fields)
        if regional_fields[region_label].duplicated().any():
            raise ValueError(f"Could not create regional field: {region_label} has non-unique "
                             "values in regional field")
        material = self.copy()
        if region_label in self._regional_fields:
            old = material._regional_fields[region_label].copy()
            if not np.array_equal(np.sort(old[region_label].to_numpy()),
                                  np.sort(regional_fields[region_label].to_numpy())):
                raise ValueError(f"Values of {region_label} do not match between new and "
                                 "existing regional field")
            regional_fields = old[[region_label]].merge(regional_fields, on=region_label,
                                                         how="left").combine_first(old)
        elif region_label not in self._fields:
            raise ValueError(f"Could not create regional field: {region_label} is not a field")
        for c in regional_fields.columns:
            if c != region_label and c in self._fields:
                raise ValueError("Could not create regional field: the provided regional fields "
                                 "include a field that already exists in the Material")
        keys = set(np.asarray(regional_fields[region_label].to_list()).tolist())
        present = set(np.unique(np.asarray(self._fields[region_label])).tolist())
        missing = sorted(present - keys)
        if missing:
            raise ValueError(f"Values of {region_label} not found in regional field: {missing}")
        material._regional_fields[region_label] = regional_fields
        return material

    def extract_regional_field(self, region_label, field_label=None):
        df = self._regional_fields[region_label]
        if field_label is None:
            return df
        data = df[field_label].to_list()
        if _is_tensorlike(data[0]):
            return type(data[0]).from_list(data)
        return data

    def export_to_evpfft(self, orientation_label="orientation", grain_label="grain",
                         phase_label="phase", output="fields.txt", euler_angles_to_degrees=True):
        """The EVP-FFT input file (material.py:1035-1091): one line per point, z slowest
        and x fastest, "e1 e2 e3 x y z grain phase" with Bunge angles to five decimals and
        1-based indices.  Warns when a dimension is not a power of two."""
        import warnings
        dims = self.dimensions
        if not all(d > 0 and (d & (d - 1)) == 0 for d in dims.tolist()):
            warnings.warn("Outputting to EVP-FFT with dimensions that are not powers of 2. Use "
                          "Material.crop_by_range() or Material.crop_by_id_range() if the "
                          "dimensions must be powers of 2.")
        o = self.extract(orientation_label)
        e = o.euler_angles_in_degrees if euler_angles_to_degrees else o.euler_angles
        e = np.asarray(e).reshape(-1, 3)
        ids = [np.asarray(self.extract(k)).astype(np.int64) + 1 for k in ("x_id", "y_id", "z_id")]
        grains = np.asarray(self.extract(grain_label))
        phases = np.asarray(self.extract(phase_label))
        order = np.lexsort((ids[0], ids[1], ids[2]))

        def fmt(a):
            if np.issubdtype(a.dtype, np.floating):
                return ["%.5f" % x for x in a[order]]
            return [str(x) for x in a[order].tolist()]

        cols = [fmt(e[:, 0]), fmt(e[:, 1]), fmt(e[:, 2]), fmt(ids[0]), fmt(ids[1]), fmt(ids[2]),
                fmt(grains), fmt(phases)]
        with open(output, "w") as f:
            f.write("".join(" ".join(row) + "\n" for row in zip(*cols)))

    def get_region_volume_fractions(self, region_label="region"):
        vals, counts = np.unique(np.asarray(self._fields[region_label]), return_counts=True)
        return dict(zip(vals.tolist(), counts / self.num_points))

    def get_region_indices(self, region_label="region"):
        """Point indices per region, regions ascending (material.py:628-646)."""
        regions = np.asarray(self._fields[region_label])
        order = np.argsort(regions, kind="stable")
        vals, starts = np.unique(regions[order], return_index=True)
        bounds = list(starts) + [len(order)]
        return {v.item() if hasattr(v, "item") else v: order[bounds[i]:bounds[i + 1]]
                for i, v in enumerate(vals)}


class Feature:
    """Geometric region used by Material.insert_feature (material.py:1095-1107)."""

    def check_inside(self, points):
        raise NotImplementedError


class Sphere(Feature):
    def __init__(self, radius, centroid):
        self.radius = np.asarray(radius, dtype=float)
        self.centroid = np.asarray(centroid, dtype=float)

    def check_inside(self, points):
        p = points.components
        if self.centroid.ndim == 1:
            return np.linalg.norm(p - self.centroid, axis=-1) <= self.radius
        d = np.linalg.norm(p[:, None, :] - self.centroid[None], axis=-1)
        return d <= self.radius[None]


class Superellipsoid(Feature):
    def __init__(self, x_radius, y_radius, z_radius, shape_exponent, centroid):
        self.radii = np.stack([np.asarray(x_radius, float), np.asarray(y_radius, float),
                               np.asarray(z_radius, float)], axis=-1)
        self.exponent = np.asarray(shape_exponent, dtype=float)
        self.centroid = np.asarray(centroid, dtype=float)

    def check_inside(self, points):
        p = points.components
        if self.centroid.ndim == 1:
            return np.sum((np.abs(p - self.centroid) / self.radii) ** self.exponent, axis=-1) <= 1
        d = np.abs(p[:, None, :] - self.centroid[None]) / self.radii[None]
        return np.sum(d ** self.exponent[None, :, None], axis=-1) <= 1


class Box(Feature):
    def __init__(self, min_corner=(-np.inf, -np.inf, -np.inf), max_corner=(np.inf, np.inf, np.inf)):
        self.min_corner = self._remove_nones(min_corner, -np.inf)
        self.max_corner = self._remove_nones(max_corner, np.inf)

    @staticmethod
    def _remove_nones(corner, default):
        if isinstance(corner, Vector):
            corner = corner.components
        arr = np.array(corner, dtype=object)
        flat = [default if x is None else x for x in arr.ravel()]
        return np.asarray(flat, dtype=float).reshape(arr.shape)

    def check_inside(self, points):
        p = points.components
        if self.min_corner.ndim == 1:
            return np.all(p >= self.min_corner, axis=-1) & np.all(p <= self.max_corner, axis=-1)
        return (np.all(p[:, None, :] >= self.min_corner[None], axis=-1)
                & np.all(p[:, None, :] <= self.max_corner[None], axis=-1))
