"""Host-side tensor objects with materialite's conventions (materialite/tensor.py).

Components follow the reference: symmetric second-order tensors are Mandel 6-vectors
[11, 22, 33, 23, 13, 12] with sqrt(2) on shears (materialite/basis_operations.py:37-48),
symmetric fourth-order tensors are 6x6 Mandel matrices.  Every tensor carries a dims
string naming its leading (non-component) axes -- "p" points, "s" slip systems, "t" time
-- and binary operations align operands by dim name, as the reference does
(tensor.py:67-120, 176-330).

These objects are plumbing for the drop-in API (inputs to SmallStrainFFT and its
outputs); the solve itself runs in libssfft.
"""

from numbers import Number

import numpy as np

SQRT2 = np.sqrt(2.0)
_MANDEL_PAIRS = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
_MANDEL_SCALE = np.array([1.0, 1.0, 1.0, SQRT2, SQRT2, SQRT2])


def _mandel_from_cartesian(M):
    M = np.asarray(M, dtype=np.float64)
    return np.stack([M[..., i, j] * _MANDEL_SCALE[k] for k, (i, j) in enumerate(_MANDEL_PAIRS)],
                    axis=-1)


def _cartesian_from_mandel(v):
    v = np.asarray(v, dtype=np.float64)
    out = np.zeros(v.shape[:-1] + (3, 3))
    for k, (i, j) in enumerate(_MANDEL_PAIRS):
        val = v[..., k] / _MANDEL_SCALE[k]
        out[..., i, j] = val
        out[..., j, i] = val
    return out


def _order_dims(a, b):
    """Union of two dims strings, keeping a's order then b's new dims
    (tensor.py:67-120)."""
    return a + "".join(c for c in b if c not in a)


def _align(data, dims, target, ncomp):
    """Transpose/expand ``data`` (leading dims ``dims``) to the leading dims ``target``."""
    lead = data.ndim - ncomp
    if lead != len(dims):
        raise ValueError(f"dims {dims!r} do not match data of shape {data.shape}")
    order = [dims.index(c) for c in target if c in dims]
    data = np.transpose(data, order + list(range(lead, data.ndim)))
    present = [c for c in target if c in dims]
    shape = []
    k = 0
    for c in target:
        if c in dims:
            shape.append(data.shape[k])
            k += 1
        else:
            shape.append(1)
    return data.reshape(tuple(shape) + data.shape[len(present):])


def _default_dims(n):
    # materialite/tensor.py:327-341: "p" for one leading dim, then "pst..." style defaults
    return "pstuvwxyz"[:n] if n > 0 else ""


class Tensor:
    """Base class: ``components`` with ``_ncomp`` trailing component axes."""

    _ncomp = 0
    __array_ufunc__ = None

    def __init__(self, components, dims=None):
        self.components = np.asarray(components, dtype=np.float64)
        lead = self.components.ndim - self._ncomp
        if lead < 0:
            raise ValueError(f"{type(self).__name__} components have too few axes")
        self.dims_str = _default_dims(lead) if dims is None else dims
        if len(self.dims_str) != lead:
            raise ValueError(f"tried to create {type(self).__name__} with dimensions "
                             f"{self.dims_str!r} but components have shape {self.components.shape}")

    # ---- containers -------------------------------------------------------------------
    @property
    def shape(self):
        return self.components.shape[:len(self.dims_str)]

    @property
    def dims(self):
        return self.dims_str

    def with_dims(self, dims):
        return type(self)(self.components, dims)

    def copy(self):
        return type(self)(self.components.copy(), self.dims_str)

    def __len__(self):
        if not self.dims_str:
            raise TypeError(f"{type(self).__name__} without dims has no length")
        return self.components.shape[0]

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def __getitem__(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        if len(key) > len(self.dims_str):
            raise IndexError("too many indices for tensor dims")
        dims = []
        for k, c in zip(key, self.dims_str):
            if isinstance(k, (int, np.integer)):
                continue
            if isinstance(k, np.ndarray) and k.ndim == 0:
                continue
            dims.append(c)
        dims += list(self.dims_str[len(key):])
        return type(self)(self.components[key], "".join(dims))

    def __setitem__(self, key, item):
        if isinstance(item, Tensor):
            self.components[key] = item.components
        else:
            self.components[key] = item

    def __repr__(self):
        return f"{type(self).__name__}(dims={self.dims_str!r}, shape={self.shape})"

    # ---- reductions -------------------------------------------------------------------
    def _reduce(self, fn, dim):
        if dim is None:
            axes = tuple(range(len(self.dims_str)))
            dims = ""
        else:
            if dim not in self.dims_str:
                raise ValueError(f"dim {dim!r} not in {self.dims_str!r}")
            axes = (self.dims_str.index(dim),)
            dims = self.dims_str.replace(dim, "")
        return type(self)(fn(self.components, axis=axes), dims)

    def mean(self, dim=None):
        return self._reduce(np.mean, dim)

    def sum(self, dim=None):
        return self._reduce(np.sum, dim)

    def repeat(self, shape, dims=None):
        shape = tuple(shape) if hasattr(shape, "__iter__") else (shape,)
        comps = np.broadcast_to(self.components, shape + self.components.shape).copy()
        return type(self)(comps, _default_dims(len(shape)) if dims is None else dims)

    @classmethod
    def from_list(cls, tensors):
        return cls(np.stack([t.components for t in tensors]), "p" + tensors[0].dims_str)

    @classmethod
    def from_stack(cls, tensors, new_dim, axis=0):
        comps = np.stack([t.components for t in tensors], axis=axis)
        dims = list(tensors[0].dims_str)
        dims.insert(axis, new_dim)
        return cls(comps, "".join(dims))

    # ---- elementwise ------------------------------------------------------------------
    def _binary(self, other, op, out_type=None):
        out_type = out_type or type(self)
        if isinstance(other, Number):
            return out_type(op(self.components, other), self.dims_str)
        if isinstance(other, Scalar) and not isinstance(self, Scalar):
            dims = _order_dims(self.dims_str, other.dims_str)
            a = _align(self.components, self.dims_str, dims, self._ncomp)
            b = _align(other.components, other.dims_str, dims, 0)
            b = b.reshape(b.shape + (1,) * self._ncomp)
            return out_type(op(a, b), dims)
        if type(other) is not type(self):
            return NotImplemented
        dims = _order_dims(self.dims_str, other.dims_str)
        a = _align(self.components, self.dims_str, dims, self._ncomp)
        b = _align(other.components, other.dims_str, dims, self._ncomp)
        return out_type(op(a, b), dims)

    def __add__(self, other):
        return self._binary(other, np.add)

    def __radd__(self, other):
        return self.__add__(other)

    def __sub__(self, other):
        return self._binary(other, np.subtract)

    def __rsub__(self, other):
        return (-self).__add__(other)

    def __neg__(self):
        return type(self)(-self.components, self.dims_str)

    def __truediv__(self, other):
        return self._binary(other, np.divide)


class Scalar(Tensor):
    """Scalar field (materialite/tensor.py:661-769)."""

    _ncomp = 0

    @classmethod
    def zero(cls):
        return cls(0.0)

    @classmethod
    def random(cls, shape, rng=None, dims=None):
        rng = np.random.default_rng() if rng is None else rng
        return cls(rng.random(shape), dims)

    @property
    def abs(self):
        return Scalar(np.abs(self.components), self.dims_str)

    @property
    def sqrt(self):
        return Scalar(np.sqrt(self.components), self.dims_str)

    def max(self, dim=None):
        return self._reduce(np.max, dim)

    def __pow__(self, other):
        if isinstance(other, Scalar):
            return self._binary(other, np.power)
        return Scalar(self.components ** other, self.dims_str)

    def __mul__(self, other):
        if isinstance(other, Number):
            return Scalar(self.components * other, self.dims_str)
        if isinstance(other, Scalar):
            return self._binary(other, np.multiply)
        if isinstance(other, Tensor):
            return other._binary(self, np.multiply)
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)

    def __rtruediv__(self, other):
        if isinstance(other, Number):
            return Scalar(other / self.components, self.dims_str)
        return NotImplemented


class Vector(Tensor):
    """Cartesian 3-vector (materialite/tensor.py:772-944)."""

    _ncomp = 1

    @classmethod
    def zero(cls):
        return cls(np.zeros(3))

    @classmethod
    def basis(cls, dim="b"):
        return cls(np.eye(3), dim)

    @property
    def norm(self):
        return Scalar(np.linalg.norm(self.components, axis=-1), self.dims_str)

    @property
    def unit(self):
        return Vector(self.components / np.linalg.norm(self.components, axis=-1, keepdims=True),
                      self.dims_str)

    def outer(self, other):
        dims = _order_dims(self.dims_str, other.dims_str)
        a = _align(self.components, self.dims_str, dims, 1)
        b = _align(other.components, other.dims_str, dims, 1)
        return Order2Tensor(a[..., :, None] * b[..., None, :], dims)

    def __mul__(self, other):
        if isinstance(other, Number):
            return Vector(self.components * other, self.dims_str)
        if isinstance(other, Vector):
            dims = _order_dims(self.dims_str, other.dims_str)
            a = _align(self.components, self.dims_str, dims, 1)
            b = _align(other.components, other.dims_str, dims, 1)
            return Scalar(np.sum(a * b, axis=-1), dims)
        if isinstance(other, Scalar):
            return self._binary(other, np.multiply)
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)


class Order2Tensor(Tensor):
    """General second-order tensor, Cartesian 3x3 (materialite/tensor.py:947-1125)."""

    _ncomp = 2

    @classmethod
    def identity(cls):
        return cls(np.eye(3))

    @property
    def cartesian(self):
        return self.components

    @property
    def sym(self):
        c = self.components
        return Order2SymmetricTensor.from_cartesian(0.5 * (c + np.swapaxes(c, -1, -2)),
                                                    self.dims_str)

    @property
    def T(self):
        return Order2Tensor(np.swapaxes(self.components, -1, -2), self.dims_str)


class Order2SymmetricTensor(Tensor):
    """Symmetric second-order tensor in Mandel form (materialite/tensor.py:1128-1382)."""

    _ncomp = 1

    @classmethod
    def identity(cls):
        return cls(np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0]))

    @classmethod
    def zero(cls):
        return cls(np.zeros(6))

    @classmethod
    def random(cls, shape=1, rng=None, dims=None):
        rng = np.random.default_rng() if rng is None else rng
        shape = tuple(shape) if hasattr(shape, "__iter__") else (shape,)
        return cls(np.squeeze(rng.random((*shape, 6))), dims)

    @classmethod
    def from_cartesian(cls, matrices, dims=None):
        m = np.asarray(matrices, dtype=np.float64)
        if not np.allclose(m, np.swapaxes(m, -1, -2), atol=1e-14):
            raise ValueError("tried to create Order2SymmetricTensor using non-symmetric input")
        return cls(_mandel_from_cartesian(m), dims)

    @classmethod
    def from_mandel(cls, components, dims=None):
        return cls(components, dims)

    @classmethod
    def from_strain_voigt(cls, vectors, dims=None):
        v = np.asarray(vectors, dtype=np.float64).copy()
        v[..., 3:] = v[..., 3:] / SQRT2  # engineering shear gamma -> sqrt(2) * eps
        return cls(v, dims)

    @classmethod
    def from_stress_voigt(cls, vectors, dims=None):
        v = np.asarray(vectors, dtype=np.float64).copy()
        v[..., 3:] = v[..., 3:] * SQRT2
        return cls(v, dims)

    @property
    def mandel(self):
        return self.components

    @property
    def cartesian(self):
        return _cartesian_from_mandel(self.components)

    @property
    def strain_voigt(self):
        v = self.components.copy()
        v[..., 3:] *= SQRT2
        return v

    @property
    def stress_voigt(self):
        v = self.components.copy()
        v[..., 3:] /= SQRT2
        return v

    @property
    def norm(self):
        return Scalar(np.sqrt(np.sum(self.components ** 2, axis=-1)), self.dims_str)

    @property
    def trace(self):
        return Scalar(np.sum(self.components[..., :3], axis=-1), self.dims_str)

    @property
    def dev(self):
        c = self.components.copy()
        c[..., :3] -= np.sum(c[..., :3], axis=-1, keepdims=True) / 3.0
        return Order2SymmetricTensor(c, self.dims_str)

    @property
    def inv(self):
        return Order2SymmetricTensor.from_cartesian(np.linalg.inv(self.cartesian), self.dims_str)

    def __mul__(self, other):
        if isinstance(other, Number):
            return Order2SymmetricTensor(self.components * other, self.dims_str)
        if isinstance(other, Order2SymmetricTensor):
            dims = _order_dims(self.dims_str, other.dims_str)
            a = _align(self.components, self.dims_str, dims, 1)
            b = _align(other.components, other.dims_str, dims, 1)
            return Scalar(np.sum(a * b, axis=-1), dims)
        if isinstance(other, Scalar):
            return self._binary(other, np.multiply)
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)

    def outer(self, other):
        dims = _order_dims(self.dims_str, other.dims_str)
        a = _align(self.components, self.dims_str, dims, 1)
        b = _align(other.components, other.dims_str, dims, 1)
        return Order4SymmetricTensor(a[..., :, None] * b[..., None, :], dims)

    def to_crystal_frame(self, orientations):
        """R eps R^T (tensor.py:1347-1360) as R_m @ eps_m."""
        return _rotate2(self, orientations, transpose=False)

    def to_specimen_frame(self, orientations):
        """R^T eps R (tensor.py:1362-1375) as R_m^T @ eps_m."""
        return _rotate2(self, orientations, transpose=True)


class Order4SymmetricTensor(Tensor):
    """Fourth-order tensor with minor symmetries, 6x6 Mandel (tensor.py:1384-1640)."""

    _ncomp = 2

    @classmethod
    def identity(cls):
        return cls(np.eye(6))

    @classmethod
    def zero(cls):
        return cls(np.zeros((6, 6)))

    @classmethod
    def from_mandel(cls, components, dims=None):
        return cls(components, dims)

    @classmethod
    def from_voigt(cls, matrix, dims=None):
        return cls(np.asarray(matrix, dtype=np.float64) * np.outer(_MANDEL_SCALE, _MANDEL_SCALE),
                   dims)

    @classmethod
    def from_cubic_constants(cls, C11, C12, C44):
        V = np.zeros((6, 6))
        V[:3, :3] = C12
        V[[0, 1, 2], [0, 1, 2]] = C11
        V[[3, 4, 5], [3, 4, 5]] = C44
        return cls.from_voigt(V)

    @classmethod
    def from_transverse_isotropic_constants(cls, C11, C12, C13, C33, C44):
        C66 = (C11 - C12) / 2.0
        V = np.array([[C11, C12, C13, 0, 0, 0], [C12, C11, C13, 0, 0, 0],
                      [C13, C13, C33, 0, 0, 0], [0, 0, 0, C44, 0, 0],
                      [0, 0, 0, 0, C44, 0], [0, 0, 0, 0, 0, C66]], dtype=float)
        return cls.from_voigt(V)

    @classmethod
    def from_isotropic_constants(cls, modulus, shear_modulus):
        E, G = modulus, shear_modulus
        L = G * (E - 2 * G) / (3 * G - E)
        V = np.zeros((6, 6))
        V[:3, :3] = L
        V[[0, 1, 2], [0, 1, 2]] = L + 2 * G
        V[[3, 4, 5], [3, 4, 5]] = G
        return cls.from_voigt(V)

    @property
    def mandel(self):
        return self.components

    @property
    def voigt(self):
        return self.components / np.outer(_MANDEL_SCALE, _MANDEL_SCALE)

    @property
    def inv(self):
        return Order4SymmetricTensor(np.linalg.inv(self.components), self.dims_str)

    @property
    def norm(self):
        return Scalar(np.sqrt(np.sum(self.components ** 2, axis=(-2, -1))), self.dims_str)

    def __mul__(self, other):
        if isinstance(other, Number):
            return Order4SymmetricTensor(self.components * other, self.dims_str)
        if isinstance(other, Scalar):
            return self._binary(other, np.multiply)
        if isinstance(other, Order4SymmetricTensor):
            dims = _order_dims(self.dims_str, other.dims_str)
            a = _align(self.components, self.dims_str, dims, 2)
            b = _align(other.components, other.dims_str, dims, 2)
            return Scalar(np.sum(a * b, axis=(-2, -1)), dims)
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)

    def __matmul__(self, other):
        dims = _order_dims(self.dims_str, other.dims_str)
        a = _align(self.components, self.dims_str, dims, 2)
        if isinstance(other, Order2SymmetricTensor):
            b = _align(other.components, other.dims_str, dims, 1)
            return Order2SymmetricTensor(np.einsum("...mn,...n->...m", a, b), dims)
        if isinstance(other, Order4SymmetricTensor):
            b = _align(other.components, other.dims_str, dims, 2)
            return Order4SymmetricTensor(np.einsum("...mn,...no->...mo", a, b), dims)
        return NotImplemented

    def directional_modulus(self, direction):
        d = Vector(direction).unit.components
        dd = _mandel_from_cartesian(np.outer(d, d))
        return Scalar(1.0 / (dd @ np.linalg.inv(self.components) @ dd))

    def to_crystal_frame(self, orientations):
        """R_m K R_m^T (tensor.py:1604-1618)."""
        Rm = orientations.rotation_matrix_mandel
        return Order4SymmetricTensor(np.einsum("...ai,ij,...bj->...ab", Rm, self.components, Rm),
                                     orientations.dims_str)

    def to_specimen_frame(self, orientations):
        """R_m^T K R_m (tensor.py:1620-1634)."""
        Rm = orientations.rotation_matrix_mandel
        return Order4SymmetricTensor(np.einsum("...ia,ij,...jb->...ab", Rm, self.components, Rm),
                                     orientations.dims_str)


def _rotate2(t, orientations, transpose):
    Rm = orientations.rotation_matrix_mandel
    dims = _order_dims(t.dims_str, orientations.dims_str)
    a = _align(t.components, t.dims_str, dims, 1)
    R = _align(Rm, orientations.dims_str, dims, 2)
    sub = "...ji,...j->...i" if transpose else "...ij,...j->...i"
    a, R = np.broadcast_arrays(a[..., None, :], R)
    return Order2SymmetricTensor(np.einsum(sub, R, a[..., 0, :]), dims)


class Orientation:
    """Crystal orientation as the rotation taking specimen components to crystal
    components (materialite/tensor.py:1643-2016)."""

    __array_ufunc__ = None

    def __init__(self, rotation_matrix, dims=None):
        if isinstance(rotation_matrix, Orientation):
            self.rotation_matrix = rotation_matrix.rotation_matrix.copy()
            self.dims_str = rotation_matrix.dims_str
            return
        self.rotation_matrix = np.asarray(rotation_matrix, dtype=np.float64)
        lead = self.rotation_matrix.ndim - 2
        self.dims_str = _default_dims(lead) if dims is None else dims
        if len(self.dims_str) != lead:
            raise ValueError(f"tried to create Orientation with dimensions {self.dims_str!r} but "
                             f"rotation matrix has shape {self.rotation_matrix.shape}")

    @property
    def shape(self):
        return self.rotation_matrix.shape[:len(self.dims_str)]

    def __len__(self):
        return self.rotation_matrix.shape[0]

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def __getitem__(self, key):
        R = self.rotation_matrix[key]
        return Orientation(R, "p"[:R.ndim - 2] if R.ndim > 2 else "")

    def copy(self):
        return Orientation(self.rotation_matrix.copy(), self.dims_str)

    @classmethod
    def identity(cls):
        return cls(np.eye(3))

    @classmethod
    def from_rotation_matrix(cls, rotation_matrix, dims=None):
        return cls(rotation_matrix, dims)

    @classmethod
    def from_euler_angles(cls, euler_angles, in_degrees=False, dims=None):
        from .microstructure import euler_to_rotation
        e = np.asarray(euler_angles, dtype=np.float64)
        if in_degrees:
            e = e * np.pi / 180.0
        return cls(np.squeeze(euler_to_rotation(e)), dims)

    @classmethod
    def random(cls, shape=1, rng=None, dims=None):
        """Uniform Bunge angles (z1, arccos(2u-1), z3), the reference's sampler and RNG
        consumption (tensor.py:1899-1912)."""
        rng = np.random.default_rng() if rng is None else rng
        shape = tuple(shape) if hasattr(shape, "__iter__") else (shape,)
        z1 = rng.random(shape) * 2.0 * np.pi
        x2 = np.arccos(rng.random(shape) * 2.0 - 1.0)
        z3 = rng.random(shape) * 2.0 * np.pi
        return cls.from_euler_angles(np.stack([z1, x2, z3], axis=-1), dims=dims)

    @classmethod
    def from_list(cls, orientations):
        return cls(np.stack([o.rotation_matrix for o in orientations]), "p")

    @property
    def euler_angles(self):
        """Bunge (z1, x2, z3) angles of the rotation matrices, the inverse of
        from_euler_angles (tensor.py:1919-1961, after D. Eberly, "Euler Angle Formulas").
        With R[2,2] = +-1 the rotation is about z alone and is reported as z1 (x2 = 0 or
        pi, z3 = 0)."""
        R = np.asarray(self.rotation_matrix, dtype=np.float64)
        r22 = R[..., 2, 2]
        default = (r22 < 1.0) & (r22 > -1.0)
        with np.errstate(invalid="ignore"):
            z1 = np.arctan2(R[..., 2, 0], -R[..., 2, 1])
            x2 = np.arccos(r22)
            z3 = np.arctan2(R[..., 0, 2], R[..., 1, 2])
        up = r22 >= 1.0
        z1 = np.where(default, z1, np.where(up, np.arctan2(-R[..., 1, 0], R[..., 0, 0]),
                                            np.arctan2(R[..., 1, 0], R[..., 0, 0])))
        x2 = np.where(default, x2, np.where(up, 0.0, np.pi))
        z3 = np.where(default, z3, 0.0)
        return np.squeeze(np.stack([z1, x2, z3], axis=-1))

    @property
    def euler_angles_in_degrees(self):
        return self.euler_angles * 180.0 / np.pi

    @property
    def rotation_matrix_mandel(self):
        """6x6 Mandel rotation (tensor.py:1668-1700)."""
        R = self.rotation_matrix
        out = np.zeros(R.shape[:-2] + (6, 6))
        out[..., :3, :3] = R ** 2
        pairs = [(1, 2), (0, 2), (0, 1)]
        for a in range(3):
            for s, (j, k) in enumerate(pairs):
                out[..., a, 3 + s] = SQRT2 * R[..., a, j] * R[..., a, k]
        for s, (i, j) in enumerate(pairs):
            for b in range(3):
                out[..., 3 + s, b] = SQRT2 * R[..., i, b] * R[..., j, b]
            for t, (k, l) in enumerate(pairs):
                out[..., 3 + s, 3 + t] = R[..., i, k] * R[..., j, l] + R[..., i, l] * R[..., j, k]
        return out

    def __repr__(self):
        return f"Orientation(dims={self.dims_str!r}, shape={self.shape})"
