"""numpy restatement of materialite 0.1.3's SmallStrainFFT solve (test infrastructure).

Every function cites the reference lines it follows (paths relative to the reference
project root).  Conventions are the reference's Mandel basis
(materialite/basis_operations.py:37-48): component order [11, 22, 33, 23, 13, 12] with
sqrt(2) on the shear components; points in C order of (x, y, z), z fastest
(materialite/util/util.py:40-42).

Inputs are plain arrays: per-point rotation matrices (specimen -> crystal, as
``Orientation.rotation_matrix``), per-point phase index, a list of model descriptions,
and load-schedule closures returning 6-vectors.  No GPU code is touched here.
"""

import math
from collections import defaultdict

import numpy as np

from .minres import minres

SQRT2 = math.sqrt(2.0)


# --------------------------------------------------------------------------------------
# Mandel tensor helpers (materialite/tensor.py)
# --------------------------------------------------------------------------------------

def rotation_matrix_mandel(R):
    """6x6 Mandel form of a rotation (materialite/tensor.py:1668-1700)."""
    R = np.asarray(R, dtype=np.float64)
    out = np.zeros(R.shape[:-2] + (6, 6))
    out[..., :3, :3] = R**2
    pairs = [(1, 2), (0, 2), (0, 1)]  # Mandel shear slots 3, 4, 5
    for a in range(3):
        for s, (j, k) in enumerate(pairs):
            out[..., a, 3 + s] = SQRT2 * R[..., a, j] * R[..., a, k]
    for s, (i, j) in enumerate(pairs):
        for b in range(3):
            out[..., 3 + s, b] = SQRT2 * R[..., i, b] * R[..., j, b]
        for t, (k, l) in enumerate(pairs):
            out[..., 3 + s, 3 + t] = R[..., i, k] * R[..., j, l] + R[..., i, l] * R[..., j, k]
    return out


def voigt_to_mandel_stiffness(C_voigt):
    """Order4SymmetricTensor.from_voigt (materialite/tensor.py:1407-1411): scale shear
    rows/columns by sqrt(2) each."""
    scale = np.array([1, 1, 1, SQRT2, SQRT2, SQRT2])
    return np.asarray(C_voigt, dtype=np.float64) * np.outer(scale, scale)


def cubic_stiffness(C11, C12, C44):
    """Order4SymmetricTensor.from_cubic_constants (materialite/tensor.py:1422-1434)."""
    V = np.zeros((6, 6))
    V[:3, :3] = C12
    V[[0, 1, 2], [0, 1, 2]] = C11
    V[[3, 4, 5], [3, 4, 5]] = C44
    return voigt_to_mandel_stiffness(V)


def isotropic_stiffness(E, G):
    """Order4SymmetricTensor.from_isotropic_constants (materialite/tensor.py:1453-1467)."""
    L = G * (E - 2 * G) / (3 * G - E)
    V = np.zeros((6, 6))
    V[:3, :3] = L
    V[[0, 1, 2], [0, 1, 2]] = L + 2 * G
    V[[3, 4, 5], [3, 4, 5]] = G
    return voigt_to_mandel_stiffness(V)


def sym_mandel(M):
    """Mandel vector of sym(M) for Cartesian 3x3 matrices (materialite/tensor.py:1003-1007)."""
    M = np.asarray(M, dtype=np.float64)
    S = 0.5 * (M + np.swapaxes(M, -1, -2))
    return np.stack(
        [S[..., 0, 0], S[..., 1, 1], S[..., 2, 2],
         SQRT2 * S[..., 1, 2], SQRT2 * S[..., 0, 2], SQRT2 * S[..., 0, 1]], axis=-1)


def schmid_mandel(normals, directions):
    """sym(d (x) n) for unit slip normals / directions
    (materialite/slip_system.py:18-22, 139-141)."""
    n = np.asarray(normals, dtype=np.float64)
    d = np.asarray(directions, dtype=np.float64)
    n = n / np.linalg.norm(n, axis=-1, keepdims=True)
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)
    return sym_mandel(np.einsum("si,sj->sij", d, n))


def octahedral_slip_systems():
    """The 12 FCC {111}<110> systems (materialite/slip_system.py:35-65)."""
    normals = [[1, 1, -1]] * 3 + [[1, -1, -1]] * 3 + [[1, -1, 1]] * 3 + [[1, 1, 1]] * 3
    directions = [[0, 1, 1], [1, 0, 1], [1, -1, 0], [0, 1, -1], [1, 0, 1], [1, 1, 0],
                  [0, 1, 1], [1, 0, -1], [1, 1, 0], [0, 1, -1], [1, 0, -1], [1, -1, 0]]
    return np.array(normals, float), np.array(directions, float)


def directional_modulus_x(C):
    """1 / (d (x) d : C^-1 : d (x) d) for d = x (materialite/tensor.py:1571-1574)."""
    dd = np.array([1.0, 0, 0, 0, 0, 0])
    return 1.0 / (dd @ np.linalg.inv(C) @ dd)


def dev_norm(s):
    """|dev s| for Mandel vectors (materialite/tensor.py:1232-1244)."""
    tr = s[..., 0] + s[..., 1] + s[..., 2]
    d = s.copy()
    d[..., :3] -= tr[..., None] / 3.0
    return np.sqrt(np.einsum("...n,...n", d, d))


# --------------------------------------------------------------------------------------
# Hardening laws (materialite/models/small_strain_fft/hardening_laws.py)
# --------------------------------------------------------------------------------------

def hardening(kind, props, Gamma_old, g_old, gdot, dt, latent=1.0):
    """Slip resistances after an increment.  ``Gamma_old`` (V,), ``g_old`` and ``gdot``
    (V, S).  Laws follow hardening_laws.py:18-90; ``latent`` != 1 is a latent-hardening
    extension with no reference counterpart, applied only by the caller."""
    dgam = dt * np.sum(np.abs(gdot), axis=-1)  # hardening_laws.py:35-38 / 49-52 / 83-86
    if kind == "perfect_plasticity":          # :18-25
        return g_old.copy()
    if kind == "linear":                      # :28-39
        return g_old + props["hardening_rate"] * dgam[:, None]
    if kind == "voce":                        # :42-72
        th0, th1, tau1 = props["theta_0"], props["theta_1"], props["tau_1"]
        ratio = abs(th0 / tau1)
        e_i = np.exp(-ratio * Gamma_old)
        e_c = np.exp(-ratio * dgam)
        inc = (th1 * dgam
               - (ratio * tau1 - th1) / ratio * e_i * (e_c - 1)
               - th1 / ratio * e_i * (e_c * (1 + ratio * (Gamma_old + dgam)) - 1 - ratio * Gamma_old))
        return g_old + inc[:, None]
    if kind == "armstrong_frederick":         # :75-90
        h, r = props["direct_hardening"], props["dynamic_recovery"]
        return g_old + (h - r * g_old) * (dgam / (1 + r * dgam))[:, None]
    raise ValueError(f"unknown hardening law {kind}")


# --------------------------------------------------------------------------------------
# Constitutive models
# --------------------------------------------------------------------------------------

class ElasticOracle:
    """Elastic (materialite/models/small_strain_fft/elastic.py:16-49)."""

    def __init__(self, C):
        self.C = np.asarray(C, dtype=np.float64)

    def initialize(self, R):
        Rm = rotation_matrix_mandel(R)
        # to_specimen_frame: R_m^T C R_m (tensor.py:1620-1634)
        self.K = np.einsum("pia,ij,pjb->pab", Rm, self.C, Rm)
        return self.K

    def calculate_stress_and_tangent(self, strain, guess, dt):
        return np.einsum("pmn,pn->pm", self.K, strain), self.K, 1

    def update_state_variables(self):
        pass

    def outputs(self):
        return {}


class EVPOracle:
    """Crystal elasto-viscoplasticity
    (materialite/models/small_strain_fft/elastic_viscoplastic.py:20-271)."""

    TOLERANCE = 2.0e-5     # elastic_viscoplastic.py:92
    MAX_ITERATIONS = 60    # :93

    def __init__(self, C, schmid, gdot0, n, g0, hardening_kind, hardening_props, latent=1.0):
        self.C = np.asarray(C, dtype=np.float64)
        self.P = np.asarray(schmid, dtype=np.float64)          # (S, 6) Mandel sym Schmid
        self.PP = np.einsum("sm,sn->smn", self.P, self.P)
        self.gdot0 = float(gdot0)
        self.n = float(n)
        self.g0 = float(g0)
        self.kind = hardening_kind
        self.props = hardening_props
        self.latent = float(latent)
        self.E_ref = directional_modulus_x(self.C)             # :32-34

    def initialize(self, R):                                   # :52-89
        V = R.shape[0]
        S = self.P.shape[0]
        self.Rm = rotation_matrix_mandel(R)
        self.g = np.full((V, S), self.g0)          # slip_resistances (trial)
        self.g_old = self.g.copy()
        self.ep = np.zeros((V, 6))                 # _plastic_strains (crystal, trial)
        self.ep_old = np.zeros((V, 6))
        self.gam = np.zeros((V, S))                # slip_system_shear_strains (trial)
        self.gam_old = np.zeros((V, S))
        self.Gam = np.zeros(V)                     # accumulated_slip (trial)
        self.Gam_old = np.zeros(V)
        self.ep_spec = np.zeros((V, 6))            # plastic_strains (specimen, committed)
        return np.einsum("pia,ij,pjb->pab", self.Rm, self.C, self.Rm)

    def _iterate(self, g, sig, ep_old, dt, eps, Gam_old, g_old):   # :190-253
        prev = sig.copy()
        tau = sig @ self.P.T                                       # :206
        ratio = np.abs(tau / g)
        pref = self.gdot0 * ratio ** (self.n - 1.0) / g            # :209-214
        gdot = pref * tau                                          # :216
        ep = ep_old + (gdot @ self.P) * dt                         # :219-222
        A = np.einsum("ps,smn->pmn", self.n * pref, self.PP)
        J = np.eye(6)[None] + dt * np.einsum("ij,pjk->pik", self.C, A)
        Jinv = np.linalg.inv(J)                                     # :225-230
        resid = sig - (eps - ep) @ self.C.T
        sig = prev - np.einsum("pij,pj->pi", Jinv, resid)          # :233-235
        g_new = hardening(self.kind, self.props, Gam_old, g_old, gdot, dt)  # :236-242
        if self.latent != 1.0:
            g_new = latent_hardening(g_old, g_new, gdot, self.latent)
        diff = np.sqrt(np.sum((sig - prev) ** 2, axis=-1))
        return sig, diff, g_new, ep, gdot * dt, Jinv

    def calculate_stress_and_tangent(self, strain, guess, dt):      # :91-188
        Rm = self.Rm
        gnorm = np.sqrt(np.sum(guess**2, axis=-1))
        sig = np.einsum("pij,pj->pi", Rm, guess)     # to_crystal_frame
        eps = np.einsum("pij,pj->pi", Rm, strain)
        g = self.g
        V = sig.shape[0]
        it = 0
        frac = 0.0
        conv = None
        while True:
            it += 1
            if frac >= 0.5:                                        # :116-136
                nc = ~conv
                s, d, gg, e, inc, Ji = self._iterate(
                    g[nc], sig[nc], self.ep_old[nc], dt, eps[nc], self.Gam_old[nc], self.g_old[nc])
                sig[nc], diff[nc], g[nc], ep[nc], slip_inc[nc], Jinv[nc] = s, d, gg, e, inc, Ji
            else:
                sig, diff, g, ep, slip_inc, Jinv = self._iterate(
                    g, sig, self.ep_old, dt, eps, self.Gam_old, self.g_old)
            with np.errstate(divide="ignore", invalid="ignore"):
                conv = np.logical_or(diff / gnorm <= self.TOLERANCE,
                                     diff / self.E_ref < 1.0e-12)  # :161-164
            frac = np.count_nonzero(conv) / V
            if np.all(conv):
                break
            if it == self.MAX_ITERATIONS:
                return None, None, 0                               # :168-170
        tangent = np.einsum("pij,jk->pik", Jinv, self.C)           # :172
        self.ep = ep
        self.g = g
        self.gam = self.gam_old + slip_inc
        self.Gam = self.Gam_old + np.sum(np.abs(slip_inc), axis=-1)
        sig_s = np.einsum("pji,pj->pi", Rm, sig)                   # to_specimen_frame
        tan_s = np.einsum("pia,pij,pjb->pab", Rm, tangent, Rm)
        return sig_s, tan_s, it

    def update_state_variables(self):                              # :255-271
        self.ep_old = self.ep.copy()
        self.ep_spec = np.einsum("pji,pj->pi", self.Rm, self.ep)
        self.g_old = self.g.copy()
        self.gam_old = self.gam.copy()
        self.Gam_old = self.Gam.copy()

    def outputs(self):
        return {"slip_resistances": self.g.copy(),
                "plastic_strains": self.ep_spec.copy(),
                "slip_system_shear_strains": self.gam.copy()}


def hardening_scalar(kind, props, eq_old, y_old, rate, dt):
    """The hardening laws called with one scalar rate per point, as IsotropicElasticPlastic
    calls them (isotropic_elastic_plastic.py:125-131): the increment is dt * |rate|
    (hardening_laws.py:35-38, the ValueError branch for a Scalar)."""
    inc = dt * np.abs(rate)
    if kind == "perfect_plasticity":
        return y_old.copy()
    if kind == "linear":
        return y_old + props["hardening_rate"] * inc
    if kind == "voce":
        th0, th1, tau1 = props["theta_0"], props["theta_1"], props["tau_1"]
        ratio = abs(th0 / tau1)
        e_i = np.exp(-ratio * eq_old)
        e_c = np.exp(-ratio * inc)
        return (y_old + th1 * inc - (ratio * tau1 - th1) / ratio * e_i * (e_c - 1)
                - th1 / ratio * e_i * (e_c * (1 + ratio * (eq_old + inc)) - 1 - ratio * eq_old))
    if kind == "armstrong_frederick":
        h, r = props["direct_hardening"], props["dynamic_recovery"]
        return y_old + (h - r * y_old) * inc / (1 + r * inc)
    raise ValueError(f"unknown hardening law {kind}")


MANDEL_IDENTITY = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])


class J2Oracle:
    """IsotropicElasticPlastic: small-strain J2 plasticity with radial return
    (materialite/models/small_strain_fft/isotropic_elastic_plastic.py:17-183).  The
    return-mapping loop is the reference's: a fixed-point update of the equivalent plastic
    strain increment with the constant inverse Jacobian -1/(3G), the residual clipped at
    zero, repeated for every point until every point has converged (:106-138)."""
    TOLERANCE = 1.0e-7
    MAX_ITERATIONS = 100

    def __init__(self, E, G, yield_stress, hardening_kind, hardening_props):
        self.E, self.G = float(E), float(G)
        self.Kb = G * E / (3 * (3 * G - E))                              # :28-30
        self.C = isotropic_stiffness(E, G)
        self.y0 = float(yield_stress)
        self.kind, self.props = hardening_kind, hardening_props

    def initialize(self, R):                                           # :55-69
        V = len(R)
        self.K = np.tile(self.C, (V, 1, 1))
        self.ep_old = np.zeros((V, 6))
        self.eq_old = np.zeros(V)
        self.y_old = np.full(V, self.y0)
        self.ep, self.eq, self.y = self.ep_old.copy(), self.eq_old.copy(), self.y_old.copy()
        return self.K

    def calculate_stress_and_tangent(self, strain, guess, dt):         # :71-164
        G = self.G
        ee = strain - self.ep_old
        tr = ee[:, 0] + ee[:, 1] + ee[:, 2]
        dev = ee - (1 / 3 * tr)[:, None] * MANDEL_IDENTITY
        s = 2.0 * G * dev
        mean = self.Kb * tr
        q = np.sqrt(1.5) * np.sqrt(np.einsum("pn,pn->p", s, s))
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio_s = s / q[:, None]
        jinv = -1.0 / (3.0 * G)
        elastic = q <= self.y_old
        if np.all(elastic):                                            # :94-99
            return s + mean[:, None] * MANDEL_IDENTITY, self.K, 1
        dp = np.zeros_like(q)
        y = self.y_old.copy()
        it = 0
        while True:
            it += 1
            r = q - 3.0 * G * dp - y
            r[r <= 0.0] = 0.0
            prev = dp.copy()
            dp = dp - jinv * r
            y = hardening_scalar(self.kind, self.props, self.eq_old, self.y_old, dp / dt, dt)
            if np.all(np.abs(dp - prev) < self.TOLERANCE):
                break
            if it == self.MAX_ITERATIONS:
                return None, None, 0
        with np.errstate(invalid="ignore"):
            self.ep = self.ep_old + 1.5 * ratio_s * dp[:, None]
        self.eq = self.eq_old + dp
        self.y = y
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = 3.0 * G / q
            stress = (1.0 - ratio * dp)[:, None] * s + mean[:, None] * MANDEL_IDENTITY
            dev_id = np.eye(6) - np.outer(MANDEL_IDENTITY, MANDEL_IDENTITY) / 3.0
            t1 = 2.0 * G * ratio * dp
            t2 = ratio**2 * (dp / q - 1 / (3 * G))
            K = (self.C[None] - t1[:, None, None] * dev_id[None]
                 + t2[:, None, None] * np.einsum("pm,pn->pmn", s, s))
        K[elastic] = self.C
        return stress, K, it

    def update_state_variables(self):                                  # :166-175
        self.ep_old = self.ep.copy()
        self.eq_old = self.eq.copy()
        self.y_old = self.y.copy()

    def outputs(self):
        return {"yield_stresses": self.y.copy(), "plastic_strains": self.ep.copy(),
                "eq_plastic_strains": self.eq.copy()}


def latent_hardening(g_old, g_iso, gdot, q):
    """Latent-hardening extension with no reference counterpart: the isotropic increment
    of the reference law is redistributed with the interaction matrix
    h_ab = q + (1 - q) delta_ab, weighted by |gdot_b| / sum |gdot|.  q = 1 recovers the
    reference exactly."""
    a = np.abs(gdot)
    tot = a.sum(axis=-1, keepdims=True)
    inc = g_iso - g_old
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(tot > 0, (q * tot + (1.0 - q) * a) / tot, 1.0)
    return g_old + inc * w


class MultiphaseOracle:
    """Per-phase dispatch (materialite/models/small_strain_fft/multiphase.py:18-95)."""

    def __init__(self, models, indices, V):
        self.models = models
        self.indices = indices
        self.V = V

    def initialize(self, R):
        K = np.zeros((self.V, 6, 6))
        for m, i in zip(self.models, self.indices):
            K[i] = m.initialize(R[i])
        return K

    def calculate_stress_and_tangent(self, strain, guess, dt):
        sig = np.zeros((self.V, 6))
        K = np.zeros((self.V, 6, 6))
        its = []
        for m, i in zip(self.models, self.indices):
            s, k, it = m.calculate_stress_and_tangent(strain[i], guess[i], dt)
            if not it:
                return None, None, 0
            sig[i] = s
            K[i] = k
            its.append(it)
        return sig, K, max(its)

    def update_state_variables(self):
        for m in self.models:
            m.update_state_variables()

    def outputs(self):
        out = {}
        for m, i in zip(self.models, self.indices):
            for k, v in m.outputs().items():
                if k not in out:
                    out[k] = np.zeros((self.V,) + v.shape[1:])
                out[k][i] = v
        return out


# --------------------------------------------------------------------------------------
# Projection operator and its apply (small_strain_fft.py:301-382)
# --------------------------------------------------------------------------------------

def projection_operator(dims, stress_mask):
    """Gamma-hat(q) as (Nx, Ny, Nz, 6, 6) Mandel matrices (small_strain_fft.py:301-368).

    Follows the reference's rotated frequencies q = i/4 tan(pi f) prod_k(1 + e^{2 pi i f_k})
    normalised, A = delta_im q_j conj(q_l), B = q_i q_j conj(q_l q_m), Gamma = sym(A) - B,
    Nyquist planes zeroed for even sizes and Gamma(0) = diag(stress_mask)."""
    Nx, Ny, Nz = (int(d) for d in dims)
    f = np.array(np.meshgrid(np.fft.fftfreq(Nx), np.fft.fftfreq(Ny), np.fft.fftfreq(Nz),
                             indexing="ij"))
    shift = lambda x: 1 + np.exp(2j * np.pi * x)
    const = shift(f[0]) * shift(f[1]) * shift(f[2])
    qv = np.array([1j / 4 * np.tan(np.pi * f[k]) * const for k in range(3)])
    nrm = np.linalg.norm(qv, axis=0)
    q = np.divide(qv, nrm, out=np.zeros_like(qv), where=nrm != 0)
    A = np.real(np.einsum("im,jxyz,lxyz->xyzijlm", np.eye(3), q, np.conj(q), optimize=True))
    B = np.real(np.einsum("ixyz,jxyz,lxyz,mxyz->xyzijlm", q, q, np.conj(q), np.conj(q),
                          optimize=True))
    G4 = 0.5 * (A + A.transpose(0, 1, 2, 3, 4, 6, 5) + A.transpose(0, 1, 2, 4, 3, 5, 6)
                + A.transpose(0, 1, 2, 4, 3, 6, 5)) - B
    if Nx % 2 == 0:
        G4[Nx // 2] = 0.0
    if Ny % 2 == 0:
        G4[:, Ny // 2] = 0.0
    if Nz % 2 == 0:
        G4[:, :, Nz // 2] = 0.0
    # Cartesian -> Mandel 6x6 (tensor.py:1413-1415 with the Mandel product basis)
    basis = np.zeros((6, 3, 3))
    r2 = 1 / SQRT2
    basis[0, 0, 0] = basis[1, 1, 1] = basis[2, 2, 2] = 1.0
    basis[3, 1, 2] = basis[3, 2, 1] = r2
    basis[4, 0, 2] = basis[4, 2, 0] = r2
    basis[5, 0, 1] = basis[5, 1, 0] = r2
    G = np.einsum("mij,nkl,xyzijkl->xyzmn", basis, basis, G4, optimize=True)
    mask = np.asarray(stress_mask, dtype=np.float64)
    if not np.array_equal(mask, np.zeros(6)):
        G[0, 0, 0] = np.diag((mask != 0).astype(np.float64))
    return G


def apply_projection(G, tau):
    """ifftn(G : fftn(tau)).real flattened (small_strain_fft.py:376-382)."""
    dims = G.shape[:3]
    grid = np.asarray(tau).reshape(*dims, 6)
    ft = np.fft.fftn(grid, axes=(0, 1, 2))
    prod = np.einsum("xyzij,xyzj->xyzi", G, ft, optimize=True)
    return np.fft.ifftn(prod, axes=(0, 1, 2)).real.ravel()


# --------------------------------------------------------------------------------------
# The solve (small_strain_fft.py:60-279)
# --------------------------------------------------------------------------------------

class LoadOracle:
    """Plain-closure load schedule: functions of (t, dt) returning Mandel 6-vectors
    (materialite/models/small_strain_fft/load_schedule.py:17-40)."""

    def __init__(self, dstrain, dstress, stress, mask):
        self.dstrain, self.dstress, self.stress = dstrain, dstress, stress
        self.mask = np.asarray(mask, dtype=np.float64)

    @classmethod
    def constant_rates(cls, strain_rate, stress_rate, mask, start_time=0.0):
        mask = np.asarray(mask, dtype=np.float64)
        er = np.asarray(strain_rate, float) * (1 - mask)
        sr = np.asarray(stress_rate, float) * mask
        return cls(lambda t, dt: er * dt, lambda t, dt: sr * dt,
                   lambda t, dt: sr * (t + dt - start_time), mask)

    @classmethod
    def uniaxial(cls, magnitude=1.0, direction="z", start_time=0.0):
        axis = "xyz".index(direction)
        rate = np.zeros(6)
        rate[axis] = magnitude
        mask = np.ones(6)
        mask[axis] = 0.0
        return cls.constant_rates(rate, np.zeros(6), mask, start_time)


def solve(dims, R, model, load, end_time=1.0, initial_time_increment=None,
          max_time_increment=None, min_time_increment=1.0e-9, start_time=0.0,
          global_tolerance=1.0e-3, strain_correction_tolerance=1.0e-2,
          linear_solver_tolerance=1.0e-5, output_times=None, output_variables=None,
          stats=None, krylov_maxiter=None, krylov_floor=0.0, krylov_forcing=0.0):
    """Oracle of ``SmallStrainFFT.run`` (small_strain_fft.py:60-264).  ``model`` is an
    Elastic/EVP/Multiphase oracle; returns a dict of final fields, or of per-output-time
    stacks when ``output_times`` is given.  ``krylov_floor`` > 0 (not part of the reference)
    adds the product's served-request floor to each MINRES solve: an absolute residual
    tolerance of krylov_floor * global_tolerance * the mean von Mises stress of the stress
    the right-hand side was computed from; ``krylov_forcing`` > 0 its relative forcing, a
    residual tolerance of krylov_forcing * |b|."""
    dims = tuple(int(d) for d in dims)
    V = int(np.prod(dims))
    dt = end_time if initial_time_increment is None else initial_time_increment
    dt_max = dt if max_time_increment is None else max_time_increment
    t = start_time
    t_tol = min_time_increment / 2.0
    if output_times is not None:
        out_idx = 0
        output_times = np.append(output_times, np.inf)
        next_out = output_times[0]
    else:
        next_out = np.inf
    history = defaultdict(list)
    G = projection_operator(dims, load.mask)
    proj = lambda tau: apply_projection(G, tau)
    tangent = model.initialize(np.asarray(R, dtype=np.float64))
    stress = np.zeros((V, 6))
    strain = np.zeros((V, 6))
    old_tangent = tangent.copy()
    old_strain = np.zeros((V, 6))
    old_stress = np.zeros((V, 6))
    old_fluct = np.zeros((V, 6))
    old_max_inc = 0.0
    summed_vm = 0.0
    step = 0
    if stats is not None:
        stats.setdefault("krylov", [])
        stats.setdefault("newton", [])
    while t < end_time - t_tol:
        dE = np.asarray(load.dstrain(t, dt), float)
        dS = np.asarray(load.dstress(t, dt), float)
        Sbar = np.asarray(load.stress(t, dt), float)
        max_inc = dE[np.argmax(np.abs(dE))]
        if max_inc * old_max_inc < 0.0:
            old_fluct = np.zeros((V, 6))
        strain = old_strain + dE + old_fluct
        if not np.all(dS < 1.0e-14):
            strain = strain + np.linalg.inv(tangent.mean(axis=0)) @ dS
        if step == 0:
            guess = dS + np.einsum("pmn,n->pm", tangent, dE)
        else:
            guess = old_stress + dS
        converged = False
        it = 0
        constit_its = []
        while not converged:
            it += 1
            if it == 1:
                stress, tangent, cit = model.calculate_stress_and_tangent(strain, guess, dt)
                if not cit:
                    tangent = old_tangent.copy()
                    break
                b = proj(Sbar - stress)
                mvm = dev_norm(stress.mean(axis=0)) * math.sqrt(1.5)
                eq_err = np.max(np.abs(b)) / mvm
                guess = stress.copy()
                constit_its.append(cit)
            old_eq = max(eq_err, global_tolerance)
            matvec = lambda v: proj(np.einsum("pmn,pn->pm", tangent, v.reshape(V, 6)))
            atol = 0.0
            if krylov_floor > 0.0:
                atol = krylov_floor * global_tolerance * \
                    dev_norm(stress.mean(axis=0)) * math.sqrt(1.5)
            if krylov_forcing > 0.0:
                bf = np.ravel(b)
                atol = max(atol, krylov_forcing * math.sqrt(float(bf @ bf)))
            x, kits = minres(matvec, b, linear_solver_tolerance, krylov_maxiter, atol=atol)
            if stats is not None:
                stats["krylov"].append(kits)
            fluct = x.reshape(V, 6)
            strain = strain + fluct
            old_fluct = old_fluct + fluct
            stress, tangent, cit = model.calculate_stress_and_tangent(strain, guess, dt)
            if not cit:
                tangent = old_tangent.copy()
                break
            constit_its.append(cit)
            b = proj(Sbar - stress)
            mvm = dev_norm(stress.mean(axis=0)) * math.sqrt(1.5)
            tavg = (summed_vm + mvm) / (step + 1)
            if mvm / tavg < 1.0e-12:
                mvm = tavg
            eq_err = np.max(np.abs(b)) / mvm
            max_ds = np.max(dev_norm(stress - old_stress)) * math.sqrt(1.5)
            if max_ds / mvm < 1.0e-12:
                max_ds = mvm
            Kdx = np.einsum("pmn,pn->pm", tangent, fluct)
            s_err = np.max(np.sqrt(np.sum(Kdx**2, axis=-1))) / max_ds
            p_err = s_err * eq_err / old_eq
            if eq_err < global_tolerance and (
                    s_err < strain_correction_tolerance or p_err < strain_correction_tolerance
                    or step == 0 or eq_err < 1e-8):
                converged = True
            guess = stress.copy()
            if it == 100 and not converged:
                break
        if stats is not None:
            stats["newton"].append(it)
        if converged:
            model.update_state_variables()
            old_stress = stress.copy()
            old_strain = strain.copy()
            old_tangent = tangent.copy()
            summed_vm += mvm
            old_max_inc = max_inc
            step += 1
            t += dt
            if t >= next_out - t_tol:
                outs = model.outputs()
                outs.update({"stress": stress.copy(), "strain": strain.copy()})
                for k, v in outs.items():
                    history[k].append(v)
                out_idx += 1
                next_out = output_times[out_idx]
            fixed = min(next_out - t, end_time - t)
            cands = [dt_max, fixed, dt * 2.0 if max(constit_its) < 11 else dt]
            new_dt = min(cands)
            old_fluct = old_fluct * new_dt / dt
            dt = new_dt
        else:
            dt = dt / 2.0
            old_fluct = old_fluct / 2.0
            if dt < min_time_increment:
                raise ValueError("min time increment reached")
    if output_times is None:
        outs = model.outputs()
        outs.update({"stress": stress, "strain": strain})
        return outs
    return {k: np.stack(v, axis=1) for k, v in history.items()}
