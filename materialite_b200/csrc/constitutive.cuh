// Per-voxel constitutive updates of materialite's SmallStrainFFT path:
//   Elastic             sigma = K_spec : eps      (elastic.py:23-31)
//   ElasticViscoplastic backward-Euler crystal plasticity in the crystal frame
//                       (elastic_viscoplastic.py:91-253) with the hardening laws of
//                       hardening_laws.py:18-90.
//
// The EVP update runs in double.  Each thread owns one voxel and keeps its slip-system
// sums in registers.  The reference's Jacobian J = I + dt C A (A = sum n p P (x) P) and
// tangent J^-1 C are evaluated through the symmetric positive definite matrix
// M = C^-1 + dt A:  J^-1 r = M^-1 C^-1 r  and  J^-1 C = M^-1, both from one Cholesky
// factorisation of M (equal to the reference's explicit inverse up to round-off).
//
// Voxels stop at their own convergence test (stress change <= 2e-5 |guess| or
// <= 1e-12 E_x, elastic_viscoplastic.py:161-164).  The reference instead iterates all
// voxels until half have converged and then only the rest (:116-158); both stop inside
// the same tolerance of the same Newton iteration.
#pragma once

#include "common.cuh"

#define EVP_TOLERANCE 2.0e-5
#define EVP_MAX_ITERATIONS 60
#define MAX_SLIP 12

enum { PHASE_ELASTIC = 0, PHASE_EVP = 1 };
enum { HARD_PERFECT = 0, HARD_LINEAR = 1, HARD_VOCE = 2, HARD_AF = 3 };

struct PhaseParams {
  int kind, nslip, hardening, pad;
  double C[36];
  double Cinv[36];
  double P[MAX_SLIP * 6];
  double gdot0, n, g0, latent;
  double props[4];
  double E_ref;
};

template <typename T> struct ConstArgs {
  long long V;
  const T *eps;            // 6 planes
  const T *guess;          // 6 planes
  T *sig;                  // 6 planes (out)
  T *kvox;                 // 21 planes (out, EVP voxels) or null (table mode)
  const T *ktab;           // table-mode tangents [n_gid][21]
  const int32_t *gid;      // table-mode tangent index
  const int32_t *phase;    // phase per voxel (null: phase 0)
  const int32_t *orient;   // orientation per voxel
  const PhaseParams *params;
  const double *rm_tab;    // [n_orient][36] Mandel rotations (specimen -> crystal)
  // EVP state (double, planes of V): g_in is read (previous trial), g_out written
  const double *g_in;
  double *g_out;
  const double *g_old;
  const double *ep_old;    // crystal frame, 6 planes
  double *ep_trial;
  const double *Gam_old;
  double *Gam_trial;
  const double *gam_old;   // optional per-system shear strains
  double *gam_trial;
  double dt;
  int *max_iters;          // atomicMax of iterations
  int *failed;             // set when a voxel does not converge
};

__device__ __forceinline__ void cholesky6(const double *M, double *L) {
  // M, L packed symmetric (sym_idx); L holds the lower factor L[i][j], i >= j
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double d = M[sym_idx(j, j)];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= L[sym_idx(j, k)] * L[sym_idx(j, k)];
    const double ljj = sqrt(d);
    L[sym_idx(j, j)] = ljj;
    const double inv = 1.0 / ljj;
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      double s = M[sym_idx(i, j)];
#pragma unroll
      for (int k = 0; k < j; ++k) s -= L[sym_idx(i, k)] * L[sym_idx(j, k)];
      L[sym_idx(i, j)] = s * inv;
    }
  }
}

__device__ __forceinline__ void chol_solve6(const double *L, const double *b, double *x) {
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = b[i];
#pragma unroll
    for (int k = 0; k < i; ++k) s -= L[sym_idx(i, k)] * y[k];
    y[i] = s / L[sym_idx(i, i)];
  }
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    double s = y[i];
#pragma unroll
    for (int k = i + 1; k < 6; ++k) s -= L[sym_idx(k, i)] * x[k];
    x[i] = s / L[sym_idx(i, i)];
  }
}

__device__ __forceinline__ double int_or_real_pow(double x, double e) {
  // x >= 0.  Integer exponents by binary powering (as accurate as pow, much cheaper in
  // double); others through pow.
  const double ei = rint(e);
  if (ei == e && ei >= 0.0 && ei <= 1024.0) {
    int k = (int)ei;
    double r = 1.0, b = x;
    while (k) {
      if (k & 1) r *= b;
      b *= b;
      k >>= 1;
    }
    return r;
  }
  return pow(x, e);
}

// Slip resistance of one system after an increment (hardening_laws.py:18-90).
// dgam = dt * sum |gdot|; Gold = accumulated slip before the increment.
__device__ __forceinline__ double harden_iso(const PhaseParams &P, double gold, double Gold,
                                             double dgam) {
  switch (P.hardening) {
    case HARD_LINEAR:
      return gold + P.props[0] * dgam;
    case HARD_VOCE: {
      const double tau1 = P.props[0], th0 = P.props[1], th1 = P.props[2];
      const double ratio = fabs(th0 / tau1);
      const double ei = exp(-ratio * Gold);
      const double ec = exp(-ratio * dgam);
      return gold + th1 * dgam - (ratio * tau1 - th1) / ratio * ei * (ec - 1.0) -
             th1 / ratio * ei * (ec * (1.0 + ratio * (Gold + dgam)) - 1.0 - ratio * Gold);
    }
    case HARD_AF: {
      const double h = P.props[0], r = P.props[1];
      return gold + (h - r * gold) * dgam / (1.0 + r * dgam);
    }
    default:
      return gold;
  }
}

template <typename T>
__device__ __forceinline__ void load6(const T *f, long long V, long long v, double *x) {
#pragma unroll
  for (int c = 0; c < 6; ++c) x[c] = (double)f[c * V + v];
}

template <typename T>
__global__ void __launch_bounds__(128) constitutive_kernel(ConstArgs<T> a) {
  __shared__ int blk_max;
  __shared__ int blk_fail;
  if (threadIdx.x == 0) {
    blk_max = 0;
    blk_fail = 0;
  }
  __syncthreads();
  int my_iters = 0;
  bool my_fail = false;
  const long long V = a.V;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const int ph = a.phase ? a.phase[v] : 0;
    const PhaseParams &P = a.params[ph];
    double eps[6];
    load6<T>(a.eps, V, v, eps);
    if (P.kind == PHASE_ELASTIC) {
      double s[6];
      if (a.kvox) {
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < 6; ++j) acc += (double)a.kvox[sym_idx(i, j) * V + v] * eps[j];
          s[i] = acc;
        }
      } else {
        const T *k = a.ktab + (long long)a.gid[v] * 21;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < 6; ++j) acc += (double)k[sym_idx(i, j)] * eps[j];
          s[i] = acc;
        }
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) a.sig[c * V + v] = (T)s[c];
      my_iters = max(my_iters, 1);
      continue;
    }
    // ---------------- crystal elasto-viscoplasticity ----------------
    const double *Rm = a.rm_tab + (long long)a.orient[v] * 36;
    double gs[6];
    load6<T>(a.guess, V, v, gs);
    double gnorm = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) gnorm += gs[c] * gs[c];
    gnorm = sqrt(gnorm);
    double sig[6], epc[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double s0 = 0.0, e0 = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        s0 += Rm[i * 6 + j] * gs[j];
        e0 += Rm[i * 6 + j] * eps[j];
      }
      sig[i] = s0;
      epc[i] = e0;
    }
    const int ns = P.nslip;
    const double dt = a.dt;
    const double Gold = a.Gam_old[v];
    double g[MAX_SLIP], gdot[MAX_SLIP];
#pragma unroll
    for (int al = 0; al < MAX_SLIP; ++al) g[al] = (al < ns) ? a.g_in[al * V + v] : 1.0;
    double epo[6];
    load6<double>(a.ep_old, V, v, epo);
    double ep[6], M[21], L[21];
    double dgam = 0.0;
    bool conv = false;
    int it = 0;
    while (it < EVP_MAX_ITERATIONS) {
      ++it;
      // slip rates at the current stress (elastic_viscoplastic.py:205-216)
#pragma unroll
      for (int c = 0; c < 6; ++c) ep[c] = epo[c];
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 6; ++j) M[sym_idx(i, j)] = P.Cinv[i * 6 + j];
      dgam = 0.0;
#pragma unroll
      for (int al = 0; al < MAX_SLIP; ++al) {
        if (al < ns) {
          const double *Pa = P.P + al * 6;
          double tau = 0.0;
#pragma unroll
          for (int c = 0; c < 6; ++c) tau += sig[c] * Pa[c];
          const double ga = g[al];
          const double pref = P.gdot0 * int_or_real_pow(fabs(tau / ga), P.n - 1.0) / ga;
          const double gd = pref * tau;
          gdot[al] = gd;
          dgam += fabs(gd);
          const double wep = dt * gd;
#pragma unroll
          for (int c = 0; c < 6; ++c) ep[c] += wep * Pa[c];
          const double wm = dt * P.n * pref;
#pragma unroll
          for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j) M[sym_idx(i, j)] += wm * Pa[i] * Pa[j];
        } else {
          gdot[al] = 0.0;
        }
      }
      dgam *= dt;
      // Newton update sigma <- sigma - J^-1 (sigma - C (eps - ep))   (:225-235)
      double r[6], cr[6], z[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double acc = sig[i];
#pragma unroll
        for (int j = 0; j < 6; ++j) acc -= P.C[i * 6 + j] * (epc[j] - ep[j]);
        r[i] = acc;
      }
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += P.Cinv[i * 6 + j] * r[j];
        cr[i] = acc;
      }
      cholesky6(M, L);
      chol_solve6(L, cr, z);
      double diff = 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        sig[c] -= z[c];
        diff += z[c] * z[c];
      }
      diff = sqrt(diff);
      // hardening (:236-242), from the state at the start of the increment
      double tot = 0.0;
      if (P.latent != 1.0) {
#pragma unroll
        for (int al = 0; al < MAX_SLIP; ++al) tot += fabs(gdot[al]);
      }
#pragma unroll
      for (int al = 0; al < MAX_SLIP; ++al) {
        if (al < ns) {
          const double go = a.g_old[al * V + v];
          double gn = harden_iso(P, go, Gold, dgam);
          if (P.latent != 1.0 && tot > 0.0)
            gn = go + (gn - go) * (P.latent * tot + (1.0 - P.latent) * fabs(gdot[al])) / tot;
          g[al] = gn;
        }
      }
      conv = (diff / gnorm <= EVP_TOLERANCE) || (diff / P.E_ref < 1.0e-12);
      if (conv) break;
    }
    my_iters = max(my_iters, it);
    if (!conv) {
      my_fail = true;
      continue;
    }
    // tangent M^-1 in the crystal frame, then both back to the specimen frame
    double Tc[21];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double e[6], col[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) e[i] = (i == j) ? 1.0 : 0.0;
      chol_solve6(L, e, col);
#pragma unroll
      for (int i = 0; i <= j; ++i) Tc[sym_idx(i, j)] = col[i];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) acc += Rm[j * 6 + i] * sig[j];
      a.sig[i * V + v] = (T)acc;
    }
    // K_s = Rm^T Tc Rm
    double TR[36];
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += Tc[sym_idx(i, j)] * Rm[j * 6 + b];
        TR[i * 6 + b] = acc;
      }
#pragma unroll
    for (int p = 0; p < 6; ++p)
#pragma unroll
      for (int b = p; b < 6; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) acc += Rm[i * 6 + p] * TR[i * 6 + b];
        a.kvox[sym_idx(p, b) * V + v] = (T)acc;
      }
#pragma unroll
    for (int al = 0; al < MAX_SLIP; ++al)
      if (al < ns) {
        a.g_out[al * V + v] = g[al];
        if (a.gam_trial) a.gam_trial[al * V + v] = a.gam_old[al * V + v] + gdot[al] * dt;
      }
#pragma unroll
    for (int c = 0; c < 6; ++c) a.ep_trial[c * V + v] = ep[c];
    a.Gam_trial[v] = Gold + dgam;
  }
  if (my_iters) atomicMax(&blk_max, my_iters);
  if (my_fail) blk_fail = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(a.max_iters, blk_max);
    if (blk_fail) atomicOr(a.failed, 1);
  }
}
