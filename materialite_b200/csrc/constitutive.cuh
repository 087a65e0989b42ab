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

#include "../../include/ssfft.h"
#include "common.cuh"
#include "slots.cuh"

#define EVP_TOLERANCE 2.0e-5
#define EVP_MAX_ITERATIONS 60
#define MAX_SLIP 12

enum { PHASE_ELASTIC = 0, PHASE_EVP = 1, PHASE_J2 = 2 };
enum { HARD_PERFECT = 0, HARD_LINEAR = 1, HARD_VOCE = 2, HARD_AF = 3 };

struct PhaseParams {
  int kind, nslip, hardening, pad;
  double C[36];
  double Cinv[36];
  double P[MAX_SLIP * 6];
  double gdot0, n, g0, latent;
  double props[4];
  double E_ref;
  double shear, bulk;  // J2: shear and bulk moduli (g0 is the initial yield stress)
};

template <typename T> struct ConstArgs {
  long long V;
  const double *eps;       // 6 planes
  const double *guess;     // 6 planes
  double *sig;             // 6 planes (out)
  T *kvox;                 // 21 planes (out, EVP voxels) or null (table mode)
  const T *ktab;           // table-mode tangents [n_gid][21]
  const int32_t *gid;      // table-mode tangent index
  const int32_t *phase;    // phase per voxel (null: phase 0)
  const int32_t *orient;   // orientation per voxel
  const PhaseParams *params;
  int n_params;            // phases staged in shared memory (highest phase id + 1)
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
  const int *j2;           // J2: [0] return-mapping iterations of every point, [1] any plastic
};

__device__ __forceinline__ void cholesky6(const double *M, double *L, double *inv_diag) {
  // M, L packed symmetric (sym_idx); L holds the lower factor L[i][j], i >= j.  L may be
  // M itself: entry (i, j) of M is read only before entry (i, j) of L is written.
  // inv_diag receives 1 / L[j][j] for the triangular solves.
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double d = M[sym_idx(j, j)];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= L[sym_idx(j, k)] * L[sym_idx(j, k)];
    const double ljj = sqrt(d);
    L[sym_idx(j, j)] = ljj;
    const double inv = 1.0 / ljj;
    inv_diag[j] = inv;
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      double s = M[sym_idx(i, j)];
#pragma unroll
      for (int k = 0; k < j; ++k) s -= L[sym_idx(i, k)] * L[sym_idx(j, k)];
      L[sym_idx(i, j)] = s * inv;
    }
  }
}

__device__ __forceinline__ void chol_solve6(const double *L, const double *inv_diag,
                                            const double *b, double *x) {
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = b[i];
#pragma unroll
    for (int k = 0; k < i; ++k) s -= L[sym_idx(i, k)] * y[k];
    y[i] = s * inv_diag[i];
  }
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    double s = y[i];
#pragma unroll
    for (int k = i + 1; k < 6; ++k) s -= L[sym_idx(k, i)] * x[k];
    x[i] = s * inv_diag[i];
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

// Increment of the slip resistance when it is the same for every system and independent
// of the system's own value: perfect plasticity, linear and Voce hardening
// (hardening_laws.py:18-72); g_new = g_old + this.
__device__ __forceinline__ double harden_increment(const PhaseParams &P, double Gold,
                                                   double dgam) {
  switch (P.hardening) {
    case HARD_LINEAR:
      return P.props[0] * dgam;
    case HARD_VOCE: {
      const double tau1 = P.props[0], th0 = P.props[1], th1 = P.props[2];
      const double ratio = fabs(th0 / tau1);
      const double ei = exp(-ratio * Gold);
      const double ec = exp(-ratio * dgam);
      return th1 * dgam - (ratio * tau1 - th1) / ratio * ei * (ec - 1.0) -
             th1 / ratio * ei * (ec * (1.0 + ratio * (Gold + dgam)) - 1.0 - ratio * Gold);
    }
    default:
      return 0.0;
  }
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

// Threads of a constitutive block, and points of one item (four per thread).
#define CONST_THREADS 128
#define CONST_POINTS (4 * CONST_THREADS)

__host__ __device__ inline int const_items(long long V) {
  return (int)((V + CONST_POINTS - 1) / CONST_POINTS);
}

// The constitutive call of one slot: strain and stress guess in, stress and tangent out,
// plastic trial state written from the committed one (elastic_viscoplastic.py:91-188).
template <typename T>
__device__ __forceinline__ ConstArgs<T> const_args(const SlotDev<T> &S, long long V) {
  ConstArgs<T> a;
  a.V = V;
  a.eps = S.eps;
  a.guess = S.sig;
  a.sig = S.sig_next;
  a.kvox = S.voxel_mode ? S.kvox : nullptr;
  a.ktab = S.ktab;
  a.gid = S.gid;
  a.phase = S.phase;
  a.orient = S.orient;
  a.params = S.params;
  a.n_params = S.n_params;
  a.rm_tab = S.rm_tab;
  a.g_in = S.g_in;
  a.g_out = S.g_out;
  a.g_old = S.g_old;
  a.ep_old = S.ep_old;
  a.ep_trial = S.ep_trial;
  a.Gam_old = S.Gam_old;
  a.Gam_trial = S.Gam_trial;
  a.gam_old = S.gam_old;
  a.gam_trial = S.gam_trial;
  a.dt = S.dt;
  a.max_iters = S.citers;
  a.failed = S.citers + 1;
  a.j2 = S.citers + 2;
  return a;
}

// ---------------- J2 plasticity (isotropic_elastic_plastic.py:71-164) ----------------
#define J2_TOLERANCE 1.0e-7
#define J2_MAX_ITERATIONS 100

// Elastic predictor of one point: deviatoric stress s (Mandel), mean stress, von Mises q.
__device__ __forceinline__ void j2_predictor(const PhaseParams &P, const double *eps,
                                             const double *ep_old, double *s, double &mean,
                                             double &q) {
  double ee[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) ee[c] = eps[c] - ep_old[c];
  const double tr = ee[0] + ee[1] + ee[2];
  const double vol = 1.0 / 3.0 * tr;  // tensor.py:1242-1244
  double n2 = 0.0;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    s[c] = 2.0 * P.shear * (c < 3 ? ee[c] - vol : ee[c]);
    n2 += s[c] * s[c];
  }
  mean = P.bulk * tr;
  q = sqrt(1.5) * sqrt(n2);
}

// Yield stress after an equivalent plastic strain increment dp, as the reference calls the
// hardening laws from IsotropicElasticPlastic: rate dp / dt, increment dt |rate|
// (hardening_laws.py:35-38, 49-52, 83-86).
__device__ __forceinline__ double j2_yield(const PhaseParams &P, double eq_old, double y_old,
                                           double dp, double dt) {
  return harden_iso(P, y_old, eq_old, dt * fabs(dp / dt));
}

// One fixed-point update of the return mapping (:110-119): residual clipped at zero,
// inverse Jacobian -1/(3G).
__device__ __forceinline__ double j2_update(const PhaseParams &P, double q, double dp,
                                            double y) {
  double r = q - 3.0 * P.shear * dp - y;
  if (r <= 0.0) r = 0.0;
  const double jinv = -1.0 / (3.0 * P.shear);
  return dp - jinv * r;
}

// Pass 1 of a J2 update: the reference iterates every point until all have converged, so
// each point's own iteration count is found first and reduced to the maximum (j2[0]),
// with j2[1] = 1 if any point is plastic.  A point that does not converge within
// J2_MAX_ITERATIONS fails the update (:133-137).
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    j2_count_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  __shared__ int blk_n, blk_any, blk_fail;
  const int per = const_items(V);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
  const int kslot = item / per;
  const int local = item - kslot * per;
  const SlotDev<T> &S = tab[list.ids[kslot]];
  const ConstArgs<T> a = const_args<T>(S, V);
  int *j2 = S.citers + 2;
  __syncthreads();
  if (threadIdx.x == 0) {
    blk_n = 0;
    blk_any = 0;
    blk_fail = 0;
  }
  __syncthreads();
  int my_n = 0, my_any = 0, my_fail = 0;
  const long long v1 = min(V, (long long)(local + 1) * CONST_POINTS);
  for (long long v = (long long)local * CONST_POINTS + threadIdx.x; v < v1; v += blockDim.x) {
    const PhaseParams &P = a.params[a.phase ? a.phase[v] : 0];
    if (P.kind != PHASE_J2) continue;
    double eps[6], epo[6], s[6], mean, q;
    load6<double>(a.eps, V, v, eps);
    load6<double>(a.ep_old, V, v, epo);
    j2_predictor(P, eps, epo, s, mean, q);
    const double y_old = a.g_old[v], eq_old = a.Gam_old[v];
    if (!(q <= y_old)) my_any = 1;
    double dp = 0.0, y = y_old;
    int it = 0;
    bool conv = false;
    while (it < J2_MAX_ITERATIONS) {
      ++it;
      const double prev = dp;
      dp = j2_update(P, q, dp, y);
      y = j2_yield(P, eq_old, y_old, dp, a.dt);
      if (fabs(dp - prev) < J2_TOLERANCE) {
        conv = true;
        break;
      }
    }
    my_n = max(my_n, it);
    if (!conv) my_fail = 1;
  }
  if (my_n) atomicMax(&blk_n, my_n);
  if (my_any) blk_any = 1;
  if (my_fail) blk_fail = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (blk_n) atomicMax(&j2[0], blk_n);
    if (blk_any) atomicOr(&j2[1], 1);
    if (blk_fail) atomicOr(a.failed, 1);
  }
  }
}

// Threads of a constitutive block, and the shared memory a block holds: the phase table
// plus per-thread slip arrays (old and current resistances, slip rates) and the two
// crystal-frame strain vectors, [entry][thread] so that a warp's accesses are contiguous.
inline size_t constitutive_smem_bytes() {
  return (size_t)SSFFT_MAX_PHASES * sizeof(PhaseParams) +
         (size_t)(3 * MAX_SLIP + 12) * CONST_THREADS * sizeof(double);
}

template <typename T>
__global__ void __launch_bounds__(CONST_THREADS, 3)
    constitutive_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  extern __shared__ __align__(16) unsigned char csm[];
  PhaseParams *sp = reinterpret_cast<PhaseParams *>(csm);
  const int tid = threadIdx.x;
  // per-thread slip arrays after the largest phase table, stride CONST_THREADS
  double *s_gold = reinterpret_cast<double *>(sp + SSFFT_MAX_PHASES) + tid;
  double *s_gdot = s_gold + MAX_SLIP * CONST_THREADS;
  double *s_g = s_gdot + MAX_SLIP * CONST_THREADS;
  double *s_epo = s_g + MAX_SLIP * CONST_THREADS;
  double *s_epc = s_epo + 6 * CONST_THREADS;
#define TS(arr, k) arr[(k) * CONST_THREADS]
  __shared__ int blk_max;
  __shared__ int blk_fail;
  const int per = const_items(V);
  const int n_items = list_items(list, per);
  int staged = -1;  // slot whose phase table is in shared memory
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
  const int kslot = item / per;
  const int local = item - kslot * per;
  const int slot = list.ids[kslot];
  const ConstArgs<T> a = const_args<T>(tab[slot], V);
  __syncthreads();
  if (slot != staged) {
    const int nw = a.n_params * (int)(sizeof(PhaseParams) / sizeof(int));
    const int *src = reinterpret_cast<const int *>(a.params);
    int *dst = reinterpret_cast<int *>(sp);
    for (int i = tid; i < nw; i += CONST_THREADS) dst[i] = src[i];
    staged = slot;
  }
  if (tid == 0) {
    blk_max = 0;
    blk_fail = 0;
  }
  __syncthreads();
  int my_iters = 0;
  bool my_fail = false;
  const long long v1 = min(V, (long long)(local + 1) * CONST_POINTS);
  for (long long v = (long long)local * CONST_POINTS + tid; v < v1; v += CONST_THREADS) {
    const int ph = a.phase ? a.phase[v] : 0;
    const PhaseParams &P = sp[ph];
    double eps[6];
    load6<double>(a.eps, V, v, eps);
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
      for (int c = 0; c < 6; ++c) a.sig[c * V + v] = s[c];
      my_iters = max(my_iters, 1);
      continue;
    }
    if (P.kind == PHASE_J2) {
      // pass 2: every point runs the common iteration count of pass 1 (:106-138)
      double epo[6], s[6], mean, q;
      load6<double>(a.ep_old, V, v, epo);
      j2_predictor(P, eps, epo, s, mean, q);
      const double y_old = a.g_old[v], eq_old = a.Gam_old[v];
      const bool elastic = q <= y_old;
      double sig[6];
      if (!a.j2[1]) {
        // every point elastic: elastic stress, elastic tangent, state untouched (:94-99);
        // the current slip-resistance plane is carried into the next trial buffer
#pragma unroll
        for (int c = 0; c < 6; ++c) sig[c] = s[c] + (c < 3 ? mean : 0.0);
#pragma unroll
        for (int c = 0; c < 6; ++c) a.sig[c * V + v] = sig[c];
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
          for (int j = i; j < 6; ++j) a.kvox[sym_idx(i, j) * V + v] = (T)P.C[i * 6 + j];
        a.g_out[v] = a.g_in[v];
        // the trial plastic state equals the committed one, so that a commit may swap
        // the trial and committed buffers
#pragma unroll
        for (int c = 0; c < 6; ++c) a.ep_trial[c * V + v] = epo[c];
        a.Gam_trial[v] = eq_old;
        my_iters = max(my_iters, 1);
        continue;
      }
      const int N = a.j2[0];
      double dp = 0.0, y = y_old;
      for (int it = 0; it < N; ++it) {
        dp = j2_update(P, q, dp, y);
        y = j2_yield(P, eq_old, y_old, dp, a.dt);
      }
      my_iters = max(my_iters, N);
      // state (:139-146); a point with no deviatoric strain keeps its plastic strain
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const double rs = q > 0.0 ? s[c] / q : 0.0;
        a.ep_trial[c * V + v] = epo[c] + 1.5 * rs * dp;
      }
      a.Gam_trial[v] = eq_old + dp;
      a.g_out[v] = y;
      const double ratio = 3.0 * P.shear / q;
#pragma unroll
      for (int c = 0; c < 6; ++c) sig[c] = (1.0 - ratio * dp) * s[c] + (c < 3 ? mean : 0.0);
#pragma unroll
      for (int c = 0; c < 6; ++c) a.sig[c * V + v] = sig[c];
      // consistent tangent C - t1 I_dev + t2 s (x) s on plastic points, C on elastic ones
      // (:148-163)
      const double t1 = elastic ? 0.0 : 2.0 * P.shear * ratio * dp;
      const double t2 = elastic ? 0.0 : ratio * ratio * (dp / q - 1.0 / (3.0 * P.shear));
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 6; ++j) {
          const double idev = (i == j ? 1.0 : 0.0) - (i < 3 && j < 3 ? 1.0 / 3.0 : 0.0);
          const double k = elastic ? P.C[i * 6 + j] : P.C[i * 6 + j] - t1 * idev + t2 * (s[i] * s[j]);
          a.kvox[sym_idx(i, j) * V + v] = (T)k;
        }
      continue;
    }
    // ---------------- crystal elasto-viscoplasticity ----------------
    const double *Rm = a.rm_tab + (long long)a.orient[v] * 36;
    double gs[6];
    load6<double>(a.guess, V, v, gs);
    double gnorm = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) gnorm += gs[c] * gs[c];
    gnorm = sqrt(gnorm);
    double sig[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double s0 = 0.0, e0 = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const double rij = Rm[i * 6 + j];
        s0 += rij * gs[j];
        e0 += rij * eps[j];
      }
      sig[i] = s0;
      TS(s_epc, i) = e0;
      TS(s_epo, i) = a.ep_old[i * V + v];
    }
    const int ns = P.nslip;
    const double dt = a.dt;
    const double Gold = a.Gam_old[v];
    for (int al = 0; al < ns; ++al) {
      TS(s_g, al) = a.g_in[al * V + v];
      TS(s_gold, al) = a.g_old[al * V + v];
    }
    // linear / Voce / perfect with no latent ratio: one increment for all systems
    const bool iso = (P.latent == 1.0) && (P.hardening != HARD_AF);
    double ep[6], M[21], idg[6];
    double dgam = 0.0;
    bool conv = false;
    int it = 0;
    while (it < EVP_MAX_ITERATIONS) {
      ++it;
      // slip rates at the current stress (elastic_viscoplastic.py:205-216)
#pragma unroll
      for (int c = 0; c < 6; ++c) ep[c] = TS(s_epo, c);
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 6; ++j) M[sym_idx(i, j)] = P.Cinv[i * 6 + j];
      dgam = 0.0;
      for (int al = 0; al < ns; ++al) {
        const double *Pa = P.P + al * 6;
        double pa[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) pa[c] = Pa[c];
        double tau = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) tau += sig[c] * pa[c];
        const double inv_g = 1.0 / TS(s_g, al);
        const double pref = P.gdot0 * int_or_real_pow(fabs(tau) * inv_g, P.n - 1.0) * inv_g;
        const double gd = pref * tau;
        TS(s_gdot, al) = gd;
        dgam += fabs(gd);
        const double wep = dt * gd;
#pragma unroll
        for (int c = 0; c < 6; ++c) ep[c] += wep * pa[c];
        const double wm = dt * P.n * pref;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const double wi = wm * pa[i];
#pragma unroll
          for (int j = i; j < 6; ++j) M[sym_idx(i, j)] += wi * pa[j];
        }
      }
      dgam *= dt;
      // Newton update sigma <- sigma - J^-1 (sigma - C (eps - ep))   (:225-235), with
      // J^-1 r = M^-1 C^-1 r and C^-1 r = C^-1 sigma - (eps - ep)
      double cr[6], z[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double acc = ep[i] - TS(s_epc, i);
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += P.Cinv[i * 6 + j] * sig[j];
        cr[i] = acc;
      }
      cholesky6(M, M, idg);
      chol_solve6(M, idg, cr, z);
      double diff = 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        sig[c] -= z[c];
        diff += z[c] * z[c];
      }
      diff = sqrt(diff);
      // hardening (:236-242), from the state at the start of the increment
      if (iso) {
        const double inc = harden_increment(P, Gold, dgam);
        for (int al = 0; al < ns; ++al) TS(s_g, al) = TS(s_gold, al) + inc;
      } else {
        double tot = 0.0;
        if (P.latent != 1.0)
          for (int al = 0; al < ns; ++al) tot += fabs(TS(s_gdot, al));
        for (int al = 0; al < ns; ++al) {
          const double go = TS(s_gold, al);
          double gn = harden_iso(P, go, Gold, dgam);
          if (P.latent != 1.0 && tot > 0.0)
            gn = go + (gn - go) * (P.latent * tot + (1.0 - P.latent) * fabs(TS(s_gdot, al))) / tot;
          TS(s_g, al) = gn;
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
    // stress back to the specimen frame
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) acc += Rm[j * 6 + i] * sig[j];
      a.sig[i * V + v] = acc;
    }
    // tangent M^-1 in the crystal frame (columns from the factor), then
    // K_s = Rm^T M^-1 Rm one row at a time
    double Tc[21];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double e[6], col[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) e[i] = (i == j) ? 1.0 : 0.0;
      chol_solve6(M, idg, e, col);
#pragma unroll
      for (int i = 0; i <= j; ++i) Tc[sym_idx(i, j)] = col[i];
    }
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      double t[6];  // row p of Rm^T Tc
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) acc += Rm[i * 6 + p] * Tc[sym_idx(i, j)];
        t[j] = acc;
      }
#pragma unroll
      for (int b = p; b < 6; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += t[j] * Rm[j * 6 + b];
        a.kvox[sym_idx(p, b) * V + v] = (T)acc;
      }
    }
    for (int al = 0; al < ns; ++al) {
      a.g_out[al * V + v] = TS(s_g, al);
      if (a.gam_trial) a.gam_trial[al * V + v] = a.gam_old[al * V + v] + TS(s_gdot, al) * dt;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) a.ep_trial[c * V + v] = ep[c];
    a.Gam_trial[v] = Gold + dgam;
  }
  if (my_iters) atomicMax(&blk_max, my_iters);
  if (my_fail) blk_fail = 1;
  __syncthreads();
  if (tid == 0) {
    atomicMax(a.max_iters, blk_max);
    if (blk_fail) atomicOr(a.failed, 1);
  }
  }
#undef TS
}
