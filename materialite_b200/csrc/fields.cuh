// Elementwise and reduction kernels around the Newton loop of SmallStrainFFT.run
// (small_strain_fft.py:106-246): strain guess, strain update, convergence norms,
// mean tangent, commit, and layout conversion for read-back.
#pragma once

#include "common.cuh"
#include "constitutive.cuh"
#include "krylov.cuh"
#include "slots.cuh"

// Tangent lookup: table mode (per (orientation, phase) pair) or voxel mode (21 planes).
template <typename T> struct TangentRef {
  const T *ktab;
  const int32_t *gid;
  const T *kvox;
  long long V;
  __device__ __forceinline__ void apply(long long v, const double *x, double *y) const {
    if (kvox) {
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += (double)kvox[sym_idx(i, j) * V + v] * x[j];
        y[i] = acc;
      }
    } else {
      const T *k = ktab + (long long)gid[v] * 21;
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += (double)k[sym_idx(i, j)] * x[j];
        y[i] = acc;
      }
    }
  }
  __device__ __forceinline__ double entry(long long v, int k) const {
    return kvox ? (double)kvox[k * V + v] : (double)ktab[(long long)gid[v] * 21 + k];
  }
};

// The slot's tangent: the committed one (start of a load increment: the tangent of the
// last converged state, or the initial one) or the latest constitutive output.
template <typename T>
__device__ __forceinline__ TangentRef<T> tangent_of(const SlotDev<T> &S, bool committed,
                                                    long long V) {
  TangentRef<T> K;
  K.ktab = S.ktab;
  K.gid = S.gid;
  K.kvox = S.voxel_mode ? (committed ? S.kvox_old : S.kvox) : nullptr;
  K.V = V;
  return K;
}

// strain = old_strain + dE + old_fluct ; guess = first ? dS + K dEbar : old_stress + dS
// (small_strain_fft.py:113-123).  The guess goes to the slot's latest-stress buffer, which
// the next constitutive call reads.  The fluctuation is first scaled by the slot's
// fluct_scale (new dt / old dt after an increment, 1/2 after a cutback,
// small_strain_fft.py:236-244) or cleared (reset_fluct: the load reversed).
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    strain_guess_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  const int per = vec_items(V);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = item / per;
    const int local = item - k * per;
    const SlotDev<T> &S = tab[list.ids[k]];
    const long long v0 = (long long)local * VEC_CHUNK;
    const long long v1 = min(V, v0 + VEC_CHUNK);
    const StepVec sv = S.sv;
    const bool first = S.first_step != 0, reset = S.reset_fluct != 0;
    const double fs = S.fluct_scale;
    const TangentRef<T> K = tangent_of<T>(S, true, V);
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        double f = S.dfl[c * V + v];
        if (reset) f = 0.0;
        else if (fs != 1.0) f = f * fs;
        if (reset || fs != 1.0) S.dfl[c * V + v] = f;
        // same association as the reference: (old + dEbar + fluct) + correction
        double e = S.eps_old[c * V + v] + sv.dEbar[c];
        S.eps[c * V + v] = (e + f) + sv.corr[c];
      }
      if (first) {
        double y[6];
        K.apply(v, sv.dEbar, y);
#pragma unroll
        for (int c = 0; c < 6; ++c) S.sig[c * V + v] = sv.dS[c] + y[c];
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) S.sig[c * V + v] = S.sig_old[c * V + v] + sv.dS[c];
      }
    }
  }
}

// strain += dx ; old_fluct += dx  (small_strain_fft.py:154-155), dx the slot's Krylov
// iterate.  (In the mixed mode the double re-projection of dx does this in its epilogue.)
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    update_strain_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  const long long n = 6 * V;
  const int per = vec_items(n);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = item / per;
    const int local = item - k * per;
    const SlotDev<T> &S = tab[list.ids[k]];
    const T *dx = S.kr[5];
    const long long i0 = (long long)local * VEC_CHUNK;
    const long long i1 = min(n, i0 + VEC_CHUNK);
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const double d = dx[i];
      S.eps[i] += d;
      S.dfl[i] += d;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    scale_kernel(long long n, T *__restrict__ x, double f) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = (T)((double)x[i] * f);
}

__device__ __forceinline__ double dev_norm6(const double *s) {
  const double tr3 = (s[0] + s[1] + s[2]) / 3.0;
  const double a = s[0] - tr3, b = s[1] - tr3, c = s[2] - tr3;
  return sqrt(a * a + b * b + c * c + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
}

// Convergence quantities of small_strain_fft.py:172-189 in one pass:
//   out[0..5]  sum of stress      out[6..11] sum of strain
//   out[12]    max |dev(stress - old_stress)|   out[13] max |K : dx|  (if norms_dx)
#define NORM_VALS 14
#define NORM_SUMS 12  // values 0..11 are sums, 12..13 maxima
#define NORM_CHUNK (4 * SSFFT_THREADS)  // points per item

// Combine one of the norm values (sum or max) in a fixed order.
__device__ __forceinline__ double norm_combine(int k, double a, double b) {
  return k < NORM_SUMS ? a + b : fmax(a, b);
}

// Warp tree reduction of value k (fixed shuffle order).
__device__ __forceinline__ double norm_warp_reduce(int k, double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = norm_combine(k, v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

__host__ __device__ inline int norm_items(long long V) { return (int)((V + NORM_CHUNK - 1) / NORM_CHUNK); }

template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    newton_norms_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  __shared__ double wred[NORM_VALS][SSFFT_THREADS / 32];
  const int per = norm_items(V);
  const int n_items = list_items(list, per);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int kslot = item / per;
    const int local = item - kslot * per;
    const SlotDev<T> &S = tab[list.ids[kslot]];
    const T *dx = S.norms_dx ? S.kr[5] : nullptr;
    const TangentRef<T> K = tangent_of<T>(S, false, V);
    double acc[NORM_VALS];
#pragma unroll
    for (int k = 0; k < NORM_VALS; ++k) acc[k] = 0.0;
    const long long v0 = (long long)local * NORM_CHUNK;
    const long long v1 = min(V, v0 + NORM_CHUNK);
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
      double s[6], d[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        s[c] = (double)S.sig[c * V + v];
        acc[c] += s[c];
        acc[6 + c] += (double)S.eps[c * V + v];
        d[c] = s[c] - (double)S.sig_old[c * V + v];
      }
      acc[12] = fmax(acc[12], dev_norm6(d));
      if (dx) {
        double x[6], y[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) x[c] = (double)dx[c * V + v];
        K.apply(v, x, y);
        double n2 = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) n2 += y[c] * y[c];
        acc[13] = fmax(acc[13], sqrt(n2));
      }
    }
    // all fourteen values through one warp pass and one barrier
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NORM_VALS; ++k) {
      const double r = norm_warp_reduce(k, acc[k]);
      if (lane == 0) wred[k][warp] = r;
    }
    __syncthreads();
    if (threadIdx.x < NORM_VALS) {
      const int k = threadIdx.x;
      double r = wred[k][0];
      for (int w = 1; w < nw; ++w) r = norm_combine(k, r, wred[k][w]);
      S.partials[(size_t)local * NORM_VALS + k] = r;
    }
    if (last_item_arrives(S.tickets + TK_NORMS, (unsigned)per)) {
      // one warp per value: lanes stride over the item partials, then a fixed tree
      for (int k = warp; k < NORM_VALS; k += nw) {
        double r = 0.0;
        for (int b = lane; b < per; b += 32)
          r = norm_combine(k, r, S.partials[(size_t)b * NORM_VALS + k]);
        r = norm_warp_reduce(k, r);
        if (lane == 0) S.results[k] = r;
      }
      if (threadIdx.x == 0) S.tickets[TK_NORMS] = 0;
    }
    __syncthreads();
  }
}

// Sum of the committed tangent over all points (21 packed entries) for
// tangent.mean().inv (small_strain_fft.py:119-120), into results[16..36].
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    tangent_sum_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  __shared__ double red[32];
  const int per = vec_items(V);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int kslot = item / per;
    const int local = item - kslot * per;
    const SlotDev<T> &S = tab[list.ids[kslot]];
    const TangentRef<T> K = tangent_of<T>(S, true, V);
    double acc[21];
#pragma unroll
    for (int k = 0; k < 21; ++k) acc[k] = 0.0;
    const long long v0 = (long long)local * VEC_CHUNK;
    const long long v1 = min(V, v0 + VEC_CHUNK);
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
#pragma unroll
      for (int k = 0; k < 21; ++k) acc[k] += K.entry(v, k);
    }
#pragma unroll
    for (int k = 0; k < 21; ++k) {
      const double r = block_sum(acc[k], red);
      if (threadIdx.x == 0) S.partials[(size_t)local * 21 + k] = r;
    }
    if (last_item_arrives(S.tickets + TK_TSUM, (unsigned)per)) {
      for (int k = 0; k < 21; ++k) {
        const double r = ordered_sum(S.partials + k, per, 21, red);
        if (threadIdx.x == 0) S.results[16 + k] = r;
      }
      if (threadIdx.x == 0) S.tickets[TK_TSUM] = 0;
    }
    __syncthreads();
  }
}

// Commit of the slip resistances (elastic_viscoplastic.py:264-266): g_old = g_in, the last
// converged trial.  The other committed fields change roles by pointer swaps; g_in must
// keep its values, since the next constitutive call starts its inner Newton from them.
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    commit_slip_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V,
                       int nslip_max) {
  const long long n = (long long)nslip_max * V;
  const int per = vec_items(n);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = item / per;
    const int local = item - k * per;
    const SlotDev<T> &S = tab[list.ids[k]];
    if (!S.any_evp) continue;
    const long long ns = (long long)S.nslip * V;
    const long long i0 = (long long)local * VEC_CHUNK;
    const long long i1 = min(ns, i0 + VEC_CHUNK);
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) S.g_old[i] = S.g_in[i];
  }
}

// Planar T (width planes of V) -> point-major float64 (V x width).
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    to_point_major_kernel(long long V, int width, const T *__restrict__ src,
                          double *__restrict__ dst) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < V * width;
       i += (long long)gridDim.x * blockDim.x) {
    const long long v = i / width;
    const int c = (int)(i - v * width);
    dst[i] = (double)src[c * V + v];
  }
}

// Point-major float64 (V x 6) -> planar T.
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    from_point_major_kernel(long long V, const double *__restrict__ src, T *__restrict__ dst) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < V * 6;
       i += (long long)gridDim.x * blockDim.x) {
    const long long v = i / 6;
    const int c = (int)(i - v * 6);
    dst[c * V + v] = (T)src[i];
  }
}

// Committed plastic strains -> specimen frame, point-major: crystal-frame EVP strains are
// rotated (elastic_viscoplastic.py:258-263); J2 strains are kept in the specimen frame.
__global__ void __launch_bounds__(SSFFT_THREADS)
    plastic_to_specimen_kernel(long long V, const double *__restrict__ ep,
                               const int32_t *__restrict__ orient,
                               const double *__restrict__ rm_tab,
                               const int32_t *__restrict__ phase,
                               const PhaseParams *__restrict__ params, double *__restrict__ dst) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    if (params[phase ? phase[v] : 0].kind == PHASE_J2) {
#pragma unroll
      for (int i = 0; i < 6; ++i) dst[v * 6 + i] = ep[i * V + v];
      continue;
    }
    const double *Rm = rm_tab + (long long)orient[v] * 36;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) acc += Rm[j * 6 + i] * ep[j * V + v];
      dst[v * 6 + i] = acc;
    }
  }
}

// Initial plastic state: slip resistances g0 on EVP voxels, the initial yield stress in
// plane 0 on J2 voxels, zero elsewhere.
__global__ void __launch_bounds__(SSFFT_THREADS)
    evp_init_kernel(long long V, int nslip_max, const int32_t *__restrict__ phase,
                    const PhaseParams *__restrict__ params, double *g_a, double *g_b,
                    double *g_old) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const PhaseParams &P = params[phase ? phase[v] : 0];
    for (int al = 0; al < nslip_max; ++al) {
      const double g = ((P.kind == PHASE_EVP && al < P.nslip) || (P.kind == PHASE_J2 && al == 0))
                           ? P.g0 : 0.0;
      g_a[al * V + v] = g;
      g_b[al * V + v] = g;
      g_old[al * V + v] = g;
    }
  }
}

// Voxel-mode tangent initialisation: K = Rm^T C Rm for every voxel of every phase
// (elastic.py:23-27, elastic_viscoplastic.py:89).
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    init_kvox_kernel(long long V, const int32_t *__restrict__ phase,
                     const int32_t *__restrict__ orient, const PhaseParams *__restrict__ params,
                     const double *__restrict__ rm_tab, T *__restrict__ kvox) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const PhaseParams &P = params[phase ? phase[v] : 0];
    if (P.kind == PHASE_J2) {
      // isotropic: the unrotated stiffness (isotropic_elastic_plastic.py:55-59)
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = a; b < 6; ++b) kvox[sym_idx(a, b) * V + v] = (T)P.C[a * 6 + b];
      continue;
    }
    const double *Rm = rm_tab + (long long)orient[v] * 36;
    double CR[36];
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += P.C[i * 6 + j] * Rm[j * 6 + b];
        CR[i * 6 + b] = acc;
      }
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
      for (int b = a; b < 6; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) acc += Rm[i * 6 + a] * CR[i * 6 + b];
        kvox[sym_idx(a, b) * V + v] = (T)acc;
      }
  }
}
