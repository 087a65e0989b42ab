// Device MINRES (Paige & Saunders 1975) for the Newton correction of
// small_strain_fft.py:281-299, which the reference delegates to scipy's minres with
// x0 = 0, no preconditioner and its default stopping tests.
//
// All scalars live in a MinresState in device memory (one per slot) and are advanced by
// the last item of each reduction, so an iteration needs no host round trip.  With u_j
// the Lanczos vector of iteration j (v_j = u_j / beta_j), one iteration is five
// (plane-fused) or seven kernels:
//
//   update        pending update of iteration j-1: u_j = y' - (alfa/beta) u_{j-1},
//                 w = (v_{j-1} - oldeps w1 - delta w2) / gamma, x += phi w;
//                 last item: |x| and the stopping tests          (minres_after_update)
//                 then tau = K (u_j / beta_j) into y''s buffer
//   forward z(y)  forward transform of tau
//   ... y/x passes ...
//   inverse z     inverse transform: P tau into y''s buffer
//   epilogue      y' = P tau - (beta_j / beta_{j-1}) u_{j-1}; u_j.y', y'.y', u_j.u_j;
//                 last item: alfa, beta_{j+1}, plane rotation    (minres_after_matvec)
//
// The update needs alfa, a global dot product of the matvec, so it cannot join the
// inverse pass; it opens the next iteration.  The last iteration's update is applied by
// one more update pass, which then finds the solve done.  Vectors are component-planar in the solve precision T, handled as one
// contiguous run of 6V values; every dot product and norm accumulates in double, in a
// fixed order (item partials summed by the slot's last item), so results depend neither on
// scheduling nor on the other slots of a launch.  Buffer roles follow the slot's own
// iteration count (kroles), so slots of one launch may be at different iterations.
#pragma once

#include "common.cuh"
#include "projector.cuh"

// Values per item of the elementwise and reduction kernels over 6V (or V) values.
#define VEC_CHUNK 4096

__host__ __device__ inline int vec_items(long long n) { return (int)((n + VEC_CHUNK - 1) / VEC_CHUNK); }

// Start of a solve on every listed slot: r1 = r2 = b, x = w = w2 = 0, |b|^2; the slot's
// last item initialises its MINRES state.
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    minres_init_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  __shared__ double red[32];
  const long long n = 6 * V;
  const int per = vec_items(n);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = item / per;
    const int local = item - k * per;
    const SlotDev<T> &S = tab[list.ids[k]];
    const KRoles<T> r = kroles<T>(S, 0);
    const long long i0 = (long long)local * VEC_CHUNK;
    const long long i1 = min(n, i0 + VEC_CHUNK);
    double acc = 0.0;
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const T bi = S.b[i];
      r.P[i] = bi;
      r.Q[i] = bi;
      r.X[i] = 0;
      r.W[i] = 0;
      r.W2[i] = 0;
      acc += (double)bi * (double)bi;
    }
    const double part = block_sum(acc, red);
    if (threadIdx.x == 0) S.partials[local] = part;
    if (last_item_arrives(S.tickets + TK_INIT, (unsigned)per)) {
      const double b2 = ordered_sum(S.partials, per, 1, red);
      if (threadIdx.x == 0) {
        S.tickets[TK_INIT] = 0;
        MinresState s;
        const double beta1 = sqrt(b2);
        s.beta1 = beta1;
        s.beta = beta1;
        s.oldb = 0.0;
        s.alfa = 0.0;
        s.dbar = 0.0;
        s.epsln = 0.0;
        s.phibar = beta1;
        s.tnorm2 = 0.0;
        s.gmax = 0.0;
        s.gmin = 1.7976931348623157e308;
        s.cs = -1.0;
        s.sn = 0.0;
        s.delta = 0.0;
        s.oldeps = 0.0;
        s.gamma = 0.0;
        s.phi = 0.0;
        s.denom = 0.0;
        s.root = 0.0;
        s.anorm = 0.0;
        s.ynorm = 0.0;
        s.rnorm = beta1;
        s.test1 = 0.0;
        s.test2 = 0.0;
        s.s = (beta1 > 0.0) ? 1.0 / beta1 : 0.0;
        s.s_prev = 0.0;
        s.c_r1 = 0.0;
        s.coef = 0.0;
        s.rtol = S.rtol;
        s.eps = 2.220446049250313e-16;
        s.itn = 0;
        s.maxiter = S.maxiter;
        s.istop = 0;
        // absolute floor (the stress scale of the residual just computed) and relative forcing
        s.atol = S.atol_scale > 0.0 ? S.atol_scale * mean_von_mises(S.results, V) : 0.0;
        s.atol = fmax(s.atol, S.forcing * beta1);
        // beta1 == 0: x = 0 is exact; beta1 under the floor: x = 0 is close enough
        s.done = (b2 == 0.0 || beta1 <= s.atol) ? 1 : 0;
        if (s.done && b2 != 0.0) s.istop = 1;
        *S.st = s;
      }
    }
    __syncthreads();
  }
}

// The forward half of a Krylov matvec, elementwise: for every listed slot whose solve is
// not done, the pending update of the previous iteration (u_j = y' - coef u_{j-1}, w, x,
// |x|^2 and, in the slot's last item, the stopping tests) and tau = K (s u_j), which
// replaces y' in its buffer point by point (y' is consumed here; the inverse pass of this
// iteration writes the next y' there).  The forward transform then copies tau from there
// (PRO_TAU).  A plain streaming kernel: each point's loads go out together and no register
// cap is imposed, so the loads of a block keep HBM busy.
template <typename T, int PRO>
__global__ void __launch_bounds__(SSFFT_THREADS)
    krylov_update_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  __shared__ double red[32];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<T>)];
  const int per = vec_items(V);
  const int n_items = list_items(list, per);
  int staged = -1;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = item / per;
    const int local = item - k * per;
    const SlotDev<T> &S = stage_slot<T>(tab, list.ids[k], sdesc, staged);
    if (slot_done(S.st)) continue;
    const KrylovIn<T, T> u = krylov_in<T, T>(S);
    const long long v0 = (long long)local * VEC_CHUNK;
    const long long v1 = min(V, v0 + VEC_CHUNK);
    T *tau_out = u.r.Y;
    double xx = 0.0;
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
      T tau[6];
      tangent_prologue<T, T, PRO, true>(S, V, v, u, 0, tau, xx);
#pragma unroll
      for (int c = 0; c < 6; ++c) tau_out[c * V + v] = tau[c];
    }
    if (u.on) finish_pending_update(S, xx, local, per, red);
  }
}

// The MINRES half of the matvec epilogue, elementwise: over the P tau that the inverse
// transform left in y''s buffer (EPI_PTAU), y' = P tau - (beta_j / beta_{j-1}) u_{j-1} in
// place, and the dot products u_j.y', y'.y', u_j.u_j; the slot's last item advances the
// recurrence (minres_after_matvec).
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    krylov_epilogue_kernel(const SlotDev<T> *__restrict__ tab, SlotList list, long long V) {
  __shared__ double red[32];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<T>)];
  const int per = vec_items(V);
  const int n_items = list_items(list, per);
  int staged = -1;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = item / per;
    const int local = item - k * per;
    const SlotDev<T> &S = stage_slot<T>(tab, list.ids[k], sdesc, staged);
    if (slot_done(S.st)) continue;
    const KRoles<T> kr = kroles<T>(S, S.st->itn);
    const T c1 = (T)S.st->c_r1;
    const long long v0 = (long long)local * VEC_CHUNK;
    const long long v1 = min(V, v0 + VEC_CHUNK);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if constexpr (sizeof(T) == 4) {
      // four consecutive points a thread, one 16-byte load per component plane and vector
      // (each plane starts on a 16-byte boundary when V is a multiple of 4, and so does every
      // item): four times the bytes in flight of one point a thread
      if ((V & 3) == 0) {
        for (long long v = v0 + 4 * threadIdx.x; v < v1; v += 4 * blockDim.x) {
          float4 pt[6], r1[6], r2[6];
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            pt[c] = *reinterpret_cast<const float4 *>(kr.Y + c * V + v);
            r1[c] = *reinterpret_cast<const float4 *>(kr.P + c * V + v);
            r2[c] = *reinterpret_cast<const float4 *>(kr.Q + c * V + v);
          }
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            const float4 y = make_float4(pt[c].x - c1 * r1[c].x, pt[c].y - c1 * r1[c].y,
                                         pt[c].z - c1 * r1[c].z, pt[c].w - c1 * r1[c].w);
            *reinterpret_cast<float4 *>(kr.Y + c * V + v) = y;
            a0 += (double)r2[c].x * (double)y.x + (double)r2[c].y * (double)y.y +
                  (double)r2[c].z * (double)y.z + (double)r2[c].w * (double)y.w;
            a1 += (double)y.x * (double)y.x + (double)y.y * (double)y.y +
                  (double)y.z * (double)y.z + (double)y.w * (double)y.w;
            a2 += (double)r2[c].x * (double)r2[c].x + (double)r2[c].y * (double)r2[c].y +
                  (double)r2[c].z * (double)r2[c].z + (double)r2[c].w * (double)r2[c].w;
          }
        }
        finish_inverse<T, EPI_MINRES>(S, a0, a1, a2, local, per, red);
        continue;
      }
    }
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
      T pt[6], r1[6], r2[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        pt[c] = kr.Y[c * V + v];
        r1[c] = kr.P[c * V + v];
        r2[c] = kr.Q[c * V + v];
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const T y = pt[c] - c1 * r1[c];
        kr.Y[c * V + v] = y;
        a0 += (double)r2[c] * (double)y;
        a1 += (double)y * (double)y;
        a2 += (double)r2[c] * (double)r2[c];
      }
    }
    finish_inverse<T, EPI_MINRES>(S, a0, a1, a2, local, per, red);
  }
}

// Upper bound on the default Krylov iteration limit (scipy's is 5 x ndof); the device-side
// loop also stops there whatever limit it was given, so it can never run unbounded.
#define KRYLOV_ITERATION_CAP 20000

// Reaching the cap ends a solve as scipy's iteration limit does (istop 6, the current
// iterate is the answer).
__device__ __forceinline__ void minres_cap(MinresState *st) {
  if (!st->done && st->itn > KRYLOV_ITERATION_CAP) {
    st->istop = 6;
    st->done = 1;
  }
}

// End of one chunk of a handle's device-side Krylov loop (a CUDA-graph while node): run
// another chunk unless the solve is done.
__global__ void minres_continue_kernel(MinresState *st, cudaGraphConditionalHandle cond) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    minres_cap(st);
    cudaGraphSetConditional(cond, st->done ? 0u : 1u);
  }
}

// End of one chunk of a group's Krylov loop: drop the slots whose solve is done from the
// active list (in place, keeping their order) and run another chunk while any is left.
// chunks[0] counts the chunks run.
template <typename T>
__global__ void group_minres_continue_kernel(const SlotDev<T> *__restrict__ tab, int *ids,
                                             int *count, cudaGraphConditionalHandle cond,
                                             unsigned long long *chunks) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *chunks += 1;
    int m = 0;
    const int n = *count;
    for (int k = 0; k < n; ++k) {
      const int s = ids[k];
      minres_cap(tab[s].st);
      if (!tab[s].st->done) ids[m++] = s;
    }
    *count = m;
    cudaGraphSetConditional(cond, m > 0 ? 1u : 0u);
  }
}
