// Device MINRES (Paige & Saunders 1975) for the Newton correction of
// small_strain_fft.py:281-299, which the reference delegates to scipy's minres with
// x0 = 0, no preconditioner and its default stopping tests.
//
// All scalars live in a MinresState in device memory and are advanced by the last
// block of each reduction kernel, so an iteration needs no host round trip:
//
//   zfwd(PRO_TANGENT_*)  v = s r2, tau = K v                          (projector.cuh)
//   ... y/x passes ...
//   zinv(EPI_MINRES)     y' = P tau - c_r1 r1 -> r1 buffer; r2.y', y'.y', r2.r2;
//                        last block: alfa, beta', plane rotation   (minres_after_matvec)
//   update               y'' = y' - (alfa/beta) r2 -> r1 buffer (the next r2),
//                        w = (v - oldeps w1 - delta w2)/gamma, x += phi w;
//                        last block: |x| and the stopping tests    (minres_after_update)
//
// Vectors are component-planar in the solve precision T, handled as one contiguous run of
// 6V values; every dot product and norm accumulates in double, in a fixed order (block
// partials summed by the last block), so results do not depend on scheduling.
#pragma once

#include "common.cuh"
#include "projector.cuh"

// VW consecutive values moved as one vector access (16 bytes for float4 / double2).
template <typename T, int VW> struct alignas(sizeof(T) * VW) Pack {
  T v[VW];
};

template <typename T> constexpr int vec_width() { return 16 / (int)sizeof(T); }

// r1 = r2 = b, x = w = w2 = 0, |b|^2; the last block initialises the MINRES state.
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    minres_init_kernel(const T *__restrict__ b, T *__restrict__ r1, T *__restrict__ r2,
                       T *__restrict__ x, T *__restrict__ w, T *__restrict__ w2, long long n,
                       MinresState *st, double rtol, long long maxiter, double *partials,
                       unsigned int *ticket) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const T bi = b[i];
    r1[i] = bi;
    r2[i] = bi;
    x[i] = 0;
    w[i] = 0;
    w2[i] = 0;
    acc += (double)bi * (double)bi;
  }
  const double part = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
  if (!last_block_arrives(ticket)) return;
  const double b2 = ordered_sum(partials, gridDim.x, 1, red);
  if (threadIdx.x == 0) {
    *ticket = 0;
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
    s.rtol = rtol;
    s.eps = 2.220446049250313e-16;
    s.itn = 0;
    s.maxiter = maxiter;
    s.istop = 0;
    s.done = (b2 == 0.0) ? 1 : 0;  // beta1 == 0: x = 0 is exact
    *st = s;
  }
}

// Stopping tests of scipy's minres after the solution update.
static __device__ __noinline__ void minres_after_update(MinresState *st, double x2) {
  MinresState s = *st;
  s.anorm = sqrt(s.tnorm2);
  s.ynorm = sqrt(x2);
  const double epsx = s.anorm * s.ynorm * s.eps;
  s.rnorm = s.phibar;
  s.test1 = (s.ynorm == 0.0 || s.anorm == 0.0) ? INFINITY : s.rnorm / (s.anorm * s.ynorm);
  s.test2 = (s.anorm == 0.0) ? INFINITY : s.root / s.anorm;
  const double acond = s.gmax / s.gmin;
  if (s.istop == 0) {
    if (1.0 + s.test2 <= 1.0) s.istop = 2;
    if (1.0 + s.test1 <= 1.0) s.istop = 1;
    if (s.itn >= s.maxiter) s.istop = 6;
    if (acond >= 0.1 / s.eps) s.istop = 4;
    if (epsx >= s.beta1) s.istop = 3;
    if (s.test2 <= s.rtol) s.istop = 2;
    if (s.test1 <= s.rtol) s.istop = 1;
  }
  if (!isfinite(s.ynorm) || !isfinite(s.beta)) s.istop = 9;  // NaN guard
  if (s.beta == 0.0 && s.istop == 0) s.istop = 1;           // exact breakdown
  if (s.istop != 0) s.done = 1;
  *st = s;
}

// y'' = y' - coef r2 (in place in y), w = (s_prev r2 - oldeps w1 - delta w2) denom into
// wout, x += phi w, partial |x|^2.  w1 / w2 are the rotated directions (the buffers of
// the previous w2 and w), wout the buffer of the discarded oldest one.
template <typename T, int VW>
__global__ void __launch_bounds__(SSFFT_THREADS)
    minres_update_kernel(T *__restrict__ y, const T *__restrict__ r2, const T *__restrict__ w1,
                         const T *__restrict__ w2, T *__restrict__ wout, T *__restrict__ x,
                         long long n, MinresState *st, double *partials, unsigned int *ticket) {
  if (st->done) return;
  __shared__ double red[32];
  const T coef = (T)st->coef, sv = (T)st->s_prev, oe = (T)st->oldeps, de = (T)st->delta;
  const T dn = (T)st->denom, ph = (T)st->phi;
  double acc = 0.0;
  using P = Pack<T, VW>;
  const long long nv = n / VW;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    P yy = reinterpret_cast<const P *>(y)[i];
    const P rr = reinterpret_cast<const P *>(r2)[i];
    const P a1 = reinterpret_cast<const P *>(w1)[i];
    const P a2 = reinterpret_cast<const P *>(w2)[i];
    P xx = reinterpret_cast<const P *>(x)[i];
    P ww;
#pragma unroll
    for (int k = 0; k < VW; ++k) {
      yy.v[k] = yy.v[k] - coef * rr.v[k];
      ww.v[k] = (sv * rr.v[k] - oe * a1.v[k] - de * a2.v[k]) * dn;
      xx.v[k] = xx.v[k] + ph * ww.v[k];
      acc += (double)xx.v[k] * (double)xx.v[k];
    }
    reinterpret_cast<P *>(y)[i] = yy;
    reinterpret_cast<P *>(wout)[i] = ww;
    reinterpret_cast<P *>(x)[i] = xx;
  }
  // tail (n not a multiple of VW)
  for (long long i = nv * VW + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    y[i] = y[i] - coef * r2[i];
    const T wn = (sv * r2[i] - oe * w1[i] - de * w2[i]) * dn;
    wout[i] = wn;
    const T xi = x[i] + ph * wn;
    x[i] = xi;
    acc += (double)xi * (double)xi;
  }
  const double part = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
  if (!last_block_arrives(ticket)) return;
  const double x2 = ordered_sum(partials, gridDim.x, 1, red);
  if (threadIdx.x == 0) {
    *ticket = 0;
    minres_after_update(st, x2);
  }
}
