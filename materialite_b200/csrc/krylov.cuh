// Device MINRES (Paige & Saunders 1975) for the Newton correction of
// small_strain_fft.py:281-299, which the reference delegates to scipy's minres with
// x0 = 0, no preconditioner and its default stopping tests.
//
// All scalars live in a MinresState in device memory and are advanced by the last
// block of each reduction kernel, so an iteration needs no host round trip:
//
//   zfwd(PRO_TANGENT_*)  v = s r2, tau = K v           (projector.cuh)
//   ... y/x passes ...
//   zinv(EPI_MINRES)     y = P tau - c_r1 r1 -> r1 buf, alfa = v . y
//   upd1                 y -= (alfa/beta) r2, beta' = |y|, plane rotation
//   upd2                 w = (v - oldeps w1 - delta w2)/gamma, x += phi w, tests
//
// Vectors are component-planar in the solve precision T; every dot product and norm
// accumulates in double, in a fixed order (block partials summed by the last block).
#pragma once

#include "common.cuh"
#include "projector.cuh"

// Partial sums over a grid-stride range of the 6V components.
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
    s.rtol = rtol;
    s.eps = 2.220446049250313e-16;
    s.itn = 0;
    s.maxiter = maxiter;
    s.istop = 0;
    s.done = (b2 == 0.0) ? 1 : 0;  // beta1 == 0: x = 0 is exact
    *st = s;
  }
}

// y -= (alfa/beta) r2 ; beta_new = |y| ; rotation update.
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    minres_upd1_kernel(T *__restrict__ y, const T *__restrict__ r2, long long n, MinresState *st,
                       double *partials, unsigned int *ticket) {
  if (st->done) return;
  __shared__ double red[32];
  const T coef = (T)(st->alfa / st->beta);
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const T yi = y[i] - coef * r2[i];
    y[i] = yi;
    acc += (double)yi * (double)yi;
  }
  const double part = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
  if (!last_block_arrives(ticket)) return;
  const double beta2 = ordered_sum(partials, gridDim.x, 1, red);
  if (threadIdx.x == 0) {
    *ticket = 0;
    MinresState s = *st;
    s.oldb = s.beta;
    s.beta = sqrt(beta2);
    s.tnorm2 += s.alfa * s.alfa + s.oldb * s.oldb + s.beta * s.beta;
    if (s.itn == 1 && s.beta / s.beta1 <= 10.0 * s.eps) s.istop = -1;
    s.oldeps = s.epsln;
    s.delta = s.cs * s.dbar + s.sn * s.alfa;
    const double gbar = s.sn * s.dbar - s.cs * s.alfa;
    s.epsln = s.sn * s.beta;
    s.dbar = -s.cs * s.beta;
    s.root = hypot(gbar, s.dbar);
    s.gamma = fmax(hypot(gbar, s.beta), s.eps);
    s.cs = gbar / s.gamma;
    s.sn = s.beta / s.gamma;
    s.phi = s.cs * s.phibar;
    s.phibar = s.sn * s.phibar;
    s.denom = 1.0 / s.gamma;
    s.gmax = fmax(s.gmax, s.gamma);
    s.gmin = fmin(s.gmin, s.gamma);
    s.s_prev = s.s;
    s.s = (s.beta > 0.0) ? 1.0 / s.beta : 0.0;
    s.c_r1 = (s.oldb > 0.0) ? s.beta / s.oldb : 0.0;
    *st = s;
  }
}

// w_new = (v - oldeps w1 - delta w2) / gamma  with v = s_prev * vprev ;  x += phi w_new ;
// then the stopping tests.  w1 / w2 / w are the rotated search directions:
// w_new is written into `wout` (the buffer of the discarded oldest direction).
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    minres_upd2_kernel(const T *__restrict__ vprev, const T *__restrict__ w1,
                       const T *__restrict__ w2, T *__restrict__ wout, T *__restrict__ x,
                       long long n, MinresState *st, double *partials, unsigned int *ticket) {
  if (st->done) return;
  __shared__ double red[32];
  const T sv = (T)st->s_prev, oe = (T)st->oldeps, de = (T)st->delta, dn = (T)st->denom;
  const T ph = (T)st->phi;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const T wn = (sv * vprev[i] - oe * w1[i] - de * w2[i]) * dn;
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
}
