// Device MINRES (Paige & Saunders 1975) for the Newton correction of
// small_strain_fft.py:281-299, which the reference delegates to scipy's minres with
// x0 = 0, no preconditioner and its default stopping tests.
//
// All scalars live in a MinresState in device memory and are advanced by the last
// block of each reduction kernel, so an iteration needs no host round trip.  With u_j the
// Lanczos vector of iteration j (v_j = u_j / beta_j), one iteration is three (plane-fused)
// or five kernels:
//
//   forward z(y)  pending update of iteration j-1: u_j = y' - (alfa/beta) u_{j-1},
//                 w = (v_{j-1} - oldeps w1 - delta w2) / gamma, x += phi w;
//                 last block: |x| and the stopping tests          (minres_after_update)
//                 then tau = K (u_j / beta_j) and its forward transform
//   ... y/x passes ...
//   inverse z     y' = P tau - (beta_j / beta_{j-1}) u_{j-1}; u_j.y', y'.y', u_j.u_j;
//                 last block: alfa, beta_{j+1}, plane rotation    (minres_after_matvec)
//
// The update needs alfa, a global dot product of the matvec, so it cannot join the
// inverse pass; it rides on the next forward pass, which reads the same vectors anyway.
// The last iteration's update is applied by one more forward pass, which then finds the
// solve done.  Vectors are component-planar in the solve precision T, handled as one
// contiguous run of 6V values; every dot product and norm accumulates in double, in a
// fixed order (block partials summed by the last block), so results do not depend on
// scheduling.
#pragma once

#include "common.cuh"
#include "projector.cuh"

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

// Upper bound on the default Krylov iteration limit (scipy's is 5 x ndof); the device-side
// loop also stops there whatever limit it was given, so it can never run unbounded.
#define KRYLOV_ITERATION_CAP 20000

// End of one chunk of the device-side Krylov loop (a CUDA-graph while node): run another
// chunk unless the solve is done.  Reaching the cap ends the solve as scipy's iteration
// limit does (istop 6, the current iterate is the answer).
__global__ void minres_continue_kernel(MinresState *st, cudaGraphConditionalHandle cond) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (!st->done && st->itn > KRYLOV_ITERATION_CAP) {
      st->istop = 6;
      st->done = 1;
    }
    cudaGraphSetConditional(cond, st->done ? 0u : 1u);
  }
}
