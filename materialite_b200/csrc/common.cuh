// Shared device helpers for libssfft: complex arithmetic, Mandel helpers, block
// reductions and the deterministic "last block finishes" reduction pattern.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#define SSFFT_THREADS 256
#define SQRT2_D 1.41421356237309504880
#define INV_SQRT2_D 0.70710678118654752440

template <typename T> struct cvec;
template <> struct cvec<float> { using type = float2; };
template <> struct cvec<double> { using type = double2; };
template <typename T> using cplx = typename cvec<T>::type;

template <typename T> __device__ __forceinline__ cplx<T> mk(T x, T y) {
  cplx<T> r;
  r.x = x;
  r.y = y;
  return r;
}
template <typename T> __device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T> __device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x - b.x, a.y - b.y);
}
template <typename T> __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cplx<T> cconj(cplx<T> a) {
  return mk<T>(a.x, -a.y);
}
template <typename T> __device__ __forceinline__ cplx<T> cscale(cplx<T> a, T s) {
  return mk<T>(a.x * s, a.y * s);
}
// multiply by -i (forward) or +i (inverse)
template <typename T, bool INV> __device__ __forceinline__ cplx<T> mul_mi(cplx<T> a) {
  return INV ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

// ---- asynchronous global-to-shared copies -------------------------------------------
// cp.async moves an element from global to shared memory without a register round trip, so
// a thread can have all of a tile's loads in flight at once (a load-then-store loop waits a
// full memory latency per element).  The caller waits with cp_async_wait_all() and then
// syncs the block.
template <typename T> __device__ __forceinline__ void cp_async_elem(cplx<T> *dst, const cplx<T> *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(cplx<T>) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
template <typename T> __device__ __forceinline__ void cp_async_scalar(T *dst, const T *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---- block reductions (double) ------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum over the block; result valid in thread 0.  `scratch` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
  if (wid == 0) v = warp_sum(v);
  return v;
}
__device__ __forceinline__ double block_max(double v, double *scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
  if (wid == 0) v = warp_max(v);
  return v;
}

// Deterministic grid reduction: every block writes its partials (nvals doubles) to
// partials[block * nvals + k]; the block that arrives last (ticket) sees all of them.
// Returns true in the last block (all threads), after which the caller sums the
// partials in block order.  The ticket counter is reset by the last block.
__device__ __forceinline__ bool last_block_arrives(unsigned int *ticket) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == gridDim.x * gridDim.y * gridDim.z - 1);
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// Sum `count` partials strided by `stride` starting at `base`, in a fixed order
// (thread-strided then tree), result in thread 0.
__device__ __forceinline__ double ordered_sum(const double *p, int count, int stride,
                                              double *scratch) {
  double v = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) v += p[(size_t)i * stride];
  return block_sum(v, scratch);
}
__device__ __forceinline__ double ordered_max(const double *p, int count, int stride,
                                              double *scratch) {
  double v = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) v = fmax(v, p[(size_t)i * stride]);
  return block_max(v, scratch);
}

// Symmetric 6x6 packed as 21 entries, upper triangle row by row:
// (0,0)(0,1)..(0,5)(1,1)..(1,5)(2,2)..(5,5)
__host__ __device__ __forceinline__ int sym_idx(int i, int j) {
  if (i > j) {
    int t = i;
    i = j;
    j = t;
  }
  return i * 6 - (i * (i - 1)) / 2 + (j - i);
}
