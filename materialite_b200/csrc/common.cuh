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

// ---- bulk copies (the TMA engine, without a tensor map) ------------------------------
// cp.async.bulk moves a contiguous run of 16-byte multiples from global to this block's
// shared memory and signals an mbarrier when the bytes have landed: one instruction per
// run instead of one per element.  The destination is the issuing block's own shared
// memory; nothing here multicasts.  A block owns one barrier for its tile loads and flips
// the parity it waits for after each use.

// Set when a bounded mbarrier wait gives up (the copy never completed); nothing clears it.
// One per translation unit (internal linkage).
static __device__ int g_bulk_wait_timeouts;

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// One thread initialises the barrier (expected arrivals: one, the issuing thread's
// arrive.expect_tx); the block syncs before any use.
__device__ __forceinline__ void bulk_barrier_init(uint64_t *bar) {
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
}

// Wait for the barrier phase with the given parity, at most about 2^22 polls (each poll may
// suspend the thread for a while); on giving up, flag it and go on rather than hang.
__device__ __forceinline__ void bulk_barrier_wait(uint64_t *bar, unsigned parity) {
  for (int i = 0; i < (1 << 22); ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return;
  }
  atomicExch(&g_bulk_wait_timeouts, 1);
}

#define BULK_MIN_BYTES 1024

// Block-cooperative copy of n_outer x n_inner runs of `bytes` bytes each, run (o, i) from
// src + o * s_outer + i * s_inner bytes to dst + o * d_outer + i * d_inner bytes, completing
// on `bar` (the caller then waits on it with its current parity).  Returns false, having
// issued nothing, unless every address, size and step is a multiple of 16 bytes and the runs
// are at least BULK_MIN_BYTES long; the caller then copies another way.  The answer is the
// same in every thread.  Call after a block barrier that ends all reads of the destination.
__device__ __forceinline__ bool bulk_copy_rows(void *dst, const void *src, int n_outer,
                                               int n_inner, unsigned bytes, long long d_outer,
                                               long long d_inner, long long s_outer,
                                               long long s_inner, uint64_t *bar) {
  const int rows = n_outer * n_inner;
  // runs under BULK_MIN_BYTES cost more as bulk copies issued from one warp than as
  // per-element cp.async spread over the block (measured: the x pass's 64-byte runs took
  // twice as long); only long runs go to the bulk engine
  const bool ok = rows > 0 && bytes >= BULK_MIN_BYTES && (bytes & 15u) == 0 &&
                  ((uintptr_t)dst & 15u) == 0 && ((uintptr_t)src & 15u) == 0 &&
                  ((d_outer | d_inner | s_outer | s_inner) & 15) == 0;
  if (!ok) return false;
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) {
      // order this block's earlier generic-proxy accesses of the destination before the
      // asynchronous writes, then announce the bytes to expect
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                   "r"((unsigned)(bytes * (unsigned)rows))
                   : "memory");
    }
    __syncwarp();
    for (int r = threadIdx.x; r < rows; r += 32) {
      const int o = r / n_inner, i = r - o * n_inner;
      const char *s = (const char *)src + o * s_outer + i * s_inner;
      char *d = (char *)dst + o * d_outer + i * d_inner;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
              smem_u32(d)),
          "l"(s), "r"(bytes), "r"(smem_u32(bar))
          : "memory");
    }
  }
  return true;
}

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

// Product rounded on its own on the device as well (no fused multiply-add), so that the
// Newton decisions taken on the device (serving groups) and on the host (handles) agree
// to the last bit.
__host__ __device__ inline double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}

// Mean von Mises stress from summed stress components (small_strain_fft.py:141-143).
__host__ __device__ inline double mean_von_mises(const double *sums, long long V) {
  double m[6];
  for (int c = 0; c < 6; ++c) m[c] = sums[c] / (double)V;
  const double tr3 = (m[0] + m[1] + m[2]) / 3.0;
  double s = 0.0;
  for (int c = 0; c < 6; ++c) {
    const double d = (c < 3) ? m[c] - tr3 : m[c];
    s += mul_rn(d, d);
  }
  return sqrt(s) * sqrt(1.5);
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
