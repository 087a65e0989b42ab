// Batched mixed-radix FFTs of lines held in shared memory (Stockham autosort, DIT
// form of Govindaraju et al., "High performance discrete Fourier transforms on graphics
// processors", SC 2008).  Every stage reads one buffer and writes the other, so a
// transform of length N = r_1 r_2 ... r_m takes m stages and no bit reversal.
//
// Radices 2, 3, 4 and 8 have hand-written butterflies; any other factor (5, 7, ...,
// up to SSFFT_MAX_GENERIC_RADIX) uses a direct DFT with the twiddle table.
#pragma once

#include "common.cuh"

#define SSFFT_MAX_STAGES 16
#define SSFFT_MAX_GENERIC_RADIX 32

// Division by an invariant unsigned integer with one multiply-high, add and shift
// (Granlund & Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994): q = (umulhi(n, m) + n) >> s with s = ceil(log2 d),
// m = floor(2^32 (2^s - d) / d) + 1; exact for n < 2^31.
struct FastDiv {
  uint32_t d, m, s;
};

__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  uint32_t s = 0;
  while ((1ull << s) < d) ++s;
  f.s = s;
  f.m = (uint32_t)(((1ull << 32) * ((1ull << s) - d)) / d + 1);
  return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  return (uint32_t)(((uint64_t)__umulhi(n, f.m) + n) >> f.s);
}

struct AxisPlan {
  int n;                          // transform length
  int nrad;                       // number of stages
  int rad[SSFFT_MAX_STAGES];      // radix of each stage
  FastDiv mdiv[SSFFT_MAX_STAGES]; // divisor n / rad[s]
  FastDiv nsdiv[SSFFT_MAX_STAGES];// divisor Ns = rad[0] * ... * rad[s-1]
};

// Factor n into stages: radix 8 first, then 4, 2, then odd factors (<= 32).
static inline bool make_axis_plan(int n, AxisPlan &p) {
  p.n = n;
  p.nrad = 0;
  int m = n;
  auto push = [&](int r) {
    if (p.nrad >= SSFFT_MAX_STAGES) return false;
    p.rad[p.nrad++] = r;
    m /= r;
    return true;
  };
  while (m % 8 == 0)
    if (!push(8)) return false;
  while (m % 4 == 0)
    if (!push(4)) return false;
  while (m % 2 == 0)
    if (!push(2)) return false;
  for (int f = 3; m > 1; f += 2) {
    while (m % f == 0) {
      if (f > SSFFT_MAX_GENERIC_RADIX) return false;
      if (!push(f)) return false;
    }
  }
  int ns = 1;
  for (int st = 0; st < p.nrad; ++st) {
    p.mdiv[st] = make_fastdiv((uint32_t)(n / p.rad[st]));
    p.nsdiv[st] = make_fastdiv((uint32_t)ns);
    ns *= p.rad[st];
  }
  return true;
}

// Shared-memory index with one pad slot per 16 elements: spreads the stride-r accesses
// of the early Stockham stages of contiguous lines over all banks.
template <bool PAD> __device__ __forceinline__ int sidx(int i) { return PAD ? i + (i >> 4) : i; }
__host__ __device__ inline int padded_len(int n) { return n + (n >> 4) + 1; }

// Line layout in shared memory: line l starts at
//   (l / lsub) * lstride_hi + (l % lsub) * lstride_lo
// and its element j sits at start + j * estride.
// The divisors of nlines and lsub come prepared from the host (a device-side make_fastdiv
// costs a 64-bit division per thread).
struct LineLayout {
  int nlines, lsub, lstride_hi, lstride_lo, estride;
  FastDiv nl_div, lsub_div;
  __device__ LineLayout(int nlines_, int lsub_, int hi, int lo, int es, const FastDiv &nld,
                        const FastDiv &lsd)
      : nlines(nlines_), lsub(lsub_), lstride_hi(hi), lstride_lo(lo), estride(es),
        nl_div(nld), lsub_div(lsd) {}
  __device__ __forceinline__ int start(int l) const {
    if (lsub == nlines) return l * lstride_lo;  // one group (block-uniform branch)
    const int g = (int)fdiv((uint32_t)l, lsub_div);
    return g * lstride_hi + (l - g * lsub) * lstride_lo;
  }
};

template <typename T, bool INV>
__device__ __forceinline__ cplx<T> twiddle(const cplx<T> *tw, int idx) {
  cplx<T> w = tw[idx];
  return INV ? cconj<T>(w) : w;
}

template <typename T, bool INV>
__device__ __forceinline__ void bfly2(cplx<T> *v) {
  cplx<T> a = v[0], b = v[1];
  v[0] = cadd<T>(a, b);
  v[1] = csub<T>(a, b);
}

template <typename T, bool INV>
__device__ __forceinline__ void bfly4(cplx<T> *v) {
  cplx<T> t0 = cadd<T>(v[0], v[2]), t1 = csub<T>(v[0], v[2]);
  cplx<T> t2 = cadd<T>(v[1], v[3]), t3 = mul_mi<T, INV>(csub<T>(v[1], v[3]));
  v[0] = cadd<T>(t0, t2);
  v[2] = csub<T>(t0, t2);
  v[1] = cadd<T>(t1, t3);
  v[3] = csub<T>(t1, t3);
}

template <typename T, bool INV>
__device__ __forceinline__ void bfly8(cplx<T> *v) {
  const T c = (T)INV_SQRT2_D;
  cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
  cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
  bfly4<T, INV>(e);
  bfly4<T, INV>(o);
  // o[k] *= w8^k  (w8 = e^{-i pi/4}, conjugated for the inverse)
  cplx<T> o1 = o[1], o3 = o[3];
  if (!INV) {
    o[1] = mk<T>(c * (o1.x + o1.y), c * (o1.y - o1.x));
    o[3] = mk<T>(c * (o3.y - o3.x), -c * (o3.x + o3.y));
  } else {
    o[1] = mk<T>(c * (o1.x - o1.y), c * (o1.x + o1.y));
    o[3] = mk<T>(-c * (o3.x + o3.y), c * (o3.x - o3.y));
  }
  o[2] = mul_mi<T, INV>(o[2]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd<T>(e[k], o[k]);
    v[k + 4] = csub<T>(e[k], o[k]);
  }
}

template <typename T, bool INV>
__device__ __forceinline__ void bfly3(cplx<T> *v) {
  const T s = (T)0.86602540378443864676;  // sqrt(3)/2
  cplx<T> t = cadd<T>(v[1], v[2]), d = csub<T>(v[1], v[2]);
  cplx<T> m = mk<T>(v[0].x - (T)0.5 * t.x, v[0].y - (T)0.5 * t.y);
  // -i s d for the forward transform, +i s d for the inverse
  cplx<T> r = INV ? mk<T>(-s * d.y, s * d.x) : mk<T>(s * d.y, -s * d.x);
  v[0] = cadd<T>(v[0], t);
  v[1] = cadd<T>(m, r);
  v[2] = csub<T>(m, r);
}

// One Stockham stage of radix R (R = 0: generic radix r).  PAD: shared-memory indices go
// through sidx<true>.
template <typename T, bool INV, bool LINES_FAST, int R, bool PAD>
__device__ __forceinline__ void fft_stage(const cplx<T> *__restrict__ src,
                                          cplx<T> *__restrict__ dst, const LineLayout &L,
                                          int N, int r, int Ns, const FastDiv &mdiv,
                                          const FastDiv &nsdiv, const cplx<T> *tw) {
  const int m = N / r;
  const int total = L.nlines * m;
  const int twstep = N / (Ns * r);
  const int rstep = N / r;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int l, j;
    if (LINES_FAST) {
      j = (int)fdiv((uint32_t)t, L.nl_div);
      l = t - j * L.nlines;
    } else {
      l = (int)fdiv((uint32_t)t, mdiv);
      j = t - l * m;
    }
    const int base = L.start(l);
    const int jn = (int)fdiv((uint32_t)j, nsdiv);
    const int k = j - jn * Ns;
    const int outj = jn * Ns * r + k;
    if (R > 0) {
      cplx<T> v[R > 0 ? R : 1];
#pragma unroll
      for (int q = 0; q < R; ++q) v[q] = src[sidx<PAD>(base + (j + q * m) * L.estride)];
      if (Ns > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul<T>(v[q], twiddle<T, INV>(tw, q * k * twstep));
      }
      if (R == 2) bfly2<T, INV>(v);
      if (R == 3) bfly3<T, INV>(v);
      if (R == 4) bfly4<T, INV>(v);
      if (R == 8) bfly8<T, INV>(v);
#pragma unroll
      for (int q = 0; q < R; ++q) dst[sidx<PAD>(base + (outj + q * Ns) * L.estride)] = v[q];
    } else {
      cplx<T> v[SSFFT_MAX_GENERIC_RADIX];
      for (int q = 0; q < r; ++q) {
        cplx<T> a = src[sidx<PAD>(base + (j + q * m) * L.estride)];
        v[q] = (Ns > 1 && q > 0) ? cmul<T>(a, twiddle<T, INV>(tw, q * k * twstep)) : a;
      }
      for (int p = 0; p < r; ++p) {
        cplx<T> acc = v[0];
        for (int q = 1; q < r; ++q)
          acc = cadd<T>(acc, cmul<T>(v[q], twiddle<T, INV>(tw, ((p * q) % r) * rstep)));
        dst[sidx<PAD>(base + (outj + p * Ns) * L.estride)] = acc;
      }
    }
  }
}

// Transform every line of `L` held in buffer `a` (scratch `b` of the same size).  The
// caller must __syncthreads() before (data ready) and uses the returned buffer after.
// Returns the buffer that holds the result.
template <typename T, bool INV, bool LINES_FAST, bool PAD = false>
__device__ cplx<T> *smem_fft(cplx<T> *a, cplx<T> *b, const LineLayout &L, const AxisPlan &P,
                             const cplx<T> *tw) {
  int Ns = 1;
  for (int s = 0; s < P.nrad; ++s) {
    const int r = P.rad[s];
    const FastDiv &md = P.mdiv[s];
    const FastDiv &nd = P.nsdiv[s];
    switch (r) {
      case 2: fft_stage<T, INV, LINES_FAST, 2, PAD>(a, b, L, P.n, r, Ns, md, nd, tw); break;
      case 3: fft_stage<T, INV, LINES_FAST, 3, PAD>(a, b, L, P.n, r, Ns, md, nd, tw); break;
      case 4: fft_stage<T, INV, LINES_FAST, 4, PAD>(a, b, L, P.n, r, Ns, md, nd, tw); break;
      case 8: fft_stage<T, INV, LINES_FAST, 8, PAD>(a, b, L, P.n, r, Ns, md, nd, tw); break;
      default: fft_stage<T, INV, LINES_FAST, 0, PAD>(a, b, L, P.n, r, Ns, md, nd, tw); break;
    }
    __syncthreads();
    cplx<T> *t = a;
    a = b;
    b = t;
    Ns *= r;
  }
  return a;
}
