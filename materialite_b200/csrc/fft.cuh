// Batched mixed-radix FFTs of lines held in shared memory (Stockham autosort, DIT
// form of Govindaraju et al., "High performance discrete Fourier transforms on graphics
// processors", SC 2008).  Every stage reads one buffer and writes the other, so a
// transform of length N = r_1 r_2 ... r_m takes m stages and no bit reversal.
//
// Radices 2, 3, 4, 8, 12 and 16 have hand-written butterflies (12 and 16 composed in
// registers from radix-3/4 butterflies and constant twiddles); any other factor (5, 7, ...,
// up to SSFFT_MAX_GENERIC_RADIX) uses a direct DFT with the twiddle table.  A plan uses the
// fewest stages its radices allow (every stage is a pass through shared memory), widest
// radix first (the first stage needs no twiddles): 128 = 16 x 8, 96 = 12 x 8, 48 = 16 x 3.
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

// Factor n into stages with the fewest passes: radices up to `maxrad` among 16, 12, 8, 4,
// 3, 2 (hand-written butterflies) and odd primes up to SSFFT_MAX_GENERIC_RADIX (direct
// DFT).  Among plans of equal length: fewer generic stages, then the widest radix first.
static inline void plan_search(int m, int maxrad, int *cur, int depth, int *best, int *best_len,
                               int *best_gen) {
  if (depth > SSFFT_MAX_STAGES) return;
  if (m == 1) {
    int gen = 0;  // stages without a hand-written butterfly
    for (int i = 0; i < depth; ++i) {
      const int r = cur[i];
      gen += (r == 2 || r == 3 || r == 4 || r == 8 || r == 12 || r == 16) ? 0 : 1;
    }
    // sort descending (widest radix first)
    int tmp[SSFFT_MAX_STAGES];
    for (int i = 0; i < depth; ++i) tmp[i] = cur[i];
    for (int i = 0; i < depth; ++i)
      for (int j = i + 1; j < depth; ++j)
        if (tmp[j] > tmp[i]) {
          const int t = tmp[i];
          tmp[i] = tmp[j];
          tmp[j] = t;
        }
    bool better = *best_len < 0 || depth < *best_len || (depth == *best_len && gen < *best_gen);
    if (!better && depth == *best_len && gen == *best_gen) {
      for (int i = 0; i < depth; ++i) {
        if (tmp[i] != best[i]) {
          better = tmp[i] > best[i];
          break;
        }
      }
    }
    if (better) {
      for (int i = 0; i < depth; ++i) best[i] = tmp[i];
      *best_len = depth;
      *best_gen = gen;
    }
    return;
  }
  if (*best_len >= 0 && depth + 1 > *best_len) return;
  static const int hand[6] = {16, 12, 8, 4, 3, 2};
  for (int i = 0; i < 6; ++i) {
    const int r = hand[i];
    if (r > maxrad || m % r) continue;
    cur[depth] = r;
    plan_search(m / r, maxrad, cur, depth + 1, best, best_len, best_gen);
  }
  for (int f = 5; f <= SSFFT_MAX_GENERIC_RADIX; f += 2) {
    bool prime = true;
    for (int d = 3; d * d <= f; d += 2)
      if (f % d == 0) prime = false;
    if (!prime || m % f) continue;
    cur[depth] = f;
    plan_search(m / f, maxrad, cur, depth + 1, best, best_len, best_gen);
  }
}

static inline bool make_axis_plan(int n, AxisPlan &p, int maxrad = 8) {
  p.n = n;
  p.nrad = 0;
  int cur[SSFFT_MAX_STAGES + 1], best[SSFFT_MAX_STAGES + 1], best_len = -1, best_gen = 0;
  if (n < 1) return false;
  if (n > 1) {
    plan_search(n, maxrad, cur, 0, best, &best_len, &best_gen);
    if (best_len < 0) return false;
    for (int i = 0; i < best_len; ++i) p.rad[p.nrad++] = best[i];
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

// Radix 16 as 4 x 4 in registers: DFT4 over n1 of x[4 n1 + n2] for each n2, twiddles
// W16^(n2 k1), DFT4 over n2 for each k1 (output k1 + 4 k2).
template <typename T, bool INV>
__device__ __forceinline__ void bfly16(cplx<T> *v) {
  const T c1 = (T)0.92387953251128675613;  // cos(pi/8)
  const T s1 = (T)0.38268343236508977173;  // sin(pi/8)
  const T h = (T)INV_SQRT2_D;
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    cplx<T> t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
    bfly4<T, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) v[4 * k1 + n2] = t[k1];  // A[n2][k1] at 4 k1 + n2
  }
  // W16^m = cos(pi m / 8) - i sin(pi m / 8) (conjugate for the inverse)
  const T sg = INV ? (T)-1 : (T)1;
  const cplx<T> w1 = mk<T>(c1, -sg * s1), w2 = mk<T>(h, -sg * h), w3 = mk<T>(s1, -sg * c1);
  const cplx<T> w6 = mk<T>(-h, -sg * h), w9 = mk<T>(-c1, sg * s1);
  v[4 * 1 + 1] = cmul<T>(v[4 * 1 + 1], w1);
  v[4 * 2 + 1] = cmul<T>(v[4 * 2 + 1], w2);
  v[4 * 3 + 1] = cmul<T>(v[4 * 3 + 1], w3);
  v[4 * 1 + 2] = cmul<T>(v[4 * 1 + 2], w2);
  v[4 * 2 + 2] = mul_mi<T, INV>(v[4 * 2 + 2]);  // W16^4 = -i
  v[4 * 3 + 2] = cmul<T>(v[4 * 3 + 2], w6);
  v[4 * 1 + 3] = cmul<T>(v[4 * 1 + 3], w3);
  v[4 * 2 + 3] = cmul<T>(v[4 * 2 + 3], w6);
  v[4 * 3 + 3] = cmul<T>(v[4 * 3 + 3], w9);
  cplx<T> o[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    cplx<T> t[4] = {v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]};
    bfly4<T, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) o[k1 + 4 * k2] = t[k2];
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = o[q];
}

// Radix 12 as 3 x 4 in registers: DFT3 over n1 of x[4 n1 + n2] for each n2, twiddles
// W12^(n2 k1), DFT4 over n2 for each k1 (output k1 + 3 k2).
template <typename T, bool INV>
__device__ __forceinline__ void bfly12(cplx<T> *v) {
  const T r3 = (T)0.86602540378443864676;  // sqrt(3)/2
  cplx<T> a[12];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    cplx<T> t[3] = {v[n2], v[4 + n2], v[8 + n2]};
    bfly3<T, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) a[4 * k1 + n2] = t[k1];  // A[n2][k1] at 4 k1 + n2
  }
  // W12^m = cos(pi m / 6) - i sin(pi m / 6) (conjugate for the inverse)
  const T sg = INV ? (T)-1 : (T)1;
  const cplx<T> w1 = mk<T>(r3, -sg * (T)0.5), w2 = mk<T>((T)0.5, -sg * r3);
  const cplx<T> w4 = mk<T>((T)-0.5, -sg * r3);
  a[4 * 1 + 1] = cmul<T>(a[4 * 1 + 1], w1);
  a[4 * 2 + 1] = cmul<T>(a[4 * 2 + 1], w2);
  a[4 * 1 + 2] = cmul<T>(a[4 * 1 + 2], w2);
  a[4 * 2 + 2] = cmul<T>(a[4 * 2 + 2], w4);
  a[4 * 1 + 3] = mul_mi<T, INV>(a[4 * 1 + 3]);  // W12^3 = -i
  a[4 * 2 + 3] = mk<T>(-a[4 * 2 + 3].x, -a[4 * 2 + 3].y);  // W12^6 = -1
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    cplx<T> t[4] = {a[4 * k1], a[4 * k1 + 1], a[4 * k1 + 2], a[4 * k1 + 3]};
    bfly4<T, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 3 * k2] = t[k2];
  }
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
      if (R == 12) bfly12<T, INV>(v);
      if (R == 16) bfly16<T, INV>(v);
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
      case 12:  // float plans only: a double radix-12/16 butterfly does not fit 64 registers
        if constexpr (sizeof(T) == 4) fft_stage<T, INV, LINES_FAST, 12, PAD>(a, b, L, P.n, r, Ns, md, nd, tw);
        break;
      case 16:
        if constexpr (sizeof(T) == 4) fft_stage<T, INV, LINES_FAST, 16, PAD>(a, b, L, P.n, r, Ns, md, nd, tw);
        break;
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
