// The compatibility projection  out = ifftn( Gamma-hat(q) : fftn(tau) ).real  of
// materialite's SmallStrainFFT (small_strain_fft.py:301-382), as five passes over a
// half spectrum held in HBM:
//
//   zfwd : per (x,y) line, build tau (prologue), real-to-complex FFT along z
//   yfwd : complex FFT along y
//   xpass: complex FFT along x, Gamma-hat apply on all six components, inverse along x
//   yinv : inverse complex FFT along y
//   zinv : complex-to-real inverse along z, then the epilogue
//
// The six real components are paired into three complex lines for the z passes
// ((0,1), (2,3), (4,5)), so the z transforms run at half length-cost.  Gamma-hat is
// never stored: with t = normalize(tan(pi f_x), tan(pi f_y), tan(pi f_z)) the reference
// operator (rotated frequencies normalised, A = delta q conj q, B = q q conj q conj q)
// reduces exactly to  Gamma-hat : T = t (x) u + u (x) t - (t . u) t (x) t,  u = T t.
// Nyquist planes of even sizes are zero (small_strain_fft.py:354-359) and
// Gamma-hat(0) = diag(stress_mask) (:363-367).
#pragma once

#include "common.cuh"
#include "fft.cuh"

// Spectrum layout: spec[c * S + (x * ny + y) * hz + kz], c = Mandel component,
// hz = nz/2 + 1, S = nx * ny * hz.  Real fields: f[c * V + (x * ny + y) * nz + z].
template <typename T> struct Grid {
  int nx, ny, nz, hz;
  long long V, S;
  AxisPlan px, py, pz;
  const cplx<T> *twx, *twy, *twz;  // e^{-2 pi i k / n}, k < n
  const T *tanx, *tany, *tanz;     // tan(pi f_k) with f = fftfreq (nx, ny, hz entries)
  T scale;                         // 1 / V
  T mask[6];                       // stress mask (0/1)
  int lz;                          // (x,y) lines per z-pass block
  int ky;                          // kz columns per y-pass block
  int kx;                          // kz columns per x-pass block
};

// Device-resident state of one MINRES solve (doubles; see krylov.cuh).
struct MinresState {
  double beta1, beta, oldb, alfa, dbar, epsln, phibar, tnorm2, gmax, gmin, cs, sn;
  double delta, oldeps, gamma, phi, denom, root, anorm, ynorm, rnorm, test1, test2;
  double s, s_prev, c_r1;
  double rtol, eps;
  long long itn, maxiter;
  int istop, done;
};

// ---- prologue modes of zfwd ----------------------------------------------------------
enum { PRO_INPUT = 0, PRO_RESIDUAL = 1, PRO_TANGENT_TABLE = 2, PRO_TANGENT_VOXEL = 3 };

template <typename T> struct ProArgs {
  const T *in;           // PRO_INPUT: tau planes; PRO_RESIDUAL: stress; TANGENT: Krylov v
  const int32_t *gid;    // TANGENT_TABLE: tangent index per point
  const T *ktab;         // TANGENT_TABLE: [n_gid][21]
  const T *kvox;         // TANGENT_VOXEL: 21 planes of V
  const MinresState *st; // TANGENT_*: scale 1/beta, early exit when done
  double sbar[6];        // PRO_RESIDUAL: applied mean stress
};

template <typename T>
__device__ __forceinline__ void sym6_apply(const T *k, long long kstride, const T *x,
                                           T *y) {
  // y = K x for K symmetric packed as 21 entries (k[i * kstride])
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    T acc = 0;
#pragma unroll
    for (int j = 0; j < 6; ++j) acc += k[sym_idx(i, j) * kstride] * x[j];
    y[i] = acc;
  }
}

template <typename T, typename TF, int PRO>
__device__ __forceinline__ void prologue(const Grid<T> &g, const ProArgs<TF> &a, long long v,
                                         T s, T *tau) {
  if constexpr (PRO == PRO_INPUT) {
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = (T)a.in[c * g.V + v];
  } else if constexpr (PRO == PRO_RESIDUAL) {
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = (T)a.sbar[c] - (T)a.in[c * g.V + v];
  } else {
    T x[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) x[c] = s * a.in[c * g.V + v];
    if constexpr (PRO == PRO_TANGENT_TABLE) {
      sym6_apply<T>(a.ktab + (long long)a.gid[v] * 21, 1, x, tau);
    } else {
      sym6_apply<T>(a.kvox + v, g.V, x, tau);
    }
  }
}

template <typename T>
__device__ __forceinline__ void load_table(cplx<T> *dst, const cplx<T> *src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// zfwd: blockIdx.x covers g.lz consecutive (x,y) lines.  TF is the storage type of the
// input fields (TF = T except when a double-precision transform reads float fields).
template <typename T, typename TF, int PRO>
__global__ void __launch_bounds__(SSFFT_THREADS)
    zfwd_kernel(Grid<T> g, ProArgs<TF> a, cplx<T> *__restrict__ spec) {
  if (PRO >= PRO_TANGENT_TABLE && a.st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nz = g.nz, hz = g.hz;
  const long long nlines_all = (long long)g.nx * g.ny;
  const long long line0 = (long long)blockIdx.x * g.lz;
  const int nl = (int)min((long long)g.lz, nlines_all - line0);
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + 3 * g.lz * nz;
  cplx<T> *tw = bufB + 3 * g.lz * nz;
  load_table<T>(tw, g.twz, nz);
  const T s = (PRO >= PRO_TANGENT_TABLE) ? (T)a.st->s : (T)1;
  for (int e = threadIdx.x; e < nl * nz; e += blockDim.x) {
    const int l = e / nz, z = e - (e / nz) * nz;
    const long long v = (line0 + l) * nz + z;
    T tau[6];
    prologue<T, TF, PRO>(g, a, v, s, tau);
#pragma unroll
    for (int p = 0; p < 3; ++p) bufA[(p * nl + l) * nz + z] = mk<T>(tau[2 * p], tau[2 * p + 1]);
  }
  __syncthreads();
  LineLayout L{3 * nl, 3 * nl, 0, nz, 1};
  cplx<T> *res = smem_fft<T, false, false>(bufA, bufB, L, g.pz, tw);
  // split the paired transform: A = (Z_k + conj Z_{-k}) / 2, B = (Z_k - conj Z_{-k}) / 2i
  for (int e = threadIdx.x; e < 3 * nl * hz; e += blockDim.x) {
    const int p = e / (nl * hz);
    const int rem = e - p * nl * hz;
    const int l = rem / hz, k = rem - (rem / hz) * hz;
    const cplx<T> Z = res[(p * nl + l) * nz + k];
    const int km = (k == 0) ? 0 : nz - k;
    const cplx<T> Zm = res[(p * nl + l) * nz + km];
    const cplx<T> A = mk<T>((T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y));
    const cplx<T> B = mk<T>((T)0.5 * (Z.y + Zm.y), (T)0.5 * (Zm.x - Z.x));
    const long long off = (line0 + l) * hz + k;
    spec[(2 * p) * g.S + off] = A;
    spec[(2 * p + 1) * g.S + off] = B;
  }
}

// y passes: grid (ceil(hz/ky), nx, 6); lines are kz columns of one (c, x) slab.
template <typename T, bool INV>
__global__ void __launch_bounds__(SSFFT_THREADS)
    ypass_kernel(Grid<T> g, cplx<T> *__restrict__ spec, const MinresState *st) {
  if (st && st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ny = g.ny, hz = g.hz;
  const int k0 = blockIdx.x * g.ky;
  const int nk = min(g.ky, hz - k0);
  const int x = blockIdx.y, c = blockIdx.z;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + g.ky * ny;
  cplx<T> *tw = bufB + g.ky * ny;
  load_table<T>(tw, g.twy, ny);
  cplx<T> *base = spec + c * g.S + (long long)x * ny * hz + k0;
  for (int e = threadIdx.x; e < ny * nk; e += blockDim.x) {
    const int y = e / nk, kk = e - (e / nk) * nk;
    bufA[y * nk + kk] = base[(long long)y * hz + kk];
  }
  __syncthreads();
  LineLayout L{nk, nk, 0, 1, nk};
  cplx<T> *res = smem_fft<T, INV, true>(bufA, bufB, L, g.py, tw);
  for (int e = threadIdx.x; e < ny * nk; e += blockDim.x) {
    const int y = e / nk, kk = e - (e / nk) * nk;
    base[(long long)y * hz + kk] = res[y * nk + kk];
  }
}

// Gamma-hat : tau-hat at one frequency, in place on the six complex components.
template <typename T>
__device__ __forceinline__ void green_apply(const Grid<T> &g, int kx, int ky, int kz,
                                            cplx<T> *m) {
  const bool nyq = ((g.nx % 2 == 0) && kx == g.nx / 2) || ((g.ny % 2 == 0) && ky == g.ny / 2) ||
                   ((g.nz % 2 == 0) && kz == g.nz / 2);
  if (kx == 0 && ky == 0 && kz == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = cscale<T>(m[c], g.mask[c] * g.scale);
    return;
  }
  if (nyq) {
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = mk<T>((T)0, (T)0);
    return;
  }
  T t0 = g.tanx[kx], t1 = g.tany[ky], t2 = g.tanz[kz];
  const T inv = (T)1 / sqrt(t0 * t0 + t1 * t1 + t2 * t2);
  t0 *= inv;
  t1 *= inv;
  t2 *= inv;
  const T h = (T)INV_SQRT2_D, r2 = (T)SQRT2_D;
  // Cartesian T from Mandel: T00=m0 T11=m1 T22=m2 T12=m3/r2 T02=m4/r2 T01=m5/r2
  // u = T t (real and imaginary parts together)
  cplx<T> u0 = mk<T>(m[0].x * t0 + h * (m[5].x * t1 + m[4].x * t2),
                     m[0].y * t0 + h * (m[5].y * t1 + m[4].y * t2));
  cplx<T> u1 = mk<T>(m[1].x * t1 + h * (m[5].x * t0 + m[3].x * t2),
                     m[1].y * t1 + h * (m[5].y * t0 + m[3].y * t2));
  cplx<T> u2 = mk<T>(m[2].x * t2 + h * (m[4].x * t0 + m[3].x * t1),
                     m[2].y * t2 + h * (m[4].y * t0 + m[3].y * t1));
  cplx<T> tu = mk<T>(t0 * u0.x + t1 * u1.x + t2 * u2.x, t0 * u0.y + t1 * u1.y + t2 * u2.y);
  const T sc = g.scale;
  // O_ij = t_i u_j + u_i t_j - tu t_i t_j ; Mandel shears carry sqrt(2)
  m[0] = mk<T>(sc * (2 * t0 * u0.x - tu.x * t0 * t0), sc * (2 * t0 * u0.y - tu.y * t0 * t0));
  m[1] = mk<T>(sc * (2 * t1 * u1.x - tu.x * t1 * t1), sc * (2 * t1 * u1.y - tu.y * t1 * t1));
  m[2] = mk<T>(sc * (2 * t2 * u2.x - tu.x * t2 * t2), sc * (2 * t2 * u2.y - tu.y * t2 * t2));
  m[3] = mk<T>(sc * r2 * (t1 * u2.x + u1.x * t2 - tu.x * t1 * t2),
               sc * r2 * (t1 * u2.y + u1.y * t2 - tu.y * t1 * t2));
  m[4] = mk<T>(sc * r2 * (t0 * u2.x + u0.x * t2 - tu.x * t0 * t2),
               sc * r2 * (t0 * u2.y + u0.y * t2 - tu.y * t0 * t2));
  m[5] = mk<T>(sc * r2 * (t0 * u1.x + u0.x * t1 - tu.x * t0 * t1),
               sc * r2 * (t0 * u1.y + u0.y * t1 - tu.y * t0 * t1));
}

// x pass: grid (ceil(hz/kx), ny); forward x-FFT of all six components, Gamma-hat,
// inverse x-FFT, store.
template <typename T>
__global__ void __launch_bounds__(SSFFT_THREADS)
    xpass_kernel(Grid<T> g, cplx<T> *__restrict__ spec, const MinresState *st) {
  if (st && st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = g.nx, ny = g.ny, hz = g.hz;
  const int k0 = blockIdx.x * g.kx;
  const int nk = min(g.kx, hz - k0);
  const int y = blockIdx.y;
  const int slab = nx * nk;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + 6 * nx * g.kx;
  cplx<T> *tw = bufB + 6 * nx * g.kx;
  load_table<T>(tw, g.twx, nx);
  for (int e = threadIdx.x; e < 6 * slab; e += blockDim.x) {
    const int c = e / slab, rem = e - c * slab;
    const int x = rem / nk, kk = rem - (rem / nk) * nk;
    bufA[c * slab + x * nk + kk] = spec[c * g.S + ((long long)x * ny + y) * hz + k0 + kk];
  }
  __syncthreads();
  LineLayout L{6 * nk, nk, slab, 1, nk};
  cplx<T> *res = smem_fft<T, false, true>(bufA, bufB, L, g.px, tw);
  cplx<T> *other = (res == bufA) ? bufB : bufA;
  for (int e = threadIdx.x; e < slab; e += blockDim.x) {
    const int x = e / nk, kk = e - (e / nk) * nk;
    cplx<T> m[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = res[c * slab + x * nk + kk];
    green_apply<T>(g, x, y, k0 + kk, m);
#pragma unroll
    for (int c = 0; c < 6; ++c) res[c * slab + x * nk + kk] = m[c];
  }
  __syncthreads();
  cplx<T> *out = smem_fft<T, true, true>(res, other, L, g.px, tw);
  for (int e = threadIdx.x; e < 6 * slab; e += blockDim.x) {
    const int c = e / slab, rem = e - c * slab;
    const int x = rem / nk, kk = rem - (rem / nk) * nk;
    spec[c * g.S + ((long long)x * ny + y) * hz + k0 + kk] = out[c * slab + x * nk + kk];
  }
}

// ---- epilogue modes of zinv ----------------------------------------------------------
enum { EPI_STORE = 0, EPI_RESIDUAL = 1, EPI_MINRES = 2 };

template <typename T> struct EpiArgs {
  T *out;                 // STORE/RESIDUAL: output planes; MINRES: r1 (read, then y)
  const T *r2;            // MINRES: current Lanczos vector (v = s * r2)
  MinresState *st;        // MINRES
  double *partials;       // per-block partial results
  unsigned int *ticket;   // last-block counter
  double *result;         // RESIDUAL: max |b|
};

template <typename T, typename TF, int EPI>
__global__ void __launch_bounds__(SSFFT_THREADS)
    zinv_kernel(Grid<T> g, EpiArgs<TF> a, const cplx<T> *__restrict__ spec) {
  if (EPI == EPI_MINRES && a.st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  const int nz = g.nz, hz = g.hz;
  const long long nlines_all = (long long)g.nx * g.ny;
  const long long line0 = (long long)blockIdx.x * g.lz;
  const int nl = (int)min((long long)g.lz, nlines_all - line0);
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + 3 * g.lz * nz;
  cplx<T> *tw = bufB + 3 * g.lz * nz;
  load_table<T>(tw, g.twz, nz);
  // rebuild the full z spectrum of Z = A + iB from the stored half (Hermitian in z)
  for (int e = threadIdx.x; e < 3 * nl * nz; e += blockDim.x) {
    const int p = e / (nl * nz);
    const int rem = e - p * nl * nz;
    const int l = rem / nz, k = rem - (rem / nz) * nz;
    const bool low = (k < hz);
    const int ks = low ? k : nz - k;
    const long long off = (line0 + l) * hz + ks;
    const cplx<T> A = spec[(2 * p) * g.S + off];
    const cplx<T> B = spec[(2 * p + 1) * g.S + off];
    bufA[(p * nl + l) * nz + k] = low ? mk<T>(A.x - B.y, A.y + B.x) : mk<T>(A.x + B.y, B.x - A.y);
  }
  __syncthreads();
  LineLayout L{3 * nl, 3 * nl, 0, nz, 1};
  cplx<T> *res = smem_fft<T, true, false>(bufA, bufB, L, g.pz, tw);
  double acc = 0.0;
  T s = 0, c1 = 0;
  if (EPI == EPI_MINRES) {
    s = (T)a.st->s;
    c1 = (T)a.st->c_r1;
  }
  for (int e = threadIdx.x; e < nl * nz; e += blockDim.x) {
    const int l = e / nz, z = e - (e / nz) * nz;
    const long long v = (line0 + l) * nz + z;
    T r[6];
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const cplx<T> Z = res[(p * nl + l) * nz + z];
      r[2 * p] = Z.x;
      r[2 * p + 1] = Z.y;
    }
    if (EPI == EPI_STORE) {
#pragma unroll
      for (int c = 0; c < 6; ++c) a.out[c * g.V + v] = (TF)r[c];
    } else if (EPI == EPI_RESIDUAL) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        a.out[c * g.V + v] = (TF)r[c];
        acc = fmax(acc, fabs((double)r[c]));
      }
    } else {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const T y = r[c] - c1 * (T)a.out[c * g.V + v];
        a.out[c * g.V + v] = (TF)y;
        acc += (double)(s * (T)a.r2[c * g.V + v]) * (double)y;
      }
    }
  }
  if (EPI == EPI_STORE) return;
  const double part = (EPI == EPI_RESIDUAL) ? block_max(acc, red) : block_sum(acc, red);
  if (threadIdx.x == 0) a.partials[blockIdx.x] = part;
  if (!last_block_arrives(a.ticket)) return;
  if (EPI == EPI_RESIDUAL) {
    const double m = ordered_max(a.partials, gridDim.x, 1, red);
    if (threadIdx.x == 0) {
      *a.result = m;
      *a.ticket = 0;
    }
  } else {
    const double alfa = ordered_sum(a.partials, gridDim.x, 1, red);
    if (threadIdx.x == 0) {
      a.st->alfa = alfa;
      a.st->itn += 1;
      *a.ticket = 0;
    }
  }
}
