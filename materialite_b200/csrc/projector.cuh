// The compatibility projection  out = ifftn( Gamma-hat(q) : fftn(tau) ).real  of
// materialite's SmallStrainFFT (small_strain_fft.py:301-382), over a half spectrum held in
// HBM, for every slot of a SlotList at once.
//
// Five passes (any grid):
//   zfwd : per tile of (x,y) lines, build tau (prologue), real-to-complex FFT along z
//   yfwd : complex FFT along y
//   xpass: complex FFT along x, Gamma-hat apply on all six components, inverse along x
//   yinv : inverse complex FFT along y
//   zinv : complex-to-real inverse along z, then the epilogue
// Three passes (grids whose yz plane fits in shared memory): zyfwd does z and y of one x
// plane, yzinv their inverse, and the spectrum crosses HBM four times instead of eight.
// Larger planes run the same three passes on thread-block clusters (zyfwd_cl, yzinv_cl):
// the C blocks of a cluster split one plane and exchange it through distributed shared
// memory between the z and the y transforms.
//
// The six real components are paired into three complex lines for the z passes
// ((0,1), (2,3), (4,5)), so the z transforms run at half length-cost.  Gamma-hat is
// never stored: with t = normalize(tan(pi f_x), tan(pi f_y), tan(pi f_z)) the reference
// operator (rotated frequencies normalised, A = delta q conj q, B = q q conj q conj q)
// reduces exactly to  Gamma-hat : T = t (x) u + u (x) t - (t . u) t (x) t,  u = T t.
// Nyquist planes of even sizes are zero (small_strain_fft.py:354-359) and
// Gamma-hat(0) = diag(stress_mask) (:363-367).
//
// Every kernel runs a persistent grid over items (slot, tile); see slots.cuh.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "fft.cuh"
#include "slots.cuh"

// Spectrum layout: spec[c * S + (x * ny + y) * hs + kz], c = Mandel component,
// S = nx * ny * hs.  Real fields: f[c * V + (x * ny + y) * nz + z].  The half spectrum
// has hz = nz/2 + 1 columns; on even grids the last one, kz = nz/2, is a Nyquist plane that
// Gamma-hat zeroes (small_strain_fft.py:354-359), so it is neither stored nor transformed
// along x and y: hs = nz/2 columns are stored (hs = hz on odd grids), and the inverse
// z passes read the Nyquist column as zero.
template <typename T> struct Grid {
  int nx, ny, nz, hz, hs;
  long long V, S;
  AxisPlan px, py, pz;
  const cplx<T> *twx, *twy, *twz;  // e^{-2 pi i k / n}, k < n
  const T *tanx, *tany, *tanz;     // tan(pi f_k) with f = fftfreq (nx, ny, hz entries)
  T scale;                         // 1 / V
  int lz;                          // (x,y) lines per z-pass tile
  int ky;                          // kz columns per y-pass tile
  int kx;                          // kz columns per x-pass tile
  int nzb, nky, nkx;               // tiles along the lines, y columns and x columns
  // Divisors of the index arithmetic, prepared on the host (grid_divisors): [0] for a full
  // tile, [1] for the last, partial one along that axis.
  FastDiv fd_nz, fd_hs, fd_ny, fd_nx, fd_2hs, fd_plane;  // plane kernels
  FastDiv fd_z3[2], fd_znh[2], fd_znz[2];               // z passes: 3 nl, nl hs, nl nz
  FastDiv fd_ky[2];                                     // y passes: nk
  FastDiv fd_kx[2], fd_x6k[2], fd_xslab[2];             // x pass: nk, 6 nk, nx nk
  // items per slot and their decomposition
  FastDiv fd_it_plane, fd_it_x, fd_nkx, fd_it_z, fd_it_y, fd_nky, fd_nkynx, fd_3;
};

// Fill the stored-column count, tile counts and divisor table of a grid whose sizes and
// tiles (lz, ky, kx) are set.
template <typename T> inline void grid_divisors(Grid<T> &g) {
  const long long lines = (long long)g.nx * g.ny;
  g.hs = (g.nz % 2 == 0) ? g.nz / 2 : g.hz;
  g.nzb = (int)((lines + g.lz - 1) / g.lz);
  g.nky = (g.hs + g.ky - 1) / g.ky;
  g.nkx = (g.hs + g.kx - 1) / g.kx;
  const int lzt = (int)(lines - (long long)(g.nzb - 1) * g.lz);
  const int kyt = g.hs - (g.nky - 1) * g.ky;
  const int kxt = g.hs - (g.nkx - 1) * g.kx;
  auto fd = [](long long d) { return make_fastdiv((uint32_t)d); };
  g.fd_nz = fd(g.nz);
  g.fd_hs = fd(g.hs);
  g.fd_ny = fd(g.ny);
  g.fd_nx = fd(g.nx);
  g.fd_2hs = fd(2 * g.hs);
  g.fd_plane = fd((long long)g.ny * g.hs);
  const int nl[2] = {g.lz, lzt}, ky[2] = {g.ky, kyt}, kx[2] = {g.kx, kxt};
  for (int t = 0; t < 2; ++t) {
    g.fd_z3[t] = fd(3LL * nl[t]);
    g.fd_znh[t] = fd((long long)nl[t] * g.hs);
    g.fd_znz[t] = fd((long long)nl[t] * g.nz);
    g.fd_ky[t] = fd(ky[t]);
    g.fd_kx[t] = fd(kx[t]);
    g.fd_x6k[t] = fd(6LL * kx[t]);
    g.fd_xslab[t] = fd((long long)g.nx * kx[t]);
  }
  g.fd_it_plane = fd(3LL * g.nx);
  g.fd_it_x = fd((long long)g.nkx * g.ny);
  g.fd_nkx = fd(g.nkx);
  g.fd_it_z = fd(g.nzb);
  g.fd_it_y = fd(6LL * g.nky * g.nx);
  g.fd_nky = fd(g.nky);
  g.fd_nkynx = fd((long long)g.nky * g.nx);
  g.fd_3 = fd(3);
}

__device__ __forceinline__ int udiv(int n, const FastDiv &f) { return (int)fdiv((uint32_t)n, f); }

// Items of one slot in each pass.
template <typename T> __host__ __device__ inline int items_plane(const Grid<T> &g) { return 3 * g.nx; }
template <typename T> __host__ __device__ inline int items_x(const Grid<T> &g) { return g.nkx * g.ny; }
template <typename T> __host__ __device__ inline int items_z(const Grid<T> &g) { return g.nzb; }
template <typename T> __host__ __device__ inline int items_y(const Grid<T> &g) { return 6 * g.nky * g.nx; }

// Shared-memory footprint of the passes (elements of cplx<T>).  The z passes hold three
// paired lines per (x,y) line, padded (sidx<true>); the x pass pads each component slab
// by 64 bytes so the six slabs start on alternating bank halves.
__host__ __device__ inline int zbuf_elems(int lz, int nz) { return padded_len(3 * lz * nz); }
template <typename T> __host__ __device__ inline int xslab_elems(int nx, int kx) {
  return nx * kx + 64 / (int)sizeof(cplx<T>);
}
template <typename T> inline size_t smem_z_bytes(int lz, int nz) {
  return (2 * (size_t)zbuf_elems(lz, nz) + nz) * sizeof(cplx<T>);
}
template <typename T> inline size_t smem_y_bytes(int ky, int ny) {
  return (2 * (size_t)ky * ny + ny) * sizeof(cplx<T>);
}
template <typename T> inline size_t smem_x_bytes(int kx, int nx) {
  return (2 * 6 * (size_t)xslab_elems<T>(nx, kx) + nx) * sizeof(cplx<T>);
}

// Device-resident state of one MINRES solve (doubles; see krylov.cuh).
struct MinresState {
  double beta1, beta, oldb, alfa, dbar, epsln, phibar, tnorm2, gmax, gmin, cs, sn;
  double delta, oldeps, gamma, phi, denom, root, anorm, ynorm, rnorm, test1, test2;
  double s, s_prev, c_r1, coef;
  double rtol, eps, atol;
  long long itn, maxiter;
  int istop, done;
};

// A slot's "solve done" flag, read by every thread from L2.  Within a launch the flag of a
// slot is written only by the slot's last item to arrive, after every item of the slot has
// read it, so all threads of a block read the same value and no barrier is needed.
__device__ __forceinline__ bool slot_done(const MinresState *st) { return __ldcg(&st->done) != 0; }

// Caller-owned input and output of the plain projection (PRO_INPUT / EPI_STORE).
template <typename TF> struct ExtIO {
  const TF *in;
  TF *out;
};

// ---- prologue modes of the forward passes ---------------------------------------------
//   PRO_INPUT          tau = caller's planes
//   PRO_RESIDUAL       tau = Sbar - sigma                    (small_strain_fft.py:140,168)
//   PRO_TANGENT_*      tau = K v of the Krylov iteration     (:370-374), table or voxel K;
//                      formed by the update kernel (krylov.cuh), not by a transform pass
//   PRO_REPROJECT      tau = x (the Newton correction)
//   PRO_TAU            tau = K v as the update kernel left it in the slot's y' buffer (the
//                      forward transform of a Krylov iteration; skips finished solves)
enum { PRO_INPUT = 0, PRO_RESIDUAL = 1, PRO_TANGENT_TABLE = 2, PRO_TANGENT_VOXEL = 3,
       PRO_REPROJECT = 4, PRO_TAU = 5 };
#define PRO_IS_KRYLOV(P) ((P) == PRO_TANGENT_TABLE || (P) == PRO_TANGENT_VOXEL)

// ---- epilogue modes of the inverse passes -----------------------------------------------
//   EPI_STORE          caller's planes = result
//   EPI_RESIDUAL       b = result, max|b|                    (:141-144)
//   EPI_MINRES         the MINRES dot products' reduction (the epilogue kernel, krylov.cuh;
//                      not a transform-pass mode)
//   EPI_REPROJECT      x = result; strain += x; fluctuation += x   (:154-155)
//   EPI_PTAU           y' buffer = P tau (the epilogue kernel, krylov.cuh, forms y' there)
enum { EPI_STORE = 0, EPI_RESIDUAL = 1, EPI_MINRES = 2, EPI_REPROJECT = 3, EPI_PTAU = 4 };
#define EPI_SKIPS_DONE(E) ((E) == EPI_PTAU)

// Stopping tests of scipy's minres after the solution update (last item of the forward
// pass that applied it, with x2 = |x|^2).
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
    if (s.rnorm <= s.atol) s.istop = 1;  // the absolute floor (0 when off)
  }
  if (!isfinite(s.ynorm) || !isfinite(s.beta)) s.istop = 9;  // NaN guard
  if (s.beta == 0.0 && s.istop == 0) s.istop = 1;           // exact breakdown
  if (s.istop != 0) s.done = 1;
  *st = s;
}

// MINRES scalar recurrence after the matvec (Paige & Saunders 1975; scipy's minres loop
// body up to the plane rotation).  d0 = r2 . y', d1 = y' . y', d2 = r2 . r2 where
// y' = A v - (beta/oldb) r1 and v = r2 / beta.  The orthogonalised y'' = y' - (alfa/beta) r2
// is formed by the next forward pass; its norm follows from the three dot products:
// |y''|^2 = d1 - 2 c d0 + c^2 d2 with c = alfa / beta.
static __device__ __noinline__ void minres_after_matvec(MinresState *st, double d0, double d1,
                                                        double d2) {
  MinresState s = *st;
  s.itn += 1;
  s.alfa = s.s * d0;
  s.coef = s.alfa / s.beta;
  double beta2 = d1 - 2.0 * s.coef * d0 + s.coef * s.coef * d2;
  if (beta2 < 0.0) beta2 = 0.0;
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

// Scalars of the update pending from the previous MINRES iteration (all iterations after
// the first: itn >= 1), and the vector roles of this iteration.
template <typename T, typename TF> struct KrylovIn {
  bool on;
  T s, coef, sp, oe, de, dn, ph;
  KRoles<TF> r;
};

template <typename T, typename TF>
__device__ __forceinline__ KrylovIn<T, TF> krylov_in(const SlotDev<TF> &S) {
  const MinresState *st = S.st;
  KrylovIn<T, TF> u;
  const long long itn = st->itn;
  u.on = itn >= 1;
  u.s = (T)st->s;
  u.coef = (T)st->coef;
  u.sp = (T)st->s_prev;
  u.oe = (T)st->oldeps;
  u.de = (T)st->delta;
  u.dn = (T)st->denom;
  u.ph = (T)st->phi;
  u.r = kroles<TF>(S, itn);
  return u;
}

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

// Non-Krylov prologues at one point.
template <typename T, typename TF, int PRO>
__device__ __forceinline__ void prologue(const SlotDev<TF> &S, const TF *ext_in, long long V,
                                         long long v, T *tau) {
  if constexpr (PRO == PRO_INPUT) {
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = (T)ext_in[c * V + v];
  } else if constexpr (PRO == PRO_REPROJECT) {
    const TF *x = S.kr[5];
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = (T)x[c * V + v];
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = (T)S.sbar[c] - (T)S.sig[c * V + v];
  }
}

// Krylov prologue at one point: apply the pending update of the previous iteration
// (u_{j+1} = y' - coef u_j, w = (v_j - oldeps w1 - delta w2) denom, x += phi w, with
// v_j = s_prev u_j), then tau = K (s u_{j+1}).  Every block forms all six components of
// u_{j+1} (the tangent couples them) but updates and stores only the components it owns:
// all six (ALL) or the pair 2 pair, 2 pair + 1; |x|^2 of those accumulates into xx.  With
// ALL, tau[0..5] is the whole tau; otherwise tau[0..1] are the owned pair's components,
// and only the two tangent rows they need are loaded.
template <typename T, typename TF, int PRO, bool ALL>
__device__ __forceinline__ void tangent_prologue(const SlotDev<TF> &S, long long V, long long v,
                                                 const KrylovIn<T, TF> &u, int pair, T *tau,
                                                 double &xx) {
  constexpr int NO = ALL ? 6 : 2;  // owned components
  const int c0 = ALL ? 0 : 2 * pair;
  // every load is issued before the first store: the stores may alias the loaded arrays
  // as far as the compiler knows, and loads held back behind them would serialise
  T r[6], yv[6], a1[NO], a2[NO], xo[NO], k[ALL ? 21 : 12];
  const TF *in = u.r.P;
#pragma unroll
  for (int c = 0; c < 6; ++c) r[c] = (T)in[c * V + v];
  const TF *kp;
  long long ks;
  if constexpr (PRO == PRO_TANGENT_TABLE) {
    kp = S.ktab + (long long)S.gid[v] * 21;
    ks = 1;
  } else {
    kp = S.kvox + v;
    ks = V;
  }
  if constexpr (ALL) {
#pragma unroll
    for (int q = 0; q < 21; ++q) k[q] = (T)kp[q * ks];
  } else {
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int j = 0; j < 6; ++j) k[q * 6 + j] = (T)kp[sym_idx(c0 + q, j) * ks];
  }
  if (u.on) {
#pragma unroll
    for (int c = 0; c < 6; ++c) yv[c] = (T)u.r.Y[c * V + v];
#pragma unroll
    for (int q = 0; q < NO; ++q) {
      const long long i = (c0 + q) * V + v;
      a1[q] = (T)u.r.W1[i];
      a2[q] = (T)u.r.W2[i];
      xo[q] = (T)u.r.X[i];
    }
  }
  T vv[6];
  if (u.on) {
    T un[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      un[c] = yv[c] - u.coef * r[c];
      vv[c] = u.s * un[c];
    }
#pragma unroll
    for (int q = 0; q < NO; ++q) {
      // the owned components, picked by selects (no run-time register indexing)
      T uo, ro;
      if constexpr (ALL) {
        uo = un[q];
        ro = r[q];
      } else {
        uo = pair == 0 ? un[q] : (pair == 1 ? un[2 + q] : un[4 + q]);
        ro = pair == 0 ? r[q] : (pair == 1 ? r[2 + q] : r[4 + q]);
      }
      const long long i = (c0 + q) * V + v;
      const T w = (u.sp * ro - u.oe * a1[q] - u.de * a2[q]) * u.dn;
      const T xn = xo[q] + u.ph * w;
      u.r.Q[i] = (TF)uo;
      u.r.W[i] = (TF)w;
      u.r.X[i] = (TF)xn;
      xx += (double)xn * (double)xn;
    }
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) vv[c] = u.s * r[c];
  }
  if constexpr (ALL) {
    sym6_apply<T>(k, 1, vv, tau);
  } else {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      T acc = 0;
#pragma unroll
      for (int j = 0; j < 6; ++j) acc += k[q * 6 + j] * vv[j];
      tau[q] = acc;
    }
  }
}

// End of a forward item that applied a pending update: the slot's |x|^2 over its items,
// then the stopping tests in the slot's last item to arrive.
template <typename TF>
__device__ __forceinline__ void finish_pending_update(const SlotDev<TF> &S, double xx, int local,
                                                      int per_slot, double *red) {
  const double part = block_sum(xx, red);
  if (threadIdx.x == 0) S.partials[local] = part;
  if (!last_item_arrives(S.tickets + TK_UPD, (unsigned)per_slot)) return;
  const double x2 = ordered_sum(S.partials, per_slot, 1, red);
  if (threadIdx.x == 0) {
    S.tickets[TK_UPD] = 0;
    minres_after_update(S.st, x2);
  }
}

template <typename T>
__device__ __forceinline__ void load_table(cplx<T> *dst, const cplx<T> *src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Block-uniform "skip this item": a Krylov item of a slot whose solve is done.
template <typename TF, int PRO> __device__ __forceinline__ bool skip_item(const SlotDev<TF> &S) {
  if constexpr (PRO == PRO_TAU) return slot_done(S.st);
  return false;
}

// Per-point epilogue of the inverse passes: r[] is the transformed value of the owned
// components c0 .. c0 + NC - 1 at point v; acc0 accumulates the residual's max |b|.
template <typename T, typename TF, int EPI, int NC>
__device__ __forceinline__ void epilogue_point(const SlotDev<TF> &S, const ExtIO<TF> &io,
                                               const KRoles<TF> &kr, long long V, long long v,
                                               int c0, const T *r, double &acc0) {
  static_assert(EPI != EPI_MINRES, "the MINRES epilogue is the epilogue kernel (krylov.cuh)");
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const long long i = (long long)(c0 + q) * V + v;
    if constexpr (EPI == EPI_STORE) {
      io.out[i] = (TF)r[q];
    } else if constexpr (EPI == EPI_RESIDUAL) {
      S.b[i] = (TF)r[q];
      acc0 = fmax(acc0, fabs((double)r[q]));
    } else if constexpr (EPI == EPI_REPROJECT) {
      // the strain fields are double: they take the re-projected correction unrounded
      kr.X[i] = (TF)r[q];
      S.eps[i] += (double)r[q];
      S.dfl[i] += (double)r[q];
    } else {  // EPI_PTAU
      kr.Y[i] = (TF)r[q];
    }
  }
}

// End of an inverse item: the slot's max |b| (residual) or its three MINRES dot products,
// finished by the slot's last item.
template <typename TF, int EPI>
__device__ __forceinline__ void finish_inverse(const SlotDev<TF> &S, double acc0, double acc1,
                                               double acc2, int local, int per_slot,
                                               double *red) {
  if constexpr (EPI == EPI_RESIDUAL) {
    const double part = block_max(acc0, red);
    if (threadIdx.x == 0) S.partials[local] = part;
  } else if constexpr (EPI == EPI_MINRES) {
    const double q0 = block_sum(acc0, red);
    const double q1 = block_sum(acc1, red);
    const double q2 = block_sum(acc2, red);
    if (threadIdx.x == 0) {
      S.partials[3 * local] = q0;
      S.partials[3 * local + 1] = q1;
      S.partials[3 * local + 2] = q2;
    }
  } else {
    return;
  }
  if (!last_item_arrives(S.tickets + TK_ZINV, (unsigned)per_slot)) return;
  if constexpr (EPI == EPI_RESIDUAL) {
    const double m = ordered_max(S.partials, per_slot, 1, red);
    if (threadIdx.x == 0) {
      S.results[40] = m;
      S.tickets[TK_ZINV] = 0;
    }
  } else {
    const double d0 = ordered_sum(S.partials, per_slot, 3, red);
    const double d1 = ordered_sum(S.partials + 1, per_slot, 3, red);
    const double d2 = ordered_sum(S.partials + 2, per_slot, 3, red);
    if (threadIdx.x == 0) {
      minres_after_matvec(S.st, d0, d1, d2);
      S.tickets[TK_ZINV] = 0;
    }
  }
}

// ---- five-pass kernels ------------------------------------------------------------------

// z kernels: three blocks per SM in float (80 registers), two in double
#define Z_MIN_BLOCKS(T) (sizeof(T) == 4 ? 3 : 2)

// zfwd: an item is (slot, tile of g.lz consecutive (x,y) lines).  TF is the storage type of
// the fields (TF = T except when a double-precision transform reads float fields).
template <typename T, typename TF, int PRO>
__global__ void __launch_bounds__(SSFFT_THREADS, Z_MIN_BLOCKS(T))
    zfwd_kernel(Grid<T> g, const SlotDev<TF> *__restrict__ tab, SlotList list, ExtIO<TF> io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<TF>)];
  const int nz = g.nz, hs = g.hs;
  const long long V = g.V;
  const long long nlines_all = (long long)g.nx * g.ny;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + zbuf_elems(g.lz, nz);
  cplx<T> *tw = bufB + zbuf_elems(g.lz, nz);
  load_table<T>(tw, g.twz, nz);
  const int per = items_z(g);
  const int n_items = list_items(list, per);
  int staged = -1;  // slot whose descriptor sdesc holds
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = udiv(item, g.fd_it_z);
    const int local = item - k * per;
    const SlotDev<TF> &S = stage_slot<TF>(tab, list.ids[k], sdesc, staged);
    if (skip_item<TF, PRO>(S)) continue;
    const long long line0 = (long long)local * g.lz;
    const int nl = (int)min((long long)g.lz, nlines_all - line0);
    const int ti = (nl == g.lz) ? 0 : 1;
    __syncthreads();  // table loaded; previous item done with the buffers
    if constexpr (PRO == PRO_TAU) {
      // the six tau planes of the tile's lines straight into the paired lines, in flight
      // together
      const T *src = reinterpret_cast<const T *>(kroles<TF>(S, S.st->itn).Y);
      for (int e = threadIdx.x; e < nl * nz; e += blockDim.x) {
        const int l = udiv(e, g.fd_nz), z = e - l * nz;
        const long long v = (line0 + l) * nz + z;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          cplx<T> *d = &bufA[sidx<true>((p * nl + l) * nz + z)];
          cp_async_scalar<T>(&d->x, src + (2 * p) * V + v);
          cp_async_scalar<T>(&d->y, src + (2 * p + 1) * V + v);
        }
      }
      cp_async_wait_all();
    } else {
      for (int e = threadIdx.x; e < nl * nz; e += blockDim.x) {
        const int l = udiv(e, g.fd_nz), z = e - l * nz;
        const long long v = (line0 + l) * nz + z;
        T tau[6];
        prologue<T, TF, PRO>(S, io.in, V, v, tau);
#pragma unroll
        for (int p = 0; p < 3; ++p)
          bufA[sidx<true>((p * nl + l) * nz + z)] = mk<T>(tau[2 * p], tau[2 * p + 1]);
      }
    }
    __syncthreads();
    const LineLayout L(3 * nl, 3 * nl, 0, nz, 1, g.fd_z3[ti], g.fd_z3[ti]);
    cplx<T> *res = smem_fft<T, false, false, true>(bufA, bufB, L, g.pz, tw);
    cplx<T> *spec = reinterpret_cast<cplx<T> *>(S.spec);
    // split the paired transform: A = (Z_k + conj Z_{-k}) / 2, B = (Z_k - conj Z_{-k}) / 2i
    for (int e = threadIdx.x; e < 3 * nl * hs; e += blockDim.x) {
      const int p = udiv(e, g.fd_znh[ti]);
      const int rem = e - p * nl * hs;
      const int l = udiv(rem, g.fd_hs), kk = rem - l * hs;
      const cplx<T> Z = res[sidx<true>((p * nl + l) * nz + kk)];
      const int km = (kk == 0) ? 0 : nz - kk;
      const cplx<T> Zm = res[sidx<true>((p * nl + l) * nz + km)];
      const cplx<T> A = mk<T>((T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y));
      const cplx<T> B = mk<T>((T)0.5 * (Z.y + Zm.y), (T)0.5 * (Zm.x - Z.x));
      const long long off = (line0 + l) * hs + kk;
      spec[(2 * p) * g.S + off] = A;
      spec[(2 * p + 1) * g.S + off] = B;
    }
  }
}

// y passes: an item is (slot, kz column tile, x, component); lines are kz columns of one
// (c, x) slab.
template <typename T, typename TF, bool INV, bool KRY>
__global__ void __launch_bounds__(SSFFT_THREADS)
    ypass_kernel(Grid<T> g, const SlotDev<TF> *__restrict__ tab, SlotList list) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ny = g.ny, hs = g.hs;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + g.ky * ny;
  cplx<T> *tw = bufB + g.ky * ny;
  __shared__ __align__(8) uint64_t tile_bar;
  load_table<T>(tw, g.twy, ny);
  bulk_barrier_init(&tile_bar);
  unsigned tile_phase = 0;
  const int per = items_y(g);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = udiv(item, g.fd_it_y);
    const int local = item - k * per;
    const SlotDev<TF> &S = tab[list.ids[k]];
    // a finished solve's items are skipped: the flag is read here and tested after the tile
    // copy, so the read's latency overlaps the copy (the flag does not change in a launch)
    const int done = KRY ? __ldcg(&S.st->done) : 0;
    const int c = udiv(local, g.fd_nkynx);
    const int r1 = local - c * g.nky * g.nx;
    const int x = udiv(r1, g.fd_nky);
    const int kb = r1 - x * g.nky;
    const int k0 = kb * g.ky;
    const int nk = min(g.ky, hs - k0);
    const int ti = (nk == g.ky) ? 0 : 1;
    cplx<T> *base = reinterpret_cast<cplx<T> *>(S.spec) + c * g.S + (long long)x * ny * hs + k0;
    __syncthreads();
    constexpr long long E = sizeof(cplx<T>);
    if (bulk_copy_rows(bufA, base, ny, 1, (unsigned)(nk * E), nk * E, 0, hs * E, 0, &tile_bar)) {
      bulk_barrier_wait(&tile_bar, tile_phase);
      tile_phase ^= 1;
    } else {
      for (int e = threadIdx.x; e < ny * nk; e += blockDim.x) {
        const int y = udiv(e, g.fd_ky[ti]), kk = e - y * nk;
        cp_async_elem<T>(&bufA[y * nk + kk], &base[(long long)y * hs + kk]);
      }
      cp_async_wait_all();
    }
    __syncthreads();
    if (done) continue;
    const LineLayout L(nk, nk, 0, 1, nk, g.fd_ky[ti], g.fd_ky[ti]);
    cplx<T> *res = smem_fft<T, INV, true>(bufA, bufB, L, g.py, tw);
    for (int e = threadIdx.x; e < ny * nk; e += blockDim.x) {
      const int y = udiv(e, g.fd_ky[ti]), kk = e - y * nk;
      base[(long long)y * hs + kk] = res[y * nk + kk];
    }
  }
}

// Gamma-hat : tau-hat at one frequency, in place on the six complex components.
template <typename T>
__device__ __forceinline__ void green_apply(const Grid<T> &g, const double *mask, int kx, int ky,
                                            int kz, cplx<T> *m) {
  const bool nyq = ((g.nx % 2 == 0) && kx == g.nx / 2) || ((g.ny % 2 == 0) && ky == g.ny / 2) ||
                   ((g.nz % 2 == 0) && kz == g.nz / 2);
  if (kx == 0 && ky == 0 && kz == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = cscale<T>(m[c], (T)mask[c] * g.scale);
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

// x pass: an item is (slot, y, kz column tile); forward x-FFT of all six components,
// Gamma-hat, inverse x-FFT, store.  KRY: skip slots whose solve is done.
// PT threads a block (any multiple of 32 up to 1024: every loop strides by blockDim.x).
#define XPASS_THREADS SSFFT_THREADS
template <typename T, typename TF, bool KRY, int PT = XPASS_THREADS>
__global__ void __launch_bounds__(PT)
    xpass_kernel(Grid<T> g, const SlotDev<TF> *__restrict__ tab, SlotList list) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = g.nx, ny = g.ny, hs = g.hs;
  const int sst = xslab_elems<T>(nx, g.kx);      // padded slab stride
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + 6 * sst;
  cplx<T> *tw = bufB + 6 * sst;
  __shared__ __align__(8) uint64_t tile_bar;
  load_table<T>(tw, g.twx, nx);
  bulk_barrier_init(&tile_bar);
  unsigned tile_phase = 0;
  const int per = items_x(g);
  const int n_items = list_items(list, per);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int kk_slot = udiv(item, g.fd_it_x);
    const int local = item - kk_slot * per;
    const SlotDev<TF> &S = tab[list.ids[kk_slot]];
    // a finished solve's items are skipped: the flag is read here and tested after the tile
    // copy, so the read's latency overlaps the copy (the flag does not change in a launch)
    const int done = KRY ? __ldcg(&S.st->done) : 0;
    const int y = udiv(local, g.fd_nkx);
    const int kb = local - y * g.nkx;
    const int k0 = kb * g.kx;
    const int nk = min(g.kx, hs - k0);
    const int ti = (nk == g.kx) ? 0 : 1;
    const int slab = nx * nk;                      // live elements per component
    cplx<T> *spec = reinterpret_cast<cplx<T> *>(S.spec);
    __syncthreads();
    constexpr long long E = sizeof(cplx<T>);
    // rows (c, x): nk columns each, from spec[c][x][y][k0..]
    if (bulk_copy_rows(bufA, spec + (long long)y * hs + k0, 6, nx, (unsigned)(nk * E), sst * E,
                       nk * E, g.S * E, (long long)ny * hs * E, &tile_bar)) {
      bulk_barrier_wait(&tile_bar, tile_phase);
      tile_phase ^= 1;
    } else {
      for (int e = threadIdx.x; e < 6 * slab; e += blockDim.x) {
        const int c = udiv(e, g.fd_xslab[ti]), rem = e - c * slab;
        const int x = udiv(rem, g.fd_kx[ti]), kk = rem - x * nk;
        cp_async_elem<T>(&bufA[c * sst + x * nk + kk], &spec[c * g.S + ((long long)x * ny + y) * hs + k0 + kk]);
      }
      cp_async_wait_all();
    }
    __syncthreads();
    if (done) continue;
    const LineLayout L(6 * nk, nk, sst, 1, nk, g.fd_x6k[ti], g.fd_kx[ti]);
    cplx<T> *res = smem_fft<T, false, true>(bufA, bufB, L, g.px, tw);
    cplx<T> *other = (res == bufA) ? bufB : bufA;
    for (int e = threadIdx.x; e < slab; e += blockDim.x) {
      const int x = udiv(e, g.fd_kx[ti]), kk = e - x * nk;
      cplx<T> m[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) m[c] = res[c * sst + x * nk + kk];
      green_apply<T>(g, S.mask, x, y, k0 + kk, m);
#pragma unroll
      for (int c = 0; c < 6; ++c) res[c * sst + x * nk + kk] = m[c];
    }
    __syncthreads();
    cplx<T> *out = smem_fft<T, true, true>(res, other, L, g.px, tw);
    for (int e = threadIdx.x; e < 6 * slab; e += blockDim.x) {
      const int c = udiv(e, g.fd_xslab[ti]), rem = e - c * slab;
      const int x = udiv(rem, g.fd_kx[ti]), kk = rem - x * nk;
      spec[c * g.S + ((long long)x * ny + y) * hs + k0 + kk] = out[c * sst + x * nk + kk];
    }
  }
}


template <typename T, typename TF, int EPI>
__global__ void __launch_bounds__(SSFFT_THREADS, Z_MIN_BLOCKS(T))
    zinv_kernel(Grid<T> g, const SlotDev<TF> *__restrict__ tab, SlotList list, ExtIO<TF> io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<TF>)];
  const int nz = g.nz, hz = g.hz;
  const long long V = g.V;
  const long long nlines_all = (long long)g.nx * g.ny;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + zbuf_elems(g.lz, nz);
  cplx<T> *tw = bufB + zbuf_elems(g.lz, nz);
  __shared__ __align__(8) uint64_t tile_bar;
  load_table<T>(tw, g.twz, nz);
  bulk_barrier_init(&tile_bar);
  unsigned tile_phase = 0;
  const int per = items_z(g);
  const int n_items = list_items(list, per);
  int staged = -1;  // slot whose descriptor sdesc holds
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = udiv(item, g.fd_it_z);
    const int local = item - k * per;
    const SlotDev<TF> &S = stage_slot<TF>(tab, list.ids[k], sdesc, staged);
    if (EPI_SKIPS_DONE(EPI) && slot_done(S.st)) continue;
    const long long line0 = (long long)local * g.lz;
    const int nl = (int)min((long long)g.lz, nlines_all - line0);
    const int ti = (nl == g.lz) ? 0 : 1;
    const int nel = nl * nz;
    KRoles<TF> kr{};
    if constexpr (EPI == EPI_PTAU) {
      kr = kroles<TF>(S, S.st->itn);
    } else if constexpr (EPI == EPI_REPROJECT) {
      kr = kroles<TF>(S, 0);
    }
    const cplx<T> *spec = reinterpret_cast<const cplx<T> *>(S.spec);
    const int hs = g.hs, nlhs = nl * hs;
    __syncthreads();
    // the tile's stored halves, [c][l][ks] in bufB, all in flight at once (the tile's lines
    // are consecutive rows of the spectrum)
    const bool staged_half = 6 * nlhs <= zbuf_elems(g.lz, nz);
    if (staged_half) {
      constexpr long long E = sizeof(cplx<T>);
      // six bulk copies, one per component, where the runs are 16-byte aligned
      if (bulk_copy_rows(bufB, spec + line0 * hs, 6, 1, (unsigned)(nlhs * E), nlhs * E, 0,
                         g.S * E, 0, &tile_bar)) {
        bulk_barrier_wait(&tile_bar, tile_phase);
        tile_phase ^= 1;
      } else {
        for (int e = threadIdx.x; e < 6 * nlhs; e += blockDim.x) {
          const int c = udiv(e, g.fd_znh[ti]), rem = e - c * nlhs;
          cp_async_elem<T>(&bufB[e], &spec[c * g.S + line0 * hs + rem]);
        }
        cp_async_wait_all();
      }
      __syncthreads();
    }
    // rebuild the full z spectrum of Z = A + iB from the stored half (Hermitian in z)
    for (int e = threadIdx.x; e < 3 * nel; e += blockDim.x) {
      const int p = udiv(e, g.fd_znz[ti]);
      const int rem = e - p * nel;
      const int l = udiv(rem, g.fd_nz), kk = rem - l * nz;
      const bool low = (kk < hz);
      const int ks = low ? kk : nz - kk;
      const bool nyq = 2 * ks == nz;  // the unstored Nyquist column is zero
      cplx<T> A = mk<T>((T)0, (T)0), B = A;
      if (!nyq) {
        if (staged_half) {
          A = bufB[(2 * p) * nlhs + l * hs + ks];
          B = bufB[(2 * p + 1) * nlhs + l * hs + ks];
        } else {
          const long long off = (line0 + l) * hs + ks;
          A = spec[(2 * p) * g.S + off];
          B = spec[(2 * p + 1) * g.S + off];
        }
      }
      bufA[sidx<true>((p * nl + l) * nz + kk)] =
          low ? mk<T>(A.x - B.y, A.y + B.x) : mk<T>(A.x + B.y, B.x - A.y);
    }
    __syncthreads();
    const LineLayout L(3 * nl, 3 * nl, 0, nz, 1, g.fd_z3[ti], g.fd_z3[ti]);
    cplx<T> *res = smem_fft<T, true, false, true>(bufA, bufB, L, g.pz, tw);
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      const long long v = line0 * nz + e;
      T r[6];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const cplx<T> Z = res[sidx<true>(p * nel + e)];
        r[2 * p] = Z.x;
        r[2 * p + 1] = Z.y;
      }
      epilogue_point<T, TF, EPI, 6>(S, io, kr, V, v, 0, r, acc0);
    }
    finish_inverse<TF, EPI>(S, acc0, acc1, acc2, local, per, red);
  }
}

// ---- plane-fused passes (grids whose yz planes fit in shared memory) -------------------
//
// zyfwd: an item is (slot, x plane, component pair p): tau of the pair over the whole
// plane (prologue), real-to-complex along z, complex FFT along y, write the half spectrum
// of both components.  yzinv is its inverse followed by the epilogue.  The three pair
// items of one plane are adjacent, so the Krylov vectors all three read come from L2.

// Shared memory of the plane passes: two buffers of the padded plane (ny (nz + 2)
// complex, enough for the paired z lines and for the split half spectra of two
// components) plus the y and z twiddles.
template <typename T> inline size_t smem_plane_bytes(int ny, int nz) {
  return (2 * (size_t)padded_len(ny * (nz + 2)) + ny + nz) * sizeof(cplx<T>);
}

// Plane kernels run PT threads (256, 512 or 1024), at most 64 registers each.
#define PLANE_MIN_BLOCKS(PT) (1024 / (PT))

// Prologue of a plane item over the points vbase .. vbase + nel - 1 (whole z lines): tau
// of the component pair p as one complex value per point, into padded z lines in buf.
// PRO_TAU copies the pair's two planes with cp.async (all in flight at once).
template <typename T, typename TF, int PRO>
__device__ __forceinline__ void plane_prologue(const SlotDev<TF> &S, const ExtIO<TF> &io,
                                               long long V, long long vbase, int nel, int p,
                                               cplx<T> *buf) {
  if constexpr (PRO == PRO_TAU) {
    const T *src = reinterpret_cast<const T *>(kroles<TF>(S, S.st->itn).Y);
    const T *s0 = src + (2 * p) * V + vbase, *s1 = src + (2 * p + 1) * V + vbase;
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      cplx<T> *d = &buf[sidx<true>(e)];
      cp_async_scalar<T>(&d->x, s0 + e);
      cp_async_scalar<T>(&d->y, s1 + e);
    }
    cp_async_wait_all();
  } else {
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      T tau[6];
      prologue<T, TF, PRO>(S, io.in, V, vbase + e, tau);
      buf[sidx<true>(e)] = mk<T>(tau[2 * p], tau[2 * p + 1]);
    }
  }
}

// Epilogue of a plane item: fin holds components 2p (real part) and 2p + 1 (imaginary
// part) of the points vbase .. vbase + nel - 1 in padded z lines; acc0 accumulates the
// residual's max |b|.
template <typename T, typename TF, int EPI>
__device__ __forceinline__ void plane_epilogue(const SlotDev<TF> &S, const ExtIO<TF> &io,
                                               long long V, long long vbase, int nel, int p,
                                               const cplx<T> *fin, double &acc0) {
  KRoles<TF> kr{};
  if constexpr (EPI == EPI_PTAU) {
    kr = kroles<TF>(S, S.st->itn);
  } else if constexpr (EPI == EPI_REPROJECT) {
    kr = kroles<TF>(S, 0);
  }
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    const cplx<T> Z = fin[sidx<true>(e)];
    const T r[2] = {Z.x, Z.y};
    epilogue_point<T, TF, EPI, 2>(S, io, kr, V, vbase + e, 2 * p, r, acc0);
  }
}

template <typename T, typename TF, int PRO, int PT>
__global__ void __launch_bounds__(PT, PLANE_MIN_BLOCKS(PT))
    zyfwd_kernel(Grid<T> g, const SlotDev<TF> *__restrict__ tab, SlotList list, ExtIO<TF> io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<TF>)];
  const int ny = g.ny, nz = g.nz, hs = g.hs;
  const long long V = g.V;
  const int cap = padded_len(ny * (nz + 2));
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + cap;
  cplx<T> *twy = bufB + cap;
  cplx<T> *twz = twy + ny;
  load_table<T>(twy, g.twy, ny);
  load_table<T>(twz, g.twz, nz);
  const int per = items_plane(g);
  const int n_items = list_items(list, per);
  const int plane = ny * hs;
  int staged = -1;  // slot whose descriptor sdesc holds
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = udiv(item, g.fd_it_plane);
    const int local = item - k * per;
    const SlotDev<TF> &S = stage_slot<TF>(tab, list.ids[k], sdesc, staged);
    if (skip_item<TF, PRO>(S)) continue;
    const int x = udiv(local, g.fd_3);
    const int p = local - 3 * x;
    const long long vbase = (long long)x * ny * nz;
    __syncthreads();
    plane_prologue<T, TF, PRO>(S, io, V, vbase, ny * nz, p, bufA);
    __syncthreads();
    const LineLayout Lz(ny, ny, 0, nz, 1, g.fd_ny, g.fd_ny);
    cplx<T> *res = smem_fft<T, false, false, true>(bufA, bufB, Lz, g.pz, twz);
    cplx<T> *oth = (res == bufA) ? bufB : bufA;
    // split the paired transform into the half spectra of components 2p and 2p+1,
    // laid out [c][y][k] for the y transform
    for (int e = threadIdx.x; e < plane; e += blockDim.x) {
      const int y = udiv(e, g.fd_hs), kk = e - y * hs;
      const cplx<T> Z = res[sidx<true>(y * nz + kk)];
      const cplx<T> Zm = res[sidx<true>(y * nz + (kk == 0 ? 0 : nz - kk))];
      oth[e] = mk<T>((T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y));
      oth[plane + e] = mk<T>((T)0.5 * (Z.y + Zm.y), (T)0.5 * (Zm.x - Z.x));
    }
    __syncthreads();
    const LineLayout Ly(2 * hs, hs, plane, 1, hs, g.fd_2hs, g.fd_hs);
    cplx<T> *out = smem_fft<T, false, true>(oth, res, Ly, g.py, twy);
    cplx<T> *spec = reinterpret_cast<cplx<T> *>(S.spec);
    for (int e = threadIdx.x; e < 2 * plane; e += blockDim.x) {
      const int c = udiv(e, g.fd_plane), rem = e - c * plane;
      spec[(2 * p + c) * g.S + (long long)x * plane + rem] = out[e];
    }
  }
}

template <typename T, typename TF, int EPI, int PT>
__global__ void __launch_bounds__(PT, PLANE_MIN_BLOCKS(PT))
    yzinv_kernel(Grid<T> g, const SlotDev<TF> *__restrict__ tab, SlotList list, ExtIO<TF> io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<TF>)];
  const int ny = g.ny, nz = g.nz, hz = g.hz, hs = g.hs;
  const long long V = g.V;
  const int cap = padded_len(ny * (nz + 2));
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + cap;
  cplx<T> *twy = bufB + cap;
  cplx<T> *twz = twy + ny;
  __shared__ __align__(8) uint64_t tile_bar;
  load_table<T>(twy, g.twy, ny);
  load_table<T>(twz, g.twz, nz);
  bulk_barrier_init(&tile_bar);
  unsigned tile_phase = 0;
  const int per = items_plane(g);
  const int n_items = list_items(list, per);
  const int plane = ny * hs;
  int staged = -1;  // slot whose descriptor sdesc holds
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int k = udiv(item, g.fd_it_plane);
    const int local = item - k * per;
    const SlotDev<TF> &S = stage_slot<TF>(tab, list.ids[k], sdesc, staged);
    if (EPI_SKIPS_DONE(EPI) && slot_done(S.st)) continue;
    const int x = udiv(local, g.fd_3);
    const int p = local - 3 * x;
    const cplx<T> *spec = reinterpret_cast<const cplx<T> *>(S.spec);
    __syncthreads();
    constexpr long long E = sizeof(cplx<T>);
    // the pair's two half-spectrum planes, one bulk copy each where 16-byte aligned
    if (bulk_copy_rows(bufA, spec + (2 * p) * g.S + (long long)x * plane, 2, 1,
                       (unsigned)(plane * E), plane * E, 0, g.S * E, 0, &tile_bar)) {
      bulk_barrier_wait(&tile_bar, tile_phase);
      tile_phase ^= 1;
    } else {
      for (int e = threadIdx.x; e < 2 * plane; e += blockDim.x) {
        const int c = udiv(e, g.fd_plane), rem = e - c * plane;
        cp_async_elem<T>(&bufA[e], &spec[(2 * p + c) * g.S + (long long)x * plane + rem]);
      }
      cp_async_wait_all();
    }
    __syncthreads();
    const LineLayout Ly(2 * hs, hs, plane, 1, hs, g.fd_2hs, g.fd_hs);
    cplx<T> *res = smem_fft<T, true, true>(bufA, bufB, Ly, g.py, twy);
    cplx<T> *oth = (res == bufA) ? bufB : bufA;
    // full z lines of Z = A + iB from the stored halves (Hermitian in z)
    for (int e = threadIdx.x; e < ny * nz; e += blockDim.x) {
      const int y = udiv(e, g.fd_nz), kk = e - y * nz;
      const bool low = (kk < hz);
      const int ks = low ? kk : nz - kk;
      const bool nyq = 2 * ks == nz;  // the unstored Nyquist column is zero
      const cplx<T> A = nyq ? mk<T>((T)0, (T)0) : res[y * hs + ks];
      const cplx<T> B = nyq ? mk<T>((T)0, (T)0) : res[plane + y * hs + ks];
      oth[sidx<true>(e)] = low ? mk<T>(A.x - B.y, A.y + B.x) : mk<T>(A.x + B.y, B.x - A.y);
    }
    __syncthreads();
    const LineLayout Lz(ny, ny, 0, nz, 1, g.fd_ny, g.fd_ny);
    cplx<T> *fin = smem_fft<T, true, false, true>(oth, res, Lz, g.pz, twz);
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    plane_epilogue<T, TF, EPI>(S, io, V, (long long)x * ny * nz, ny * nz, p, fin, acc0);
    finish_inverse<TF, EPI>(S, acc0, acc1, acc2, local, per, red);
  }
}

// ---- cluster plane passes (planes that fit the shared memory of a block cluster) ---------
//
// C blocks (a thread-block cluster) share one (x plane, pair) item.  Block r transforms
// the R = ny / C rows y in [rR, rR + R) along z, and along y the Lq = 2 hs / C half-spectrum
// columns with c hs + kz in [r Lq, r Lq + Lq) (c: component 2p + c of the pair).  Between
// the two transforms each block stores its split half spectra straight into the owning
// block's shared memory (distributed shared memory: no round trip through HBM or L2), and
// the inverse does the same in reverse.  Two cluster barriers per item order the exchange:
// the first finds every block's free buffer free, the second finds the exchange complete.
// Every block of a cluster runs the same items and reaches every barrier, also for an item
// it skips; the buffer that takes the exchange follows from the stage count of the
// transform before it, not from whether the block ran it.
struct ClusterGeo {
  int C, R, Lq, cap;  // cluster size, rows and columns per block, elements per buffer
  FastDiv fd_R, fd_Lq;
};

// Elements of one buffer: R padded z lines, the split half spectra of R rows (2 R hs), or
// the Lq columns of ny points a block transforms along y.
__host__ __device__ inline int cplane_buf_elems(int ny, int nz, int hs, int C) {
  const int R = ny / C, Lq = 2 * hs / C;
  int n = padded_len(R * nz);
  n = n > 2 * R * hs ? n : 2 * R * hs;
  return n > ny * Lq ? n : ny * Lq;
}
template <typename T> inline size_t smem_cplane_bytes(int ny, int nz, int hs, int C) {
  return (2 * (size_t)cplane_buf_elems(ny, nz, hs, C) + ny + nz) * sizeof(cplx<T>);
}

// Blocks of PT = 1024 threads (one per SM), 512 (two per SM when their shared memory
// fits, so that one block's loads overlap the other's transforms) or 256, at most 64
// registers.
template <typename T, typename TF, int PRO, int PT>
__global__ void __launch_bounds__(PT, PLANE_MIN_BLOCKS(PT))
    zyfwd_cl_kernel(Grid<T> g, ClusterGeo cq, const SlotDev<TF> *__restrict__ tab,
                    SlotList list, ExtIO<TF> io) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<TF>)];
  cg::cluster_group cl = cg::this_cluster();
  const int C = cq.C, R = cq.R, Lq = cq.Lq;
  const int rank = (int)cl.block_rank();
  const int ny = g.ny, nz = g.nz, hs = g.hs;
  const long long V = g.V;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + cq.cap;
  cplx<T> *twy = bufB + cq.cap;
  cplx<T> *twz = twy + ny;
  load_table<T>(twy, g.twy, ny);
  load_table<T>(twz, g.twz, nz);
  // after the z transform the result is in bufA for an even stage count
  cplx<T> *res = (g.pz.nrad & 1) ? bufB : bufA;
  cplx<T> *oth = (g.pz.nrad & 1) ? bufA : bufB;
  const int per = items_plane(g);
  const int n_items = list_items(list, per);
  const int plane = ny * hs;
  const int y0 = rank * R;
  const int cown = (rank * Lq) / hs, k0 = rank * Lq - cown * hs;  // owned columns
  const int ncl = gridDim.x / C;
  int staged = -1;  // slot whose descriptor sdesc holds
  for (int item = blockIdx.x / C; item < n_items; item += ncl) {
    const int k = udiv(item, g.fd_it_plane);
    const int local = item - k * per;
    const SlotDev<TF> &S = stage_slot<TF>(tab, list.ids[k], sdesc, staged);
    const bool skip = skip_item<TF, PRO>(S);
    const int x = udiv(local, g.fd_3);
    const int p = local - 3 * x;
    if (!skip) {
      __syncthreads();
      plane_prologue<T, TF, PRO>(S, io, V, ((long long)x * ny + y0) * nz, R * nz, p, bufA);
      __syncthreads();
      const LineLayout Lz(R, R, 0, nz, 1, cq.fd_R, cq.fd_R);
      smem_fft<T, false, false, true>(bufA, bufB, Lz, g.pz, twz);
    }
    cl.sync();  // every block's z transform is done: its other buffer is free
    if (!skip) {
      // split the paired transform; column (c, kz) goes to block (c hs + kz) / Lq, which
      // holds it at [y][column - its first column]
      for (int e = threadIdx.x; e < R * hs; e += blockDim.x) {
        const int yl = udiv(e, g.fd_hs), kk = e - yl * hs;
        const cplx<T> Z = res[sidx<true>(yl * nz + kk)];
        const cplx<T> Zm = res[sidx<true>(yl * nz + (kk == 0 ? 0 : nz - kk))];
        const cplx<T> A = mk<T>((T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y));
        const cplx<T> B = mk<T>((T)0.5 * (Z.y + Zm.y), (T)0.5 * (Zm.x - Z.x));
        const int qa = udiv(kk, cq.fd_Lq), qb = udiv(hs + kk, cq.fd_Lq);
        cplx<T> *da = cl.map_shared_rank(oth, qa);
        cplx<T> *db = cl.map_shared_rank(oth, qb);
        da[(y0 + yl) * Lq + (kk - qa * Lq)] = A;
        db[(y0 + yl) * Lq + (hs + kk - qb * Lq)] = B;
      }
    }
    cl.sync();  // the owned columns are complete
    if (!skip) {
      const LineLayout Ly(Lq, Lq, 0, 1, Lq, cq.fd_Lq, cq.fd_Lq);
      cplx<T> *out = smem_fft<T, false, true>(oth, res, Ly, g.py, twy);
      cplx<T> *spec = reinterpret_cast<cplx<T> *>(S.spec) + (2 * p + cown) * g.S +
                      (long long)x * plane + k0;
      for (int e = threadIdx.x; e < ny * Lq; e += blockDim.x) {
        const int y = udiv(e, cq.fd_Lq), kl = e - y * Lq;
        spec[(long long)y * hs + kl] = out[e];
      }
    }
  }
}

template <typename T, typename TF, int EPI, int PT>
__global__ void __launch_bounds__(PT, PLANE_MIN_BLOCKS(PT))
    yzinv_cl_kernel(Grid<T> g, ClusterGeo cq, const SlotDev<TF> *__restrict__ tab,
                    SlotList list, ExtIO<TF> io) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ __align__(16) unsigned char sdesc[sizeof(SlotDev<TF>)];
  cg::cluster_group cl = cg::this_cluster();
  const int C = cq.C, R = cq.R, Lq = cq.Lq;
  const int rank = (int)cl.block_rank();
  const int ny = g.ny, nz = g.nz, hz = g.hz, hs = g.hs;
  const long long V = g.V;
  cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *bufB = bufA + cq.cap;
  cplx<T> *twy = bufB + cq.cap;
  cplx<T> *twz = twy + ny;
  __shared__ __align__(8) uint64_t tile_bar;
  load_table<T>(twy, g.twy, ny);
  load_table<T>(twz, g.twz, nz);
  bulk_barrier_init(&tile_bar);
  unsigned tile_phase = 0;
  // after the y transform the result is in bufA for an even stage count
  cplx<T> *res = (g.py.nrad & 1) ? bufB : bufA;
  cplx<T> *oth = (g.py.nrad & 1) ? bufA : bufB;
  const int per = items_plane(g);
  const int n_items = list_items(list, per);
  const int plane = ny * hs;
  const int y0 = rank * R;
  const int lam0 = rank * Lq;
  const int cown = lam0 / hs, k0 = lam0 - cown * hs;
  const int ncl = gridDim.x / C;
  int staged = -1;  // slot whose descriptor sdesc holds
  for (int item = blockIdx.x / C; item < n_items; item += ncl) {
    const int k = udiv(item, g.fd_it_plane);
    const int local = item - k * per;
    const SlotDev<TF> &S = stage_slot<TF>(tab, list.ids[k], sdesc, staged);
    const bool skip = EPI_SKIPS_DONE(EPI) && slot_done(S.st);
    const int x = udiv(local, g.fd_3);
    const int p = local - 3 * x;
    if (!skip) {
      const cplx<T> *spec = reinterpret_cast<const cplx<T> *>(S.spec) + (2 * p + cown) * g.S +
                            (long long)x * plane + k0;
      __syncthreads();
      constexpr long long E = sizeof(cplx<T>);
      // the block's Lq columns of every row y: one bulk copy per row where 16-byte aligned
      if (bulk_copy_rows(bufA, spec, ny, 1, (unsigned)(Lq * E), Lq * E, 0, hs * E, 0,
                         &tile_bar)) {
        bulk_barrier_wait(&tile_bar, tile_phase);
        tile_phase ^= 1;
      } else {
        for (int e = threadIdx.x; e < ny * Lq; e += blockDim.x) {
          const int y = udiv(e, cq.fd_Lq), kl = e - y * Lq;
          cp_async_elem<T>(&bufA[e], &spec[(long long)y * hs + kl]);
        }
        cp_async_wait_all();
      }
      __syncthreads();
      const LineLayout Ly(Lq, Lq, 0, 1, Lq, cq.fd_Lq, cq.fd_Lq);
      smem_fft<T, true, true>(bufA, bufB, Ly, g.py, twy);
    }
    cl.sync();  // every block's y transform is done: its other buffer is free
    if (!skip) {
      // row y goes to block y / R, which holds the half spectra of its rows at [c][y][kz]
      for (int e = threadIdx.x; e < ny * Lq; e += blockDim.x) {
        const int y = udiv(e, cq.fd_Lq), kl = e - y * Lq;
        const int q = udiv(y, cq.fd_R), yl = y - q * R;
        const int lam = lam0 + kl;
        const int c = lam >= hs ? 1 : 0, kk = lam - c * hs;
        cplx<T> *d = cl.map_shared_rank(oth, q);
        d[(c * R + yl) * hs + kk] = res[e];
      }
    }
    cl.sync();  // the owned rows are complete
    if (!skip) {
      // full z lines of Z = A + iB from the stored halves (Hermitian in z)
      for (int e = threadIdx.x; e < R * nz; e += blockDim.x) {
        const int yl = udiv(e, g.fd_nz), kk = e - yl * nz;
        const bool low = (kk < hz);
        const int ks = low ? kk : nz - kk;
        const bool nyq = 2 * ks == nz;  // the unstored Nyquist column is zero
        const cplx<T> A = nyq ? mk<T>((T)0, (T)0) : oth[yl * hs + ks];
        const cplx<T> B = nyq ? mk<T>((T)0, (T)0) : oth[(R + yl) * hs + ks];
        res[sidx<true>(e)] = low ? mk<T>(A.x - B.y, A.y + B.x) : mk<T>(A.x + B.y, B.x - A.y);
      }
      __syncthreads();
      const LineLayout Lz(R, R, 0, nz, 1, cq.fd_R, cq.fd_R);
      cplx<T> *fin = smem_fft<T, true, false, true>(res, oth, Lz, g.pz, twz);
      double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
      plane_epilogue<T, TF, EPI>(S, io, V, ((long long)x * ny + y0) * nz, R * nz, p, fin, acc0);
      finish_inverse<TF, EPI>(S, acc0, acc1, acc2, local * C + rank, per * C, red);
    }
  }
}
