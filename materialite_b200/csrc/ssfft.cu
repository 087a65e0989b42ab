// libssfft: C ABI and host driver of the sm_100a SmallStrainFFT solver.
//
// The Newton / Krylov structure follows materialite's SmallStrainFFT.run
// (materialite/models/small_strain_fft/small_strain_fft.py:106-246): one call to
// ssfft_step is one load increment (strain guess, Newton loop, MINRES per Newton
// iteration, convergence tests); the time loop, adaptive dt and output collection stay
// with the caller, as in the reference.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ssfft.h"
#include "common.cuh"
#include "constitutive.cuh"
#include "fft.cuh"
#include "fields.cuh"
#include "krylov.cuh"
#include "projector.cuh"

// ---------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(SSFFT_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

#define CKR(expr)          \
  do {                     \
    int r_ = (expr);       \
    if (r_ != 0) return r_; \
  } while (0)

// NVTX range for the lifetime of a scope (visible in Nsight tools; free otherwise).
struct NvtxScope {
  explicit NvtxScope(const char *name) { nvtxRangePushA(name); }
  ~NvtxScope() { nvtxRangePop(); }
};

extern "C" const char *ssfft_last_error(void) { return g_last_error.c_str(); }

// Lets other translation units of the library report through ssfft_last_error().
__attribute__((visibility("hidden"))) int ssfft_internal_fail(int code, const std::string &msg) {
  return fail(code, msg);
}

// ---------------------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------------------
enum { TK_INIT = 0, TK_ZINV, TK_UPD, TK_SPARE, TK_NORMS, TK_TSUM, TK_COUNT };
#define MAX_PARTIAL_BLOCKS 65536

struct ssfft_handle {
  ssfft_config cfg;
  bool fp64;
  size_t rs;  // sizeof(real)
  cudaStream_t stream;
  int nx, ny, nz, hz;
  long long V, S;
  AxisPlan px, py, pz;
  int lz, ky, kx;
  size_t smem_z, smem_y, smem_x;
  int red_blocks;  // grid of grid-stride reduction kernels
  void *tw[2][3], *tn[2][3];  // [0]: float, [1]: double tables per axis
  // fields (planar, real type)
  void *eps, *sig, *sig_old, *eps_old, *dfl, *guess, *b;
  void *kr[7];  // Krylov vectors: u (two), y', three directions, x
  void *spec;
  // microstructure
  bool micro_set;
  bool voxel_mode;
  // capacities of the microstructure-dependent buffers (bytes; grow-only on rebinding)
  size_t cap_rm, cap_ktab, cap_stage;
  int cap_nslip;
  bool have_phase_buf, have_gid_buf, have_kvox;
  double *stage;  // device staging for point-major read-back
  int n_orient, n_gid;
  int32_t *orient, *phase, *gid;
  double *rm_tab;
  void *ktab, *kvox, *kvox_old;
  PhaseParams hparams[SSFFT_MAX_PHASES];
  bool phase_set[SSFFT_MAX_PHASES];
  PhaseParams *dparams;
  bool any_evp;   // a phase with plastic state (crystal EVP or J2): voxel tangents, state buffers
  bool any_j2;
  int nslip_max;  // planes of the slip-state buffers (J2 uses plane 0 for the yield stress)
  // EVP state
  double *g_buf[2];
  int g_cur;
  double *g_old, *ep_old, *ep_trial, *Gam_old, *Gam_trial, *gam_old, *gam_trial;
  // reductions / scalars
  double *partials;
  unsigned int *tickets;
  double *results;   // [0..13] norms, [16..36] tangent sum, [40] max|b|
  MinresState *st;
  int *citers, *cfail;
  double *h_results;  // pinned mirror
  MinresState *h_st;
  int *h_cint;
  cudaGraphExec_t krylov_graph;  // one Krylov chunk, captured on first use
  bool use_graphs;
  bool use_plane;                 // plane-fused z/y passes where they fit
  cudaGraphExec_t krylov_loop;    // while node over the chunk: the whole solve on device
  bool use_device_loop;
  int chunk_kernels;              // kernels launched by one chunk
  cudaEvent_t ev0, ev1, tev0, tev1;
  cudaEvent_t pev[9];
  double last_step_seconds;
  long long launches;
};

// ---------------------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------------------
static bool make_plan(int n, AxisPlan &p) { return make_axis_plan(n, p); }

template <typename T> static std::vector<T> twiddles(int n) {
  std::vector<T> tw(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * k / n;
    tw[2 * k] = (T)std::cos(a);
    tw[2 * k + 1] = (T)std::sin(a);
  }
  return tw;
}

// tan(pi f) for numpy's fftfreq ordering (first `count` entries).
template <typename T> static std::vector<T> tan_table(int n, int count) {
  std::vector<T> t(count);
  for (int k = 0; k < count; ++k) {
    const int kk = (k < (n + 1) / 2) ? k : k - n;  // fftfreq index
    const long double f = (long double)kk / n;
    if (2 * kk == -n || 2 * kk == n)
      t[k] = (T)0;  // Nyquist plane: operator is zeroed there
    else
      t[k] = (T)std::tan(3.14159265358979323846264338327950288L * f);
  }
  return t;
}

template <typename T> static Grid<T> make_grid(const ssfft_handle *h) {
  Grid<T> g;
  g.nx = h->nx;
  g.ny = h->ny;
  g.nz = h->nz;
  g.hz = h->hz;
  g.V = h->V;
  g.S = h->S;
  g.px = h->px;
  g.py = h->py;
  g.pz = h->pz;
  const int p = sizeof(T) == 8 ? 1 : 0;
  g.twx = (const cplx<T> *)h->tw[p][0];
  g.twy = (const cplx<T> *)h->tw[p][1];
  g.twz = (const cplx<T> *)h->tw[p][2];
  g.tanx = (const T *)h->tn[p][0];
  g.tany = (const T *)h->tn[p][1];
  g.tanz = (const T *)h->tn[p][2];
  g.scale = (T)(1.0 / (double)h->V);
  for (int c = 0; c < 6; ++c) g.mask[c] = (T)((h->cfg.stress_mask[c] != 0.0) ? 1.0 : 0.0);
  g.lz = h->lz;
  g.ky = h->ky;
  g.kx = h->kx;
  grid_divisors(g);
  return g;
}

static int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Per-point phase index of the current binding (null: every point is phase 0).
static const int32_t *phase_ptr(const ssfft_handle *h) {
  return h->have_phase_buf ? h->phase : nullptr;
}

static size_t field_bytes(const ssfft_handle *h, int planes) {
  return (size_t)planes * (size_t)h->V * h->rs;
}

template <typename F> static int smem_attr(F f, int m) {
  CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
  return 0;
}

template <typename T, typename TF, int PT> static int plane_attrs(int m) {
  CKR(smem_attr(zyfwd_kernel<T, TF, PRO_INPUT, PT>, m));
  CKR(smem_attr(zyfwd_kernel<T, TF, PRO_RESIDUAL, PT>, m));
  CKR(smem_attr(yzinv_kernel<T, TF, EPI_STORE, PT>, m));
  CKR(smem_attr(yzinv_kernel<T, TF, EPI_RESIDUAL, PT>, m));
  if (sizeof(T) == sizeof(TF)) {
    CKR(smem_attr(zyfwd_kernel<T, T, PRO_TANGENT_TABLE, PT>, m));
    CKR(smem_attr(zyfwd_kernel<T, T, PRO_TANGENT_VOXEL, PT>, m));
    CKR(smem_attr(yzinv_kernel<T, T, EPI_MINRES, PT>, m));
  }
  return 0;
}

// Opt every shared-memory-hungry kernel instantiation into up to `smax` bytes.
template <typename T, typename TF> static int set_kernel_attrs(size_t smax) {
  const int m = (int)smax;
  CKR(smem_attr(zfwd_kernel<T, TF, PRO_INPUT>, m));
  CKR(smem_attr(zfwd_kernel<T, TF, PRO_RESIDUAL>, m));
  CKR(smem_attr(ypass_kernel<T, false>, m));
  CKR(smem_attr(ypass_kernel<T, true>, m));
  CKR(smem_attr(xpass_kernel<T>, m));
  CKR(smem_attr(zinv_kernel<T, TF, EPI_STORE>, m));
  CKR(smem_attr(zinv_kernel<T, TF, EPI_RESIDUAL>, m));
  CKR((plane_attrs<T, TF, 512>(m)));
  CKR((plane_attrs<T, TF, 1024>(m)));
  if (sizeof(T) == sizeof(TF)) {
    CKR(smem_attr(constitutive_kernel<T>, (int)constitutive_smem_bytes(SSFFT_MAX_PHASES)));
    CKR(smem_attr(zfwd_kernel<T, T, PRO_TANGENT_TABLE>, m));
    CKR(smem_attr(zfwd_kernel<T, T, PRO_TANGENT_VOXEL>, m));
    CKR(smem_attr(zinv_kernel<T, T, EPI_MINRES>, m));
  }
  return 0;
}

static const size_t SMEM_LIMIT = 200 * 1024;

static int plan_tiles(ssfft_handle *h) {
  // tiles are sized for double-precision transforms, which both modes run (the mixed mode
  // computes its equilibrium residual in double)
  h->lz = std::max(1, std::min(32, 2048 / (3 * h->nz)));
  h->lz = (int)std::min<long long>(h->lz, (long long)h->nx * h->ny);
  h->ky = std::min(h->hz, 16);
  while (h->ky > 1 && smem_y_bytes<double>(h->ky, h->ny) > 96 * 1024) h->ky /= 2;
  // kz columns per x-pass block: 8 (64-byte runs of the spectrum per x), 4 on grids of up
  // to 64 points along x, where 8 would leave about two blocks per SM
  h->kx = std::min(h->hz, h->nx <= 64 ? 4 : 8);
  while (h->kx > 1 && smem_x_bytes<double>(h->kx, h->nx) > 100 * 1024) h->kx /= 2;
  h->smem_z = smem_z_bytes<double>(h->lz, h->nz);
  h->smem_y = smem_y_bytes<double>(h->ky, h->ny);
  h->smem_x = smem_x_bytes<double>(h->kx, h->nx);
  if (h->smem_z > SMEM_LIMIT || h->smem_y > SMEM_LIMIT || h->smem_x > SMEM_LIMIT)
    return fail(SSFFT_E_UNSUPPORTED, "grid too large for the shared-memory FFT passes");
  if (div_up((long long)h->nx * h->ny, h->lz) > MAX_PARTIAL_BLOCKS)
    return fail(SSFFT_E_UNSUPPORTED, "grid too large for the reduction partials");
  return 0;
}

// ---------------------------------------------------------------------------------------
// projector launches
// ---------------------------------------------------------------------------------------
// The plane-fused passes apply when a padded yz plane pair fits in shared memory.
#define PLANE_SMEM_LIMIT (200 * 1024)
template <typename T> static bool plane_ok(const ssfft_handle *h) {
  return h->use_plane && smem_plane_bytes<T>(h->ny, h->nz) <= PLANE_SMEM_LIMIT;
}

// Threads of a plane block: 1024 when a single block fits an SM (228 KB of shared memory),
// else 512.
template <typename T> static int plane_threads(const ssfft_handle *h) {
  return smem_plane_bytes<T>(h->ny, h->nz) > 113 * 1024 ? 1024 : 512;
}

// Launch the passes of one projection.  ev (optional, 6 events) is recorded before the
// first pass and after each of the five pass slots z-fwd, y-fwd, x, y-inv, z-inv; with
// the plane-fused passes the y slots are empty (zero time).
template <typename T, typename TF, int PRO, int EPI>
static int launch_projector(ssfft_handle *h, const ProArgs<TF> &pa, const EpiArgs<TF> &ea,
                            const MinresState *st, cudaEvent_t *ev = nullptr) {
  Grid<T> g = make_grid<T>(h);
  cplx<T> *spec = (cplx<T> *)h->spec;
  auto rec = [&](int k) {
    if (ev) cudaEventRecord(ev[k], h->stream);
  };
  const size_t sx = smem_x_bytes<T>(h->kx, h->nx);
  rec(0);
  if (plane_ok<T>(h)) {
    const size_t sp = smem_plane_bytes<T>(h->ny, h->nz);
    const int pt = plane_threads<T>(h);
    if (pt == 1024)
      zyfwd_kernel<T, TF, PRO, 1024><<<dim3(h->nx, 3), 1024, sp, h->stream>>>(g, pa, spec);
    else
      zyfwd_kernel<T, TF, PRO, 512><<<dim3(h->nx, 3), 512, sp, h->stream>>>(g, pa, spec);
    rec(1);
    rec(2);
    xpass_kernel<T><<<dim3(div_up(h->hz, h->kx), h->ny), XPASS_THREADS, sx, h->stream>>>(
        g, spec, st);
    rec(3);
    rec(4);
    if (pt == 1024)
      yzinv_kernel<T, TF, EPI, 1024><<<dim3(h->nx, 3), 1024, sp, h->stream>>>(g, ea, spec);
    else
      yzinv_kernel<T, TF, EPI, 512><<<dim3(h->nx, 3), 512, sp, h->stream>>>(g, ea, spec);
    rec(5);
    h->launches += 3;
  } else {
    const size_t sz = smem_z_bytes<T>(h->lz, h->nz);
    const size_t sy = smem_y_bytes<T>(h->ky, h->ny);
    const int nzb = div_up((long long)h->nx * h->ny, h->lz);
    zfwd_kernel<T, TF, PRO><<<nzb, SSFFT_THREADS, sz, h->stream>>>(g, pa, spec);
    rec(1);
    ypass_kernel<T, false><<<dim3(div_up(h->hz, h->ky), h->nx, 6), SSFFT_THREADS, sy,
                             h->stream>>>(g, spec, st);
    rec(2);
    xpass_kernel<T><<<dim3(div_up(h->hz, h->kx), h->ny), XPASS_THREADS, sx, h->stream>>>(
        g, spec, st);
    rec(3);
    ypass_kernel<T, true><<<dim3(div_up(h->hz, h->ky), h->nx, 6), SSFFT_THREADS, sy,
                            h->stream>>>(g, spec, st);
    rec(4);
    zinv_kernel<T, TF, EPI><<<nzb, SSFFT_THREADS, sz, h->stream>>>(g, ea, spec);
    rec(5);
    h->launches += 5;
  }
  CK(cudaGetLastError());
  return 0;
}

template <typename T> static TangentRef<T> tangent_ref(const ssfft_handle *h) {
  TangentRef<T> K;
  K.ktab = (const T *)h->ktab;
  K.gid = h->gid;
  K.kvox = h->voxel_mode ? (const T *)h->kvox : nullptr;
  K.V = h->V;
  return K;
}

// b = P(Sbar - sigma) into h->b, max|b| into results[40].  The transform always runs in
// double: in the mixed mode the float stress field is read and b is stored as float, but
// the equilibrium residual and its norm are double-precision quantities.
template <typename T> static int residual(ssfft_handle *h, const double sbar[6]) {
  ProArgs<T> pa{};
  pa.in = (const T *)h->sig;
  for (int c = 0; c < 6; ++c) pa.sbar[c] = sbar[c];
  EpiArgs<T> ea{};
  ea.out = (T *)h->b;
  ea.partials = h->partials;
  ea.ticket = h->tickets + TK_ZINV;
  ea.result = h->results + 40;
  return launch_projector<double, T, PRO_RESIDUAL, EPI_RESIDUAL>(h, pa, ea, nullptr);
}

// Mixed mode only: project a Newton correction back onto compatible strain fields with a
// double-precision transform (x <- Gamma-hat : x, an identity in exact arithmetic).  Float
// Krylov iterates pick up round-off in the null space of Gamma-hat K, which the
// equilibrium test cannot see; this removes it.
template <typename T> static int reproject(ssfft_handle *h, T *x) {
  ProArgs<T> pa{};
  pa.in = x;
  EpiArgs<T> ea{};
  ea.out = x;
  return launch_projector<double, T, PRO_INPUT, EPI_STORE>(h, pa, ea, nullptr);
}

// ---------------------------------------------------------------------------------------
// MINRES driver
// ---------------------------------------------------------------------------------------
// Krylov vectors of one solve (krylov.cuh).  At the start of iteration j, P holds u_{j-1},
// Q holds u_{j-2} (dead) and receives u_j from the forward pass, Y holds y' of iteration
// j-1; W1 and W2 are the two previous directions and W receives the new one.  After the
// iteration P and Q swap and the directions rotate (periods 2 and 3).  minres_init_kernel
// writes b into both P and Q, so the first iteration (no pending update) reads u_1 = b
// from either.
template <typename T> struct KrylovBufs {
  T *P, *Q, *Y, *W, *W1, *W2, *X;
  void advance() {
    std::swap(P, Q);
    T *old_w1 = W1;
    W1 = W2;
    W2 = W;
    W = old_w1;
  }
};

template <typename T> static KrylovBufs<T> krylov_bufs(ssfft_handle *h) {
  KrylovBufs<T> k;
  k.P = (T *)h->kr[0];
  k.Q = (T *)h->kr[1];
  k.W = (T *)h->kr[2];
  k.W1 = (T *)h->kr[3];
  k.W2 = (T *)h->kr[4];
  k.X = (T *)h->kr[5];
  k.Y = (T *)h->kr[6];
  return k;
}

// r1 = r2 = b, x = w = w2 = 0 (in the names of the first iteration) and the MINRES state.
template <typename T>
static int launch_minres_init(ssfft_handle *h, const KrylovBufs<T> &k, double rtol,
                              long long maxiter) {
  minres_init_kernel<T><<<h->red_blocks, SSFFT_THREADS, 0, h->stream>>>(
      (const T *)h->b, k.P, k.Q, k.X, k.W, k.W2, 6 * h->V, h->st, rtol, maxiter, h->partials,
      h->tickets + TK_INIT);
  h->launches += 1;
  CK(cudaGetLastError());
  return 0;
}

// One MINRES iteration: the projector passes with the pending vector update in the
// forward prologue and the scalar recurrence in the inverse epilogue.  ev as in
// launch_projector.
template <typename T>
static int krylov_iteration(ssfft_handle *h, const KrylovBufs<T> &k, cudaEvent_t *ev = nullptr) {
  ProArgs<T> pa{};
  pa.in = k.P;
  pa.gid = h->gid;
  pa.ktab = (const T *)h->ktab;
  pa.kvox = (const T *)h->kvox;
  pa.st = h->st;
  pa.y = k.Y;
  pa.unew = k.Q;
  pa.w1 = k.W1;
  pa.w2 = k.W2;
  pa.wout = k.W;
  pa.x = k.X;
  pa.partials = h->partials;
  pa.ticket = h->tickets + TK_UPD;
  EpiArgs<T> ea{};
  ea.out = k.Y;
  ea.r1 = k.P;
  ea.r2 = k.Q;
  ea.st = h->st;
  ea.partials = h->partials;
  ea.ticket = h->tickets + TK_ZINV;
  if (h->voxel_mode)
    return launch_projector<T, T, PRO_TANGENT_VOXEL, EPI_MINRES>(h, pa, ea, h->st, ev);
  return launch_projector<T, T, PRO_TANGENT_TABLE, EPI_MINRES>(h, pa, ea, h->st, ev);
}

#define KRYLOV_CHUNK 6  // a multiple of both buffer-rotation periods (2 and 3)
#define MIXED_RTOL_FLOOR 1.0e-6

template <typename T>
static int finish_minres(ssfft_handle *h, long long *iters, T **xout, T *X) {
  if (h->h_st->istop == 9) return fail(SSFFT_E_NAN, "non-finite value in the Krylov solve");
  *iters = h->h_st->itn;
  *xout = X;
  return 0;
}

template <typename T> static int run_minres(ssfft_handle *h, long long *iters, T **xout) {
  NvtxScope range("ssfft_minres");
  const long long n = 6 * h->V;
  const KrylovBufs<T> k0 = krylov_bufs<T>(h);
  // scipy's default limit is 5 x ndof; past KRYLOV_ITERATION_CAP a solve is not going to
  // converge in any useful time, so every limit is clamped there (the device-side loop
  // must end by itself)
  const long long maxiter = std::min<long long>(
      h->cfg.max_krylov_iterations > 0 ? h->cfg.max_krylov_iterations : 5 * n,
      KRYLOV_ITERATION_CAP);
  // float Krylov vectors cannot resolve relative residuals much below 1e-6
  const double rtol = h->fp64 ? h->cfg.linear_solver_tolerance
                              : std::max(h->cfg.linear_solver_tolerance, MIXED_RTOL_FLOOR);
  CKR(launch_minres_init<T>(h, k0, rtol, maxiter));
  T *X = k0.X;
  // One chunk of KRYLOV_CHUNK iterations.  A chunk of 6 leaves the buffer roles where they
  // started, so the same launch sequence (and a CUDA graph captured from it) repeats until
  // the solve is done.  Kernels return at once when the device state says done.
  auto chunk = [&]() -> int {
    KrylovBufs<T> k = k0;
    for (int i = 0; i < KRYLOV_CHUNK; ++i) {
      CKR(krylov_iteration<T>(h, k));
      k.advance();
    }
    return 0;
  };
  if (h->use_device_loop) {
    // the whole Krylov loop on the device: a while node whose body is one chunk followed
    // by minres_continue_kernel, which sets the loop condition from the MINRES state
    if (!h->krylov_loop) {
      const long long launches_before = h->launches;
      cudaGraph_t graph = nullptr;
      CK(cudaGraphCreate(&graph, 0));
      cudaGraphConditionalHandle cond;
      cudaError_t e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault);
      cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
      np.conditional.handle = cond;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &np);
      cudaGraph_t body = (e == cudaSuccess) ? np.conditional.phGraph_out[0] : nullptr;
      if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(SSFFT_E_CUDA, std::string("device loop setup: ") + cudaGetErrorString(e));
      }
      const int rc = chunk();
      minres_continue_kernel<<<1, 32, 0, h->stream>>>(h->st, cond);
      cudaGraph_t captured = nullptr;
      e = cudaStreamEndCapture(h->stream, &captured);
      h->chunk_kernels = (int)(h->launches - launches_before);
      h->launches = launches_before;
      if (rc || e != cudaSuccess) {
        cudaGraphDestroy(graph);
        if (rc) return rc;
        return fail(SSFFT_E_CUDA, std::string("device loop capture: ") + cudaGetErrorString(e));
      }
      e = cudaGraphInstantiate(&h->krylov_loop, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        h->krylov_loop = nullptr;
        return fail(SSFFT_E_CUDA, std::string("device loop instantiate: ") + cudaGetErrorString(e));
      }
    }
    CK(cudaGraphLaunch(h->krylov_loop, h->stream));
    CK(cudaMemcpyAsync(h->h_st, h->st, sizeof(MinresState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const long long chunks = (h->h_st->itn + KRYLOV_CHUNK - 1) / KRYLOV_CHUNK;
    h->launches += std::max(1LL, chunks) * (h->chunk_kernels + 1);
    return finish_minres(h, iters, xout, X);
  }
  if (h->use_graphs && !h->krylov_graph) {
    cudaGraph_t graph = nullptr;
    const long long launches_before = h->launches;  // capture records, it does not launch
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = chunk();
    h->chunk_kernels = (int)(h->launches - launches_before);
    h->launches = launches_before;
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return fail(SSFFT_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&h->krylov_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      h->krylov_graph = nullptr;
      return fail(SSFFT_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
  }
  for (int round = 0;; ++round) {
    // two chunks before the first look at the state: most solves need more than one
    for (int c = 0; c < (round == 0 ? 2 : 1); ++c) {
      if (h->krylov_graph) {
        CK(cudaGraphLaunch(h->krylov_graph, h->stream));
        h->launches += h->chunk_kernels;
      } else {
        CKR(chunk());
      }
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_st, h->st, sizeof(MinresState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->h_st->done) break;
  }
  return finish_minres(h, iters, xout, X);
}

// ---------------------------------------------------------------------------------------
// constitutive call
// ---------------------------------------------------------------------------------------
// Launch the constitutive update; its iteration count and failure flag reach the host
// with the next norms() read-back (no synchronisation here).
template <typename T>
static int constitutive(ssfft_handle *h, double dt) {
  CK(cudaMemsetAsync(h->citers, 0, 4 * sizeof(int), h->stream));
  ConstArgs<T> a{};
  a.V = h->V;
  a.eps = (const T *)h->eps;
  a.guess = (const T *)h->guess;
  a.sig = (T *)h->sig;
  a.kvox = h->voxel_mode ? (T *)h->kvox : nullptr;
  a.ktab = (const T *)h->ktab;
  a.gid = h->gid;
  a.phase = phase_ptr(h);
  a.orient = h->orient;
  a.params = h->dparams;
  a.n_params = 1;
  for (int p = 0; p < SSFFT_MAX_PHASES; ++p)
    if (h->phase_set[p]) a.n_params = p + 1;
  a.rm_tab = h->rm_tab;
  if (h->any_evp) {
    a.g_in = h->g_buf[h->g_cur];
    a.g_out = h->g_buf[1 - h->g_cur];
    a.g_old = h->g_old;
    a.ep_old = h->ep_old;
    a.ep_trial = h->ep_trial;
    a.Gam_old = h->Gam_old;
    a.Gam_trial = h->Gam_trial;
    a.gam_old = h->gam_old;
    a.gam_trial = h->gam_trial;
  }
  a.dt = dt;
  a.max_iters = h->citers;
  a.failed = h->cfail;
  a.j2 = h->citers + 2;
  if (h->any_j2) {
    const int nb = std::max(1, std::min(div_up(h->V, SSFFT_THREADS), 148 * 8));
    j2_count_kernel<T><<<nb, SSFFT_THREADS, 0, h->stream>>>(a, h->citers + 2);
    h->launches += 1;
    CK(cudaGetLastError());
  }
  const int blocks = std::max(1, std::min(div_up(h->V, CONST_THREADS), 148 * 16));
  constitutive_kernel<T><<<blocks, CONST_THREADS, constitutive_smem_bytes(a.n_params),
                           h->stream>>>(a);
  h->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_cint, h->citers, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  return 0;
}

// After the read-back that follows constitutive(): iteration count and failure flag; a
// successful update makes its slip resistances the current trial state.
static void constitutive_result(ssfft_handle *h, int *iters, int *failed) {
  *iters = h->h_cint[0];
  *failed = h->h_cint[1];
  if (!*failed && h->any_evp) h->g_cur = 1 - h->g_cur;
}

template <typename T> static int norms(ssfft_handle *h, const T *dx) {
  // about four points per thread: the fourteen block partials are cheap to combine
  const int nb = std::max(1, std::min(div_up(h->V, 4 * SSFFT_THREADS), 2 * 148));
  newton_norms_kernel<T><<<nb, SSFFT_THREADS, 0, h->stream>>>(
      h->V, (const T *)h->sig, (const T *)h->sig_old, (const T *)h->eps, dx, tangent_ref<T>(h),
      h->partials, h->tickets + TK_NORMS, h->results);
  h->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_results, h->results, 48 * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

static double mean_von_mises(const double *sums, long long V) {
  double m[6];
  for (int c = 0; c < 6; ++c) m[c] = sums[c] / (double)V;
  const double tr3 = (m[0] + m[1] + m[2]) / 3.0;
  double s = 0.0;
  for (int c = 0; c < 6; ++c) {
    const double d = (c < 3) ? m[c] - tr3 : m[c];
    s += d * d;
  }
  return std::sqrt(s) * std::sqrt(1.5);
}

// 6x6 inverse by Gauss-Jordan with partial pivoting (host, double).
static bool inv6(const double *A, double *Ainv) {
  double a[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 12; ++j) a[i][j] = (j < 6) ? A[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
    if (a[p][c] == 0.0) return false;
    if (p != c)
      for (int j = 0; j < 12; ++j) std::swap(a[p][j], a[c][j]);
    const double d = a[c][c];
    for (int j = 0; j < 12; ++j) a[c][j] /= d;
    for (int r = 0; r < 6; ++r)
      if (r != c) {
        const double f = a[r][c];
        if (f != 0.0)
          for (int j = 0; j < 12; ++j) a[r][j] -= f * a[c][j];
      }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ainv[i * 6 + j] = a[i][j + 6];
  return true;
}

template <typename T> static void restore_tangent(ssfft_handle *h) {
  if (h->voxel_mode)
    cudaMemcpyAsync(h->kvox, h->kvox_old, field_bytes(h, 21), cudaMemcpyDeviceToDevice,
                    h->stream);
}

// One load increment (small_strain_fft.py:106-211).
template <typename T> static int step_impl(ssfft_handle *h, const ssfft_step_in *in,
                                           ssfft_step_out *out) {
  NvtxScope range("ssfft_step");
  memset(out, 0, sizeof(*out));
  CK(cudaEventRecord(h->ev0, h->stream));
  const long long V = h->V;
  const int eb = std::max(1, std::min(div_up(V, SSFFT_THREADS), 148 * 16));
  StepVec sv{};
  for (int c = 0; c < 6; ++c) {
    sv.dEbar[c] = in->strain_increment[c];
    sv.dS[c] = in->stress_increment[c];
    sv.corr[c] = 0.0;
  }
  bool all_small = true;
  for (int c = 0; c < 6; ++c)
    if (!(in->stress_increment[c] < 1.0e-14)) all_small = false;
  if (!all_small) {  // strain += tangent.mean().inv @ stress_increment
    tangent_sum_kernel<T><<<h->red_blocks, SSFFT_THREADS, 0, h->stream>>>(
        V, tangent_ref<T>(h), h->partials, h->tickets + TK_TSUM, h->results + 16);
    h->launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_results, h->results, 48 * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double Km[36], Ki[36];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) Km[i * 6 + j] = h->h_results[16 + sym_idx(i, j)] / (double)V;
    if (!inv6(Km, Ki)) return fail(SSFFT_E_INVALID, "mean tangent is singular");
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 6; ++j) acc += Ki[i * 6 + j] * in->stress_increment[j];
      sv.corr[i] = acc;
    }
  }
  strain_guess_kernel<T><<<eb, SSFFT_THREADS, 0, h->stream>>>(
      V, sv, in->time_step_id == 0, in->reset_fluctuation, (const T *)h->eps_old, (T *)h->dfl,
      (const T *)h->sig_old, (T *)h->eps, (T *)h->guess, tangent_ref<T>(h));
  h->launches += 1;
  CK(cudaGetLastError());

  const double gtol = h->cfg.global_tolerance;
  const double stol = h->cfg.strain_correction_tolerance;
  const int max_newton = h->cfg.max_newton_iterations > 0 ? h->cfg.max_newton_iterations : 100;
  bool converged = false;
  int it = 0, max_cit = 0;
  double eq_err = 0.0, mvm = 0.0, s_err = 0.0;
  long long kits_total = 0;
  int solves = 0;
  while (!converged) {
    ++it;
    if (it == 1) {
      int cit, cf;
      CKR(constitutive<T>(h, in->dt));
      CKR(residual<T>(h, in->mean_applied_stress));
      CKR(norms<T>(h, nullptr));
      constitutive_result(h, &cit, &cf);
      if (cf) {
        restore_tangent<T>(h);
        out->constitutive_failed = 1;
        break;
      }
      max_cit = std::max(max_cit, cit);
      mvm = mean_von_mises(h->h_results, V);
      eq_err = h->h_results[40] / mvm;
      CK(cudaMemcpyAsync(h->guess, h->sig, field_bytes(h, 6), cudaMemcpyDeviceToDevice,
                         h->stream));
    }
    const double old_eq = std::max(eq_err, gtol);
    long long kits = 0;
    T *X = nullptr;
    CKR(run_minres<T>(h, &kits, &X));
    kits_total += kits;
    ++solves;
    if (!h->fp64) CKR(reproject<T>(h, X));
    update_strain_kernel<T><<<eb, SSFFT_THREADS, 0, h->stream>>>(6 * V, X, (T *)h->eps,
                                                                  (T *)h->dfl);
    h->launches += 1;
    int cit, cf;
    CKR(constitutive<T>(h, in->dt));
    CKR(residual<T>(h, in->mean_applied_stress));
    CKR(norms<T>(h, X));
    constitutive_result(h, &cit, &cf);
    if (cf) {
      restore_tangent<T>(h);
      out->constitutive_failed = 1;
      break;
    }
    max_cit = std::max(max_cit, cit);
    mvm = mean_von_mises(h->h_results, V);
    const double tavg = (in->summed_von_mises_stress + mvm) / (double)(in->time_step_id + 1);
    if (mvm / tavg < 1.0e-12) mvm = tavg;
    eq_err = h->h_results[40] / mvm;
    double max_ds = h->h_results[12] * std::sqrt(1.5);
    if (max_ds / mvm < 1.0e-12) max_ds = mvm;
    s_err = h->h_results[13] / max_ds;
    const double p_err = s_err * eq_err / old_eq;
    if (eq_err < gtol && (s_err < stol || p_err < stol || in->time_step_id == 0 || eq_err < 1e-8))
      converged = true;
    CK(cudaMemcpyAsync(h->guess, h->sig, field_bytes(h, 6), cudaMemcpyDeviceToDevice,
                       h->stream));
    if (it == max_newton && !converged) break;
  }
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_step_seconds = ms * 1e-3;
  out->converged = converged ? 1 : 0;
  out->newton_iterations = it;
  out->max_constitutive_iterations = max_cit;
  out->krylov_iterations = kits_total;
  out->linear_solves = solves;
  out->equilibrium_error = eq_err;
  out->scaled_strain_error = s_err;
  out->mean_von_mises_stress = mvm;
  for (int c = 0; c < 6; ++c) {
    out->mean_stress[c] = h->h_results[c] / (double)V;
    out->mean_strain[c] = h->h_results[6 + c] / (double)V;
  }
  if (!std::isfinite(eq_err) && converged) out->status = SSFFT_E_NAN;
  return 0;
}

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
static void free_handle(ssfft_handle *h) {
  if (!h) return;
  for (int p = 0; p < 2; ++p)
    for (int a = 0; a < 3; ++a) {
      if (h->tw[p][a]) cudaFree(h->tw[p][a]);
      if (h->tn[p][a]) cudaFree(h->tn[p][a]);
    }
  void *ptrs[] = {h->eps, h->sig,
                  h->sig_old, h->eps_old, h->dfl, h->guess, h->b, h->kr[0], h->kr[1],
                  h->kr[2], h->kr[3], h->kr[4], h->kr[5], h->kr[6], h->spec, h->orient, h->phase,
                  h->gid, h->rm_tab, h->ktab, h->kvox, h->kvox_old, h->dparams,
                  h->g_buf[0], h->g_buf[1], h->g_old, h->ep_old, h->ep_trial, h->Gam_old,
                  h->Gam_trial, h->gam_old, h->gam_trial, h->partials, h->tickets,
                  h->results, h->st, h->citers, h->stage};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (h->krylov_graph) cudaGraphExecDestroy(h->krylov_graph);
  if (h->krylov_loop) cudaGraphExecDestroy(h->krylov_loop);
  if (h->h_results) cudaFreeHost(h->h_results);
  if (h->h_st) cudaFreeHost(h->h_st);
  if (h->h_cint) cudaFreeHost(h->h_cint);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->tev0) cudaEventDestroy(h->tev0);
  if (h->tev1) cudaEventDestroy(h->tev1);
  for (int k = 0; k < 9; ++k)
    if (h->pev[k]) cudaEventDestroy(h->pev[k]);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

#define ALLOC(ptr, bytes)                                                           \
  do {                                                                              \
    cudaError_t e_ = cudaMalloc((void **)&(ptr), (bytes));                          \
    if (e_ != cudaSuccess) {                                                        \
      cudaGetLastError();                                                           \
      return fail(SSFFT_E_NOMEM, std::string("cudaMalloc ") + #ptr + ": " +         \
                                     cudaGetErrorString(e_));                       \
    }                                                                               \
  } while (0)

static int validate_config(const ssfft_config *cfg) {
  if (!cfg) return fail(SSFFT_E_INVALID, "null config");
  for (int d = 0; d < 3; ++d)
    if (cfg->n[d] < 1 || cfg->n[d] > 1024) return fail(SSFFT_E_UNSUPPORTED, "grid size out of range");
  if (cfg->precision != SSFFT_FP64 && cfg->precision != SSFFT_MIXED)
    return fail(SSFFT_E_INVALID, "precision must be SSFFT_FP64 or SSFFT_MIXED");
  for (int c = 0; c < 6; ++c)
    if (cfg->stress_mask[c] != 0.0 && cfg->stress_mask[c] != 1.0)
      return fail(SSFFT_E_INVALID, "stress mask can only have zeros and ones");
  AxisPlan p;
  for (int d = 0; d < 3; ++d)
    if (!make_plan(cfg->n[d], p))
      return fail(SSFFT_E_UNSUPPORTED, "grid size has a prime factor above 32");
  return 0;
}

extern "C" int ssfft_estimate_bytes(const ssfft_config *cfg, int any_evp, int n_slip,
                                    size_t *bytes) {
  CKR(validate_config(cfg));
  const size_t V = (size_t)cfg->n[0] * cfg->n[1] * cfg->n[2];
  const size_t rs = cfg->precision == SSFFT_FP64 ? 8 : 4;
  const size_t S = (size_t)cfg->n[0] * cfg->n[1] * (cfg->n[2] / 2 + 1);
  size_t b = 14 * 6 * V * rs + 6 * S * 16 + 3 * V * 4;
  if (any_evp) b += 2 * 21 * V * rs + (5 * (size_t)n_slip + 12 + 2) * V * 8;
  b += (size_t)MAX_PARTIAL_BLOCKS * 21 * 8 + (1 << 20);
  *bytes = b;
  return 0;
}

extern "C" int ssfft_create(const ssfft_config *cfg, ssfft_handle **out) {
  if (!out) return fail(SSFFT_E_INVALID, "null output pointer");
  *out = nullptr;
  CKR(validate_config(cfg));
  CK(cudaSetDevice(cfg->device));
  ssfft_handle *h = new ssfft_handle();
  memset((void *)h, 0, sizeof(ssfft_handle));
  h->cfg = *cfg;
  h->fp64 = cfg->precision == SSFFT_FP64;
  h->rs = h->fp64 ? 8 : 4;
  h->nx = cfg->n[0];
  h->ny = cfg->n[1];
  h->nz = cfg->n[2];
  h->hz = h->nz / 2 + 1;
  h->V = (long long)h->nx * h->ny * h->nz;
  h->S = (long long)h->nx * h->ny * h->hz;
  make_plan(h->nx, h->px);
  make_plan(h->ny, h->py);
  make_plan(h->nz, h->pz);
  int rc = plan_tiles(h);
  if (rc) {
    free_handle(h);
    return rc;
  }
  h->red_blocks = std::max(1, std::min(div_up(6 * h->V, SSFFT_THREADS), 148 * 8));
  {
    const char *ng = getenv("SSFFT_NO_GRAPHS");
    h->use_graphs = !(ng && ng[0] == '1');
    const char *np = getenv("SSFFT_NO_PLANE");
    h->use_plane = !(np && np[0] == '1');
    const char *nl = getenv("SSFFT_NO_DEVICE_LOOP");
    h->use_device_loop = h->use_graphs && !(nl && nl[0] == '1');
  }
  auto body = [&]() -> int {
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    CK(cudaEventCreate(&h->tev0));
    CK(cudaEventCreate(&h->tev1));
    for (int k = 0; k < 9; ++k) CK(cudaEventCreate(&h->pev[k]));
    // FFT tables: float ones for the mixed-mode Krylov transforms, double ones for every
    // double-precision transform (all transforms of the FP64 mode, residual and
    // re-projection of the mixed mode)
    const int dims[3] = {h->nx, h->ny, h->nz};
    const int tcount[3] = {h->nx, h->ny, h->hz};
    for (int p = (h->fp64 ? 1 : 0); p < 2; ++p)
      for (int a = 0; a < 3; ++a) {
        const size_t es = p ? 8 : 4;
        ALLOC(h->tw[p][a], (size_t)dims[a] * 2 * es);
        ALLOC(h->tn[p][a], (size_t)tcount[a] * es);
        if (p) {
          auto tw = twiddles<double>(dims[a]);
          auto tn = tan_table<double>(dims[a], tcount[a]);
          CK(cudaMemcpyAsync(h->tw[p][a], tw.data(), tw.size() * es, cudaMemcpyHostToDevice, h->stream));
          CK(cudaMemcpyAsync(h->tn[p][a], tn.data(), tn.size() * es, cudaMemcpyHostToDevice, h->stream));
        } else {
          auto tw = twiddles<float>(dims[a]);
          auto tn = tan_table<float>(dims[a], tcount[a]);
          CK(cudaMemcpyAsync(h->tw[p][a], tw.data(), tw.size() * es, cudaMemcpyHostToDevice, h->stream));
          CK(cudaMemcpyAsync(h->tn[p][a], tn.data(), tn.size() * es, cudaMemcpyHostToDevice, h->stream));
        }
      }
    CKR((set_kernel_attrs<double, double>(SMEM_LIMIT)));
    CKR((set_kernel_attrs<float, float>(SMEM_LIMIT)));
    CKR((set_kernel_attrs<double, float>(SMEM_LIMIT)));
    void **fields[] = {&h->eps, &h->sig, &h->sig_old, &h->eps_old, &h->dfl, &h->guess, &h->b,
                       &h->kr[0], &h->kr[1], &h->kr[2], &h->kr[3], &h->kr[4], &h->kr[5],
                       &h->kr[6]};
    for (void **f : fields) {
      ALLOC(*f, field_bytes(h, 6));
      CK(cudaMemsetAsync(*f, 0, field_bytes(h, 6), h->stream));
    }
    ALLOC(h->spec, (size_t)6 * h->S * 16);  // sized for double-precision transforms
    ALLOC(h->partials, (size_t)MAX_PARTIAL_BLOCKS * 21 * sizeof(double));
    ALLOC(h->tickets, 16 * sizeof(unsigned int));
    CK(cudaMemsetAsync(h->tickets, 0, 16 * sizeof(unsigned int), h->stream));
    ALLOC(h->results, 64 * sizeof(double));
    CK(cudaMemsetAsync(h->results, 0, 64 * sizeof(double), h->stream));
    ALLOC(h->st, sizeof(MinresState));
    ALLOC(h->citers, 4 * sizeof(int));
    ALLOC(h->dparams, SSFFT_MAX_PHASES * sizeof(PhaseParams));
    CK(cudaMallocHost((void **)&h->h_results, 64 * sizeof(double)));
    CK(cudaMallocHost((void **)&h->h_st, sizeof(MinresState)));
    CK(cudaMallocHost((void **)&h->h_cint, 4 * sizeof(int)));
    h->cfail = h->citers + 1;
    // every upload and clear above is ordered on the handle's stream (a non-blocking
    // stream is not ordered with the legacy default stream that cudaMemcpy uses)
    CK(cudaStreamSynchronize(h->stream));
    return 0;
  };
  rc = body();
  if (rc) {
    free_handle(h);
    return rc;
  }
  *out = h;
  return 0;
}

extern "C" int ssfft_destroy(ssfft_handle *h) {
  if (!h) return 0;
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_handle(h);
  return 0;
}

static int check_phase(ssfft_handle *h, int phase) {
  if (!h) return fail(SSFFT_E_INVALID, "null handle");
  if (phase < 0 || phase >= SSFFT_MAX_PHASES) return fail(SSFFT_E_INVALID, "phase index out of range");
  return 0;
}

extern "C" int ssfft_set_phase_elastic(ssfft_handle *h, int phase, const double stiffness[36]) {
  CKR(check_phase(h, phase));
  PhaseParams &P = h->hparams[phase];
  memset(&P, 0, sizeof(P));
  P.kind = PHASE_ELASTIC;
  memcpy(P.C, stiffness, 36 * sizeof(double));
  P.latent = 1.0;
  h->phase_set[phase] = true;
  return 0;
}

extern "C" int ssfft_set_phase_evp(ssfft_handle *h, int phase, const double stiffness[36],
                                   int n_slip, const double *schmid, double reference_slip_rate,
                                   double rate_exponent, double slip_resistance, int hardening,
                                   const double *hardening_props, int n_props,
                                   double latent_ratio) {
  CKR(check_phase(h, phase));
  if (n_slip < 1 || n_slip > SSFFT_MAX_SLIP)
    return fail(SSFFT_E_UNSUPPORTED, "number of slip systems must be 1..12");
  if (hardening < 0 || hardening > 3) return fail(SSFFT_E_INVALID, "unknown hardening law");
  if (n_props < 0 || n_props > 4) return fail(SSFFT_E_INVALID, "at most 4 hardening properties");
  PhaseParams &P = h->hparams[phase];
  memset(&P, 0, sizeof(P));
  P.kind = PHASE_EVP;
  P.nslip = n_slip;
  P.hardening = hardening;
  memcpy(P.C, stiffness, 36 * sizeof(double));
  if (!inv6(P.C, P.Cinv)) return fail(SSFFT_E_INVALID, "EVP stiffness is singular");
  // the packed M uses the upper triangle of C^-1; symmetrise against round-off
  for (int i = 0; i < 6; ++i)
    for (int j = i + 1; j < 6; ++j) {
      const double s = 0.5 * (P.Cinv[i * 6 + j] + P.Cinv[j * 6 + i]);
      P.Cinv[i * 6 + j] = P.Cinv[j * 6 + i] = s;
    }
  memcpy(P.P, schmid, (size_t)n_slip * 6 * sizeof(double));
  P.gdot0 = reference_slip_rate;
  P.n = rate_exponent;
  P.g0 = slip_resistance;
  P.latent = latent_ratio;
  for (int k = 0; k < n_props; ++k) P.props[k] = hardening_props[k];
  // directional modulus along x: 1 / (C^-1)_00 (elastic_viscoplastic.py:32-34)
  P.E_ref = 1.0 / P.Cinv[0];
  h->phase_set[phase] = true;
  return 0;
}

extern "C" int ssfft_set_phase_j2(ssfft_handle *h, int phase, double modulus,
                                  double shear_modulus, double yield_stress, int hardening,
                                  const double *hardening_props, int n_props) {
  CKR(check_phase(h, phase));
  if (hardening < 0 || hardening > 3) return fail(SSFFT_E_INVALID, "unknown hardening law");
  if (n_props < 0 || n_props > 4) return fail(SSFFT_E_INVALID, "at most 4 hardening properties");
  if (n_props > 0 && !hardening_props) return fail(SSFFT_E_INVALID, "null hardening properties");
  const double E = modulus, G = shear_modulus;
  if (!(G > 0.0) || !(E > 0.0) || 3.0 * G - E == 0.0)
    return fail(SSFFT_E_INVALID, "J2 moduli must be positive with 3G != E");
  PhaseParams &P = h->hparams[phase];
  memset(&P, 0, sizeof(P));
  P.kind = PHASE_J2;
  P.nslip = 1;
  P.hardening = hardening;
  // Order4SymmetricTensor.from_isotropic_constants (tensor.py:1453-1467), Mandel
  const double L = G * (E - 2.0 * G) / (3.0 * G - E);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P.C[i * 6 + j] = (i == j) ? L + 2.0 * G : L;
  for (int i = 3; i < 6; ++i) P.C[i * 6 + i] = 2.0 * G;
  P.shear = G;
  P.bulk = G * E / (3.0 * (3.0 * G - E));  // isotropic_elastic_plastic.py:28-30
  P.g0 = yield_stress;
  P.latent = 1.0;
  for (int k = 0; k < n_props; ++k) P.props[k] = hardening_props[k];
  P.E_ref = E;
  h->phase_set[phase] = true;
  return 0;
}

template <typename T> static void build_ktab(const ssfft_handle *h, const std::vector<double> &Rm,
                                             const std::vector<int> &gid_orient,
                                             const std::vector<int> &gid_phase,
                                             std::vector<T> &tab) {
  const int n = (int)gid_orient.size();
  tab.assign((size_t)n * 21, (T)0);
  for (int g = 0; g < n; ++g) {
    const double *R = &Rm[(size_t)gid_orient[g] * 36];
    const double *C = h->hparams[gid_phase[g]].C;
    double CR[36];
    for (int i = 0; i < 6; ++i)
      for (int b = 0; b < 6; ++b) {
        double acc = 0.0;
        for (int j = 0; j < 6; ++j) acc += C[i * 6 + j] * R[j * 6 + b];
        CR[i * 6 + b] = acc;
      }
    for (int a = 0; a < 6; ++a)
      for (int b = a; b < 6; ++b) {
        double acc = 0.0;
        for (int i = 0; i < 6; ++i) acc += R[i * 6 + a] * CR[i * 6 + b];
        tab[(size_t)g * 21 + sym_idx(a, b)] = (T)acc;
      }
  }
}

// Mandel form of a rotation (materialite/tensor.py:1668-1700).
static void rotation_mandel(const double *R, double *M) {
  const double r2 = SQRT2_D;
  auto r = [&](int i, int j) { return R[i * 3 + j]; };
  const int pr[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  for (int a = 0; a < 3; ++a) {
    for (int b = 0; b < 3; ++b) M[a * 6 + b] = r(a, b) * r(a, b);
    for (int s = 0; s < 3; ++s) M[a * 6 + 3 + s] = r2 * r(a, pr[s][0]) * r(a, pr[s][1]);
  }
  for (int s = 0; s < 3; ++s) {
    const int i = pr[s][0], j = pr[s][1];
    for (int b = 0; b < 3; ++b) M[(3 + s) * 6 + b] = r2 * r(i, b) * r(j, b);
    for (int t = 0; t < 3; ++t) {
      const int k = pr[t][0], l = pr[t][1];
      M[(3 + s) * 6 + 3 + t] = r(i, k) * r(j, l) + r(i, l) * r(j, k);
    }
  }
}

// (Re)allocate *p to hold `bytes` unless its capacity *cap already does.
static int ensure_buffer(void **p, size_t *cap, size_t bytes) {
  if (*p && *cap >= bytes) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(SSFFT_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  *cap = bytes;
  return 0;
}

static void drop_graph(ssfft_handle *h) {
  if (h->krylov_graph) {
    cudaGraphExecDestroy(h->krylov_graph);
    h->krylov_graph = nullptr;
  }
  if (h->krylov_loop) {
    cudaGraphExecDestroy(h->krylov_loop);
    h->krylov_loop = nullptr;
  }
}

extern "C" int ssfft_set_options(ssfft_handle *h, const ssfft_config *cfg) {
  if (!h || !cfg) return fail(SSFFT_E_INVALID, "null argument");
  CKR(validate_config(cfg));
  for (int d = 0; d < 3; ++d)
    if (cfg->n[d] != h->cfg.n[d]) return fail(SSFFT_E_INVALID, "grid size differs from the handle's");
  if (cfg->precision != h->cfg.precision)
    return fail(SSFFT_E_INVALID, "precision differs from the handle's");
  const int device = h->cfg.device;
  h->cfg = *cfg;
  h->cfg.device = device;
  drop_graph(h);  // the captured launches carry the stress mask
  return 0;
}

extern "C" int ssfft_set_microstructure(ssfft_handle *h, int n_orient, const double *rotations,
                                        const int32_t *orient_of_point,
                                        const int32_t *phase_of_point) {
  if (!h) return fail(SSFFT_E_INVALID, "null handle");
  if (n_orient < 1 || !rotations || !orient_of_point)
    return fail(SSFFT_E_INVALID, "rotations and orientation indices are required");
  CK(cudaSetDevice(h->cfg.device));
  const long long V = h->V;
  int max_phase = 0;
  for (long long v = 0; v < V; ++v) {
    const int o = orient_of_point[v];
    const int p = phase_of_point ? phase_of_point[v] : 0;
    if (o < 0 || o >= n_orient) return fail(SSFFT_E_INVALID, "orientation index out of range");
    if (p < 0 || p >= SSFFT_MAX_PHASES || !h->phase_set[p])
      return fail(SSFFT_E_INVALID, "point refers to an undefined phase");
    max_phase = std::max(max_phase, p);
  }
  h->any_evp = false;
  h->any_j2 = false;
  h->nslip_max = 0;
  for (int p = 0; p < SSFFT_MAX_PHASES; ++p) {
    if (!h->phase_set[p]) continue;
    if (h->hparams[p].kind == PHASE_EVP) {
      h->any_evp = true;
      h->nslip_max = std::max(h->nslip_max, h->hparams[p].nslip);
    } else if (h->hparams[p].kind == PHASE_J2) {
      h->any_evp = true;
      h->any_j2 = true;
      h->nslip_max = std::max(h->nslip_max, 1);
    }
  }
  // a handle may be rebound to a new microstructure (serving reuses handles): buffers of
  // the previous binding are kept when large enough, and the captured Krylov launches,
  // which carry their addresses, are dropped
  drop_graph(h);
  h->micro_set = false;
  h->voxel_mode = h->any_evp;
  h->n_orient = n_orient;
  std::vector<double> Rm((size_t)n_orient * 36);
  for (int o = 0; o < n_orient; ++o) rotation_mandel(rotations + (size_t)o * 9, &Rm[(size_t)o * 36]);
  CKR(ensure_buffer((void **)&h->rm_tab, &h->cap_rm, Rm.size() * sizeof(double)));
  CK(cudaMemcpyAsync(h->rm_tab, Rm.data(), Rm.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (!h->orient) ALLOC(h->orient, V * sizeof(int32_t));
  CK(cudaMemcpyAsync(h->orient, orient_of_point, V * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
  if (phase_of_point) {
    if (!h->phase) ALLOC(h->phase, V * sizeof(int32_t));
    CK(cudaMemcpyAsync(h->phase, phase_of_point, V * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
  }
  h->have_phase_buf = phase_of_point != nullptr;
  CK(cudaMemcpyAsync(h->dparams, h->hparams, sizeof(h->hparams), cudaMemcpyHostToDevice, h->stream));
  if (!h->voxel_mode) {
    // tangent table over the distinct (orientation, phase) pairs present
    std::vector<int> key_to_gid((size_t)n_orient * (max_phase + 1), -1);
    std::vector<int> g_or, g_ph;
    std::vector<int32_t> gid(V);
    for (long long v = 0; v < V; ++v) {
      const int o = orient_of_point[v], p = phase_of_point ? phase_of_point[v] : 0;
      int &slot = key_to_gid[(size_t)p * n_orient + o];
      if (slot < 0) {
        slot = (int)g_or.size();
        g_or.push_back(o);
        g_ph.push_back(p);
      }
      gid[v] = slot;
    }
    h->n_gid = (int)g_or.size();
    if (!h->gid) ALLOC(h->gid, V * sizeof(int32_t));
    CK(cudaMemcpyAsync(h->gid, gid.data(), V * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    if (h->fp64) {
      std::vector<double> tab;
      build_ktab<double>(h, Rm, g_or, g_ph, tab);
      CKR(ensure_buffer(&h->ktab, &h->cap_ktab, tab.size() * sizeof(double)));
      CK(cudaMemcpyAsync(h->ktab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    } else {
      std::vector<float> tab;
      build_ktab<float>(h, Rm, g_or, g_ph, tab);
      CKR(ensure_buffer(&h->ktab, &h->cap_ktab, tab.size() * sizeof(float)));
      CK(cudaMemcpyAsync(h->ktab, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    }
  } else {
    if (!h->kvox) {
      ALLOC(h->kvox, field_bytes(h, 21));
      ALLOC(h->kvox_old, field_bytes(h, 21));
    }
    const int S = h->nslip_max;
    if (h->cap_nslip < S) {
      double **bufs[] = {&h->g_buf[0], &h->g_buf[1], &h->g_old, &h->gam_old, &h->gam_trial};
      for (double **b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
      }
      for (double **b : bufs) ALLOC(*b, (size_t)S * V * 8);
      h->cap_nslip = S;
    }
    if (!h->ep_old) {
      ALLOC(h->ep_old, (size_t)6 * V * 8);
      ALLOC(h->ep_trial, (size_t)6 * V * 8);
      ALLOC(h->Gam_old, (size_t)V * 8);
      ALLOC(h->Gam_trial, (size_t)V * 8);
    }
  }
  h->micro_set = true;
  return ssfft_reset(h);
}

extern "C" int ssfft_reset(ssfft_handle *h) {
  if (!h || !h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  void *fields[] = {h->eps, h->sig, h->sig_old, h->eps_old, h->dfl, h->guess, h->b};
  for (void *f : fields) CK(cudaMemsetAsync(f, 0, field_bytes(h, 6), h->stream));
  const long long V = h->V;
  const int eb = std::max(1, std::min(div_up(V, SSFFT_THREADS), 148 * 16));
  if (h->voxel_mode) {
    if (h->fp64)
      init_kvox_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(
          V, phase_ptr(h), h->orient, h->dparams, h->rm_tab, (double *)h->kvox);
    else
      init_kvox_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(
          V, phase_ptr(h), h->orient, h->dparams, h->rm_tab, (float *)h->kvox);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->kvox_old, h->kvox, field_bytes(h, 21), cudaMemcpyDeviceToDevice,
                       h->stream));
  }
  if (h->any_evp) {
    const int S = h->nslip_max;
    evp_init_kernel<<<eb, SSFFT_THREADS, 0, h->stream>>>(V, S, phase_ptr(h), h->dparams,
                                                         h->g_buf[0], h->g_buf[1], h->g_old);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(h->gam_old, 0, (size_t)S * V * 8, h->stream));
    CK(cudaMemsetAsync(h->gam_trial, 0, (size_t)S * V * 8, h->stream));
    CK(cudaMemsetAsync(h->ep_old, 0, (size_t)6 * V * 8, h->stream));
    CK(cudaMemsetAsync(h->ep_trial, 0, (size_t)6 * V * 8, h->stream));
    CK(cudaMemsetAsync(h->Gam_old, 0, (size_t)V * 8, h->stream));
    CK(cudaMemsetAsync(h->Gam_trial, 0, (size_t)V * 8, h->stream));
    h->g_cur = 0;
  }
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

extern "C" int ssfft_step(ssfft_handle *h, const ssfft_step_in *in, ssfft_step_out *out) {
  if (!h || !in || !out) return fail(SSFFT_E_INVALID, "null argument");
  if (!h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  if (!(in->dt > 0.0)) return fail(SSFFT_E_INVALID, "time increment must be positive");
  CK(cudaSetDevice(h->cfg.device));
  return h->fp64 ? step_impl<double>(h, in, out) : step_impl<float>(h, in, out);
}

extern "C" int ssfft_commit(ssfft_handle *h, double fluctuation_scale) {
  if (!h || !h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  const size_t f6 = field_bytes(h, 6);
  CK(cudaMemcpyAsync(h->sig_old, h->sig, f6, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->eps_old, h->eps, f6, cudaMemcpyDeviceToDevice, h->stream));
  if (h->voxel_mode)
    CK(cudaMemcpyAsync(h->kvox_old, h->kvox, field_bytes(h, 21), cudaMemcpyDeviceToDevice,
                       h->stream));
  if (h->any_evp) {
    const size_t V = (size_t)h->V, S = (size_t)h->nslip_max;
    CK(cudaMemcpyAsync(h->g_old, h->g_buf[h->g_cur], S * V * 8, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->gam_old, h->gam_trial, S * V * 8, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->ep_old, h->ep_trial, 6 * V * 8, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->Gam_old, h->Gam_trial, V * 8, cudaMemcpyDeviceToDevice, h->stream));
  }
  return ssfft_scale_fluctuation(h, fluctuation_scale);
}

extern "C" int ssfft_scale_fluctuation(ssfft_handle *h, double factor) {
  if (!h || !h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  const long long n = 6 * h->V;
  const int eb = std::max(1, std::min(div_up(n, SSFFT_THREADS), 148 * 16));
  if (factor != 1.0) {
    if (h->fp64)
      scale_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(n, (double *)h->dfl, factor);
    else
      scale_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(n, (float *)h->dfl, factor);
    CK(cudaGetLastError());
  }
  return 0;  // ordered on the handle's stream; no host synchronisation needed
}

extern "C" int ssfft_num_slip(ssfft_handle *h) { return h ? h->nslip_max : 0; }

// The time loop of SmallStrainFFT.run (small_strain_fft.py:106-246) for a constant-rate
// schedule; mirrors materialite_b200/engine.py::solve without output collection.
extern "C" int ssfft_solve_constant_rates(ssfft_handle *h, const ssfft_rate_schedule *sc,
                                          ssfft_solve_out *out) {
  if (!h || !sc || !out) return fail(SSFFT_E_INVALID, "null argument");
  if (!h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  memset(out, 0, sizeof(*out));
  struct LaunchTally {  // kernel launches of this solve, on every return path
    ssfft_handle *h;
    ssfft_solve_out *o;
    long long l0;
    ~LaunchTally() { o->kernel_launches = h->launches - l0; }
  } tally{h, out, h->launches};
  const double *mask = h->cfg.stress_mask;
  double er[6], sr[6];
  for (int c = 0; c < 6; ++c) {  // apply_stress_mask (load_schedule.py:26-30)
    er[c] = sc->strain_rate[c] * (1.0 - mask[c]);
    sr[c] = sc->stress_rate[c] * mask[c];
  }
  double dt = sc->initial_time_increment > 0 ? sc->initial_time_increment
                                             : sc->end_time - sc->start_time;
  const double dt_max = sc->max_time_increment > 0 ? sc->max_time_increment : dt;
  const double dt_min = sc->min_time_increment > 0 ? sc->min_time_increment : 1.0e-9;
  const double t_tol = dt_min / 2.0;
  double t = sc->start_time, summed = 0.0, old_max_inc = 0.0;
  int step_id = 0;
  CKR(ssfft_reset(h));
  while (t < sc->end_time - t_tol) {
    ssfft_step_in in;
    memset(&in, 0, sizeof(in));
    int imax = 0;
    for (int c = 0; c < 6; ++c) {
      in.strain_increment[c] = er[c] * dt;
      in.stress_increment[c] = sr[c] * dt;
      in.mean_applied_stress[c] = sr[c] * (t + dt - sc->start_time);
      if (std::fabs(in.strain_increment[c]) > std::fabs(in.strain_increment[imax])) imax = c;
    }
    const double max_inc = in.strain_increment[imax];
    in.dt = dt;
    in.summed_von_mises_stress = summed;
    in.time_step_id = step_id;
    in.reset_fluctuation = (max_inc * old_max_inc < 0.0) ? 1 : 0;
    ssfft_step_out so;
    CKR(ssfft_step(h, &in, &so));
    out->newton_iterations += so.newton_iterations;
    out->krylov_iterations += so.krylov_iterations;
    out->device_seconds += h->last_step_seconds;
    if (so.status) {
      out->status = so.status;
      return fail(so.status, "non-finite equilibrium error");
    }
    if (so.converged) {
      CKR(ssfft_commit(h, 1.0));
      summed += so.mean_von_mises_stress;
      old_max_inc = max_inc;
      ++step_id;
      t += dt;
      const double fixed = sc->end_time - t;  // no output times in this loop
      double nd = std::min(dt_max, fixed);
      nd = std::min(nd, so.max_constitutive_iterations < 11 ? dt * 2.0 : dt);
      CKR(ssfft_scale_fluctuation(h, nd / dt));
      dt = nd;
      for (int c = 0; c < 6; ++c) {
        out->mean_stress[c] = so.mean_stress[c];
        out->mean_strain[c] = so.mean_strain[c];
      }
    } else {
      dt /= 2.0;
      ++out->cutbacks;
      CKR(ssfft_scale_fluctuation(h, 0.5));
      if (dt < dt_min) {
        out->status = SSFFT_E_INVALID;
        return fail(SSFFT_E_INVALID, "min time increment reached");
      }
    }
  }
  out->steps = step_id;
  return 0;
}

extern "C" int ssfft_get_field(ssfft_handle *h, int field, double *dst, int to_host) {
  if (!h || !dst) return fail(SSFFT_E_INVALID, "null argument");
  if (!h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  const long long V = h->V;
  int width = 6;
  const void *src = nullptr;
  bool is_double = false;
  switch (field) {
    case SSFFT_FIELD_STRESS: src = h->sig; break;
    case SSFFT_FIELD_STRAIN: src = h->eps; break;
    case SSFFT_FIELD_RESIDUAL: src = h->b; break;
    case SSFFT_FIELD_SLIP_RESISTANCES:
    case SSFFT_FIELD_SLIP_SHEAR_STRAINS:
    case SSFFT_FIELD_PLASTIC_STRAINS:
    case SSFFT_FIELD_YIELD_STRESSES:
    case SSFFT_FIELD_EQ_PLASTIC_STRAINS:
      if (!h->any_evp) return fail(SSFFT_E_INVALID, "no plastic phase in this solve");
      is_double = true;
      if (field == SSFFT_FIELD_SLIP_RESISTANCES) {
        src = h->g_buf[h->g_cur];
        width = h->nslip_max;
      } else if (field == SSFFT_FIELD_SLIP_SHEAR_STRAINS) {
        src = h->gam_trial;
        width = h->nslip_max;
      } else if (field == SSFFT_FIELD_YIELD_STRESSES) {
        src = h->g_buf[h->g_cur];  // plane 0
        width = 1;
      } else if (field == SSFFT_FIELD_EQ_PLASTIC_STRAINS) {
        src = h->Gam_trial;
        width = 1;
      }
      break;
    default: return fail(SSFFT_E_INVALID, "unknown field id");
  }
  double *ddst = dst;
  if (to_host) {
    CKR(ensure_buffer((void **)&h->stage, &h->cap_stage, (size_t)V * width * sizeof(double)));
    ddst = h->stage;
  }
  const int eb = std::max(1, std::min(div_up(V * width, SSFFT_THREADS), 148 * 16));
  if (field == SSFFT_FIELD_PLASTIC_STRAINS) {
    plastic_to_specimen_kernel<<<eb, SSFFT_THREADS, 0, h->stream>>>(
        V, h->ep_old, h->orient, h->rm_tab, phase_ptr(h), h->dparams, ddst);
  } else if (is_double || h->fp64) {
    to_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, width,
                                                                       (const double *)src, ddst);
  } else {
    to_point_major_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, width,
                                                                      (const float *)src, ddst);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && to_host) {
    e = cudaMemcpyAsync(dst, ddst, (size_t)V * width * sizeof(double), cudaMemcpyDeviceToHost,
                        h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(SSFFT_E_CUDA, std::string("get_field: ") + cudaGetErrorString(e));
  return 0;
}

template <typename T> static int apply_projection_dev(ssfft_handle *h, const T *in, T *out) {
  ProArgs<T> pa{};
  pa.in = in;
  EpiArgs<T> ea{};
  ea.out = out;
  return launch_projector<T, T, PRO_INPUT, EPI_STORE>(h, pa, ea, nullptr);
}

extern "C" int ssfft_apply_projection_device(ssfft_handle *h, const void *in_dev, void *out_dev) {
  if (!h || !in_dev || !out_dev) return fail(SSFFT_E_INVALID, "null argument");
  CK(cudaSetDevice(h->cfg.device));
  if (h->fp64)
    CKR(apply_projection_dev<double>(h, (const double *)in_dev, (double *)out_dev));
  else
    CKR(apply_projection_dev<float>(h, (const float *)in_dev, (float *)out_dev));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

extern "C" int ssfft_apply_projection(ssfft_handle *h, const double *in_host, double *out_host) {
  if (!h || !in_host || !out_host) return fail(SSFFT_E_INVALID, "null argument");
  CK(cudaSetDevice(h->cfg.device));
  const long long V = h->V;
  double *tmp = nullptr;
  ALLOC(tmp, (size_t)V * 6 * sizeof(double));
  const int eb = std::max(1, std::min(div_up(V * 6, SSFFT_THREADS), 148 * 16));
  int rc = 0;
  cudaError_t e = cudaMemcpyAsync(tmp, in_host, (size_t)V * 6 * sizeof(double),
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    if (h->fp64) {
      from_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, tmp, (double *)h->kr[0]);
      rc = apply_projection_dev<double>(h, (const double *)h->kr[0], (double *)h->kr[1]);
      to_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, 6, (const double *)h->kr[1], tmp);
    } else {
      from_point_major_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, tmp, (float *)h->kr[0]);
      rc = apply_projection_dev<float>(h, (const float *)h->kr[0], (float *)h->kr[1]);
      to_point_major_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, 6, (const float *)h->kr[1], tmp);
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && rc == 0)
    e = cudaMemcpyAsync(out_host, tmp, (size_t)V * 6 * sizeof(double), cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(SSFFT_E_CUDA, std::string("apply_projection: ") + cudaGetErrorString(e));
  return 0;
}

extern "C" int ssfft_stats(ssfft_handle *h, double *step_seconds, int64_t *kernel_launches) {
  if (!h) return fail(SSFFT_E_INVALID, "null handle");
  if (step_seconds) *step_seconds = h->last_step_seconds;
  if (kernel_launches) *kernel_launches = h->launches;
  return 0;
}

extern "C" int ssfft_timer(ssfft_handle *h, int start, double *seconds) {
  if (!h) return fail(SSFFT_E_INVALID, "null handle");
  CK(cudaSetDevice(h->cfg.device));
  if (start) {
    CK(cudaEventRecord(h->tev0, h->stream));
    return 0;
  }
  CK(cudaEventRecord(h->tev1, h->stream));
  CK(cudaEventSynchronize(h->tev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, h->tev0, h->tev1));
  if (seconds) *seconds = ms * 1e-3;
  return 0;
}

template <typename T> static int profile_impl(ssfft_handle *h, int reps, double *sec) {
  KrylovBufs<T> k = krylov_bufs<T>(h);
  // a live MINRES state on the residual of the current stress (never marked done); call
  // after a solve so that the stress field is not uniform
  const double zero[6] = {0, 0, 0, 0, 0, 0};
  CKR(residual<T>(h, zero));
  CKR(launch_minres_init<T>(h, k, 0.0, (long long)1 << 60));
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  NvtxScope range("ssfft_profile_krylov");  // only the timed Krylov kernels
  for (int r = 0; r < reps; ++r) {
    CKR(krylov_iteration<T>(h, k, h->pev));
    CK(cudaEventRecord(h->pev[6], h->stream));
    k.advance();
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(h->pev[6]));
    for (int i = 0; i < 6; ++i) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->pev[i], h->pev[i + 1]));
      acc[i] += ms * 1e-3;
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->pev[0], h->pev[6]));
    acc[7] += ms * 1e-3;
  }
  for (int i = 0; i < 8; ++i) sec[i] = acc[i] / reps;
  sec[6] = 0.0;
  return 0;
}

extern "C" int ssfft_profile_krylov(ssfft_handle *h, int reps, double seconds[8]) {
  if (!h || !seconds || reps < 1) return fail(SSFFT_E_INVALID, "bad argument");
  if (!h->micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  return h->fp64 ? profile_impl<double>(h, reps, seconds) : profile_impl<float>(h, reps, seconds);
}
