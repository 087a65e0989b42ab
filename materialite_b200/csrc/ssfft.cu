// libssfft: C ABI and host driver of the sm_100a SmallStrainFFT solver.
//
// The Newton / Krylov structure follows materialite's SmallStrainFFT.run
// (materialite/models/small_strain_fft/small_strain_fft.py:106-246): one call to
// ssfft_step is one load increment (strain guess, Newton loop, MINRES per Newton
// iteration, convergence tests); the time loop, adaptive dt and output collection stay
// with the caller, as in the reference.
//
// A handle is one slot (plan.cuh) driven from the host: the kernels are the batched ones
// of the serving groups (group.cuh), launched over a one-entry slot list, so a request
// solved through a handle and the same request solved inside a group run the same
// arithmetic.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "plan.cuh"

// ---------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

extern "C" const char *ssfft_last_error(void) { return g_last_error.c_str(); }

// Lets other translation units of the library report through ssfft_last_error().
__attribute__((visibility("hidden"))) int ssfft_internal_fail(int code, const std::string &msg) {
  return fail(code, msg);
}

// NVTX range for the lifetime of a scope (visible in Nsight tools; free otherwise).
struct NvtxScope {
  explicit NvtxScope(const char *name) { nvtxRangePushA(name); }
  ~NvtxScope() { nvtxRangePop(); }
};

// ---------------------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------------------
struct ssfft_handle {
  ssfft_config cfg;
  GridPlan plan;
  SlotBufs sb;
  cudaStream_t stream;
  void *dtab;       // SlotDev<T>[1] on the device
  int *dlist;       // {0, 1}: slot ids then count
  cudaGraphExec_t krylov_graph;  // one Krylov chunk, captured on first use
  cudaGraphExec_t krylov_loop;   // while node over the chunk: the whole solve on device
  bool use_graphs, use_device_loop;
  bool debug_minres;             // SSFFT_DEBUG_MINRES=1: each solve's stop reason to stderr
  int chunk_kernels;             // kernels launched by one chunk
  bool committed_view;           // last call was a commit: outputs read committed buffers
  double *h_results;             // pinned mirrors
  MinresState *h_st;
  int *h_cint;
  cudaEvent_t ev0, ev1, tev0, tev1;
  cudaEvent_t pev[9];
  double *stage;                 // device staging of point-major read-back
  size_t cap_stage;
  double last_step_seconds;
  long long launches;
};

static LaunchCtx ctx(ssfft_handle *h) {
  LaunchCtx c;
  c.p = &h->plan;
  c.list.ids = h->dlist;
  c.list.count = h->dlist + 1;
  c.cap = 1;
  c.stream = h->stream;
  c.launches = &h->launches;
  return c;
}

template <typename T> static const SlotDev<T> *dtab(ssfft_handle *h) {
  return (const SlotDev<T> *)h->dtab;
}

// The descriptor mirror to the device (stream-ordered; the mirror may change right after).
static int upload(ssfft_handle *h) {
  if (h->plan.fp64)
    CK(cudaMemcpyAsync(h->dtab, &h->sb.md, sizeof(SlotDev<double>), cudaMemcpyHostToDevice,
                       h->stream));
  else
    CK(cudaMemcpyAsync(h->dtab, &h->sb.mf, sizeof(SlotDev<float>), cudaMemcpyHostToDevice,
                       h->stream));
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

// ---------------------------------------------------------------------------------------
// MINRES driver
// ---------------------------------------------------------------------------------------
#define KRYLOV_CHUNK 6
#define MIXED_RTOL_FLOOR 1.0e-6

// The MINRES absolute floor per unit of mean von Mises stress (ssfft_config::krylov_floor).
static inline double krylov_atol_scale(const ssfft_config &cfg) {
  return cfg.krylov_floor > 0.0 ? cfg.krylov_floor * cfg.global_tolerance : 0.0;
}

template <typename T> static int run_minres(ssfft_handle *h, long long *iters) {
  NvtxScope range("ssfft_minres");
  const LaunchCtx c = ctx(h);
  const SlotDev<T> *tab = dtab<T>(h);
  const bool voxel = h->sb.voxel_mode;
  CKR(launch_minres_init<T>(c, tab));
  // One chunk of KRYLOV_CHUNK iterations; kernels return at once when the slot's MINRES
  // state says done, and the vector roles follow the state's iteration count.
  auto chunk = [&]() -> int {
    for (int i = 0; i < KRYLOV_CHUNK; ++i) CKR(launch_krylov_iteration<T>(c, tab, voxel));
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
      minres_continue_kernel<<<1, 32, 0, h->stream>>>(h->sb.st, cond);
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
    CK(cudaMemcpyAsync(h->h_st, h->sb.st, sizeof(MinresState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const long long chunks = (h->h_st->itn + KRYLOV_CHUNK - 1) / KRYLOV_CHUNK;
    h->launches += std::max(1LL, chunks) * (h->chunk_kernels + 1);
  } else {
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
      for (int k = 0; k < (round == 0 ? 2 : 1); ++k) {
        if (h->krylov_graph) {
          CK(cudaGraphLaunch(h->krylov_graph, h->stream));
          h->launches += h->chunk_kernels;
        } else {
          CKR(chunk());
        }
      }
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h->h_st, h->sb.st, sizeof(MinresState), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
      if (h->h_st->done) break;
      if (h->h_st->itn > KRYLOV_ITERATION_CAP) {
        // the host-polled loop stops at the same cap as the device loop
        h->h_st->istop = 6;
        break;
      }
    }
  }
  if (h->h_st->istop == 9) return fail(SSFFT_E_NAN, "non-finite value in the Krylov solve");
  *iters = h->h_st->itn;
  if (h->debug_minres) {
    const MinresState &s = *h->h_st;
    fprintf(stderr,
            "ssfft minres: itn %lld istop %d test1 %.3e test2 %.3e rnorm %.3e anorm %.3e "
            "ynorm %.3e beta1 %.3e acond %.3e\n",
            s.itn, s.istop, s.test1, s.test2, s.rnorm, s.anorm, s.ynorm, s.beta1,
            s.gmin > 0 ? s.gmax / s.gmin : 0.0);
  }
  return 0;
}

// ---------------------------------------------------------------------------------------
// Newton-level calls
// ---------------------------------------------------------------------------------------
// Constitutive update (its iteration count and failure flag reach the host with the next
// norms() read-back).  The new stress becomes the slot's latest stress (the next call's
// guess, small_strain_fft.py:169) by a role swap.
template <typename T> static int constitutive(ssfft_handle *h, double dt) {
  SlotDev<T> &m = mirror<T>(h->sb);
  m.dt = dt;
  CKR(upload(h));
  CK(cudaMemsetAsync(h->sb.citers, 0, 4 * sizeof(int), h->stream));
  CKR(launch_constitutive<T>(ctx(h), dtab<T>(h), h->sb.any_j2));
  CK(cudaMemcpyAsync(h->h_cint, h->sb.citers, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  std::swap(m.sig, m.sig_next);
  return upload(h);
}

// After the read-back that follows constitutive(): iteration count and failure flag; a
// successful update makes its slip resistances the current trial state.
template <typename T> static int constitutive_result(ssfft_handle *h, int *iters, int *failed) {
  *iters = h->h_cint[0];
  *failed = h->h_cint[1];
  if (!*failed && h->sb.any_evp) {
    SlotDev<T> &m = mirror<T>(h->sb);
    std::swap(m.g_in, m.g_out);
    CKR(upload(h));
  }
  return 0;
}

template <typename T> static int norms(ssfft_handle *h, bool with_dx) {
  SlotDev<T> &m = mirror<T>(h->sb);
  if (m.norms_dx != (with_dx ? 1 : 0)) {
    m.norms_dx = with_dx ? 1 : 0;
    CKR(upload(h));
  }
  CKR(launch_norms<T>(ctx(h), dtab<T>(h)));
  CK(cudaMemcpyAsync(h->h_results, h->sb.results, 48 * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

// One load increment (small_strain_fft.py:106-211).
template <typename T> static int step_impl(ssfft_handle *h, const ssfft_step_in *in,
                                           ssfft_step_out *out) {
  NvtxScope range("ssfft_step");
  memset(out, 0, sizeof(*out));
  h->committed_view = false;
  CK(cudaEventRecord(h->ev0, h->stream));
  const long long V = h->plan.V;
  const LaunchCtx c = ctx(h);
  SlotDev<T> &m = mirror<T>(h->sb);
  StepVec sv{};
  for (int k = 0; k < 6; ++k) {
    sv.dEbar[k] = in->strain_increment[k];
    sv.dS[k] = in->stress_increment[k];
    sv.corr[k] = 0.0;
    m.sbar[k] = in->mean_applied_stress[k];
  }
  bool all_small = true;
  for (int k = 0; k < 6; ++k)
    if (!(in->stress_increment[k] < 1.0e-14)) all_small = false;
  if (!all_small) {  // strain += tangent.mean().inv @ stress_increment
    CKR(upload(h));
    CKR(launch_tangent_sum<T>(c, dtab<T>(h)));
    CK(cudaMemcpyAsync(h->h_results, h->sb.results, 48 * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double Km[36], Ki[36];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) Km[i * 6 + j] = h->h_results[16 + sym_idx(i, j)] / (double)V;
    if (!inv6(Km, Ki)) return fail(SSFFT_E_INVALID, "mean tangent is singular");
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 6; ++j) acc += mul_rn(Ki[i * 6 + j], in->stress_increment[j]);
      sv.corr[i] = acc;
    }
  }
  m.sv = sv;
  m.first_step = in->time_step_id == 0 ? 1 : 0;
  m.reset_fluct = in->reset_fluctuation ? 1 : 0;
  m.fluct_scale = 1.0;  // the handle's caller scales through ssfft_scale_fluctuation
  // scipy's default limit is 5 x ndof; past KRYLOV_ITERATION_CAP a solve is not going to
  // converge in any useful time, so every limit is clamped there (the device-side loop
  // must end by itself)
  m.maxiter = std::min<long long>(
      h->cfg.max_krylov_iterations > 0 ? h->cfg.max_krylov_iterations : 30 * V,
      KRYLOV_ITERATION_CAP);
  // float Krylov vectors cannot resolve relative residuals much below 1e-6
  m.rtol = h->plan.fp64 ? h->cfg.linear_solver_tolerance
                        : std::max(h->cfg.linear_solver_tolerance, MIXED_RTOL_FLOOR);
  m.atol_scale = krylov_atol_scale(h->cfg);
  m.forcing = h->cfg.krylov_forcing;
  CKR(upload(h));
  CKR(launch_strain_guess<T>(c, dtab<T>(h)));

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
      CKR(launch_residual<T>(c, dtab<T>(h)));
      CKR(norms<T>(h, false));
      CKR(constitutive_result<T>(h, &cit, &cf));
      if (cf) {
        out->constitutive_failed = 1;
        break;
      }
      max_cit = std::max(max_cit, cit);
      mvm = mean_von_mises(h->h_results, V);
      eq_err = h->h_results[40] / mvm;
    }
    const double old_eq = std::max(eq_err, gtol);
    long long kits = 0;
    CKR(run_minres<T>(h, &kits));
    kits_total += kits;
    ++solves;
    if (!h->plan.fp64)
      CKR(launch_reproject_update<T>(c, dtab<T>(h)));
    else
      CKR(launch_update_strain<T>(c, dtab<T>(h)));
    int cit, cf;
    CKR(constitutive<T>(h, in->dt));
    CKR(launch_residual<T>(c, dtab<T>(h)));
    CKR(norms<T>(h, true));
    CKR(constitutive_result<T>(h, &cit, &cf));
    if (cf) {
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
  for (int k = 0; k < 6; ++k) {
    out->mean_stress[k] = h->h_results[k] / (double)V;
    out->mean_strain[k] = h->h_results[6 + k] / (double)V;
  }
  if (!std::isfinite(eq_err) && converged) out->status = SSFFT_E_NAN;
  return 0;
}

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
static void free_handle(ssfft_handle *h) {
  if (!h) return;
  plan_free(h->plan);
  slot_free(h->sb);
  if (h->dtab) cudaFree(h->dtab);
  if (h->dlist) cudaFree(h->dlist);
  if (h->stage) cudaFree(h->stage);
  drop_graph(h);
  if (h->h_results) cudaFreeHost(h->h_results);
  if (h->h_st) cudaFreeHost(h->h_st);
  if (h->h_cint) cudaFreeHost(h->h_cint);
  cudaEvent_t evs[] = {h->ev0, h->ev1, h->tev0, h->tev1};
  for (cudaEvent_t e : evs)
    if (e) cudaEventDestroy(e);
  for (int k = 0; k < 9; ++k)
    if (h->pev[k]) cudaEventDestroy(h->pev[k]);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

// Device bytes of one slot of this config (fields, spectrum, partials, tangent, plastic
// state), as slot_alloc and slot_bind allocate them.
extern "C" int ssfft_estimate_bytes(const ssfft_config *cfg, int any_evp, int n_slip,
                                    size_t *bytes) {
  CKR(validate_config(cfg));
  const size_t V = (size_t)cfg->n[0] * cfg->n[1] * cfg->n[2];
  const size_t rs = cfg->precision == SSFFT_FP64 ? 8 : 4;
  const size_t S = (size_t)cfg->n[0] * cfg->n[1] * (cfg->n[2] / 2 + 1);
  // strain and stress fields double in both precisions, the rest in the solve precision
  size_t b = 6 * 6 * V * 8 + 8 * 6 * V * rs + 6 * S * 16 + 3 * V * 4;
  if (any_evp) b += 2 * 21 * V * rs + (5 * (size_t)n_slip + 12 + 2) * V * 8;
  b += (size_t)21 * ((V + VEC_CHUNK - 1) / VEC_CHUNK + 1) * 8 + 3 * 3 * (size_t)cfg->n[0] * 8;
  b += (size_t)1 << 20;  // tables, scalars, orientation table
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
  {
    const char *ng = getenv("SSFFT_NO_GRAPHS");
    h->use_graphs = !(ng && ng[0] == '1');
    const char *nl = getenv("SSFFT_NO_DEVICE_LOOP");
    h->use_device_loop = h->use_graphs && !(nl && nl[0] == '1');
    const char *dm = getenv("SSFFT_DEBUG_MINRES");
    h->debug_minres = dm && dm[0] == '1';
  }
  auto body = [&]() -> int {
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CKR(plan_create(h->plan, cfg, h->stream));
    CKR(slot_alloc(h->sb, h->plan, h->stream));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    CK(cudaEventCreate(&h->tev0));
    CK(cudaEventCreate(&h->tev1));
    for (int k = 0; k < 9; ++k) CK(cudaEventCreate(&h->pev[k]));
    ALLOC(h->dtab, std::max(sizeof(SlotDev<double>), sizeof(SlotDev<float>)));
    ALLOC(h->dlist, 2 * sizeof(int));
    const int list[2] = {0, 1};
    CK(cudaMemcpyAsync(h->dlist, list, sizeof(list), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMallocHost((void **)&h->h_results, 64 * sizeof(double)));
    CK(cudaMallocHost((void **)&h->h_st, sizeof(MinresState)));
    CK(cudaMallocHost((void **)&h->h_cint, 4 * sizeof(int)));
    // every upload and clear above is ordered on the handle's stream (a non-blocking
    // stream is not ordered with the legacy default stream that cudaMemcpy uses)
    CK(cudaStreamSynchronize(h->stream));
    return 0;
  };
  int rc = body();
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

// Phase parameters (host side, shared with the serving groups).
static int phase_elastic(PhaseParams &P, const double stiffness[36]) {
  memset(&P, 0, sizeof(P));
  P.kind = PHASE_ELASTIC;
  memcpy(P.C, stiffness, 36 * sizeof(double));
  P.latent = 1.0;
  return 0;
}

static int phase_evp(PhaseParams &P, const double stiffness[36], int n_slip, const double *schmid,
                     double reference_slip_rate, double rate_exponent, double slip_resistance,
                     int hardening, const double *hardening_props, int n_props,
                     double latent_ratio) {
  if (n_slip < 1 || n_slip > SSFFT_MAX_SLIP)
    return fail(SSFFT_E_UNSUPPORTED, "number of slip systems must be 1..12");
  if (hardening < 0 || hardening > 3) return fail(SSFFT_E_INVALID, "unknown hardening law");
  if (n_props < 0 || n_props > 4) return fail(SSFFT_E_INVALID, "at most 4 hardening properties");
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
  return 0;
}

extern "C" int ssfft_set_phase_elastic(ssfft_handle *h, int phase, const double stiffness[36]) {
  CKR(check_phase(h, phase));
  phase_elastic(h->sb.hparams[phase], stiffness);
  h->sb.phase_set[phase] = true;
  return 0;
}

extern "C" int ssfft_set_phase_evp(ssfft_handle *h, int phase, const double stiffness[36],
                                   int n_slip, const double *schmid, double reference_slip_rate,
                                   double rate_exponent, double slip_resistance, int hardening,
                                   const double *hardening_props, int n_props,
                                   double latent_ratio) {
  CKR(check_phase(h, phase));
  CKR(phase_evp(h->sb.hparams[phase], stiffness, n_slip, schmid, reference_slip_rate,
                rate_exponent, slip_resistance, hardening, hardening_props, n_props,
                latent_ratio));
  h->sb.phase_set[phase] = true;
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
  PhaseParams &P = h->sb.hparams[phase];
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
  h->sb.phase_set[phase] = true;
  return 0;
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
  if (h->plan.fp64)
    mirror_options<double>(h->sb.md, h->cfg);
  else
    mirror_options<float>(h->sb.mf, h->cfg);
  if (h->sb.micro_set) CKR(upload(h));
  return 0;
}

extern "C" int ssfft_set_microstructure(ssfft_handle *h, int n_orient, const double *rotations,
                                        const int32_t *orient_of_point,
                                        const int32_t *phase_of_point) {
  if (!h) return fail(SSFFT_E_INVALID, "null handle");
  CK(cudaSetDevice(h->cfg.device));
  CKR(slot_bind(h->sb, h->cfg, n_orient, rotations, orient_of_point, phase_of_point, h->stream));
  // the captured Krylov launches are specific to the tangent kind (table or per voxel)
  drop_graph(h);
  return ssfft_reset(h);
}

extern "C" int ssfft_reset(ssfft_handle *h) {
  if (!h || !h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  CKR(slot_reset(h->sb, h->cfg, h->stream));
  h->committed_view = false;
  CKR(upload(h));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

extern "C" int ssfft_step(ssfft_handle *h, const ssfft_step_in *in, ssfft_step_out *out) {
  if (!h || !in || !out) return fail(SSFFT_E_INVALID, "null argument");
  if (!h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  if (!(in->dt > 0.0)) return fail(SSFFT_E_INVALID, "time increment must be positive");
  CK(cudaSetDevice(h->cfg.device));
  return h->plan.fp64 ? step_impl<double>(h, in, out) : step_impl<float>(h, in, out);
}

extern "C" int ssfft_commit(ssfft_handle *h, double fluctuation_scale) {
  if (!h || !h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  // old_* <- current by role swaps; the slip resistances are copied (the next
  // constitutive call starts from the current trial values)
  if (h->plan.fp64) {
    CKR(launch_commit_slip<double>(ctx(h), dtab<double>(h), h->sb.nslip_max));
    mirror_commit<double>(h->sb.md);
  } else {
    CKR(launch_commit_slip<float>(ctx(h), dtab<float>(h), h->sb.nslip_max));
    mirror_commit<float>(h->sb.mf);
  }
  CKR(upload(h));
  h->committed_view = true;
  return ssfft_scale_fluctuation(h, fluctuation_scale);
}

extern "C" int ssfft_scale_fluctuation(ssfft_handle *h, double factor) {
  if (!h || !h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  const long long n = 6 * h->plan.V;
  const int eb = std::max(1, std::min(div_up(n, SSFFT_THREADS), 148 * 16));
  if (factor != 1.0) {
    // the fluctuation field is double in both precisions
    double *dfl = h->plan.fp64 ? h->sb.md.dfl : h->sb.mf.dfl;
    scale_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(n, dfl, factor);
    CK(cudaGetLastError());
  }
  return 0;  // ordered on the handle's stream; no host synchronisation needed
}

extern "C" int ssfft_num_slip(ssfft_handle *h) { return h ? h->sb.nslip_max : 0; }

// The time loop of SmallStrainFFT.run (small_strain_fft.py:106-246) for a constant-rate
// schedule; mirrors materialite_b200/engine.py::solve without output collection.
extern "C" int ssfft_solve_constant_rates(ssfft_handle *h, const ssfft_rate_schedule *sc,
                                          ssfft_solve_out *out) {
  if (!h || !sc || !out) return fail(SSFFT_E_INVALID, "null argument");
  if (!h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
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

// Field read-back as float64, point-major; `committed` selects the committed buffers of
// the fields that commits swap (after a commit they hold the converged state).
template <typename T>
static int read_field(const SlotBufs &b, const SlotDev<T> &m, bool committed, int field,
                      const void **src, bool *is_double, int *width) {
  *width = 6;
  *is_double = false;
  switch (field) {
    case SSFFT_FIELD_STRESS:  // stress and strain are double in both precisions
      *is_double = true;
      *src = committed ? m.sig_old : m.sig;
      return 0;
    case SSFFT_FIELD_STRAIN:
      *is_double = true;
      *src = committed ? m.eps_old : m.eps;
      return 0;
    case SSFFT_FIELD_RESIDUAL: *src = m.b; return 0;
    case SSFFT_FIELD_SLIP_RESISTANCES:
    case SSFFT_FIELD_SLIP_SHEAR_STRAINS:
    case SSFFT_FIELD_PLASTIC_STRAINS:
    case SSFFT_FIELD_YIELD_STRESSES:
    case SSFFT_FIELD_EQ_PLASTIC_STRAINS:
      if (!b.any_evp) return fail(SSFFT_E_INVALID, "no plastic phase in this solve");
      *is_double = true;
      if (field == SSFFT_FIELD_SLIP_RESISTANCES) {
        *src = m.g_in;
        *width = b.nslip_max;
      } else if (field == SSFFT_FIELD_SLIP_SHEAR_STRAINS) {
        *src = committed ? m.gam_old : m.gam_trial;
        *width = b.nslip_max;
      } else if (field == SSFFT_FIELD_YIELD_STRESSES) {
        *src = m.g_in;  // plane 0
        *width = 1;
      } else if (field == SSFFT_FIELD_EQ_PLASTIC_STRAINS) {
        *src = committed ? m.Gam_old : m.Gam_trial;
        *width = 1;
      } else {
        *src = m.ep_old;
      }
      return 0;
    default: return fail(SSFFT_E_INVALID, "unknown field id");
  }
}

extern "C" int ssfft_get_field(ssfft_handle *h, int field, double *dst, int to_host) {
  if (!h || !dst) return fail(SSFFT_E_INVALID, "null argument");
  if (!h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  const long long V = h->plan.V;
  const void *src = nullptr;
  bool is_double = false;
  int width = 6;
  if (h->plan.fp64)
    CKR(read_field<double>(h->sb, h->sb.md, h->committed_view, field, &src, &is_double, &width));
  else
    CKR(read_field<float>(h->sb, h->sb.mf, h->committed_view, field, &src, &is_double, &width));
  double *ddst = dst;
  if (to_host) {
    CKR(ensure_buffer((void **)&h->stage, &h->cap_stage, (size_t)V * width * sizeof(double)));
    ddst = h->stage;
  }
  const int eb = std::max(1, std::min(div_up(V * width, SSFFT_THREADS), 148 * 16));
  if (field == SSFFT_FIELD_PLASTIC_STRAINS) {
    plastic_to_specimen_kernel<<<eb, SSFFT_THREADS, 0, h->stream>>>(
        V, (const double *)src, h->sb.orient, h->sb.rm_tab,
        h->sb.have_phase_buf ? h->sb.phase : nullptr, h->sb.dparams, ddst);
  } else if (is_double || h->plan.fp64) {
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
  if (!h->sb.micro_set) {
    // the descriptor needs no microstructure for a plain projection: spectrum and mask
    mirror_init<T>(h->sb, h->cfg);
  }
  CKR(upload(h));
  ExtIO<T> io;
  io.in = in;
  io.out = out;
  return launch_projector<T, T, PRO_INPUT, EPI_STORE>(ctx(h), dtab<T>(h), io);
}

extern "C" int ssfft_apply_projection_device(ssfft_handle *h, const void *in_dev, void *out_dev) {
  if (!h || !in_dev || !out_dev) return fail(SSFFT_E_INVALID, "null argument");
  CK(cudaSetDevice(h->cfg.device));
  if (h->plan.fp64)
    CKR(apply_projection_dev<double>(h, (const double *)in_dev, (double *)out_dev));
  else
    CKR(apply_projection_dev<float>(h, (const float *)in_dev, (float *)out_dev));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

extern "C" int ssfft_apply_projection(ssfft_handle *h, const double *in_host, double *out_host) {
  if (!h || !in_host || !out_host) return fail(SSFFT_E_INVALID, "null argument");
  CK(cudaSetDevice(h->cfg.device));
  const long long V = h->plan.V;
  double *tmp = nullptr;
  ALLOC(tmp, (size_t)V * 6 * sizeof(double));
  const int eb = std::max(1, std::min(div_up(V * 6, SSFFT_THREADS), 148 * 16));
  int rc = 0;
  void *a = h->sb.field[7], *bb = h->sb.field[8];  // two Krylov buffers as scratch
  cudaError_t e = cudaMemcpyAsync(tmp, in_host, (size_t)V * 6 * sizeof(double),
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    if (h->plan.fp64) {
      from_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, tmp, (double *)a);
      rc = apply_projection_dev<double>(h, (const double *)a, (double *)bb);
      to_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, 6, (const double *)bb, tmp);
    } else {
      from_point_major_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, tmp, (float *)a);
      rc = apply_projection_dev<float>(h, (const float *)a, (float *)bb);
      to_point_major_kernel<float><<<eb, SSFFT_THREADS, 0, h->stream>>>(V, 6, (const float *)bb, tmp);
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
  SlotDev<T> &m = mirror<T>(h->sb);
  const SlotDev<T> saved = m;
  const LaunchCtx c = ctx(h);
  // a live MINRES state on the residual of the committed stress (never marked done); call
  // after a solve so that the stress field is not uniform.  After a commit the latest-stress
  // buffer holds the previous increment's field, so the committed one stands in for it.
  m.sig = m.sig_old;
  for (int k = 0; k < 6; ++k) m.sbar[k] = 0.0;
  m.rtol = 0.0;
  m.atol_scale = 0.0;
  m.forcing = 0.0;
  m.maxiter = (long long)1 << 60;
  CKR(upload(h));
  CKR(launch_residual<T>(c, dtab<T>(h)));
  CKR(launch_minres_init<T>(c, dtab<T>(h)));
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  NvtxScope range("ssfft_profile_krylov");  // only the timed Krylov kernels
  for (int r = 0; r < reps; ++r) {
    CKR(launch_krylov_iteration<T>(c, dtab<T>(h), h->sb.voxel_mode, h->pev));
    CK(cudaEventRecord(h->pev[6], h->stream));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(h->pev[6]));
    // pev[7]: before the update kernel; pev[0..5]: the projector's pass slots; pev[6]:
    // after the epilogue kernel
    for (int i = 0; i < 5; ++i) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->pev[i], h->pev[i + 1]));
      acc[i] += ms * 1e-3;
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->pev[7], h->pev[0]));
    acc[5] += ms * 1e-3;
    CK(cudaEventElapsedTime(&ms, h->pev[5], h->pev[6]));
    acc[6] += ms * 1e-3;
    CK(cudaEventElapsedTime(&ms, h->pev[7], h->pev[6]));
    acc[7] += ms * 1e-3;
  }
  for (int i = 0; i < 8; ++i) sec[i] = acc[i] / reps;
  // every timed iteration must have done its work: a state that stopped (a zero or
  // exactly solved residual) would time kernels that skip their items
  CK(cudaMemcpyAsync(h->h_st, h->sb.st, sizeof(MinresState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const bool live = !h->h_st->done && h->h_st->itn == reps;
  m = saved;
  CKR(upload(h));
  if (!live) return fail(SSFFT_E_INVALID, "profiled Krylov state stopped early: timings void");
  return 0;
}

extern "C" int ssfft_profile_krylov(ssfft_handle *h, int reps, double seconds[8]) {
  if (!h || !seconds || reps < 1) return fail(SSFFT_E_INVALID, "bad argument");
  if (!h->sb.micro_set) return fail(SSFFT_E_INVALID, "microstructure not set");
  CK(cudaSetDevice(h->cfg.device));
  return h->plan.fp64 ? profile_impl<double>(h, reps, seconds) : profile_impl<float>(h, reps, seconds);
}

#include "group.cuh"
