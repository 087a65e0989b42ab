// Batched solves: a group holds up to B RVE requests of one grid size, precision and
// tangent kind (table or per-voxel) as slots, and advances all of them together through the
// reference's time and Newton loops (small_strain_fft.py:106-246), each slot at its own
// pace.  One pass of the device loop is
//
//   schedule: slots whose MINRES solve finished and slots starting a load increment are
//     listed for service;
//   service (a conditional subgraph, skipped when the list is empty): for a finished solve
//     the strain update (:154-155); for an increment start the strain guess (:108-123);
//     then, for all listed slots, the constitutive call, the residual and the norms
//     (:130-146, :157-200), and the per-slot decisions -- convergence tests, the commit
//     (as role swaps) with the dt update of _get_new_time_increment (:266-279), the
//     cutback of :242-246 -- and the start of the next MINRES solve (:151);
//   one Krylov chunk over every slot whose solve is live (MINRES, :281-299);
//
// so a slot never waits for another slot's solve: a slot whose solve finishes is served
// at the next pass while the others keep iterating.  The passes repeat in a CUDA-graph
// while node until a slot finishes its whole solve (the host then hands its result back and
// may load a new request into the slot) or the host raises the group's wake flag (a
// request waits for a free slot).  No host round trip happens per Newton iteration.
#pragma once

#include <memory>

#include "group_api.h"

struct GroupCtl {
  int state, step_id, newton_it, max_cit;
  int cutbacks, steps, status, max_newton;
  int need_tsum, pad;
  double t, dt, dt_max, dt_min, start_time, end_time;
  double er[6], sr[6];          // masked strain and stress rates (load_schedule.py:26-40)
  double summed, old_max_inc, max_inc, pending_scale;
  double eq_err, old_eq, s_err, mvm;
  double gtol, stol;
  long long newton_total, krylov_total;
  double mean_stress[6], mean_strain[6];
};

// Slot lists of the loop: KRY (live MINRES solves; kept across passes), and the lists of
// one service: FRESH (increment starts), TAIL (finished solves), NEWTON (both), TSUM
// (increment starts under a stress increment), COMMIT (slots committed by the last
// service: slip resistances to copy), ENTER (slots that start a MINRES solve).
enum { GL_KRY = 0, GL_FRESH, GL_TAIL, GL_NEWTON, GL_TSUM, GL_COMMIT, GL_ENTER, GL_COUNT };

// Loop state of a group in device memory: slots finished and passes run since the launch
// (reset by the host before each launch); passes and services since the group began.
struct GroupLoop {
  int finished, pad;
  unsigned long long launch_passes, passes, services;
};

// Passes per graph launch at most (a launch also ends when a slot finishes its solve).
#define GROUP_PASS_CAP 200000

// Per-increment inputs of a slot that starts an increment: the load_schedule closures at
// (t, dt) (small_strain_fft.py:108-123) and the flags of the strain guess.
template <typename T> __device__ void group_begin_slot(GroupCtl &c, SlotDev<T> &S) {
  int imax = 0;
  bool all_small = true;
  for (int k = 0; k < 6; ++k) {
    const double ei = c.er[k] * c.dt;
    const double si = c.sr[k] * c.dt;
    S.sv.dEbar[k] = ei;
    S.sv.dS[k] = si;
    S.sv.corr[k] = 0.0;
    S.sbar[k] = c.sr[k] * (c.t + c.dt - c.start_time);
    if (fabs(ei) > fabs(c.er[imax] * c.dt)) imax = k;
    if (!(si < 1.0e-14)) all_small = false;
  }
  c.max_inc = c.er[imax] * c.dt;
  S.reset_fluct = (c.max_inc * c.old_max_inc < 0.0) ? 1 : 0;
  S.first_step = c.step_id == 0 ? 1 : 0;
  S.fluct_scale = c.pending_scale;
  c.pending_scale = 1.0;
  S.dt = c.dt;
  S.norms_dx = 0;
  c.newton_it = 0;
  c.max_cit = 0;
  c.need_tsum = all_small ? 0 : 1;
}

// Start of a pass: finished MINRES solves leave the live list (in place, keeping its
// order) for the tail list; slots in FRESH state are listed for an increment start; the
// service runs when either list is non-empty.
template <typename T>
__global__ void group_sched_kernel(SlotDev<T> *tab, GroupCtl *ctl, int *ids, int *counts, int B,
                                   cudaGraphConditionalHandle cond_srv, int use_cond,
                                   GroupLoop *loop) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int n[GL_COUNT];
  for (int l = 0; l < GL_COUNT; ++l) n[l] = 0;
  int *kry = ids + GL_KRY * B;
  const int nk = counts[GL_KRY];
  for (int k = 0; k < nk; ++k) {
    const int s = kry[k];
    minres_cap(tab[s].st);
    if (tab[s].st->done) {
      SlotDev<T> &S = tab[s];
      S.norms_dx = 1;
      for (int q = 0; q < 4; ++q) S.citers[q] = 0;
      ids[GL_TAIL * B + n[GL_TAIL]++] = s;
    } else {
      kry[n[GL_KRY]++] = s;
    }
  }
  for (int s = 0; s < B; ++s) {
    GroupCtl &c = ctl[s];
    if (c.state != GS_FRESH) continue;
    SlotDev<T> &S = tab[s];
    group_begin_slot<T>(c, S);
    for (int q = 0; q < 4; ++q) S.citers[q] = 0;
    ids[GL_FRESH * B + n[GL_FRESH]++] = s;
    if (c.need_tsum) ids[GL_TSUM * B + n[GL_TSUM]++] = s;
  }
  // NEWTON = FRESH then TAIL
  for (int k = 0; k < n[GL_FRESH]; ++k) ids[GL_NEWTON * B + n[GL_NEWTON]++] = ids[GL_FRESH * B + k];
  for (int k = 0; k < n[GL_TAIL]; ++k) ids[GL_NEWTON * B + n[GL_NEWTON]++] = ids[GL_TAIL * B + k];
  counts[GL_KRY] = n[GL_KRY];
  counts[GL_FRESH] = n[GL_FRESH];
  counts[GL_TAIL] = n[GL_TAIL];
  counts[GL_NEWTON] = n[GL_NEWTON];
  counts[GL_TSUM] = n[GL_TSUM];
  counts[GL_ENTER] = 0;
  loop->passes += 1;
  loop->launch_passes += 1;
  if (n[GL_NEWTON] > 0) loop->services += 1;
  if (use_cond) cudaGraphSetConditional(cond_srv, n[GL_NEWTON] > 0 ? 1u : 0u);
}

// strain += tangent.mean().inv @ stress_increment (small_strain_fft.py:119-120) for the
// slots that start an increment under a stress increment.
template <typename T>
__global__ void group_corr_kernel(SlotDev<T> *tab, GroupCtl *ctl, const int *ids,
                                  const int *counts, int B, long long V) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < counts[GL_TSUM]; ++k) {
    const int s = ids[GL_TSUM * B + k];
    SlotDev<T> &S = tab[s];
    double Km[36], Ki[36];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) Km[i * 6 + j] = S.results[16 + sym_idx(i, j)] / (double)V;
    if (!inv6(Km, Ki)) {
      ctl[s].status = SSFFT_E_INVALID;
      ctl[s].state = GS_FAILED;
      continue;
    }
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 6; ++j) acc += mul_rn(Ki[i * 6 + j], S.sv.dS[j]);
      S.sv.corr[i] = acc;
    }
  }
}

// After the constitutive call: its stress becomes the slot's latest stress (and the next
// call's guess, small_strain_fft.py:169).
template <typename T>
__global__ void group_swap_stress_kernel(SlotDev<T> *tab, const int *ids, const int *counts,
                                         int B) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < counts[GL_NEWTON]; ++k) {
    SlotDev<T> &S = tab[ids[GL_NEWTON * B + k]];
    double *t = S.sig;
    S.sig = S.sig_next;
    S.sig_next = t;
  }
}

// Cutback after a failed increment (small_strain_fft.py:242-246).
__device__ inline void group_cutback(GroupCtl &c) {
  c.dt /= 2.0;
  c.cutbacks += 1;
  c.pending_scale *= 0.5;
  if (c.dt < c.dt_min) {
    c.status = SSFFT_E_INVALID;
    c.state = GS_FAILED;
  } else {
    c.state = GS_FRESH;
  }
}

// End of a service: the Newton decisions of every listed slot.  A slot that goes on
// solving (an increment start whose residual is known, or a Newton iteration that did not
// converge) is listed to start a MINRES solve and joins the live list; a committed slot
// starts its next increment at the next service.
template <typename T>
__global__ void group_decide_kernel(SlotDev<T> *tab, GroupCtl *ctl, int *ids, int *counts,
                                    int B, long long V, GroupLoop *loop) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int n_commit = 0, n_enter = 0, finished = 0;
  int nk = counts[GL_KRY];
  for (int k = 0; k < counts[GL_NEWTON]; ++k) {
    const int s = ids[GL_NEWTON * B + k];
    GroupCtl &c = ctl[s];
    SlotDev<T> &S = tab[s];
    if (c.state == GS_FAILED) {
      ++finished;
      continue;
    }
    const int cit = S.citers[0], cf = S.citers[1];
    if (!cf && S.any_evp) {  // the trial slip resistances of a successful call
      double *t = S.g_in;
      S.g_in = S.g_out;
      S.g_out = t;
    }
    const double *r = S.results;
    bool solve = false;
    if (c.state == GS_FRESH) {
      if (cf) {
        group_cutback(c);
      } else {
        c.max_cit = max(c.max_cit, cit);
        c.mvm = mean_von_mises(r, V);
        c.eq_err = r[40] / c.mvm;
        c.old_eq = fmax(c.eq_err, c.gtol);
        c.state = GS_SOLVE;
        solve = true;
      }
    } else {  // GS_SOLVE, its MINRES solve finished
      c.newton_it += 1;
      c.newton_total += 1;
      c.krylov_total += S.st->itn;
      if (S.st->istop == 9) {
        c.status = SSFFT_E_NAN;
        c.state = GS_FAILED;
      } else if (cf) {
        group_cutback(c);
      } else {
        c.max_cit = max(c.max_cit, cit);
        double mvm = mean_von_mises(r, V);
        const double tavg = (c.summed + mvm) / (double)(c.step_id + 1);
        if (mvm / tavg < 1.0e-12) mvm = tavg;
        c.mvm = mvm;
        c.eq_err = r[40] / mvm;
        double max_ds = r[12] * sqrt(1.5);
        if (max_ds / mvm < 1.0e-12) max_ds = mvm;
        c.s_err = r[13] / max_ds;
        const double p_err = c.s_err * c.eq_err / c.old_eq;
        const bool conv = c.eq_err < c.gtol &&
                          (c.s_err < c.stol || p_err < c.stol || c.step_id == 0 || c.eq_err < 1e-8);
        if (conv && !isfinite(c.eq_err)) {
          c.status = SSFFT_E_NAN;
          c.state = GS_FAILED;
        } else if (conv) {
          // commit (update_state_variables; old_* <- current) by role swaps
          double *f6;
          f6 = S.sig_old; S.sig_old = S.sig; S.sig = f6;
          f6 = S.eps_old; S.eps_old = S.eps; S.eps = f6;
          T *t6 = S.kvox_old; S.kvox_old = S.kvox; S.kvox = t6;
          double *td;
          td = S.gam_old; S.gam_old = S.gam_trial; S.gam_trial = td;
          td = S.ep_old; S.ep_old = S.ep_trial; S.ep_trial = td;
          td = S.Gam_old; S.Gam_old = S.Gam_trial; S.Gam_trial = td;
          for (int q = 0; q < 6; ++q) {
            c.mean_stress[q] = r[q] / (double)V;
            c.mean_strain[q] = r[6 + q] / (double)V;
          }
          c.summed += c.mvm;
          c.old_max_inc = c.max_inc;
          c.step_id += 1;
          c.steps += 1;
          c.t += c.dt;
          // _get_new_time_increment (:266-279) with no output times
          double nd = fmin(c.dt_max, c.end_time - c.t);
          nd = fmin(nd, c.max_cit < 11 ? c.dt * 2.0 : c.dt);
          c.pending_scale *= nd / c.dt;
          c.dt = nd;
          if (c.t < c.end_time - c.dt_min / 2.0) {
            c.state = GS_FRESH;
            if (S.any_evp) ids[GL_COMMIT * B + n_commit++] = s;
          } else {
            c.state = GS_DONE;
          }
        } else if (c.newton_it >= c.max_newton) {
          group_cutback(c);
        } else {
          c.old_eq = fmax(c.eq_err, c.gtol);
          solve = true;
        }
      }
    }
    if (solve) {
      ids[GL_ENTER * B + n_enter++] = s;
      ids[GL_KRY * B + nk++] = s;
    }
    if (c.state == GS_DONE || c.state == GS_FAILED) ++finished;
  }
  counts[GL_COMMIT] = n_commit;
  counts[GL_ENTER] = n_enter;
  counts[GL_KRY] = nk;
  loop->finished += finished;
}

// End of a pass: the loop goes on while a slot is live, none has finished since the
// launch, the host has not asked for the device (a request waits for a free slot), and the
// pass cap is not reached.
__global__ void group_loop_kernel(const GroupCtl *ctl, int B, GroupLoop *loop,
                                  const volatile int *wake, cudaGraphConditionalHandle cond_loop,
                                  int use_cond) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int live = 0;
  for (int s = 0; s < B; ++s)
    if (ctl[s].state == GS_FRESH || ctl[s].state == GS_SOLVE) ++live;
  const bool more = live > 0 && loop->finished == 0 && *wake == 0 &&
                    loop->launch_passes < GROUP_PASS_CAP;
  if (use_cond) cudaGraphSetConditional(cond_loop, more ? 1u : 0u);
}

// Krylov iterations per pass (between looks at the slots' MINRES states).
#define GROUP_KRYLOV_CHUNK 4

// ---------------------------------------------------------------------------------------
// host side of a group
// ---------------------------------------------------------------------------------------
struct Group {
  int device = 0;
  ssfft_config proto{};        // grid and precision of every slot
  bool voxel = false;          // per-voxel tangents (crystal plasticity)
  bool stress_rates = false;   // some request has stress rates (tangent-mean correction)
  int B = 0;                   // slots
  GridPlan plan{};
  cudaStream_t stream = nullptr, cap_stream = nullptr;
  std::vector<SlotBufs> slots;
  std::vector<bool> allocated;
  void *dtab = nullptr;        // SlotDev<T>[B]
  GroupCtl *dctl = nullptr;
  GroupCtl *hctl = nullptr;    // pinned mirror
  int *dids = nullptr;         // [GL_COUNT][B]
  int *dcounts = nullptr;      // [GL_COUNT]
  GroupLoop *dloop = nullptr;
  GroupLoop *hloop = nullptr;  // pinned mirror
  int *hwake = nullptr;        // host-mapped wake flag (a request waits for a free slot)
  int *dwake = nullptr;        // its device address
  cudaGraphExec_t exec = nullptr;
  bool nested = false;         // passes loop on the device (else one pass per launch)
  bool conditional_service = false;  // the service is a conditional node (else always runs)
  int pass_kernels = 0, service_kernels = 0;
  long long launches = 0;
  double *stage = nullptr;
  size_t cap_stage = 0;

  ~Group() { release(); }

  void release() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    for (size_t s = 0; s < slots.size(); ++s)
      if (allocated[s]) slot_free(slots[s]);
    slots.clear();
    allocated.clear();
    void *ptrs[] = {dtab, dctl, dids, dcounts, dloop, stage};
    for (void *p : ptrs)
      if (p) cudaFree(p);
    dtab = nullptr;
    dctl = nullptr;
    dids = dcounts = nullptr;
    dloop = nullptr;
    stage = nullptr;
    if (hctl) cudaFreeHost(hctl);
    if (hloop) cudaFreeHost(hloop);
    if (hwake) cudaFreeHost(hwake);
    hctl = nullptr;
    hloop = nullptr;
    hwake = dwake = nullptr;
    plan_free(plan);
    if (stream) cudaStreamDestroy(stream);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    stream = cap_stream = nullptr;
  }

  size_t desc_bytes() const { return plan.fp64 ? sizeof(SlotDev<double>) : sizeof(SlotDev<float>); }

  int init(const ssfft_config &cfg, int nslots, bool voxel_mode, bool rates, int dev) {
    device = dev;
    proto = cfg;
    proto.device = dev;
    voxel = voxel_mode;
    stress_rates = rates;
    B = nslots;
    CK(cudaSetDevice(dev));
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    CKR(plan_create(plan, &proto, stream));
    slots.resize(B);
    allocated.assign(B, false);
    ALLOC(dtab, desc_bytes() * B);
    CK(cudaMemsetAsync(dtab, 0, desc_bytes() * B, stream));
    ALLOC(dctl, sizeof(GroupCtl) * B);
    CK(cudaMemsetAsync(dctl, 0, sizeof(GroupCtl) * B, stream));
    ALLOC(dids, sizeof(int) * GL_COUNT * B);
    ALLOC(dcounts, sizeof(int) * GL_COUNT);
    CK(cudaMemsetAsync(dcounts, 0, sizeof(int) * GL_COUNT, stream));
    ALLOC(dloop, sizeof(GroupLoop));
    CK(cudaMemsetAsync(dloop, 0, sizeof(GroupLoop), stream));
    CK(cudaMallocHost((void **)&hctl, sizeof(GroupCtl) * B));
    memset(hctl, 0, sizeof(GroupCtl) * B);
    CK(cudaMallocHost((void **)&hloop, sizeof(GroupLoop)));
    memset(hloop, 0, sizeof(GroupLoop));
    CK(cudaHostAlloc((void **)&hwake, sizeof(int), cudaHostAllocMapped));
    *(volatile int *)hwake = 0;
    CK(cudaHostGetDevicePointer((void **)&dwake, hwake, 0));
    CK(cudaStreamSynchronize(stream));
    return 0;
  }

  // Ask a running launch to end at its next pass boundary (any thread).
  void wake() { __atomic_store_n(hwake, 1, __ATOMIC_RELEASE); }

  SlotList list(int l) const {
    SlotList L;
    L.ids = dids + l * B;
    L.count = dcounts + l;
    return L;
  }

  LaunchCtx lctx(int l, cudaStream_t s) {
    LaunchCtx c;
    c.p = &plan;
    c.list = list(l);
    c.cap = B;
    c.stream = s;
    c.launches = &launches;
    return c;
  }

  int plan_nslip() const {
    int n = 0;
    for (size_t s = 0; s < slots.size(); ++s)
      if (allocated[s]) n = std::max(n, slots[s].nslip_max);
    return std::max(n, 1);
  }

  // The service of a pass: tail of the finished solves, head of the increment starts,
  // their constitutive calls, residuals, norms and decisions, and the start of the next
  // MINRES solves.
  template <typename T> int issue_service(cudaStream_t s) {
    SlotDev<T> *tab = (SlotDev<T> *)dtab;
    if (voxel) CKR(launch_commit_slip<T>(lctx(GL_COMMIT, s), tab, plan_nslip()));
    if (stress_rates) {
      CKR(launch_tangent_sum<T>(lctx(GL_TSUM, s), tab));
      group_corr_kernel<T><<<1, 32, 0, s>>>(tab, dctl, dids, dcounts, B, plan.V);
      ++launches;
      CK(cudaGetLastError());
    }
    CKR(launch_strain_guess<T>(lctx(GL_FRESH, s), tab));
    if (plan.fp64)
      CKR(launch_update_strain<T>(lctx(GL_TAIL, s), tab));
    else
      CKR(launch_reproject_update<T>(lctx(GL_TAIL, s), tab));
    CKR(launch_constitutive<T>(lctx(GL_NEWTON, s), tab, false));
    group_swap_stress_kernel<T><<<1, 32, 0, s>>>(tab, dids, dcounts, B);
    ++launches;
    CKR(launch_residual<T>(lctx(GL_NEWTON, s), tab));
    CKR(launch_norms<T>(lctx(GL_NEWTON, s), tab));
    group_decide_kernel<T><<<1, 32, 0, s>>>(tab, dctl, dids, dcounts, B, plan.V, dloop);
    ++launches;
    CK(cudaGetLastError());
    CKR(launch_minres_init<T>(lctx(GL_ENTER, s), tab));
    return 0;
  }

  template <typename T> int issue_chunk(cudaStream_t s) {
    SlotDev<T> *tab = (SlotDev<T> *)dtab;
    for (int i = 0; i < GROUP_KRYLOV_CHUNK; ++i)
      CKR(launch_krylov_iteration<T>(lctx(GL_KRY, s), tab, voxel));
    return 0;
  }

  // One pass captured into `into` on cap_stream: schedule, the service (a conditional node
  // when `cond_service`, else unconditional), the Krylov chunk, and the loop condition.
  template <typename T>
  cudaError_t capture_pass(cudaGraph_t into, cudaGraphConditionalHandle cond_loop, bool use_loop,
                           bool cond_service, int *rc) {
    SlotDev<T> *tab = (SlotDev<T> *)dtab;
    cudaGraphConditionalHandle cond_srv = 0;
    cudaError_t e = cudaSuccess;
    if (cond_service) e = cudaGraphConditionalHandleCreate(&cond_srv, into, 0, 0);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(cap_stream, into, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const long long l0 = launches;
    group_sched_kernel<T><<<1, 32, 0, cap_stream>>>(tab, dctl, dids, dcounts, B, cond_srv,
                                                     cond_service ? 1 : 0, dloop);
    ++launches;
    e = cudaGetLastError();
    if (e == cudaSuccess && cond_service) {
      // the service as an IF node appended to the capture's current dependencies, its body
      // captured on the group's own stream
      cudaStreamCaptureStatus cs;
      const cudaGraphNode_t *deps = nullptr;
      size_t ndeps = 0;
      cudaGraph_t capg = nullptr;
      e = cudaStreamGetCaptureInfo(cap_stream, &cs, nullptr, &capg, &deps, &ndeps);
      cudaGraphNodeParams ip = {cudaGraphNodeTypeConditional};
      ip.conditional.handle = cond_srv;
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      cudaGraphNode_t inode = nullptr;
      if (e == cudaSuccess) e = cudaGraphAddNode(&inode, capg, deps, ndeps, &ip);
      if (e == cudaSuccess)
        e = cudaStreamUpdateCaptureDependencies(cap_stream, &inode, 1, cudaStreamSetCaptureDependencies);
      if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(stream, ip.conditional.phGraph_out[0], nullptr, nullptr,
                                          0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          const long long ls = launches;
          *rc = issue_service<T>(stream);
          service_kernels = (int)(launches - ls);
          cudaGraph_t g2 = nullptr;
          const cudaError_t e2 = cudaStreamEndCapture(stream, &g2);
          if (e == cudaSuccess) e = e2;
        }
      }
    } else if (e == cudaSuccess) {
      const long long ls = launches;
      *rc = issue_service<T>(cap_stream);
      service_kernels = (int)(launches - ls);
    }
    if (e == cudaSuccess && !*rc) *rc = issue_chunk<T>(cap_stream);
    if (e == cudaSuccess && !*rc) {
      group_loop_kernel<<<1, 32, 0, cap_stream>>>(dctl, B, dloop, dwake, cond_loop,
                                                  use_loop ? 1 : 0);
      ++launches;
      e = cudaGetLastError();
    }
    pass_kernels = (int)(launches - l0) - service_kernels;
    cudaGraph_t g1 = nullptr;
    const cudaError_t e1 = cudaStreamEndCapture(cap_stream, &g1);
    return e != cudaSuccess ? e : e1;
  }

  // The passes loop as a while node holding an IF node (the service), or, when conditional
  // nodes are not available (SSFFT_NO_DEVICE_LOOP=1 or an error), one pass per launch with
  // the service always run.
  template <typename T> int build() {
    const char *nl = getenv("SSFFT_NO_DEVICE_LOOP");
    const bool allow_nested = !(nl && nl[0] == '1');
    for (int attempt = allow_nested ? 0 : 1; attempt < 2; ++attempt) {
      const bool want_nested = attempt == 0;
      const long long l0 = launches;
      cudaGraph_t graph = nullptr;
      CK(cudaGraphCreate(&graph, 0));
      cudaError_t e = cudaSuccess;
      int rc = 0;
      if (want_nested) {
        cudaGraphConditionalHandle cond_loop;
        e = cudaGraphConditionalHandleCreate(&cond_loop, graph, 1, cudaGraphCondAssignDefault);
        cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
        np.conditional.handle = cond_loop;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &np);
        if (e == cudaSuccess)
          e = capture_pass<T>(np.conditional.phGraph_out[0], cond_loop, true, true, &rc);
      } else {
        e = capture_pass<T>(graph, 0, false, false, &rc);
      }
      if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      launches = l0;
      if (rc) return rc;
      if (e == cudaSuccess) {
        nested = want_nested;
        conditional_service = want_nested;
        return 0;
      }
      exec = nullptr;
      cudaGetLastError();
      if (!want_nested)
        return ssfft_internal_fail(SSFFT_E_CUDA, std::string("group graph: ") + cudaGetErrorString(e));
    }
    return 0;
  }

  // Load a request into a free slot: buffers (allocated on first use of the slot),
  // phases, microstructure, initial state, and the slot's time-loop control.
  int load(int s, const GroupJob &j) {
    CK(cudaSetDevice(device));
    SlotBufs &b = slots[s];
    if (!allocated[s]) {
      CKR(slot_alloc(b, plan, stream));
      allocated[s] = true;
    }
    ssfft_config cfg = j.req.config;
    cfg.device = device;
    for (int p = 0; p < SSFFT_MAX_PHASES; ++p) b.phase_set[p] = false;
    for (int p = 0; p < j.req.n_phases; ++p) {
      const ssfft_phase &ph = j.req.phases[p];
      if (ph.kind == 0)
        CKR(phase_elastic(b.hparams[p], ph.stiffness));
      else
        CKR(phase_evp(b.hparams[p], ph.stiffness, ph.n_slip, ph.schmid, ph.reference_slip_rate,
                      ph.rate_exponent, ph.slip_resistance, ph.hardening, ph.hardening_props,
                      ph.n_props, ph.latent_ratio));
      b.phase_set[p] = true;
    }
    CKR(slot_bind(b, cfg, j.req.n_orient, j.rotations.data(), j.orient.data(),
                  j.phase.empty() ? nullptr : j.phase.data(), stream));
    CKR(slot_reset(b, cfg, stream));
    const long long n = 6 * plan.V;
    const long long maxiter = std::min<long long>(
        cfg.max_krylov_iterations > 0 ? cfg.max_krylov_iterations : 5 * n, KRYLOV_ITERATION_CAP);
    if (plan.fp64) {
      b.md.rtol = cfg.linear_solver_tolerance;
      b.md.maxiter = maxiter;
      b.md.atol_scale = krylov_atol_scale(cfg);
      b.md.forcing = cfg.krylov_forcing;
      CK(cudaMemcpyAsync((char *)dtab + s * desc_bytes(), &b.md, sizeof(b.md),
                         cudaMemcpyHostToDevice, stream));
    } else {
      b.mf.rtol = std::max(cfg.linear_solver_tolerance, MIXED_RTOL_FLOOR);
      b.mf.maxiter = maxiter;
      b.mf.atol_scale = krylov_atol_scale(cfg);
      b.mf.forcing = cfg.krylov_forcing;
      CK(cudaMemcpyAsync((char *)dtab + s * desc_bytes(), &b.mf, sizeof(b.mf),
                         cudaMemcpyHostToDevice, stream));
    }
    GroupCtl c;
    memset(&c, 0, sizeof(c));
    const ssfft_rate_schedule &sc = j.req.schedule;
    for (int k = 0; k < 6; ++k) {  // apply_stress_mask (load_schedule.py:26-30)
      c.er[k] = sc.strain_rate[k] * (1.0 - cfg.stress_mask[k]);
      c.sr[k] = sc.stress_rate[k] * cfg.stress_mask[k];
    }
    c.dt = sc.initial_time_increment > 0 ? sc.initial_time_increment : sc.end_time - sc.start_time;
    c.dt_max = sc.max_time_increment > 0 ? sc.max_time_increment : c.dt;
    c.dt_min = sc.min_time_increment > 0 ? sc.min_time_increment : 1.0e-9;
    c.t = sc.start_time;
    c.start_time = sc.start_time;
    c.end_time = sc.end_time;
    c.pending_scale = 1.0;
    c.gtol = cfg.global_tolerance;
    c.stol = cfg.strain_correction_tolerance;
    c.max_newton = cfg.max_newton_iterations > 0 ? cfg.max_newton_iterations : 100;
    c.state = (c.t < c.end_time - c.dt_min / 2.0) ? GS_FRESH : GS_DONE;
    hctl[s] = c;
    CK(cudaMemcpyAsync(dctl + s, &hctl[s], sizeof(GroupCtl), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    return 0;
  }

  // Advance the live slots until one finishes, the host raises the wake flag, or the pass
  // cap.  The control blocks come back to hctl.
  int run() {
    CK(cudaSetDevice(device));
    if (!exec) {
      const int rc = plan.fp64 ? build<double>() : build<float>();
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(hloop, dloop, sizeof(GroupLoop), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    const unsigned long long p0 = hloop->passes, s0 = hloop->services;
    hloop->finished = 0;
    hloop->launch_passes = 0;
    CK(cudaMemcpyAsync(dloop, hloop, sizeof(GroupLoop), cudaMemcpyHostToDevice, stream));
    for (;;) {
      CK(cudaGraphLaunch(exec, stream));
      CK(cudaMemcpyAsync(hctl, dctl, sizeof(GroupCtl) * B, cudaMemcpyDeviceToHost, stream));
      CK(cudaMemcpyAsync(hloop, dloop, sizeof(GroupLoop), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      if (nested) break;
      int live = 0;
      for (int s = 0; s < B; ++s)
        if (hctl[s].state == GS_FRESH || hctl[s].state == GS_SOLVE) ++live;
      if (live == 0 || hloop->finished > 0 || __atomic_load_n(hwake, __ATOMIC_ACQUIRE) ||
          hloop->launch_passes >= GROUP_PASS_CAP)
        break;
    }
    const unsigned long long passes = hloop->passes - p0, services = hloop->services - s0;
    launches += (long long)passes * pass_kernels +
                (long long)(conditional_service ? services : passes) * service_kernels;
    return 0;
  }

  // Final (committed) stress of slot s, point-major float64, to host memory.
  int read_stress(int s, double *dst) {
    CK(cudaSetDevice(device));
    const long long V = plan.V;
    CKR(ensure_buffer((void **)&stage, &cap_stage, (size_t)V * 6 * sizeof(double)));
    const int eb = std::max(1, std::min(div_up(V * 6, SSFFT_THREADS), 148 * 16));
    // the committed stress is the descriptor's sig_old (read back the current roles)
    if (plan.fp64) {
      SlotDev<double> m;
      CK(cudaMemcpyAsync(&m, (char *)dtab + s * desc_bytes(), sizeof(m), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      to_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, stream>>>(V, 6, m.sig_old, stage);
    } else {
      SlotDev<float> m;
      CK(cudaMemcpyAsync(&m, (char *)dtab + s * desc_bytes(), sizeof(m), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      to_point_major_kernel<double><<<eb, SSFFT_THREADS, 0, stream>>>(V, 6, m.sig_old, stage);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, stage, (size_t)V * 6 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return 0;
  }

  int set_state(int s, int state) {
    hctl[s].state = state;
    CK(cudaMemcpyAsync(&dctl[s].state, &hctl[s].state, sizeof(int), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    return 0;
  }
};

// Entry points for the serving loop (server.cu).
__attribute__((visibility("hidden"))) Group *group_new() { return new Group(); }
__attribute__((visibility("hidden"))) void group_delete(Group *g) { delete g; }
__attribute__((visibility("hidden"))) int group_init(Group *g, const ssfft_config &cfg, int slots,
                                                     bool voxel, bool rates, int dev) {
  return g->init(cfg, slots, voxel, rates, dev);
}
__attribute__((visibility("hidden"))) int group_load(Group *g, int s, const GroupJob &j) {
  return g->load(s, j);
}
__attribute__((visibility("hidden"))) int group_run(Group *g) { return g->run(); }
__attribute__((visibility("hidden"))) int group_slot_state(Group *g, int s) { return g->hctl[s].state; }
__attribute__((visibility("hidden"))) void group_slot_result(Group *g, int s, ssfft_solve_out *o) {
  const GroupCtl &c = g->hctl[s];
  memset(o, 0, sizeof(*o));
  o->status = c.status;
  o->steps = c.steps;
  o->cutbacks = c.cutbacks;
  o->newton_iterations = c.newton_total;
  o->krylov_iterations = c.krylov_total;
  for (int k = 0; k < 6; ++k) {
    o->mean_stress[k] = c.mean_stress[k];
    o->mean_strain[k] = c.mean_strain[k];
  }
}
__attribute__((visibility("hidden"))) int group_read_stress(Group *g, int s, double *dst) {
  return g->read_stress(s, dst);
}
__attribute__((visibility("hidden"))) int group_release_slot(Group *g, int s) {
  return g->set_state(s, GS_EMPTY);
}
__attribute__((visibility("hidden"))) long long group_launches(Group *g) { return g->launches; }
__attribute__((visibility("hidden"))) void group_wake(Group *g) {
  if (g && g->hwake) g->wake();
}
__attribute__((visibility("hidden"))) void group_clear_wake(Group *g) {
  if (g && g->hwake) __atomic_store_n(g->hwake, 0, __ATOMIC_RELEASE);
}
