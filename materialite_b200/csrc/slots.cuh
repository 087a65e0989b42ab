// Slots: the unit of batching.  Every kernel of the solve works on a list of slots, each
// one RVE request with its own fields, Krylov vectors, spectrum, tangent, plastic state,
// reduction partials and MINRES scalars.  A slot's descriptor (SlotDev) lives in device
// memory, so whoever drives the solve -- the host for a single handle, the decision kernel
// of a batched group -- changes buffer roles (commits, the stress guess hand-off) by
// swapping pointers in the descriptor instead of copying fields.
//
// Work is split into items: (slot, plane), (slot, line tile), (slot, chunk of points).
// Kernels run a persistent grid that strides over the items of the slots listed in a
// SlotList; every reduction is private to its slot (partials indexed by the item's index
// within the slot, summed in that order by the slot's last item to arrive), so a slot's
// results do not depend on which other slots share the launch.
#pragma once

#include "common.cuh"

struct MinresState;
struct PhaseParams;

// Inputs of the strain guess at the start of a load increment (small_strain_fft.py:113-123).
struct StepVec {
  double corr[6];  // tangent.mean().inv @ stress_increment, or zero
  double dEbar[6]; // strain increment alone (first-step stress guess)
  double dS[6];    // stress increment
};

// Ticket counters of a slot's last-item reductions.
enum { TK_INIT = 0, TK_ZINV, TK_UPD, TK_CONST, TK_NORMS, TK_TSUM, TK_COUNT };

template <typename T> struct SlotDev {
  // strain and stress fields, 6 component planes of V points each, double in both
  // precisions: the equilibrium residual is computed from them, and float storage would put
  // its noise floor at the 1e-6 tolerance once stresses grow (Newton then stalls)
  double *eps, *eps_old, *dfl;       // strain, committed strain, accumulated fluctuation
  double *sig, *sig_next, *sig_old;  // latest stress, constitutive output, committed stress
  T *b;                         // equilibrium residual
  T *kr[7];                     // Krylov vectors; roles by iteration (kroles)
  void *spec;                   // half spectrum, sized for double-precision transforms
  // tangent: table mode (one entry per (orientation, phase) pair) or voxel mode
  const int32_t *gid;
  const T *ktab;                // [n_gid][21]
  T *kvox, *kvox_old;           // 21 planes: current, committed
  int voxel_mode;
  // microstructure and phases
  const int32_t *phase;         // phase per point (null: phase 0 everywhere)
  const int32_t *orient;        // orientation per point
  const double *rm_tab;         // [n_orient][36] Mandel rotations (specimen -> crystal)
  const PhaseParams *params;
  int n_params;                 // highest phase id + 1
  int nslip;                    // planes of the slip-state buffers
  int any_evp, any_j2;
  // plastic state (double): slip resistances in (previous trial) and out, committed;
  // plastic strain, accumulated slip and per-system shear, trial and committed
  double *g_in, *g_out, *g_old;
  double *ep_old, *ep_trial, *Gam_old, *Gam_trial, *gam_old, *gam_trial;
  // reductions and scalars
  MinresState *st;
  double *partials;
  unsigned int *tickets;        // TK_COUNT counters
  double *results;              // [0..13] norms, [16..36] tangent sum, [40] max|b|
  int *citers;                  // [0] max constitutive iterations, [1] failed, [2..3] J2
  // per-increment inputs
  double mask[6];               // stress mask: Gamma-hat(0) = diag(mask)
  double sbar[6];               // applied mean stress of the residual
  StepVec sv;
  int first_step, reset_fluct;
  double fluct_scale;           // strain guess scales the fluctuation by this first
  int norms_dx;                 // Newton norms include max |K : dx|
  double dt;
  double rtol;                  // MINRES relative tolerance and iteration limit
  long long maxiter;
  double atol_scale;            // MINRES also stops once |r| <= atol_scale x mean von Mises
                                // stress (0: off)
  double forcing;               // ... or once |r| <= forcing x |b| (0: off)
};

// The slots a launch works on: ids[0 .. *count).  Both live in device memory, so a kernel
// captured in a CUDA graph sees the list of the moment it runs.
struct SlotList {
  const int *ids;
  const int *count;
};

// Krylov vector roles at iteration itn (itn matrix-vector products done): P holds u_{j-1},
// Q receives u_j, W the new search direction, W1 and W2 the previous two, X the iterate,
// Y the matvec y'.  P and Q swap every iteration and the directions rotate every three,
// as a fixed buffer set read through these roles.
template <typename T> struct KRoles {
  T *P, *Q, *W, *W1, *W2, *X, *Y;
};

template <typename T> __device__ __forceinline__ KRoles<T> kroles(const SlotDev<T> &s, long long itn) {
  const int r2 = (int)(itn & 1);
  const int r3 = (int)(itn % 3);
  KRoles<T> k;
  k.P = s.kr[r2];
  k.Q = s.kr[1 - r2];
  k.W = s.kr[2 + r3];
  k.W1 = s.kr[2 + (r3 + 1) % 3];
  k.W2 = s.kr[2 + (r3 + 2) % 3];
  k.X = s.kr[5];
  k.Y = s.kr[6];
  return k;
}

// A slot's reduction: every item stores its partials, and the item that arrives last
// (ticket == total - 1) sees all of them.  Returns true in every thread of that item's
// block; the ticket is reset by the caller.  Callers store their partials from the first
// warp, which alone fences them before the ticket: a fence in every thread would wait for
// all of the block's outstanding field stores.
__device__ __forceinline__ bool last_item_arrives(unsigned int *ticket, unsigned int total) {
  __shared__ bool is_last;
  if (threadIdx.x < 32) __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == total - 1);
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// Copy one slot's descriptor into shared memory (raw: sizeof(SlotDev<T>) bytes, 16-byte
// aligned) unless it holds that slot already, and return it.  `staged` is the slot raw
// holds (the same in every thread of the block; -1 at the start of a kernel); the
// descriptors do not change during a launch.  Pointers read from there occupy registers
// only where they are used, not across a whole item.  The block syncs around a copy.
template <typename T>
__device__ __forceinline__ const SlotDev<T> &stage_slot(const SlotDev<T> *tab, int slot,
                                                        unsigned char *raw, int &staged) {
  if (slot != staged) {
    __syncthreads();
    const uint32_t *src = reinterpret_cast<const uint32_t *>(tab + slot);
    uint32_t *dst = reinterpret_cast<uint32_t *>(raw);
    for (int i = threadIdx.x; i < (int)(sizeof(SlotDev<T>) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    staged = slot;
  }
  return *reinterpret_cast<const SlotDev<T> *>(raw);
}

// Number of items of a launch: listed slots x items per slot.
__device__ __forceinline__ int list_items(const SlotList &L, int per_slot) {
  return *L.count * per_slot;
}
