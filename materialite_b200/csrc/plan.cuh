// Host side shared by a single solver handle (ssfft.cu) and a batched group of slots
// (group.cuh): the grid plan (FFT factorisations, tiles, twiddle and tangent tables),
// the device buffers of one slot, and the launches of every kernel over a slot list with
// persistent, occupancy-sized grids.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ssfft.h"
#include "common.cuh"
#include "constitutive.cuh"
#include "fft.cuh"
#include "fields.cuh"
#include "krylov.cuh"
#include "projector.cuh"
#include "slots.cuh"

int ssfft_internal_fail(int code, const std::string &msg);

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return ssfft_internal_fail(SSFFT_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define CKR(expr)           \
  do {                      \
    int r_ = (expr);        \
    if (r_ != 0) return r_; \
  } while (0)

#define ALLOC(ptr, bytes)                                                                 \
  do {                                                                                    \
    cudaError_t e_ = cudaMalloc((void **)&(ptr), (bytes));                                \
    if (e_ != cudaSuccess) {                                                              \
      cudaGetLastError();                                                                 \
      return ssfft_internal_fail(SSFFT_E_NOMEM, std::string("cudaMalloc ") + #ptr + ": " + \
                                                    cudaGetErrorString(e_));              \
    }                                                                                     \
  } while (0)

static int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------------------
// persistent grids
// ---------------------------------------------------------------------------------------
// Blocks of a persistent launch: as many as are resident at once on the device (occupancy
// x SMs), but no more than there are items.
struct OccKey {
  const void *f;
  int threads;
  size_t smem;
  int dev;
  int cluster;  // 0: blocks; C: clusters of C blocks
  bool operator<(const OccKey &o) const {
    if (f != o.f) return f < o.f;
    if (threads != o.threads) return threads < o.threads;
    if (smem != o.smem) return smem < o.smem;
    if (dev != o.dev) return dev < o.dev;
    return cluster < o.cluster;
  }
};

static std::mutex g_occ_mutex;
static std::map<OccKey, int> g_occ;

template <typename F> static int resident_blocks(F f, int threads, size_t smem, int dev) {
  const OccKey key{(const void *)f, threads, smem, dev, 0};
  {
    std::lock_guard<std::mutex> lk(g_occ_mutex);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) return it->second;
  }
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, smem) != cudaSuccess)
    per_sm = 1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  cudaGetLastError();
  const int n = std::max(1, per_sm) * std::max(1, sms);
  std::lock_guard<std::mutex> lk(g_occ_mutex);
  g_occ[key] = n;
  return n;
}

template <typename F>
static int persistent_grid(F f, int threads, size_t smem, long long items, int dev) {
  return (int)std::max(1LL, std::min<long long>(items, resident_blocks(f, threads, smem, dev)));
}

// Clusters of C blocks resident at once (a cluster must fit the SMs of one GPC).
template <typename... A>
static int resident_clusters(void (*f)(A...), int C, int threads, size_t smem, int dev) {
  const OccKey key{(const void *)f, threads, smem, dev, C};
  {
    std::lock_guard<std::mutex> lk(g_occ_mutex);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) return it->second;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, f, &cfg) != cudaSuccess || n < 1) n = 1;
  cudaGetLastError();
  std::lock_guard<std::mutex> lk(g_occ_mutex);
  g_occ[key] = n;
  return n;
}

// Persistent launch of a cluster kernel of `threads` threads a block: as many clusters as
// are resident at once, but no more than there are items.
template <typename... P, typename... A>
static int launch_clustered(void (*f)(P...), int C, int threads, size_t smem, long long items,
                            int dev, cudaStream_t stream, A &&...args) {
  const int ncl = (int)std::max(1LL, std::min<long long>(items, resident_clusters(f, C, threads, smem, dev)));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(ncl * C));
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, f, std::forward<A>(args)...);
  if (e != cudaSuccess)
    return ssfft_internal_fail(SSFFT_E_CUDA, std::string("cluster launch: ") + cudaGetErrorString(e));
  return 0;
}

// ---------------------------------------------------------------------------------------
// grid plan
// ---------------------------------------------------------------------------------------
static const size_t SMEM_LIMIT = 200 * 1024;
#define PLANE_SMEM_LIMIT (200 * 1024)
#define CLUSTER_MAX 8  // largest portable cluster
#define MAX_ITEMS_PER_SLOT 65536

struct GridPlan {
  int dev;
  bool fp64;                  // solve precision
  int nx, ny, nz, hz;
  long long V, S;             // points; stored half-spectrum points
  AxisPlan px, py, pz;
  int lz, ky, kx;
  int kx_f;                   // kz columns per x-pass tile of the float transforms
  bool use_plane;             // plane-fused passes allowed (SSFFT_NO_PLANE=1 forbids)
  void *tw[2][3], *tn[2][3];  // [0]: float, [1]: double tables per axis
  Grid<float> gf;
  Grid<double> gd;
  size_t partial_doubles;     // reduction partials per slot
};

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

template <typename T> static Grid<T> &grid_of(GridPlan &p);
template <> Grid<float> &grid_of<float>(GridPlan &p) { return p.gf; }
template <> Grid<double> &grid_of<double>(GridPlan &p) { return p.gd; }
template <typename T> static const Grid<T> &grid_of(const GridPlan &p) {
  return grid_of<T>(const_cast<GridPlan &>(p));
}

template <typename T> static void fill_grid(GridPlan &p) {
  Grid<T> &g = grid_of<T>(p);
  memset(&g, 0, sizeof(g));
  g.nx = p.nx;
  g.ny = p.ny;
  g.nz = p.nz;
  g.hz = p.hz;
  g.V = p.V;
  g.S = p.S;
  // float transforms take radix 16 and 12 butterflies (two stages for every length up to
  // 256 the solver uses); double ones stop at radix 8, whose registers fit 64 a thread
  const int maxrad = sizeof(T) == 4 ? 16 : 8;
  make_axis_plan(p.nx, g.px, maxrad);
  make_axis_plan(p.ny, g.py, maxrad);
  make_axis_plan(p.nz, g.pz, maxrad);
  const int k = sizeof(T) == 8 ? 1 : 0;
  g.twx = (const cplx<T> *)p.tw[k][0];
  g.twy = (const cplx<T> *)p.tw[k][1];
  g.twz = (const cplx<T> *)p.tw[k][2];
  g.tanx = (const T *)p.tn[k][0];
  g.tany = (const T *)p.tn[k][1];
  g.tanz = (const T *)p.tn[k][2];
  g.scale = (T)(1.0 / (double)p.V);
  g.lz = p.lz;
  g.ky = p.ky;
  g.kx = sizeof(T) == 4 ? p.kx_f : p.kx;
  grid_divisors(g);
}

template <typename T> static bool plane_ok(const GridPlan &p) {
  return p.use_plane && smem_plane_bytes<T>(p.ny, p.nz) <= PLANE_SMEM_LIMIT;
}

// Blocks per cluster of the cluster plane passes (0: not used), for grids whose plane does
// not fit one block: the smallest C in 2, 4, 8 whose blocks fit two to an SM, else the
// smallest whose blocks fit at all (a single block per SM leaves its loads and its
// transforms without overlap).  SSFFT_CLUSTER=C asks for clusters of at least C blocks,
// also where one block would hold the plane.
static int env_int(const char *name) {
  const char *v = getenv(name);
  return v ? atoi(v) : 0;
}

template <typename T> static int cluster_size(const GridPlan &p) {
  if (!p.use_plane) return 0;
  const int want = env_int("SSFFT_CLUSTER");
  if (want <= 0 && plane_ok<T>(p)) return 0;
  const int hs = (p.nz % 2 == 0) ? p.nz / 2 : p.hz;
  auto fits = [&](int C, size_t lim) {
    return p.ny % C == 0 && (2 * hs) % C == 0 && C >= want &&
           smem_cplane_bytes<T>(p.ny, p.nz, hs, C) <= lim;
  };
  // the smallest cluster whose blocks fit two to an SM (512 threads each), else the
  // smallest whose blocks fit at all
  for (int C = 2; C <= CLUSTER_MAX; C *= 2)
    if (fits(C, 113 * 1024)) return C;
  for (int C = 2; C <= CLUSTER_MAX; C *= 2)
    if (fits(C, PLANE_SMEM_LIMIT)) return C;
  return 0;
}

template <typename T> static ClusterGeo cluster_geo(const GridPlan &p, int C) {
  ClusterGeo q;
  const int hs = (p.nz % 2 == 0) ? p.nz / 2 : p.hz;
  q.C = C;
  q.R = p.ny / C;
  q.Lq = 2 * hs / C;
  q.cap = cplane_buf_elems(p.ny, p.nz, hs, C);
  q.fd_R = make_fastdiv((uint32_t)q.R);
  q.fd_Lq = make_fastdiv((uint32_t)q.Lq);
  return q;
}

// Threads of a cluster block: for float transforms 256 when three blocks fit an SM's
// shared memory (128^3 on 4-block clusters: each radix-16 stage then has one butterfly per
// thread, where 512 threads left half of them idle; measured 7-8% faster per pass), else
// 512 when two fit, else 1024 (SSFFT_CLUSTER_THREADS=256, 512 or 1024 overrides).
template <typename T> static int cluster_threads(const GridPlan &p, int C) {
  const int hs = (p.nz % 2 == 0) ? p.nz / 2 : p.hz;
  const size_t bytes = smem_cplane_bytes<T>(p.ny, p.nz, hs, C);
  const int want = env_int("SSFFT_CLUSTER_THREADS");
  if (want == 1024 || want == 512 || want == 256) return want;
  if (sizeof(T) == 4 && bytes <= 75 * 1024) return 256;
  return bytes <= 113 * 1024 ? 512 : 1024;
}

// Threads of an x-pass block: 256, or 192 / 384 on float grids when SSFFT_XPASS_THREADS
// asks for them.
template <typename T> static int xpass_threads() {
  if (sizeof(T) != 4) return XPASS_THREADS;
  const int want = env_int("SSFFT_XPASS_THREADS");
  return (want == 192 || want == 384) ? want : XPASS_THREADS;
}

template <typename T, typename TF, bool KRY>
static void launch_xpass(const Grid<T> &g, size_t sx, long long items, int dev,
                         cudaStream_t stream, const SlotDev<TF> *tab, SlotList list) {
  const int pt = xpass_threads<T>();
  if constexpr (sizeof(T) == 4) {
    if (pt == 384) {
      auto k = xpass_kernel<T, TF, KRY, 384>;
      k<<<persistent_grid(k, 384, sx, items, dev), 384, sx, stream>>>(g, tab, list);
      return;
    }
    if (pt == 192) {
      auto k = xpass_kernel<T, TF, KRY, 192>;
      k<<<persistent_grid(k, 192, sx, items, dev), 192, sx, stream>>>(g, tab, list);
      return;
    }
  }
  auto k = xpass_kernel<T, TF, KRY>;
  k<<<persistent_grid(k, XPASS_THREADS, sx, items, dev), XPASS_THREADS, sx, stream>>>(g, tab, list);
}

// The projection runs as three passes (z and y fused, in one block or one cluster).
template <typename T> static bool three_pass(const GridPlan &p) {
  return plane_ok<T>(p) || cluster_size<T>(p) > 0;
}

// Threads of a plane block: 1024 when a single block fits an SM (228 KB of shared memory),
// else 512.
template <typename T> static int plane_threads(const GridPlan &p) {
  return smem_plane_bytes<T>(p.ny, p.nz) > 113 * 1024 ? 1024 : 512;
}

static int validate_config(const ssfft_config *cfg) {
  if (!cfg) return ssfft_internal_fail(SSFFT_E_INVALID, "null config");
  for (int d = 0; d < 3; ++d)
    if (cfg->n[d] < 1 || cfg->n[d] > 1024)
      return ssfft_internal_fail(SSFFT_E_UNSUPPORTED, "grid size out of range");
  if (cfg->precision != SSFFT_FP64 && cfg->precision != SSFFT_MIXED)
    return ssfft_internal_fail(SSFFT_E_INVALID, "precision must be SSFFT_FP64 or SSFFT_MIXED");
  for (int c = 0; c < 6; ++c)
    if (cfg->stress_mask[c] != 0.0 && cfg->stress_mask[c] != 1.0)
      return ssfft_internal_fail(SSFFT_E_INVALID, "stress mask can only have zeros and ones");
  if (!(cfg->krylov_floor >= 0.0 && cfg->krylov_floor < 1.0))
    return ssfft_internal_fail(SSFFT_E_INVALID, "krylov_floor must be in [0, 1)");
  if (!(cfg->krylov_forcing >= 0.0 && cfg->krylov_forcing < 1.0))
    return ssfft_internal_fail(SSFFT_E_INVALID, "krylov_forcing must be in [0, 1)");
  AxisPlan p;
  for (int d = 0; d < 3; ++d)
    if (!make_axis_plan(cfg->n[d], p))
      return ssfft_internal_fail(SSFFT_E_UNSUPPORTED, "grid size has a prime factor above 32");
  return 0;
}

// Tiles are sized for double-precision transforms, which both modes run (the mixed mode
// computes its equilibrium residual in double).
static int plan_tiles(GridPlan &p) {
  p.lz = std::max(1, std::min(32, 2048 / (3 * p.nz)));
  p.lz = (int)std::min<long long>(p.lz, (long long)p.nx * p.ny);
  p.ky = std::min(p.hz, 16);
  while (p.ky > 1 && smem_y_bytes<double>(p.ky, p.ny) > 96 * 1024) p.ky /= 2;
  // kz columns per x-pass tile: 8 (64-byte runs of the spectrum per x), 4 on grids of up
  // to 64 points along x, where 8 would leave about two blocks per SM
  p.kx = std::min(p.hz, p.nx <= 64 ? 4 : 8);
  while (p.kx > 1 && smem_x_bytes<double>(p.kx, p.nx) > 100 * 1024) p.kx /= 2;
  // float x tiles: the double tile unless SSFFT_XPASS_KX asks for another power of two
  // that fits
  p.kx_f = p.kx;
  const int want_kx = env_int("SSFFT_XPASS_KX");
  if (want_kx >= 1 && want_kx <= 32 && (want_kx & (want_kx - 1)) == 0 &&
      smem_x_bytes<float>(std::min(want_kx, p.hz), p.nx) <= SMEM_LIMIT)
    p.kx_f = std::min(want_kx, p.hz);
  if (smem_z_bytes<double>(p.lz, p.nz) > SMEM_LIMIT || smem_y_bytes<double>(p.ky, p.ny) > SMEM_LIMIT ||
      smem_x_bytes<double>(p.kx, p.nx) > SMEM_LIMIT)
    return ssfft_internal_fail(SSFFT_E_UNSUPPORTED, "grid too large for the shared-memory FFT passes");
  return 0;
}

static void plan_free(GridPlan &p) {
  for (int k = 0; k < 2; ++k)
    for (int a = 0; a < 3; ++a) {
      if (p.tw[k][a]) cudaFree(p.tw[k][a]);
      if (p.tn[k][a]) cudaFree(p.tn[k][a]);
      p.tw[k][a] = p.tn[k][a] = nullptr;
    }
}

template <typename T, typename TF> static int set_kernel_attrs(size_t smax);

static int plan_create(GridPlan &p, const ssfft_config *cfg, cudaStream_t stream) {
  memset(&p, 0, sizeof(p));
  p.dev = cfg->device;
  p.fp64 = cfg->precision == SSFFT_FP64;
  p.nx = cfg->n[0];
  p.ny = cfg->n[1];
  p.nz = cfg->n[2];
  p.hz = p.nz / 2 + 1;
  p.V = (long long)p.nx * p.ny * p.nz;
  // stored half-spectrum columns: the Nyquist column of an even grid is not stored
  p.S = (long long)p.nx * p.ny * ((p.nz % 2 == 0) ? p.nz / 2 : p.hz);
  make_axis_plan(p.nx, p.px);
  make_axis_plan(p.ny, p.py);
  make_axis_plan(p.nz, p.pz);
  p.use_plane = env_int("SSFFT_NO_PLANE") != 1;
  CKR(plan_tiles(p));
  // FFT tables: float ones for the mixed-mode Krylov transforms, double ones for every
  // double-precision transform
  const int dims[3] = {p.nx, p.ny, p.nz};
  const int tcount[3] = {p.nx, p.ny, p.hz};
  for (int k = (p.fp64 ? 1 : 0); k < 2; ++k)
    for (int a = 0; a < 3; ++a) {
      const size_t es = k ? 8 : 4;
      ALLOC(p.tw[k][a], (size_t)dims[a] * 2 * es);
      ALLOC(p.tn[k][a], (size_t)tcount[a] * es);
      if (k) {
        auto tw = twiddles<double>(dims[a]);
        auto tn = tan_table<double>(dims[a], tcount[a]);
        CK(cudaMemcpyAsync(p.tw[k][a], tw.data(), tw.size() * es, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(p.tn[k][a], tn.data(), tn.size() * es, cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));  // the host vectors go out of scope
      } else {
        auto tw = twiddles<float>(dims[a]);
        auto tn = tan_table<float>(dims[a], tcount[a]);
        CK(cudaMemcpyAsync(p.tw[k][a], tw.data(), tw.size() * es, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(p.tn[k][a], tn.data(), tn.size() * es, cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
      }
    }
  fill_grid<double>(p);
  if (!p.fp64) fill_grid<float>(p);
  // items of one slot per reduction, times the values each stores
  const Grid<double> &g = p.gd;
  size_t need = 0;
  need = std::max(need, (size_t)3 * items_z(g));
  need = std::max(need, (size_t)3 * CLUSTER_MAX * items_plane(g));
  need = std::max(need, (size_t)NORM_VALS * norm_items(p.V));
  need = std::max(need, (size_t)21 * vec_items(p.V));
  need = std::max(need, (size_t)vec_items(6 * p.V));
  if (items_z(g) > MAX_ITEMS_PER_SLOT || vec_items(6 * p.V) > MAX_ITEMS_PER_SLOT ||
      items_y(g) > (1 << 30) / 2)
    return ssfft_internal_fail(SSFFT_E_UNSUPPORTED, "grid too large for the reduction partials");
  p.partial_doubles = need;
  CKR((set_kernel_attrs<double, double>(SMEM_LIMIT)));
  CKR((set_kernel_attrs<float, float>(SMEM_LIMIT)));
  CKR((set_kernel_attrs<double, float>(SMEM_LIMIT)));
  return 0;
}

// ---------------------------------------------------------------------------------------
// kernel attributes
// ---------------------------------------------------------------------------------------
template <typename F> static int smem_attr(F f, int m) {
  CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
  return 0;
}

template <typename T, typename TF, int PT> static int plane_attrs(int m) {
  CKR(smem_attr(zyfwd_kernel<T, TF, PRO_INPUT, PT>, m));
  CKR(smem_attr(zyfwd_kernel<T, TF, PRO_RESIDUAL, PT>, m));
  CKR(smem_attr(zyfwd_kernel<T, TF, PRO_REPROJECT, PT>, m));
  CKR(smem_attr(yzinv_kernel<T, TF, EPI_STORE, PT>, m));
  CKR(smem_attr(yzinv_kernel<T, TF, EPI_RESIDUAL, PT>, m));
  CKR(smem_attr(yzinv_kernel<T, TF, EPI_REPROJECT, PT>, m));
  if (sizeof(T) == sizeof(TF)) {
    CKR(smem_attr(zyfwd_kernel<T, T, PRO_TAU, PT>, m));
    CKR(smem_attr(yzinv_kernel<T, T, EPI_PTAU, PT>, m));
  }
  return 0;
}

template <typename T, typename TF, int PT> static int cluster_attrs(int m) {
  CKR(smem_attr(zyfwd_cl_kernel<T, TF, PRO_INPUT, PT>, m));
  CKR(smem_attr(zyfwd_cl_kernel<T, TF, PRO_RESIDUAL, PT>, m));
  CKR(smem_attr(zyfwd_cl_kernel<T, TF, PRO_REPROJECT, PT>, m));
  CKR(smem_attr(yzinv_cl_kernel<T, TF, EPI_STORE, PT>, m));
  CKR(smem_attr(yzinv_cl_kernel<T, TF, EPI_RESIDUAL, PT>, m));
  CKR(smem_attr(yzinv_cl_kernel<T, TF, EPI_REPROJECT, PT>, m));
  if (sizeof(T) == sizeof(TF)) {
    CKR(smem_attr(zyfwd_cl_kernel<T, T, PRO_TAU, PT>, m));
    CKR(smem_attr(yzinv_cl_kernel<T, T, EPI_PTAU, PT>, m));
  }
  return 0;
}

// Opt every shared-memory-hungry kernel instantiation into up to `smax` bytes.
template <typename T, typename TF> static int set_kernel_attrs(size_t smax) {
  const int m = (int)smax;
  CKR(smem_attr(zfwd_kernel<T, TF, PRO_INPUT>, m));
  CKR(smem_attr(zfwd_kernel<T, TF, PRO_RESIDUAL>, m));
  CKR(smem_attr(zfwd_kernel<T, TF, PRO_REPROJECT>, m));
  CKR((smem_attr(ypass_kernel<T, TF, false, false>, m)));
  CKR((smem_attr(ypass_kernel<T, TF, true, false>, m)));
  CKR((smem_attr(ypass_kernel<T, TF, false, true>, m)));
  CKR((smem_attr(ypass_kernel<T, TF, true, true>, m)));
  CKR((smem_attr(xpass_kernel<T, TF, false>, m)));
  CKR((smem_attr(xpass_kernel<T, TF, true>, m)));
  if constexpr (sizeof(T) == 4) {
    CKR((smem_attr(xpass_kernel<T, TF, false, 192>, m)));
    CKR((smem_attr(xpass_kernel<T, TF, true, 192>, m)));
    CKR((smem_attr(xpass_kernel<T, TF, false, 384>, m)));
    CKR((smem_attr(xpass_kernel<T, TF, true, 384>, m)));
  }
  CKR(smem_attr(zinv_kernel<T, TF, EPI_STORE>, m));
  CKR(smem_attr(zinv_kernel<T, TF, EPI_RESIDUAL>, m));
  CKR(smem_attr(zinv_kernel<T, TF, EPI_REPROJECT>, m));
  CKR((plane_attrs<T, TF, 512>(m)));
  CKR((plane_attrs<T, TF, 1024>(m)));
  CKR((cluster_attrs<T, TF, 256>(m)));
  CKR((cluster_attrs<T, TF, 512>(m)));
  CKR((cluster_attrs<T, TF, 1024>(m)));
  if (sizeof(T) == sizeof(TF)) {
    CKR(smem_attr(constitutive_kernel<T>, (int)constitutive_smem_bytes()));
    CKR(smem_attr(zfwd_kernel<T, T, PRO_TAU>, m));
    CKR(smem_attr(zinv_kernel<T, T, EPI_PTAU>, m));
  }
  return 0;
}

// ---------------------------------------------------------------------------------------
// one slot's device buffers
// ---------------------------------------------------------------------------------------
// Allocations are owned here (freed by slot_free); the descriptor mirror holds the same
// pointers in their current roles, which swaps change.
struct SlotBufs {
  bool fp64;
  size_t rs;                   // sizeof(real)
  long long V;
  void *field[14];             // 6-plane fields: eps, eps_old, dfl, sig x3 (double), b, kr[7]
  void *spec;
  double *partials;
  unsigned int *tickets;
  double *results;
  MinresState *st;
  int *citers;
  // microstructure (capacities grow on rebinding)
  PhaseParams hparams[SSFFT_MAX_PHASES];
  bool phase_set[SSFFT_MAX_PHASES];
  PhaseParams *dparams;
  int32_t *orient, *phase, *gid;
  double *rm_tab;
  size_t cap_rm, cap_ktab;
  void *ktab;
  void *kvox_buf[2];
  double *slip_buf[5];         // g_in, g_out, g_old, gam (two)
  int cap_nslip;
  double *ep_buf[2], *Gam_buf[2];
  bool micro_set, have_phase_buf, voxel_mode, any_evp, any_j2;
  int nslip_max, n_orient, n_gid;
  SlotDev<float> mf;           // descriptor mirror (the one of the solve precision is used)
  SlotDev<double> md;
};

template <typename T> static SlotDev<T> &mirror(SlotBufs &b);
template <> SlotDev<float> &mirror<float>(SlotBufs &b) { return b.mf; }
template <> SlotDev<double> &mirror<double>(SlotBufs &b) { return b.md; }

static size_t field_bytes(const SlotBufs &b, int planes) {
  return (size_t)planes * (size_t)b.V * b.rs;
}

// Bytes of field[i]: the strain and stress fields (0..5) are double in both precisions.
static size_t field_bytes_of(const SlotBufs &b, int i) {
  return i < 6 ? (size_t)6 * (size_t)b.V * sizeof(double) : field_bytes(b, 6);
}

static int slot_alloc(SlotBufs &b, const GridPlan &p, cudaStream_t stream) {
  memset((void *)&b, 0, sizeof(b));
  b.fp64 = p.fp64;
  b.rs = p.fp64 ? 8 : 4;
  b.V = p.V;
  for (int i = 0; i < 14; ++i) {
    ALLOC(b.field[i], field_bytes_of(b, i));
    CK(cudaMemsetAsync(b.field[i], 0, field_bytes_of(b, i), stream));
  }
  ALLOC(b.spec, (size_t)6 * p.S * 16);  // sized for double-precision transforms
  ALLOC(b.partials, p.partial_doubles * sizeof(double));
  ALLOC(b.tickets, 16 * sizeof(unsigned int));
  CK(cudaMemsetAsync(b.tickets, 0, 16 * sizeof(unsigned int), stream));
  ALLOC(b.results, 64 * sizeof(double));
  CK(cudaMemsetAsync(b.results, 0, 64 * sizeof(double), stream));
  ALLOC(b.st, sizeof(MinresState));
  CK(cudaMemsetAsync(b.st, 0, sizeof(MinresState), stream));
  ALLOC(b.citers, 4 * sizeof(int));
  CK(cudaMemsetAsync(b.citers, 0, 4 * sizeof(int), stream));
  ALLOC(b.dparams, SSFFT_MAX_PHASES * sizeof(PhaseParams));
  return 0;
}

static void slot_free(SlotBufs &b) {
  void *ptrs[] = {b.spec, b.partials, b.tickets, b.results, b.st, b.citers, b.dparams,
                  b.orient, b.phase, b.gid, b.rm_tab, b.ktab, b.kvox_buf[0], b.kvox_buf[1],
                  b.slip_buf[0], b.slip_buf[1], b.slip_buf[2], b.slip_buf[3], b.slip_buf[4],
                  b.ep_buf[0], b.ep_buf[1], b.Gam_buf[0], b.Gam_buf[1]};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  for (int i = 0; i < 14; ++i)
    if (b.field[i]) cudaFree(b.field[i]);
  memset((void *)&b, 0, sizeof(b));
}

// The descriptor in its initial roles (after allocation or rebinding), with the solve
// options of cfg.
template <typename T> static void mirror_init(SlotBufs &b, const ssfft_config &cfg) {
  SlotDev<T> &m = mirror<T>(b);
  memset((void *)&m, 0, sizeof(m));
  T **f = reinterpret_cast<T **>(b.field);
  double **fd = reinterpret_cast<double **>(b.field);
  m.eps = fd[0];
  m.eps_old = fd[1];
  m.dfl = fd[2];
  m.sig = fd[3];
  m.sig_next = fd[4];
  m.sig_old = fd[5];
  m.b = f[6];
  for (int i = 0; i < 7; ++i) m.kr[i] = f[7 + i];
  m.spec = b.spec;
  m.gid = b.gid;
  m.ktab = (const T *)b.ktab;
  m.kvox = (T *)b.kvox_buf[0];
  m.kvox_old = (T *)b.kvox_buf[1];
  m.voxel_mode = b.voxel_mode ? 1 : 0;
  m.phase = b.have_phase_buf ? b.phase : nullptr;
  m.orient = b.orient;
  m.rm_tab = b.rm_tab;
  m.params = b.dparams;
  m.n_params = 1;
  for (int k = 0; k < SSFFT_MAX_PHASES; ++k)
    if (b.phase_set[k]) m.n_params = k + 1;
  m.nslip = b.nslip_max;
  m.any_evp = b.any_evp ? 1 : 0;
  m.any_j2 = b.any_j2 ? 1 : 0;
  m.g_in = b.slip_buf[0];
  m.g_out = b.slip_buf[1];
  m.g_old = b.slip_buf[2];
  m.gam_old = b.slip_buf[3];
  m.gam_trial = b.slip_buf[4];
  m.ep_old = b.ep_buf[0];
  m.ep_trial = b.ep_buf[1];
  m.Gam_old = b.Gam_buf[0];
  m.Gam_trial = b.Gam_buf[1];
  m.st = b.st;
  m.partials = b.partials;
  m.tickets = b.tickets;
  m.results = b.results;
  m.citers = b.citers;
  for (int c = 0; c < 6; ++c) m.mask[c] = (cfg.stress_mask[c] != 0.0) ? 1.0 : 0.0;
  m.fluct_scale = 1.0;
  m.dt = 1.0;
}

// Commit of a converged increment (update_state_variables; old_* <- current,
// small_strain_fft.py:213-218): roles swap; the slip resistances are copied by
// commit_slip_kernel.
template <typename T> static void mirror_commit(SlotDev<T> &m) {
  std::swap(m.sig_old, m.sig);
  std::swap(m.eps_old, m.eps);
  std::swap(m.kvox_old, m.kvox);
  std::swap(m.gam_old, m.gam_trial);
  std::swap(m.ep_old, m.ep_trial);
  std::swap(m.Gam_old, m.Gam_trial);
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

template <typename T>
static void build_ktab(const SlotBufs &b, const std::vector<double> &Rm,
                       const std::vector<int> &gid_orient, const std::vector<int> &gid_phase,
                       std::vector<T> &tab) {
  const int n = (int)gid_orient.size();
  tab.assign((size_t)n * 21, (T)0);
  for (int g = 0; g < n; ++g) {
    const double *R = &Rm[(size_t)gid_orient[g] * 36];
    const double *C = b.hparams[gid_phase[g]].C;
    double CR[36];
    for (int i = 0; i < 6; ++i)
      for (int c = 0; c < 6; ++c) {
        double acc = 0.0;
        for (int j = 0; j < 6; ++j) acc += C[i * 6 + j] * R[j * 6 + c];
        CR[i * 6 + c] = acc;
      }
    for (int a = 0; a < 6; ++a)
      for (int c = a; c < 6; ++c) {
        double acc = 0.0;
        for (int i = 0; i < 6; ++i) acc += R[i * 6 + a] * CR[i * 6 + c];
        tab[(size_t)g * 21 + sym_idx(a, c)] = (T)acc;
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
    return ssfft_internal_fail(SSFFT_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  *cap = bytes;
  return 0;
}

// Bind a microstructure to a slot whose phases are set (Elastic/ElasticViscoplastic/
// Multiphase initialize, small_strain_fft.py:94): rotations, orientation and phase per
// point, and the tangent table (elastic phases only) or per-voxel tangent and plastic
// state buffers.  Host pointers are read during the call (uploads are synchronised).
static int slot_bind(SlotBufs &b, const ssfft_config &cfg, int n_orient, const double *rotations,
                     const int32_t *orient_of_point, const int32_t *phase_of_point,
                     cudaStream_t stream) {
  if (n_orient < 1 || !rotations || !orient_of_point)
    return ssfft_internal_fail(SSFFT_E_INVALID, "rotations and orientation indices are required");
  const long long V = b.V;
  int max_phase = 0;
  for (long long v = 0; v < V; ++v) {
    const int o = orient_of_point[v];
    const int ph = phase_of_point ? phase_of_point[v] : 0;
    if (o < 0 || o >= n_orient)
      return ssfft_internal_fail(SSFFT_E_INVALID, "orientation index out of range");
    if (ph < 0 || ph >= SSFFT_MAX_PHASES || !b.phase_set[ph])
      return ssfft_internal_fail(SSFFT_E_INVALID, "point refers to an undefined phase");
    max_phase = std::max(max_phase, ph);
  }
  b.any_evp = false;
  b.any_j2 = false;
  b.nslip_max = 0;
  for (int ph = 0; ph < SSFFT_MAX_PHASES; ++ph) {
    if (!b.phase_set[ph]) continue;
    if (b.hparams[ph].kind == PHASE_EVP) {
      b.any_evp = true;
      b.nslip_max = std::max(b.nslip_max, b.hparams[ph].nslip);
    } else if (b.hparams[ph].kind == PHASE_J2) {
      b.any_evp = true;
      b.any_j2 = true;
      b.nslip_max = std::max(b.nslip_max, 1);
    }
  }
  b.micro_set = false;
  b.voxel_mode = b.any_evp;
  b.n_orient = n_orient;
  std::vector<double> Rm((size_t)n_orient * 36);
  for (int o = 0; o < n_orient; ++o) rotation_mandel(rotations + (size_t)o * 9, &Rm[(size_t)o * 36]);
  CKR(ensure_buffer((void **)&b.rm_tab, &b.cap_rm, Rm.size() * sizeof(double)));
  CK(cudaMemcpyAsync(b.rm_tab, Rm.data(), Rm.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  if (!b.orient) ALLOC(b.orient, V * sizeof(int32_t));
  CK(cudaMemcpyAsync(b.orient, orient_of_point, V * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
  if (phase_of_point) {
    if (!b.phase) ALLOC(b.phase, V * sizeof(int32_t));
    CK(cudaMemcpyAsync(b.phase, phase_of_point, V * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
  }
  b.have_phase_buf = phase_of_point != nullptr;
  CK(cudaMemcpyAsync(b.dparams, b.hparams, sizeof(b.hparams), cudaMemcpyHostToDevice, stream));
  if (!b.voxel_mode) {
    // tangent table over the distinct (orientation, phase) pairs present
    std::vector<int> key_to_gid((size_t)n_orient * (max_phase + 1), -1);
    std::vector<int> g_or, g_ph;
    std::vector<int32_t> gid(V);
    for (long long v = 0; v < V; ++v) {
      const int o = orient_of_point[v], ph = phase_of_point ? phase_of_point[v] : 0;
      int &slot = key_to_gid[(size_t)ph * n_orient + o];
      if (slot < 0) {
        slot = (int)g_or.size();
        g_or.push_back(o);
        g_ph.push_back(ph);
      }
      gid[v] = slot;
    }
    b.n_gid = (int)g_or.size();
    if (!b.gid) ALLOC(b.gid, V * sizeof(int32_t));
    CK(cudaMemcpyAsync(b.gid, gid.data(), V * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
    if (b.fp64) {
      std::vector<double> tab;
      build_ktab<double>(b, Rm, g_or, g_ph, tab);
      CKR(ensure_buffer(&b.ktab, &b.cap_ktab, tab.size() * sizeof(double)));
      CK(cudaMemcpyAsync(b.ktab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
      CK(cudaStreamSynchronize(stream));
    } else {
      std::vector<float> tab;
      build_ktab<float>(b, Rm, g_or, g_ph, tab);
      CKR(ensure_buffer(&b.ktab, &b.cap_ktab, tab.size() * sizeof(float)));
      CK(cudaMemcpyAsync(b.ktab, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
      CK(cudaStreamSynchronize(stream));
    }
  } else {
    if (!b.kvox_buf[0]) {
      ALLOC(b.kvox_buf[0], field_bytes(b, 21));
      ALLOC(b.kvox_buf[1], field_bytes(b, 21));
    }
    const int S = b.nslip_max;
    if (b.cap_nslip < S) {
      for (double *&q : b.slip_buf) {
        if (q) cudaFree(q);
        q = nullptr;
      }
      for (double *&q : b.slip_buf) ALLOC(q, (size_t)S * V * 8);
      b.cap_nslip = S;
    }
    if (!b.ep_buf[0]) {
      ALLOC(b.ep_buf[0], (size_t)6 * V * 8);
      ALLOC(b.ep_buf[1], (size_t)6 * V * 8);
      ALLOC(b.Gam_buf[0], (size_t)V * 8);
      ALLOC(b.Gam_buf[1], (size_t)V * 8);
    }
  }
  CK(cudaStreamSynchronize(stream));  // host arrays of this call go out of scope
  b.micro_set = true;
  if (b.fp64)
    mirror_init<double>(b, cfg);
  else
    mirror_init<float>(b, cfg);
  return 0;
}

// Solve state at t = start: zero strain, stress and fluctuation, initial tangents and
// slip resistances (the descriptor returns to its initial roles).
static int slot_reset(SlotBufs &b, const ssfft_config &cfg, cudaStream_t stream) {
  if (!b.micro_set) return ssfft_internal_fail(SSFFT_E_INVALID, "microstructure not set");
  if (b.fp64)
    mirror_init<double>(b, cfg);
  else
    mirror_init<float>(b, cfg);
  for (int i = 0; i < 7; ++i) CK(cudaMemsetAsync(b.field[i], 0, field_bytes_of(b, i), stream));
  const long long V = b.V;
  const int eb = std::max(1, std::min(div_up(V, SSFFT_THREADS), 148 * 16));
  const int32_t *ph = b.have_phase_buf ? b.phase : nullptr;
  if (b.voxel_mode) {
    if (b.fp64)
      init_kvox_kernel<double><<<eb, SSFFT_THREADS, 0, stream>>>(V, ph, b.orient, b.dparams,
                                                               b.rm_tab, (double *)b.kvox_buf[0]);
    else
      init_kvox_kernel<float><<<eb, SSFFT_THREADS, 0, stream>>>(V, ph, b.orient, b.dparams,
                                                              b.rm_tab, (float *)b.kvox_buf[0]);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(b.kvox_buf[1], b.kvox_buf[0], field_bytes(b, 21), cudaMemcpyDeviceToDevice,
                       stream));
  }
  if (b.any_evp) {
    const int S = b.nslip_max;
    evp_init_kernel<<<eb, SSFFT_THREADS, 0, stream>>>(V, S, ph, b.dparams, b.slip_buf[0],
                                                      b.slip_buf[1], b.slip_buf[2]);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(b.slip_buf[3], 0, (size_t)S * V * 8, stream));
    CK(cudaMemsetAsync(b.slip_buf[4], 0, (size_t)S * V * 8, stream));
    for (int k = 0; k < 2; ++k) {
      CK(cudaMemsetAsync(b.ep_buf[k], 0, (size_t)6 * V * 8, stream));
      CK(cudaMemsetAsync(b.Gam_buf[k], 0, (size_t)V * 8, stream));
    }
  }
  return 0;
}

// Slot options (stress mask) into the descriptor.
template <typename T> static void mirror_options(SlotDev<T> &m, const ssfft_config &cfg) {
  for (int c = 0; c < 6; ++c) m.mask[c] = (cfg.stress_mask[c] != 0.0) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------------------
// launches over a slot list (cap: slots the list can hold; the grid is sized for it)
// ---------------------------------------------------------------------------------------
struct LaunchCtx {
  const GridPlan *p;
  SlotList list;
  int cap;
  cudaStream_t stream;
  long long *launches;
};

// The passes of one projection.  ev (optional, 6 events) is recorded before the first pass
// and after each of the five pass slots z-fwd, y-fwd, x, y-inv, z-inv; with the
// plane-fused passes the y slots are empty (zero time).
template <typename T, typename TF, int PRO, int EPI>
static int launch_projector(const LaunchCtx &c, const SlotDev<TF> *tab, ExtIO<TF> io = {},
                            cudaEvent_t *ev = nullptr) {
  const GridPlan &p = *c.p;
  const Grid<T> &g = grid_of<T>(p);
  // the middle passes of a Krylov matvec skip finished solves as the outer ones do (a
  // device-side loop runs its chunk of iterations to the end after a solve finishes)
  constexpr bool KRY = PRO_IS_KRYLOV(PRO) || PRO == PRO_TAU;
  auto rec = [&](int k) {
    if (ev) cudaEventRecord(ev[k], c.stream);
  };
  const size_t sx = smem_x_bytes<T>(g.kx, p.nx);
  const int dev = p.dev;
  rec(0);
  if (const int C = cluster_size<T>(p)) {
    const ClusterGeo q = cluster_geo<T>(p, C);
    const size_t sp = smem_cplane_bytes<T>(p.ny, p.nz, g.hs, C);
    const long long it = (long long)c.cap * items_plane(g);
    const int pt = cluster_threads<T>(p, C);
    if (pt == 1024)
      CKR(launch_clustered(zyfwd_cl_kernel<T, TF, PRO, 1024>, C, 1024, sp, it, dev, c.stream, g, q, tab, c.list, io));
    else if (pt == 256)
      CKR(launch_clustered(zyfwd_cl_kernel<T, TF, PRO, 256>, C, 256, sp, it, dev, c.stream, g, q, tab, c.list, io));
    else
      CKR(launch_clustered(zyfwd_cl_kernel<T, TF, PRO, 512>, C, 512, sp, it, dev, c.stream, g, q, tab, c.list, io));
    rec(1);
    rec(2);
    launch_xpass<T, TF, KRY>(g, sx, (long long)c.cap * items_x(g), dev, c.stream, tab, c.list);
    rec(3);
    rec(4);
    if (pt == 1024)
      CKR(launch_clustered(yzinv_cl_kernel<T, TF, EPI, 1024>, C, 1024, sp, it, dev, c.stream, g, q, tab, c.list, io));
    else if (pt == 256)
      CKR(launch_clustered(yzinv_cl_kernel<T, TF, EPI, 256>, C, 256, sp, it, dev, c.stream, g, q, tab, c.list, io));
    else
      CKR(launch_clustered(yzinv_cl_kernel<T, TF, EPI, 512>, C, 512, sp, it, dev, c.stream, g, q, tab, c.list, io));
    rec(5);
    if (c.launches) *c.launches += 3;
  } else if (plane_ok<T>(p)) {
    const size_t sp = smem_plane_bytes<T>(p.ny, p.nz);
    const long long it = (long long)c.cap * items_plane(g);
    if (plane_threads<T>(p) == 1024) {
      auto kf = zyfwd_kernel<T, TF, PRO, 1024>;
      kf<<<persistent_grid(kf, 1024, sp, it, dev), 1024, sp, c.stream>>>(g, tab, c.list, io);
    } else {
      auto kf = zyfwd_kernel<T, TF, PRO, 512>;
      kf<<<persistent_grid(kf, 512, sp, it, dev), 512, sp, c.stream>>>(g, tab, c.list, io);
    }
    rec(1);
    rec(2);
    launch_xpass<T, TF, KRY>(g, sx, (long long)c.cap * items_x(g), dev, c.stream, tab, c.list);
    rec(3);
    rec(4);
    if (plane_threads<T>(p) == 1024) {
      auto ki = yzinv_kernel<T, TF, EPI, 1024>;
      ki<<<persistent_grid(ki, 1024, sp, it, dev), 1024, sp, c.stream>>>(g, tab, c.list, io);
    } else {
      auto ki = yzinv_kernel<T, TF, EPI, 512>;
      ki<<<persistent_grid(ki, 512, sp, it, dev), 512, sp, c.stream>>>(g, tab, c.list, io);
    }
    rec(5);
    if (c.launches) *c.launches += 3;
  } else {
    const size_t sz = smem_z_bytes<T>(p.lz, p.nz);
    const size_t sy = smem_y_bytes<T>(p.ky, p.ny);
    const long long itz = (long long)c.cap * items_z(g);
    const long long ity = (long long)c.cap * items_y(g);
    auto kz = zfwd_kernel<T, TF, PRO>;
    kz<<<persistent_grid(kz, SSFFT_THREADS, sz, itz, dev), SSFFT_THREADS, sz, c.stream>>>(g, tab, c.list, io);
    rec(1);
    auto ky = ypass_kernel<T, TF, false, KRY>;
    ky<<<persistent_grid(ky, SSFFT_THREADS, sy, ity, dev), SSFFT_THREADS, sy, c.stream>>>(g, tab, c.list);
    rec(2);
    launch_xpass<T, TF, KRY>(g, sx, (long long)c.cap * items_x(g), dev, c.stream, tab, c.list);
    rec(3);
    auto kyi = ypass_kernel<T, TF, true, KRY>;
    kyi<<<persistent_grid(kyi, SSFFT_THREADS, sy, ity, dev), SSFFT_THREADS, sy, c.stream>>>(g, tab, c.list);
    rec(4);
    auto kzi = zinv_kernel<T, TF, EPI>;
    kzi<<<persistent_grid(kzi, SSFFT_THREADS, sz, itz, dev), SSFFT_THREADS, sz, c.stream>>>(g, tab, c.list, io);
    rec(5);
    if (c.launches) *c.launches += 5;
  }
  CK(cudaGetLastError());
  return 0;
}

// One MINRES iteration on every listed slot whose solve is not done: the projector passes
// with the pending vector update in the forward prologue and the scalar recurrence in the
// inverse epilogue.
// ev (optional, 8 events): ev[7] before the update kernel, ev[0..5] by the projector (the
// epilogue kernel follows ev[5]).
template <typename T>
static int launch_krylov_iteration(const LaunchCtx &c, const SlotDev<T> *tab, bool voxel,
                                   cudaEvent_t *ev = nullptr) {
  if (ev) cudaEventRecord(ev[7], c.stream);
  const long long it = (long long)c.cap * vec_items(c.p->V);
  if (voxel) {
    auto k = krylov_update_kernel<T, PRO_TANGENT_VOXEL>;
    k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  } else {
    auto k = krylov_update_kernel<T, PRO_TANGENT_TABLE>;
    k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  }
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  CKR((launch_projector<T, T, PRO_TAU, EPI_PTAU>(c, tab, {}, ev)));
  auto ke = krylov_epilogue_kernel<T>;
  ke<<<persistent_grid(ke, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

// b = P(Sbar - sigma) into each slot's b, max|b| into results[40].  The transform always
// runs in double: in the mixed mode the float stress field is read and b is stored as
// float, but the equilibrium residual and its norm are double-precision quantities.
template <typename T> static int launch_residual(const LaunchCtx &c, const SlotDev<T> *tab) {
  return launch_projector<double, T, PRO_RESIDUAL, EPI_RESIDUAL>(c, tab);
}

// Mixed mode: project each slot's Newton correction x back onto compatible strain fields
// with a double-precision transform (x <- Gamma-hat : x, an identity in exact arithmetic),
// then strain += x and fluctuation += x.  Float Krylov iterates pick up round-off in the
// null space of Gamma-hat K, which the equilibrium test cannot see; this removes it.
template <typename T> static int launch_reproject_update(const LaunchCtx &c, const SlotDev<T> *tab) {
  return launch_projector<double, T, PRO_REPROJECT, EPI_REPROJECT>(c, tab);
}

template <typename T>
static int launch_minres_init(const LaunchCtx &c, const SlotDev<T> *tab) {
  auto k = minres_init_kernel<T>;
  const long long it = (long long)c.cap * vec_items(6 * c.p->V);
  k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

template <typename T> static int launch_strain_guess(const LaunchCtx &c, const SlotDev<T> *tab) {
  auto k = strain_guess_kernel<T>;
  const long long it = (long long)c.cap * vec_items(c.p->V);
  k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

template <typename T> static int launch_update_strain(const LaunchCtx &c, const SlotDev<T> *tab) {
  auto k = update_strain_kernel<T>;
  const long long it = (long long)c.cap * vec_items(6 * c.p->V);
  k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

template <typename T> static int launch_norms(const LaunchCtx &c, const SlotDev<T> *tab) {
  auto k = newton_norms_kernel<T>;
  const long long it = (long long)c.cap * norm_items(c.p->V);
  k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

template <typename T> static int launch_tangent_sum(const LaunchCtx &c, const SlotDev<T> *tab) {
  auto k = tangent_sum_kernel<T>;
  const long long it = (long long)c.cap * vec_items(c.p->V);
  k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

// Constitutive update of every listed slot (j2: with the J2 counting pass first).  Each
// slot's citers must be cleared before.
template <typename T>
static int launch_constitutive(const LaunchCtx &c, const SlotDev<T> *tab, bool j2) {
  const long long it = (long long)c.cap * const_items(c.p->V);
  if (j2) {
    auto kj = j2_count_kernel<T>;
    kj<<<persistent_grid(kj, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(tab, c.list, c.p->V);
    if (c.launches) *c.launches += 1;
    CK(cudaGetLastError());
  }
  const size_t sm = constitutive_smem_bytes();
  auto k = constitutive_kernel<T>;
  k<<<persistent_grid(k, CONST_THREADS, sm, it, c.p->dev), CONST_THREADS, sm, c.stream>>>(tab, c.list, c.p->V);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}

template <typename T>
static int launch_commit_slip(const LaunchCtx &c, const SlotDev<T> *tab, int nslip_max) {
  if (nslip_max < 1) return 0;
  auto k = commit_slip_kernel<T>;
  const long long it = (long long)c.cap * vec_items((long long)nslip_max * c.p->V);
  k<<<persistent_grid(k, SSFFT_THREADS, 0, it, c.p->dev), SSFFT_THREADS, 0, c.stream>>>(
      tab, c.list, c.p->V, nslip_max);
  if (c.launches) *c.launches += 1;
  CK(cudaGetLastError());
  return 0;
}


// 6x6 inverse by Gauss-Jordan with partial pivoting (host and device, double).
__host__ __device__ inline bool inv6(const double *A, double *Ainv) {
  double a[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 12; ++j) a[i][j] = (j < 6) ? A[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
    if (a[p][c] == 0.0) return false;
    if (p != c)
      for (int j = 0; j < 12; ++j) {
        const double t = a[p][j];
        a[p][j] = a[c][j];
        a[c][j] = t;
      }
    const double d = a[c][c];
    for (int j = 0; j < 12; ++j) a[c][j] /= d;
    for (int r = 0; r < 6; ++r)
      if (r != c) {
        const double f = a[r][c];
        if (f != 0.0)
          for (int j = 0; j < 12; ++j) a[r][j] -= mul_rn(f, a[c][j]);
      }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ainv[i * 6 + j] = a[i][j + 6];
  return true;
}

