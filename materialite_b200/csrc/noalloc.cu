// ssfft_apply_projection_noalloc: the compatibility projection
//   out = ifftn( Gamma-hat : fftn(in) ).real
// in double precision, for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not allowed -- for
// example inside a host callback or a library hook that must not touch the allocator,
// a process whose memory pool is owned by someone else (a framework's caching allocator
// that forbids foreign allocations), or a real-time loop that may not block on an
// allocation.  The handle-based entry points allocate their spectrum, twiddle tables
// and reduction buffers in ssfft_create; this one instead uses the file-scope device
// array below, which every GPU that loads libssfft holds until the process exits.
//
// Limits and rules:
//   * at most NOALLOC_MAX_SPEC_POINTS half-spectrum points (nx * ny * (nz/2 + 1)), i.e.
//     grids up to 64^3, and at most 1024 points per axis; larger grids are rejected;
//   * the first call on a device looks up the array's device address and sets kernel
//     attributes (once per device, kept for the life of the process); make that first
//     call before any stream capture.  The cached address belongs to the device's primary
//     context: after cudaDeviceReset() on that device, do not call this entry point again
//     in the same process;
//   * every call shares the one array: calls that overlap on the GPU (for example on two
//     streams) race and corrupt each other's results.  The spectrum is completely
//     overwritten by each call, so nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/ssfft.h"
#include "common.cuh"
#include "fft.cuh"
#include "projector.cuh"

#define NOALLOC_MAX_SPEC_POINTS (64 * 64 * 33)
#define NOALLOC_MAX_AXIS 1024
#define NOALLOC_MAX_DEVICES 64
#define NOALLOC_TABLE_OFFSET (6 * NOALLOC_MAX_SPEC_POINTS)
#define NOALLOC_DESC_OFFSET (NOALLOC_TABLE_OFFSET + 3 * NOALLOC_MAX_AXIS + 2 * NOALLOC_MAX_AXIS)
#define NOALLOC_DESC_ELEMS 64  // room for the one-slot descriptor
#define NOALLOC_LIST_OFFSET (NOALLOC_DESC_OFFSET + NOALLOC_DESC_ELEMS)
#define NOALLOC_ELEMS (NOALLOC_LIST_OFFSET + 1)

static_assert(sizeof(SlotDev<double>) <= NOALLOC_DESC_ELEMS * sizeof(double2),
              "slot descriptor does not fit its scratch space");

// spectrum (6 components), then 3 twiddle tables (double2), then 3 tan tables (double),
// then the slot descriptor the transform kernels read and the slot list {0, 1}
static __device__ __align__(256) double2 g_noalloc_scratch[NOALLOC_ELEMS];

// Failure messages go to ssfft_last_error() (defined in ssfft.cu).
int ssfft_internal_fail(int code, const std::string &msg);

static std::mutex g_noalloc_mutex;
static double2 *g_noalloc_addr[NOALLOC_MAX_DEVICES];

static int noalloc_fail(int code, const std::string &msg) { return ssfft_internal_fail(code, msg); }

// Twiddles e^{-2 pi i k/n} and tan(pi f) (f = fftfreq) for the three axes.
__global__ void noalloc_tables_kernel(int nx, int ny, int nz, double2 *tw, double *tn) {
  const int n[3] = {nx, ny, nz};
  const int cnt[3] = {nx, ny, nz / 2 + 1};
  for (int a = 0; a < 3; ++a) {
    for (int k = threadIdx.x; k < n[a]; k += blockDim.x) {
      double s, c;
      sincospi(-2.0 * (double)k / (double)n[a], &s, &c);
      tw[a * NOALLOC_MAX_AXIS + k] = make_double2(c, s);
    }
    for (int k = threadIdx.x; k < cnt[a]; k += blockDim.x) {
      const int kk = (k < (n[a] + 1) / 2) ? k : k - n[a];
      double t = 0.0;
      if (2 * kk != n[a] && 2 * kk != -n[a]) {
        double s, c;
        sincospi((double)kk / (double)n[a], &s, &c);
        t = s / c;
      }
      tn[a * NOALLOC_MAX_AXIS + k] = t;
    }
  }
}

// Once per device, with that device current: the device address of the scratch array
// (the host-side symbol is only a stand-in and must never be passed to a kernel) and
// the shared-memory opt-in of the transform kernels.
static int noalloc_setup(int dev, double2 **out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    double2 *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return noalloc_fail(SSFFT_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    const int m = 200 * 1024;
    cudaError_t a[5] = {
        cudaFuncSetAttribute(zfwd_kernel<double, double, PRO_INPUT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, m),
        cudaFuncSetAttribute(ypass_kernel<double, double, false, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, m),
        cudaFuncSetAttribute(xpass_kernel<double, double, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, m),
        cudaFuncSetAttribute(ypass_kernel<double, double, true, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, m),
        cudaFuncSetAttribute(zinv_kernel<double, double, EPI_STORE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, m)};
    for (cudaError_t x : a)
      if (x != cudaSuccess)
        return noalloc_fail(SSFFT_E_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(x));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

extern "C" int ssfft_apply_projection_noalloc(const int32_t n[3], const double stress_mask[6],
                                              const double *in_dev, double *out_dev,
                                              void *stream) {
  if (!n || !stress_mask || !in_dev || !out_dev)
    return noalloc_fail(SSFFT_E_INVALID, "null argument");
  const int nx = n[0], ny = n[1], nz = n[2];
  if (nx < 1 || ny < 1 || nz < 1 || nx > NOALLOC_MAX_AXIS || ny > NOALLOC_MAX_AXIS ||
      nz > NOALLOC_MAX_AXIS)
    return noalloc_fail(SSFFT_E_UNSUPPORTED, "each grid size must be 1..1024");
  const int hz = nz / 2 + 1;
  const long long S = (long long)nx * ny * hz;
  if (S > NOALLOC_MAX_SPEC_POINTS)
    return noalloc_fail(SSFFT_E_UNSUPPORTED,
                        "grid too large for the allocation-free projection: nx*ny*(nz/2+1) "
                        "must be at most 135168 (a 64^3 grid)");
  for (int c = 0; c < 6; ++c)
    if (stress_mask[c] != 0.0 && stress_mask[c] != 1.0)
      return noalloc_fail(SSFFT_E_INVALID, "stress mask can only have zeros and ones");
  Grid<double> g;
  if (!make_axis_plan(nx, g.px) || !make_axis_plan(ny, g.py) || !make_axis_plan(nz, g.pz))
    return noalloc_fail(SSFFT_E_UNSUPPORTED, "grid size has a prime factor above 32");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(SSFFT_E_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return noalloc_fail(SSFFT_E_UNSUPPORTED, "device ordinal");
  double2 *base = nullptr;
  int rc = noalloc_setup(dev, &base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  double2 *spec = base;
  double2 *tw = base + NOALLOC_TABLE_OFFSET;
  double *tn = (double *)(tw + 3 * NOALLOC_MAX_AXIS);
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.hz = hz;
  g.V = (long long)nx * ny * nz;
  g.S = (long long)nx * ny * ((nz % 2 == 0) ? nz / 2 : hz);  // stored columns (no Nyquist)
  g.twx = tw;
  g.twy = tw + NOALLOC_MAX_AXIS;
  g.twz = tw + 2 * NOALLOC_MAX_AXIS;
  g.tanx = tn;
  g.tany = tn + NOALLOC_MAX_AXIS;
  g.tanz = tn + 2 * NOALLOC_MAX_AXIS;
  g.scale = 1.0 / (double)g.V;
  // tiles of the handle-based path's double-precision transforms, except that the x pass
  // always takes 8 kz columns per block (the handle path takes 4 on axes of up to 64)
  g.lz = nz >= 3 * 2048 ? 1 : std::max(1, std::min(32, 2048 / (3 * nz)));
  g.lz = (int)std::min<long long>(g.lz, (long long)nx * ny);
  g.ky = std::min(hz, 16);
  while (g.ky > 1 && smem_y_bytes<double>(g.ky, ny) > 96 * 1024) g.ky /= 2;
  g.kx = std::min(hz, 8);
  while (g.kx > 1 && smem_x_bytes<double>(g.kx, nx) > 100 * 1024) g.kx /= 2;
  grid_divisors(g);
  const size_t sz = smem_z_bytes<double>(g.lz, nz);
  const size_t sy = smem_y_bytes<double>(g.ky, ny);
  const size_t sx = smem_x_bytes<double>(g.kx, nx);
  if (sz > 200 * 1024 || sy > 200 * 1024 || sx > 200 * 1024)
    return noalloc_fail(SSFFT_E_UNSUPPORTED, "grid too large for the shared-memory FFT passes");
  // the one-slot descriptor: the transforms read the spectrum and the stress mask from it
  SlotDev<double> desc;
  memset((void *)&desc, 0, sizeof(desc));
  desc.spec = spec;
  for (int c = 0; c < 6; ++c) desc.mask[c] = stress_mask[c];
  SlotDev<double> *dtab = reinterpret_cast<SlotDev<double> *>(base + NOALLOC_DESC_OFFSET);
  int *dlist = reinterpret_cast<int *>(base + NOALLOC_LIST_OFFSET);
  const int list[2] = {0, 1};
  e = cudaMemcpyAsync(dtab, &desc, sizeof(desc), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dlist, list, sizeof(list), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess)
    return noalloc_fail(SSFFT_E_CUDA, std::string("projection set-up: ") + cudaGetErrorString(e));
  SlotList L;
  L.ids = dlist;
  L.count = dlist + 1;
  ExtIO<double> io;
  io.in = in_dev;
  io.out = out_dev;
  // one block per item of the single slot
  noalloc_tables_kernel<<<1, 256, 0, s>>>(nx, ny, nz, tw, tn);
  zfwd_kernel<double, double, PRO_INPUT><<<items_z(g), SSFFT_THREADS, sz, s>>>(g, dtab, L, io);
  ypass_kernel<double, double, false, false><<<items_y(g), SSFFT_THREADS, sy, s>>>(g, dtab, L);
  xpass_kernel<double, double, false><<<items_x(g), SSFFT_THREADS, sx, s>>>(g, dtab, L);
  ypass_kernel<double, double, true, false><<<items_y(g), SSFFT_THREADS, sy, s>>>(g, dtab, L);
  zinv_kernel<double, double, EPI_STORE><<<items_z(g), SSFFT_THREADS, sz, s>>>(g, dtab, L, io);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    return noalloc_fail(SSFFT_E_CUDA, std::string("projection: ") + cudaGetErrorString(e));
  return 0;
}
