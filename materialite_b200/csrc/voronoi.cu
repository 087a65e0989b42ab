// Voronoi region of every grid point on the device: the nearest of G seeds, over the 27
// periodic images when periodic (Material.create_voronoi, materialite/material.py:337-383,
// with the images of util.repeat_data, util.py:57-88).
//
// The reference builds a cKDTree over the 27 tiled seed sets and queries every point.  The
// squared distance to a tiled seed is a sum over axes, and each axis offers three image
// coordinates (s - L, s, s + L, with L the material's sizes, spacing * (N - 1)), so the
// nearest of the 27 images is the per-axis nearest.  Every coordinate and distance term is
// formed with the same IEEE operations as the host path (point = i * spacing + origin,
// image = seed + shift, d = point - image, sum of d * d in axis order, no contraction into
// fused multiply-adds), so the chosen region matches the tree query except for exact
// distance ties between two seeds, which random seeds do not produce.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/ssfft.h"

int ssfft_internal_fail(int code, const std::string &msg);

#define VORONOI_THREADS 256
#define VORONOI_TILE 1024  // seeds staged in shared memory per pass (24 KB)

__device__ __forceinline__ double axis_sq(double p, double s, double L, bool periodic) {
  const double d0 = __dsub_rn(p, s);
  double best = __dmul_rn(d0, d0);
  if (periodic) {
    const double dm = __dsub_rn(p, __dadd_rn(s, -L));
    const double dp = __dsub_rn(p, __dadd_rn(s, L));
    best = fmin(best, __dmul_rn(dm, dm));
    best = fmin(best, __dmul_rn(dp, dp));
  }
  return best;
}

__global__ void __launch_bounds__(VORONOI_THREADS)
    voronoi_kernel(int nx, int ny, int nz, double3 origin, double3 spacing, double3 L,
                   const double *__restrict__ seeds, int G, int periodic,
                   int32_t *__restrict__ region) {
  __shared__ double sx[VORONOI_TILE], sy[VORONOI_TILE], sz[VORONOI_TILE];
  const long long V = (long long)nx * ny * nz;
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = v < V;
  double px = 0.0, py = 0.0, pz = 0.0;
  if (live) {
    const long long plane = (long long)ny * nz;
    const int i = (int)(v / plane);
    const long long r = v - (long long)i * plane;
    const int j = (int)(r / nz);
    const int k = (int)(r - (long long)j * nz);
    px = __dadd_rn(__dmul_rn((double)i, spacing.x), origin.x);
    py = __dadd_rn(__dmul_rn((double)j, spacing.y), origin.y);
    pz = __dadd_rn(__dmul_rn((double)k, spacing.z), origin.z);
  }
  const bool per = periodic != 0;
  double best = INFINITY;
  int arg = 0;
  for (int t0 = 0; t0 < G; t0 += VORONOI_TILE) {
    const int nt = min(VORONOI_TILE, G - t0);
    __syncthreads();
    for (int q = threadIdx.x; q < nt; q += blockDim.x) {
      sx[q] = seeds[3 * (t0 + q)];
      sy[q] = seeds[3 * (t0 + q) + 1];
      sz[q] = seeds[3 * (t0 + q) + 2];
    }
    __syncthreads();
    if (live) {
      for (int q = 0; q < nt; ++q) {
        const double d2 = __dadd_rn(__dadd_rn(axis_sq(px, sx[q], L.x, per),
                                               axis_sq(py, sy[q], L.y, per)),
                                     axis_sq(pz, sz[q], L.z, per));
        if (d2 < best) {  // strict: the lowest seed index among exact ties
          best = d2;
          arg = t0 + q;
        }
      }
    }
  }
  if (live) region[v] = arg;
}

#define VCK(call)                                                                       \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      rc = ssfft_internal_fail(SSFFT_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
      goto done;                                                                        \
    }                                                                                   \
  } while (0)

extern "C" int ssfft_voronoi(const int32_t dims[3], const double origin[3],
                             const double spacing[3], const double period[3],
                             const double *seeds, int num_regions, int periodic, int device,
                             int32_t *region_of_point) {
  if (!dims || !origin || !spacing || !period || !seeds || !region_of_point)
    return ssfft_internal_fail(SSFFT_E_INVALID, "null argument");
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || num_regions < 1)
    return ssfft_internal_fail(SSFFT_E_INVALID, "dimensions and number of regions must be positive");
  const long long V = (long long)dims[0] * dims[1] * dims[2];
  if (V > (1LL << 31) - 1)
    return ssfft_internal_fail(SSFFT_E_UNSUPPORTED, "grid has more than 2^31 - 1 points");
  int rc = 0;
  double *d_seeds = nullptr;
  int32_t *d_region = nullptr;
  cudaStream_t s = nullptr;
  const double3 L = make_double3(period[0], period[1], period[2]);
  const int blocks = (int)((V + VORONOI_THREADS - 1) / VORONOI_THREADS);
  VCK(cudaSetDevice(device));
  VCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  VCK(cudaMalloc((void **)&d_seeds, (size_t)num_regions * 3 * sizeof(double)));
  VCK(cudaMalloc((void **)&d_region, (size_t)V * sizeof(int32_t)));
  VCK(cudaMemcpyAsync(d_seeds, seeds, (size_t)num_regions * 3 * sizeof(double),
                      cudaMemcpyHostToDevice, s));
  voronoi_kernel<<<blocks, VORONOI_THREADS, 0, s>>>(
      dims[0], dims[1], dims[2], make_double3(origin[0], origin[1], origin[2]),
      make_double3(spacing[0], spacing[1], spacing[2]), L, d_seeds, num_regions, periodic,
      d_region);
  VCK(cudaGetLastError());
  VCK(cudaMemcpyAsync(region_of_point, d_region, (size_t)V * sizeof(int32_t),
                      cudaMemcpyDeviceToHost, s));
  VCK(cudaStreamSynchronize(s));
done:
  if (d_seeds) cudaFree(d_seeds);
  if (d_region) cudaFree(d_region);
  if (s) cudaStreamDestroy(s);
  return rc;
}
