// surface.cu -- particle-to-level-set surface reconstruction on a dense
// grid, the operations of the reference's post-processing tool
// (PostProcessing/OpenVDB/src/ConstructSurface.cc:39-72): voxel size = r/2,
// spheres of radius r rasterised as phi = min_p (|x - p| - r), then "dilate"
// by r, smooth, "erode" by r (the tool's offset(-r), gaussian(),
// offset(+r)).  The reference does this with OpenVDB's sparse narrow-band
// grids on the CPU; here the grid is dense on the device:
//   * rasterisation: one thread per particle over the voxels within r + band
//     of its centre, phi kept as fixed-point integers (2^-20 length units)
//     so that the minimum is one atomicMin; a voxel is only written when it
//     would decrease;
//   * values are clamped to +-band (band = (halfWidth voxels + r), wide
//     enough that the offsets by r stay inside it);
//   * dilate: phi - r; smooth: three passes of a 3-tap mean along x, y, z
//     (a box-filter approximation of a Gaussian); erode: phi + r.
#include <cmath>
#include <cuda_runtime.h>

#include "host_internal.h"

namespace sphpc {
namespace {

constexpr float kFixScale = 1048576.0f;  // 2^20 units per length

__global__ void k_fill_int(int* __restrict__ a, long long n, int v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}

__global__ void k_rasterise(const double* __restrict__ xyz, int np, int nx, int ny, int nz,
                            double ox, double oy, double oz, float voxel, float radius,
                            float band, int* __restrict__ phi) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float px = (float)(xyz[3 * (size_t)p] - ox), py = (float)(xyz[3 * (size_t)p + 1] - oy),
              pz = (float)(xyz[3 * (size_t)p + 2] - oz);
  const float reach = radius + band;
  const int i0 = max(0, (int)ceilf((px - reach) / voxel)), i1 = min(nx - 1, (int)floorf((px + reach) / voxel));
  const int j0 = max(0, (int)ceilf((py - reach) / voxel)), j1 = min(ny - 1, (int)floorf((py + reach) / voxel));
  const int k0 = max(0, (int)ceilf((pz - reach) / voxel)), k1 = min(nz - 1, (int)floorf((pz + reach) / voxel));
  for (int k = k0; k <= k1; ++k) {
    const float dz = k * voxel - pz;
    for (int j = j0; j <= j1; ++j) {
      const float dy = j * voxel - py;
      int* row = phi + ((size_t)k * ny + j) * nx;
      for (int i = i0; i <= i1; ++i) {
        const float dx = i * voxel - px;
        const float d = sqrtf(dx * dx + dy * dy + dz * dz) - radius;
        if (d > band) continue;
        const int q = __float2int_rn(fmaxf(d, -band) * kFixScale);
        if (q < row[i]) atomicMin(row + i, q);
      }
    }
  }
}

// dilate (shift < 0) / erode (shift > 0) with the fixed-point -> float step
__global__ void k_to_float(const int* __restrict__ in, float* __restrict__ out, long long n,
                           float shift) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i] * (1.0f / kFixScale) + shift;
}

__global__ void k_shift(float* __restrict__ a, long long n, float shift) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] += shift;
}

// 3-tap mean along one axis (stride s, extent m along it), edges replicated.
__global__ void k_mean3(const float* __restrict__ in, float* __restrict__ out, long long n,
                        long long s, int m) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)((i / s) % m);
    const float a = in[c > 0 ? i - s : i], b = in[i], d = in[c < m - 1 ? i + s : i];
    out[i] = (a + b + d) * (1.0f / 3.0f);
  }
}

}  // namespace
}  // namespace sphpc

using namespace sphpc;

// Level set of particles xyz[3 * np] (interleaved doubles, host memory, as
// WriteParticles writes them) on the dense grid dims at origin with voxel
// size radius / 2: phi[i + dims[0] * (j + dims[1] * k)] (host), negative
// inside.  half_width is the narrow band in voxels (the tool uses 2).
extern "C" int sphpc_particle_surface(const double* xyz, int np, double radius, int half_width,
                                      const int* dims, const double* origin, float* phi) {
  if (!xyz || np <= 0 || !(radius > 0.0) || half_width < 1 || !dims || !origin || !phi)
    return set_error(SPHPC_EINVAL, "sphpc_particle_surface: bad arguments");
  for (int d = 0; d < 3; ++d)
    if (dims[d] <= 0) return set_error(SPHPC_EINVAL, "sphpc_particle_surface: empty grid");
  const long long n = (long long)dims[0] * dims[1] * dims[2];
  const float voxel = (float)(radius / 2.0);
  const float r = (float)radius;
  const float band = half_width * voxel + r;
  if ((double)band * kFixScale > 2.0e9)
    return set_error(SPHPC_EINVAL, "sphpc_particle_surface: radius too large for the grid units");
  double* d_xyz = nullptr;
  int* d_fix = nullptr;
  float *d_a = nullptr, *d_b = nullptr;
  cudaError_t e = cudaMalloc(&d_xyz, sizeof(double) * 3 * (size_t)np);
  if (e == cudaSuccess) e = cudaMalloc(&d_fix, sizeof(int) * (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(&d_a, sizeof(float) * (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(&d_b, sizeof(float) * (size_t)n);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_xyz, xyz, sizeof(double) * 3 * (size_t)np, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int g = 148 * 8;
    k_fill_int<<<g, 256>>>(d_fix, n, (int)lrintf(band * kFixScale));
    k_rasterise<<<(np + 127) / 128, 128>>>(d_xyz, np, dims[0], dims[1], dims[2], origin[0],
                                           origin[1], origin[2], voxel, r, band, d_fix);
    // dilate by r, smooth, erode by r (ConstructSurface.cc:54-63)
    k_to_float<<<g, 256>>>(d_fix, d_a, n, -r);
    const long long strides[3] = {1, dims[0], (long long)dims[0] * dims[1]};
    for (int it = 0; it < 3; ++it)
      for (int ax = 0; ax < 3; ++ax) {
        k_mean3<<<g, 256>>>(d_a, d_b, n, strides[ax], dims[ax]);
        float* t = d_a;
        d_a = d_b;
        d_b = t;
      }
    k_shift<<<g, 256>>>(d_a, n, r);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(phi, d_a, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
  cudaFree(d_xyz);
  cudaFree(d_fix);
  cudaFree(d_a);
  cudaFree(d_b);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(SPHPC_ECUDA, "sphpc_particle_surface: %s", cudaGetErrorString(e));
  }
  return SPHPC_OK;
}
