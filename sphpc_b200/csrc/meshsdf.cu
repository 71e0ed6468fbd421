// meshsdf.cu -- signed distance field of a closed triangle mesh on the
// device, in the sample layout of the SDFGen files the reference's obstacle
// loader reads (obstacle.c:13-79): samples at origin + (i, j, k) * dx, i
// fastest, negative inside.  The reference runtime names such a file
// (Runtime/sim-config.ini: bunny_watertight.sdf) but ships only the mesh.
//
// |phi| is the exact distance to the nearest triangle (closest point on a
// triangle by Voronoi regions: Ericson, "Real-Time Collision Detection",
// 2005, section 5.1.5); the sign comes from the generalized winding number
// (Jacobson, Kavan, Sorkine-Hornung, SIGGRAPH 2013): the sum of the
// triangles' solid angles (Van Oosterom and Strackee, IEEE TBME 1983) is
// 4 pi inside a closed mesh and 0 outside, and a sample is inside when it
// exceeds 2 pi.  Brute force over all triangles: one thread per sample,
// triangles staged through shared memory in tiles.
#include <cmath>
#include <cuda_runtime.h>

#include "host_internal.h"

namespace sphpc {
namespace {

constexpr int kSdfBlock = 256;
constexpr int kTriTile = 256;

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// Squared distance from p to triangle abc (Ericson 5.1.5).
__device__ float tri_dist2(float3 p, float3 a, float3 b, float3 c) {
  const float3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  float3 q;
  if (d1 <= 0.f && d2 <= 0.f) {
    q = a;
  } else {
    const float3 bp = sub3(p, b);
    const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.f && d4 <= d3) {
      q = b;
    } else {
      const float vc = d1 * d4 - d3 * d2;
      if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = d1 / (d1 - d3);
        q = make_float3(a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z);
      } else {
        const float3 cp = sub3(p, c);
        const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
        if (d6 >= 0.f && d5 <= d6) {
          q = c;
        } else {
          const float vb = d5 * d2 - d1 * d6;
          if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
            const float w = d2 / (d2 - d6);
            q = make_float3(a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z);
          } else {
            const float va = d3 * d6 - d5 * d4;
            if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
              const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
              q = make_float3(b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z));
            } else {
              const float denom = 1.f / (va + vb + vc);
              const float v = vb * denom, w = vc * denom;
              q = make_float3(a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w,
                              a.z + ab.z * v + ac.z * w);
            }
          }
        }
      }
    }
  }
  const float3 d = sub3(p, q);
  return dot3(d, d);
}

// Signed solid angle of triangle abc seen from the origin (a, b, c relative
// to the sample), Van Oosterom and Strackee.
__device__ __forceinline__ float solid_angle(float3 a, float3 b, float3 c) {
  const float la = sqrtf(dot3(a, a)), lb = sqrtf(dot3(b, b)), lc = sqrtf(dot3(c, c));
  const float num = dot3(a, cross3(b, c));
  const float den = la * lb * lc + dot3(a, b) * lc + dot3(a, c) * lb + dot3(b, c) * la;
  return 2.0f * atan2f(num, den);
}

__global__ void __launch_bounds__(kSdfBlock)
    k_mesh_sdf(const float3* __restrict__ tv, int nt, int ni, int nj, int nk, double ox,
               double oy, double oz, double dx, float* __restrict__ phi) {
  __shared__ float3 s[3 * kTriTile];
  const long long total = (long long)ni * nj * nk;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = idx < total;
  const int i = live ? (int)(idx % ni) : 0;
  const int j = live ? (int)((idx / ni) % nj) : 0;
  const int k = live ? (int)(idx / ((long long)ni * nj)) : 0;
  const float3 p = make_float3((float)(ox + i * dx), (float)(oy + j * dx), (float)(oz + k * dx));
  float best = 3.0e38f, wind = 0.0f;
  for (int t0 = 0; t0 < nt; t0 += kTriTile) {
    const int cnt = min(kTriTile, nt - t0);
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * cnt; e += blockDim.x) s[e] = tv[3 * (size_t)t0 + e];
    __syncthreads();
    if (live) {
      for (int t = 0; t < cnt; ++t) {
        const float3 a = s[3 * t], b = s[3 * t + 1], c = s[3 * t + 2];
        best = fminf(best, tri_dist2(p, a, b, c));
        wind += solid_angle(sub3(a, p), sub3(b, p), sub3(c, p));
      }
    }
  }
  if (live) phi[idx] = (fabsf(wind) > 6.283185307f ? -1.0f : 1.0f) * sqrtf(best);
}

}  // namespace
}  // namespace sphpc

using namespace sphpc;

// Signed distance of the closed mesh (vertices[3 * nv], triangles[3 * nt]
// vertex indices, host memory) at the samples origin + (i, j, k) * dx of a
// dims[0] x dims[1] x dims[2] grid, into phi (host, i fastest).
extern "C" int sphpc_mesh_sdf(const float* vertices, int n_vertices, const int* triangles,
                              int n_triangles, const int* dims, const double* origin, double dx,
                              float* phi) {
  if (!vertices || !triangles || !dims || !origin || !phi || n_vertices <= 0 ||
      n_triangles <= 0 || !(dx > 0.0))
    return set_error(SPHPC_EINVAL, "sphpc_mesh_sdf: bad arguments");
  for (int d = 0; d < 3; ++d)
    if (dims[d] <= 0) return set_error(SPHPC_EINVAL, "sphpc_mesh_sdf: empty grid");
  const long long total = (long long)dims[0] * dims[1] * dims[2];
  // triangle corners, gathered on the host (validates the indices)
  float* corners = (float*)malloc(sizeof(float) * 9 * (size_t)n_triangles);
  if (!corners) return set_error(SPHPC_ENOMEM, "sphpc_mesh_sdf: host buffer");
  for (int t = 0; t < n_triangles; ++t)
    for (int v = 0; v < 3; ++v) {
      const int id = triangles[3 * t + v];
      if (id < 0 || id >= n_vertices) {
        free(corners);
        return set_error(SPHPC_EINVAL, "sphpc_mesh_sdf: triangle %d has vertex index %d", t, id);
      }
      for (int c = 0; c < 3; ++c) corners[9 * t + 3 * v + c] = vertices[3 * id + c];
    }
  float3* d_tri = nullptr;
  float* d_phi = nullptr;
  cudaError_t e = cudaMalloc(&d_tri, sizeof(float) * 9 * (size_t)n_triangles);
  if (e == cudaSuccess) e = cudaMalloc(&d_phi, sizeof(float) * (size_t)total);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_tri, corners, sizeof(float) * 9 * (size_t)n_triangles, cudaMemcpyHostToDevice);
  free(corners);
  if (e == cudaSuccess) {
    const long long blocks = (total + kSdfBlock - 1) / kSdfBlock;
    k_mesh_sdf<<<(unsigned)blocks, kSdfBlock>>>(d_tri, n_triangles, dims[0], dims[1], dims[2],
                                                origin[0], origin[1], origin[2], dx, d_phi);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(phi, d_phi, sizeof(float) * (size_t)total, cudaMemcpyDeviceToHost);
  if (d_tri) cudaFree(d_tri);
  if (d_phi) cudaFree(d_phi);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(SPHPC_ECUDA, "sphpc_mesh_sdf: %s", cudaGetErrorString(e));
  }
  return SPHPC_OK;
}
