/*
 * pbf_oracle.c -- CPU restatement of SPHPC's per-step PBF pipeline.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * pbf_oracle.h for the contract and how this file is pinned to the
 * reference.  Each function names the reference lines it restates; the
 * arithmetic follows the reference expression by expression (operand order
 * included) so that, compiled with -ffp-contract=off, the FP64 build equals
 * the verbatim reference bit for bit on the reference-compat parameters.
 */
#include "pbf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_REAL_FLOAT
typedef float real;
#else
typedef double real;
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

int oracle_real_size(void) { return (int)sizeof(real); }

/* ------------------------------------------------------------------------ */
/* Smoothing kernels, particles.c:18-65                                      */
/* ------------------------------------------------------------------------ */

/* poly6, particles.c:20-26 */
static inline real W(const real r, const real h, const real norm) {
  if (r > h) return (real)0.0;
  return norm * (h * h - r * r) * (h * h - r * r) * (h * h - r * r);
}

/* poly6 gradient magnitude, particles.c:29-35 */
static inline real DelWPoly(const real r, const real h, const real norm) {
  if (r > h) return (real)0.0;
  return norm * (h * h - r * r) * (h * h - r * r) * r;
}

/* spiky gradient magnitude, particles.c:40-46 */
static inline real DelW(const real r, const real h, const real norm) {
  if (r > h) return (real)0.0;
  return norm * (h - r) * (h - r);
}

/* Akinci cohesion spline, particles.c:54-65 */
static inline real Ccoh(const real r, const real h, const real norm) {
  real C;
  if (r > h)
    C = (real)0.0;
  else if (r <= h / (real)2.0)
    C = ((real)2.0 * (h - r) * (h - r) * (h - r) * r * r * r) -
        (h * h * h * h * h * h / (real)64.0);
  else
    C = (h - r) * (h - r) * (h - r) * r * r * r;
  return norm * C;
}

/* ------------------------------------------------------------------------ */
/* Parameters                                                               */
/* ------------------------------------------------------------------------ */

/* simulation.c:153-177 */
void oracle_set_kernel_norms(OracleParams *p, double h) {
  p->h = h;
  p->dq = 0.1 * h;
  p->W_norm = 315.0 / (64.0 * M_PI * pow(h, 9.0));
  p->DelW_poly_norm = -3.0 * 2.0 * p->W_norm;
  p->DelW_norm = -45.0 / (M_PI * pow(h, 6.0));
}

void oracle_params_reference_compat(OracleParams *p) {
  p->solve_iterations = 10;          /* simulation.c:72 */
  p->lambda_epsilon = 0.01;          /* particles.c:663 */
  p->scorr_k = 0.0;                  /* particles.c:730 */
  p->scorr_n = 4;
  p->scorr_dq = p->dq;               /* simulation.c:155 */
  p->k_stiff = 0.95;                 /* particles.c:693 */
  p->vorticity_eps = 0.1 * p->h;     /* particles.c:289 */
  p->v_max = 100.0;                  /* particles.c:791 */
  p->gravity_axis = 2;               /* particles.c:519-525 */
  p->xsph_mode = 0;                  /* particles.c:404-458, in place */
  p->enable_tension = 1;
  p->enable_vorticity = 1;
}

/* neighbors.c:23-28 */
void oracle_set_grid(OracleParams *p) {
  p->nx = (int)(ceil((p->bmax[0] - p->bmin[0]) / p->h) + 1);
  p->ny = (int)(ceil((p->bmax[1] - p->bmin[1]) / p->h) + 1);
  p->nz = (int)(ceil((p->bmax[2] - p->bmin[2]) / p->h) + 1);
}

/* ------------------------------------------------------------------------ */
/* Scene                                                                    */
/* ------------------------------------------------------------------------ */

static inline uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

double oracle_uniform01(uint64_t seed, uint64_t index, uint32_t axis) {
  uint64_t k = splitmix64(seed ^ splitmix64(index * 4u + axis));
  return (double)(k >> 11) * (1.0 / 9007199254740992.0);
}

/* geometry.c:42-55 (cell-centred lattice), plus seeded jitter */
void oracle_lattice(int nxl, int nyl, int nzl, double spacing,
                    const double origin[3], double jitter, uint64_t seed,
                    double *x, double *y, double *z) {
  int64_t i = 0;
  for (int kz = 0; kz < nzl; ++kz)
    for (int ky = 0; ky < nyl; ++ky)
      for (int kx = 0; kx < nxl; ++kx) {
        double jx = jitter * spacing * (2.0 * oracle_uniform01(seed, i, 0) - 1.0);
        double jy = jitter * spacing * (2.0 * oracle_uniform01(seed, i, 1) - 1.0);
        double jz = jitter * spacing * (2.0 * oracle_uniform01(seed, i, 2) - 1.0);
        x[i] = origin[0] + kx * spacing + spacing / 2.0 + jx;
        y[i] = origin[1] + ky * spacing + spacing / 2.0 + jy;
        z[i] = origin[2] + kz * spacing + spacing / 2.0 + jz;
        ++i;
      }
}

double oracle_lattice_poly6_sum(const OracleParams *p, double spacing) {
  const double h = p->h;
  const int R = (int)ceil(h / spacing) + 1;
  double s = 0.0;
  for (int k = -R; k <= R; ++k)
    for (int j = -R; j <= R; ++j)
      for (int i = -R; i <= R; ++i) {
        double r2 = (i * i + j * j + k * k) * spacing * spacing;
        if (r2 < h * h || (i == 0 && j == 0 && k == 0))
          s += W(sqrt(r2), h, p->W_norm);
      }
  return s;
}

/* ------------------------------------------------------------------------ */
/* Neighbour search, neighbors.c                                            */
/* ------------------------------------------------------------------------ */

/* HashVal, neighbors.c:79-98 */
uint32_t oracle_hash_val(const OracleParams *p, double x, double y, double z) {
  const double spacing = p->h;
  const unsigned int grid_x = (unsigned int)floor(x / spacing);
  const unsigned int grid_y = (unsigned int)floor(y / spacing);
  const unsigned int grid_z = (unsigned int)floor(z / spacing);
  const unsigned int num_x = (unsigned int)p->nx;
  const unsigned int num_y = (unsigned int)p->ny;
  return (num_x * num_y * grid_z) + (grid_y * num_x + grid_x);
}

/* HashParticles, neighbors.c:101-125 */
void oracle_hash_particles(const OracleParams *p, const OracleState *s,
                           OracleNeighbors *nb) {
  for (int i = 0; i < s->n; ++i) {
    nb->keys[i] = oracle_hash_val(p, s->xs[i], s->ys[i], s->zs[i]);
    nb->ids[i] = (uint32_t)i;
  }
}

/* SortByKey, thrust_c.cu:86-91: thrust::sort_by_key on u32 keys is CUB's
 * radix sort, which is stable; restated as a stable LSD counting sort. */
void oracle_sort_by_key(uint32_t *keys, uint32_t *vals, int n) {
  if (n <= 1) return;
  uint32_t *k2 = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
  uint32_t *v2 = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
  uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (int i = 0; i < n; ++i) cnt[((ka[i] >> shift) & 0xFFu) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (int i = 0; i < n; ++i) {
      size_t pos = cnt[(ka[i] >> shift) & 0xFFu]++;
      kb[pos] = ka[i];
      vb[pos] = va[i];
    }
    uint32_t *t = ka; ka = kb; kb = t;
    t = va; va = vb; vb = t;
  }
  /* 4 passes: result is back in keys/vals */
  free(k2);
  free(v2);
}

/* FindLowerBounds, thrust_c.cu:93-105 */
void oracle_lower_bounds(const uint32_t *keys, int n, int search_count,
                         uint32_t *out) {
  int lo = 0;
  for (int c = 0; c < search_count; ++c) {
    while (lo < n && keys[lo] < (uint32_t)c) ++lo;
    out[c] = (uint32_t)lo;
  }
}

/* FindUpperBounds, thrust_c.cu:107-120 */
void oracle_upper_bounds(const uint32_t *keys, int n, int search_count,
                         uint32_t *out) {
  int lo = 0;
  for (int c = 0; c < search_count; ++c) {
    while (lo < n && keys[lo] <= (uint32_t)c) ++lo;
    out[c] = (uint32_t)lo;
  }
}

/* FillNeighbors, neighbors.c:217-298 */
void oracle_fill_neighbors(const OracleParams *p, const OracleState *s,
                           OracleNeighbors *nb) {
  const double smoothing_radius2 = p->h * p->h;
  const double spacing = p->h;
  for (int i = 0; i < s->n; ++i) {
    const int p_index = i;
    int count = 0;
    uint32_t *bucket = nb->nbr + (size_t)p_index * ORACLE_MAX_NEIGHBORS;
    const double x_star_p = s->xs[p_index];
    const double y_star_p = s->ys[p_index];
    const double z_star_p = s->zs[p_index];
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const double x = x_star_p + dx * spacing;
          const double y = y_star_p + dy * spacing;
          const double z = z_star_p + dz * spacing;
          if (floor(x / spacing) > p->nx - 1 || x < 0.0 ||
              floor(y / spacing) > p->ny - 1 || y < 0.0 ||
              floor(z / spacing) > p->nz - 1 || z < 0.0)
            continue;
          const int neighbor_index = (int)oracle_hash_val(p, x, y, z);
          const unsigned int start_index = nb->start[neighbor_index];
          const unsigned int end_index = nb->end[neighbor_index];
          if (start_index != end_index) {
            for (unsigned int j = start_index; j < end_index; ++j) {
              const int q_index = (int)nb->ids[j];
              if (p_index == q_index) continue;
              const double x_diff = x_star_p - s->xs[q_index];
              const double y_diff = y_star_p - s->ys[q_index];
              const double z_diff = z_star_p - s->zs[q_index];
              const double r2 = x_diff * x_diff + y_diff * y_diff + z_diff * z_diff;
              if (r2 < smoothing_radius2 && count < ORACLE_MAX_NEIGHBORS) {
                bucket[count] = (uint32_t)q_index;
                ++count;
              }
            }
          }
        }
    nb->count[p_index] = count;
  }
}

/* FindAllNeighbors, neighbors.c:68-75 (SortHash :128-155, FindCellBounds
 * :182-215) */
void oracle_find_all_neighbors(const OracleParams *p, const OracleState *s,
                               OracleNeighbors *nb) {
  const int C = p->nx * p->ny * p->nz;
  oracle_hash_particles(p, s, nb);
  oracle_sort_by_key(nb->keys, nb->ids, s->n);
  oracle_lower_bounds(nb->keys, s->n, C, nb->start);
  oracle_upper_bounds(nb->keys, s->n, C, nb->end);
  oracle_fill_neighbors(p, s, nb);
}

/* ------------------------------------------------------------------------ */
/* SDF obstacle, obstacle_cuda.cu                                           */
/* ------------------------------------------------------------------------ */

static inline float sdf_at(const OracleParams *p, int i, int j, int k) {
  if (i < 0) i = 0;
  if (i > p->sdim[0] - 1) i = p->sdim[0] - 1;
  if (j < 0) j = 0;
  if (j > p->sdim[1] - 1) j = p->sdim[1] - 1;
  if (k < 0) k = 0;
  if (k > p->sdim[2] - 1) k = p->sdim[2] - 1;
  return p->sdf[((size_t)k * p->sdim[1] + j) * p->sdim[0] + i];
}

static inline float lerpf_(float a, float b, float t) { return fmaf(t, b - a, a); }

/* tex3D<float> with cudaFilterModeLinear, cudaAddressModeClamp and
 * normalizedCoords = 1 (obstacle_cuda.cu:166-181): texel-centre convention
 * xB = u*N - 0.5, clamp addressing of the two taps.  The weights are exact
 * FP32 (the hardware uses 9-bit fixed-point weights). */
float oracle_sdf_sample(const OracleParams *p, float u, float v, float w) {
  float xb = u * (float)p->sdim[0] - 0.5f;
  float yb = v * (float)p->sdim[1] - 0.5f;
  float zb = w * (float)p->sdim[2] - 0.5f;
  float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
  float ax = xb - fx, ay = yb - fy, az = zb - fz;
  int i = (int)fx, j = (int)fy, k = (int)fz;
  float c00 = lerpf_(sdf_at(p, i, j, k), sdf_at(p, i + 1, j, k), ax);
  float c10 = lerpf_(sdf_at(p, i, j + 1, k), sdf_at(p, i + 1, j + 1, k), ax);
  float c01 = lerpf_(sdf_at(p, i, j, k + 1), sdf_at(p, i + 1, j, k + 1), ax);
  float c11 = lerpf_(sdf_at(p, i, j + 1, k + 1), sdf_at(p, i + 1, j + 1, k + 1), ax);
  float c0 = lerpf_(c00, c10, ay);
  float c1 = lerpf_(c01, c11, ay);
  return lerpf_(c0, c1, az);
}

/* CalculateParticleCollisions_kernel, obstacle_cuda.cu:56-116, with
 * InsideObstacleBounds :20-31 and CalculateNormal :33-53.  normalize() uses
 * a correctly rounded 1/sqrt (the reference uses rsqrtf). */
void oracle_particle_collisions(const OracleParams *p, double *x, double *y,
                                double *z, int n) {
  if (!p->sdf) return;
  for (int i = 0; i < n; ++i) {
    const double x_world = x[i];
    const double y_world = y[i];
    const double z_world = z[i];
    if (!(x_world > p->ob_min[0] && x_world < p->ob_max[0] &&
          y_world > p->ob_min[1] && y_world < p->ob_max[1] &&
          z_world > p->ob_min[2] && z_world < p->ob_max[2]))
      continue;
    const float obstacle_length_world = (float)(p->ob_max[0] - p->ob_min[0]);
    const float x_tex = (float)((x_world - p->ob_min[0]) / obstacle_length_world);
    const float obstacle_height_world = (float)(p->ob_max[1] - p->ob_min[1]);
    const float y_tex = (float)((y_world - p->ob_min[1]) / obstacle_height_world);
    const float obstacle_depth_world = (float)(p->ob_max[2] - p->ob_min[2]);
    const float z_tex = (float)((z_world - p->ob_min[2]) / obstacle_depth_world);
    const float d = oracle_sdf_sample(p, x_tex, y_tex, z_tex);
    if (d < 0) {
      const float x_spacing = (float)(1.0 / (float)p->sdim[0]);
      const float y_spacing = (float)(1.0 / (float)p->sdim[1]);
      const float z_spacing = (float)(1.0 / (float)p->sdim[2]);
      const float gx = oracle_sdf_sample(p, x_tex + x_spacing, y_tex, z_tex) -
                       oracle_sdf_sample(p, x_tex - x_spacing, y_tex, z_tex);
      const float gy = oracle_sdf_sample(p, x_tex, y_tex + y_spacing, z_tex) -
                       oracle_sdf_sample(p, x_tex, y_tex - y_spacing, z_tex);
      const float gz = oracle_sdf_sample(p, x_tex, y_tex, z_tex + z_spacing) -
                       oracle_sdf_sample(p, x_tex, y_tex, z_tex - z_spacing);
      const float dot = gx * gx + gy * gy + gz * gz;
      const float inv_length = 1.0f / sqrtf(dot);
      const float nx = gx * inv_length, ny = gy * inv_length, nz = gz * inv_length;
      const float obstacle_length_model = (float)(p->sdim[0] * p->sdf_spacing);
      const float model_to_world = obstacle_length_world / obstacle_length_model;
      const float dist_world = fabsf(d) * model_to_world;
      y[i] += dist_world * ny;
      x[i] += dist_world * nx;
      z[i] += dist_world * nz;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Step functions, particles.c                                              */
/* ------------------------------------------------------------------------ */

/* ApplyBoundaryConditions, particles.c:842-867 */
static inline void boundary(const OracleParams *p, double *x, double *y, double *z) {
  const real h = (real)p->h;
  const real epsion = h * (real)0.0001;
  if (*x < p->bmin[0]) *x = p->bmin[0];
  else if (*x >= p->bmax[0]) *x = (real)p->bmax[0] - epsion;
  if (*y < p->bmin[1]) *y = p->bmin[1];
  else if (*y >= p->bmax[1]) *y = (real)p->bmax[1] - epsion;
  if (*z < p->bmin[2]) *z = p->bmin[2];
  else if (*z >= p->bmax[2]) *z = (real)p->bmax[2] - epsion;
}

/* ApplyGravity, particles.c:516-527 (axis parameterised) */
void oracle_apply_gravity(const OracleParams *p, OracleState *s) {
  const real dt = (real)p->dt;
  const real g = (real)-p->g;
  double *v = p->gravity_axis == 0 ? s->vx : (p->gravity_axis == 1 ? s->vy : s->vz);
  for (int i = 0; i < s->n; ++i) v[i] = (real)v[i] + g * dt;
}

/* PredictPositions, particles.c:748-784 */
void oracle_predict_positions(const OracleParams *p, OracleState *s) {
  const real dt = (real)p->dt;
  for (int i = 0; i < s->n; ++i) {
    s->xs[i] = (real)s->x[i] + ((real)s->vx[i] * dt);
    s->ys[i] = (real)s->y[i] + ((real)s->vy[i] * dt);
    s->zs[i] = (real)s->z[i] + ((real)s->vz[i] * dt);
    boundary(p, &s->xs[i], &s->ys[i], &s->zs[i]);
  }
}

/* ComputeDensities, particles.c:461-514 */
void oracle_compute_densities(const OracleParams *p, OracleState *s,
                              const OracleNeighbors *nb) {
  const real h = (real)p->h;
  const real rest_mass = (real)p->rest_mass;
  const real W_norm = (real)p->W_norm;
  const real W_0 = W((real)0.0, h, W_norm);
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    const real mass_p = rest_mass;
    real tmp_density = mass_p * W_0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      const real mass_q = rest_mass;
      const real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      tmp_density += mass_q * W(r_mag, h, W_norm);
    }
    s->rho[i] = tmp_density;
  }
}

/* ComputeLambda, particles.c:588-666 (epsilon parameterised) */
void oracle_compute_lambda(const OracleParams *p, OracleState *s,
                           const OracleNeighbors *nb) {
  const real rest_density = (real)p->rest_density;
  const real rest_mass = (real)p->rest_mass;
  const real h = (real)p->h;
  const real DelW_norm = (real)p->DelW_norm;
  const real epsilon = (real)p->lambda_epsilon;
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real Constraint = (real)s->rho[i] / rest_density - (real)1.0;
    const real Ci = (Constraint < (real)0.0 ? (real)0.0 : Constraint);
    real sum_C = 0.0, sum_grad_x = 0.0, sum_grad_y = 0.0, sum_grad_z = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      if (r_mag < h * (real)0.0001) r_mag = h * (real)0.0001;
      const real mass_q = rest_mass;
      const real grad = DelW(r_mag, h, DelW_norm);
      const real grad_x = mass_q * grad * x_diff / r_mag;
      const real grad_y = mass_q * grad * y_diff / r_mag;
      const real grad_z = mass_q * grad * z_diff / r_mag;
      sum_grad_x += grad_x;
      sum_grad_y += grad_y;
      sum_grad_z += grad_z;
      sum_C += (grad_x * grad_x + grad_y * grad_y + grad_z * grad_z);
    }
    sum_C += (sum_grad_x * sum_grad_x + sum_grad_y * sum_grad_y +
              sum_grad_z * sum_grad_z);
    sum_C /= (rest_density * rest_density);
    s->lam[i] = -Ci / (sum_C + epsilon);
  }
}

/* UpdateDPs, particles.c:668-746 (s_corr restored from the commented-out
 * line :729-730 with k, n and delta-q as parameters) */
void oracle_update_dps(const OracleParams *p, OracleState *s,
                       const OracleNeighbors *nb, int substep) {
  const real h = (real)p->h;
  const real rest_density = (real)p->rest_density;
  const real rest_mass = (real)p->rest_mass;
  const real W_norm = (real)p->W_norm;
  const real DelW_norm = (real)p->DelW_norm;
  const real Wdq = W((real)p->scorr_dq, h, W_norm);
  const real k = (real)p->scorr_k;
  const real k_stiff = (real)p->k_stiff;
  const real stiffness = (real)1.0 - pow(((real)1.0 - k_stiff), (real)1.0 / (real)substep);
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real dpx = 0.0, dpy = 0.0, dpz = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      if (r_mag < h * (real)0.0001) r_mag = h * (real)0.0001;
      const real mass_q = rest_mass;
      real s_corr = (real)0.0;
      if (k != (real)0.0) {
        const real WdWdq = W(r_mag, h, W_norm) / Wdq;
        s_corr = -k;
        for (int e = 0; e < p->scorr_n; ++e) s_corr = s_corr * WdWdq;
      }
      const real delW = DelW(r_mag, h, DelW_norm);
      const real dp = mass_q * ((real)s->lam[i] + (real)s->lam[q] + s_corr) * delW;
      dpx += dp * x_diff / r_mag;
      dpy += dp * y_diff / r_mag;
      dpz += dp * z_diff / r_mag;
    }
    s->dpx[i] = stiffness * dpx / rest_density;
    s->dpy[i] = stiffness * dpy / rest_density;
    s->dpz[i] = stiffness * dpz / rest_density;
  }
}

/* UpdatePositionStars, particles.c:529-564 */
void oracle_update_position_stars(const OracleParams *p, OracleState *s) {
  for (int i = 0; i < s->n; ++i) {
    s->xs[i] = (real)s->xs[i] + (real)s->dpx[i];
    s->ys[i] = (real)s->ys[i] + (real)s->dpy[i];
    s->zs[i] = (real)s->zs[i] + (real)s->dpz[i];
    boundary(p, &s->xs[i], &s->ys[i], &s->zs[i]);
  }
  oracle_particle_collisions(p, s->xs, s->ys, s->zs, s->n);
}

/* UpdateVelocities, particles.c:787-838 */
void oracle_update_velocities(const OracleParams *p, OracleState *s) {
  const real dt = (real)p->dt;
  const real v_max = (real)p->v_max;
  for (int i = 0; i < s->n; ++i) {
    real vx = ((real)s->xs[i] - (real)s->x[i]) / dt;
    real vy = ((real)s->ys[i] - (real)s->y[i]) / dt;
    real vz = ((real)s->zs[i] - (real)s->z[i]) / dt;
    if (vx > v_max) vx = v_max; else if (vx < -v_max) vx = -v_max;
    if (vy > v_max) vy = v_max; else if (vy < -v_max) vy = -v_max;
    if (vz > v_max) vz = v_max; else if (vz < -v_max) vz = -v_max;
    s->vx[i] = vx;
    s->vy[i] = vy;
    s->vz[i] = vz;
  }
}

/* ComputeSurfaceTension, particles.c:67-205 (colour pass :94-140, force
 * pass :142-204) */
void oracle_surface_tension(const OracleParams *p, OracleState *s,
                            const OracleNeighbors *nb) {
  const real rest_density = (real)p->rest_density;
  const real rest_mass = (real)p->rest_mass;
  const real h = (real)p->h;
  const real DelW_poly_norm = (real)p->DelW_poly_norm;
  const real dt = (real)p->dt;
  const real C_norm = (real)32.0 / ((real)M_PI * pow(h, (real)9.0));
  const real gama = (real)p->gamma;
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real color_dx = 0.0, color_dy = 0.0, color_dz = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      if (r_mag < h * (real)0.0001) r_mag = h * (real)0.0001;
      const real grad = DelWPoly(r_mag, h, DelW_poly_norm);
      const real mass_q = rest_mass;
      color_dx += grad * mass_q / (real)s->rho[q] * x_diff / r_mag;
      color_dy += grad * mass_q / (real)s->rho[q] * y_diff / r_mag;
      color_dz += grad * mass_q / (real)s->rho[q] * z_diff / r_mag;
    }
    s->cx[i] = h * color_dx;
    s->cy[i] = h * color_dy;
    s->cz[i] = h * color_dz;
  }
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real Fx = 0.0, Fy = 0.0, Fz = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    const real density_p = (real)s->rho[i];
    const real color_x_p = (real)s->cx[i];
    const real color_y_p = (real)s->cy[i];
    const real color_z_p = (real)s->cz[i];
    const real mass_p = rest_mass;
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      if (r_mag < h * (real)0.0001) r_mag = h * (real)0.0001;
      const real mass_q = rest_mass;
      const real c = Ccoh(r_mag, h, C_norm);
      const real F_cohesion_x = (real)-20.0 * gama * mass_p * mass_q * c * x_diff / r_mag;
      const real F_cohesion_y = (real)-20.0 * gama * mass_p * mass_q * c * y_diff / r_mag;
      const real F_cohesion_z = (real)-20.0 * gama * mass_p * mass_q * c * z_diff / r_mag;
      const real F_curvature_x = -gama * mass_p * (color_x_p - (real)s->cx[q]);
      const real F_curvature_y = -gama * mass_p * (color_y_p - (real)s->cy[q]);
      const real F_curvature_z = -gama * mass_p * (color_z_p - (real)s->cz[q]);
      const real K = (real)2.0 * rest_density / (density_p + (real)s->rho[q]);
      Fx += K * (F_cohesion_x + F_curvature_x);
      Fy += K * (F_cohesion_y + F_curvature_y);
      Fz += K * (F_cohesion_z + F_curvature_z);
    }
    s->vx[i] = (real)s->vx[i] + dt * Fx / density_p;
    s->vy[i] = (real)s->vy[i] + dt * Fy / density_p;
    s->vz[i] = (real)s->vz[i] + dt * Fz / density_p;
  }
}

/* ApplyViscosity, particles.c:383-459.  Mode 0 is the verbatim in-place
 * update (Gauss-Seidel in index order on the CPU; a data race under OpenACC
 * on the GPU).  Modes 1 and 2 are Jacobi: every particle reads the
 * velocities from before the pass. */
void oracle_apply_viscosity(const OracleParams *p, OracleState *s,
                            const OracleNeighbors *nb) {
  const real c = (real)p->c;
  const real h = (real)p->h;
  const real rest_mass = (real)p->rest_mass;
  const real W_norm = (real)p->W_norm;
  const int n = s->n;
  const double *vx = s->vx, *vy = s->vy, *vz = s->vz;
  double *out = NULL;
  if (p->xsph_mode != 0) {
    out = (double *)malloc(sizeof(double) * 3 * (size_t)n);
  }
  for (int i = 0; i < n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real sx = 0.0, sy = 0.0, sz = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    const real v_x_p = (real)vx[i];
    const real v_y_p = (real)vy[i];
    const real v_z_p = (real)vz[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      const real vx_diff = (real)vx[q] - v_x_p;
      const real vy_diff = (real)vy[q] - v_y_p;
      const real vz_diff = (real)vz[q] - v_z_p;
      real r_mag;
      if (p->xsph_mode == 2)
        r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      else /* particles.c:439 as written */
        r_mag = sqrt(x_diff * x_diff + y_diff * y_diff * z_diff * z_diff);
      const real w = W(r_mag, h, W_norm);
      const real mass_q = rest_mass;
      sx += vx_diff * w * mass_q / (real)s->rho[q];
      sy += vy_diff * w * mass_q / (real)s->rho[q];
      sz += vz_diff * w * mass_q / (real)s->rho[q];
    }
    sx *= c;
    sy *= c;
    sz *= c;
    if (out) {
      out[3 * (size_t)i + 0] = v_x_p + sx;
      out[3 * (size_t)i + 1] = v_y_p + sy;
      out[3 * (size_t)i + 2] = v_z_p + sz;
    } else {
      s->vx[i] = v_x_p + sx;
      s->vy[i] = v_y_p + sy;
      s->vz[i] = v_z_p + sz;
    }
  }
  if (out) {
    for (int i = 0; i < n; ++i) {
      s->vx[i] = out[3 * (size_t)i + 0];
      s->vy[i] = out[3 * (size_t)i + 1];
      s->vz[i] = out[3 * (size_t)i + 2];
    }
    free(out);
  }
}

/* ComputeVorticity, particles.c:207-283 */
void oracle_compute_vorticity(const OracleParams *p, OracleState *s,
                              const OracleNeighbors *nb) {
  const real h = (real)p->h;
  const real DelW_norm = (real)p->DelW_norm;
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real vort_x = 0.0, vort_y = 0.0, vort_z = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    const real v_x_p = (real)s->vx[i];
    const real v_y_p = (real)s->vy[i];
    const real v_z_p = (real)s->vz[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      const real vx_diff = (real)s->vx[q] - v_x_p;
      const real vy_diff = (real)s->vy[q] - v_y_p;
      const real vz_diff = (real)s->vz[q] - v_z_p;
      real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      if (r_mag < h * (real)0.0001) r_mag = h * (real)0.0001;
      const real dw = DelW(r_mag, h, DelW_norm);
      const real dw_x = dw * x_diff / r_mag;
      const real dw_y = dw * y_diff / r_mag;
      const real dw_z = dw * z_diff / r_mag;
      vort_x += vy_diff * dw_z - vz_diff * dw_y;
      vort_y += vz_diff * dw_x - vx_diff * dw_z;
      vort_z += vx_diff * dw_y - vy_diff * dw_x;
    }
    s->wx[i] = vort_x;
    s->wy[i] = vort_y;
    s->wz[i] = vort_z;
  }
}

/* ApplyVorticityConfinement, particles.c:285-381 (eps parameterised) */
void oracle_vorticity_confinement(const OracleParams *p, OracleState *s,
                                  const OracleNeighbors *nb) {
  const real dt = (real)p->dt;
  const real eps = (real)p->vorticity_eps;
  const real h = (real)p->h;
  const real rest_mass = (real)p->rest_mass;
  const real DelW_norm = (real)p->DelW_norm;
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    real eta_x = 0.0, eta_y = 0.0, eta_z = 0.0;
    const real x_star_p = (real)s->xs[i];
    const real y_star_p = (real)s->ys[i];
    const real z_star_p = (real)s->zs[i];
    for (int j = 0; j < nb->count[i]; ++j) {
      const int q = (int)nbr[j];
      const real x_diff = x_star_p - (real)s->xs[q];
      const real y_diff = y_star_p - (real)s->ys[q];
      const real z_diff = z_star_p - (real)s->zs[q];
      real r_mag = sqrt(x_diff * x_diff + y_diff * y_diff + z_diff * z_diff);
      if (r_mag < h * (real)0.0001) r_mag = h * (real)0.0001;
      const real dw = DelW(r_mag, h, DelW_norm);
      const real dw_x = dw * x_diff / r_mag;
      const real dw_y = dw * y_diff / r_mag;
      const real dw_z = dw * z_diff / r_mag;
      const real wqx = (real)s->wx[q], wqy = (real)s->wy[q], wqz = (real)s->wz[q];
      const real vort_mag = sqrt(wqx * wqx + wqy * wqy + wqz * wqz);
      eta_x += vort_mag * dw_x;
      eta_y += vort_mag * dw_y;
      eta_z += vort_mag * dw_z;
    }
    real eta_mag = sqrt(eta_x * eta_x + eta_y * eta_y + eta_z * eta_z);
    if (eta_mag < h * (real)0.0001) eta_mag = h * (real)0.0001;
    const real N_x = eta_x / eta_mag;
    const real N_y = eta_y / eta_mag;
    const real N_z = eta_z / eta_mag;
    const real wx = (real)s->wx[i], wy = (real)s->wy[i], wz = (real)s->wz[i];
    const real mass_p = rest_mass;
    s->vx[i] = (real)s->vx[i] + dt * eps * (N_y * wz - N_z * wy) / mass_p;
    s->vy[i] = (real)s->vy[i] + dt * eps * (N_z * wx - N_x * wz) / mass_p;
    s->vz[i] = (real)s->vz[i] + dt * eps * (N_x * wy - N_y * wx) / mass_p;
  }
}

/* UpdatePositions, particles.c:566-586 */
void oracle_update_positions(OracleState *s) {
  for (int i = 0; i < s->n; ++i) {
    s->x[i] = s->xs[i];
    s->y[i] = s->ys[i];
    s->z[i] = s->zs[i];
  }
}

/* Loop body of main, simulation.c:56-116 */
void oracle_step(const OracleParams *p, OracleState *s, OracleNeighbors *nb) {
  oracle_apply_gravity(p, s);
  oracle_predict_positions(p, s);
  oracle_find_all_neighbors(p, s, nb);
  for (int sub_i = 0; sub_i < p->solve_iterations; ++sub_i) {
    oracle_compute_densities(p, s, nb);
    oracle_compute_lambda(p, s, nb);
    oracle_update_dps(p, s, nb, sub_i);
    oracle_update_position_stars(p, s);
  }
  oracle_update_velocities(p, s);
  if (p->enable_tension) oracle_surface_tension(p, s, nb);
  oracle_apply_viscosity(p, s, nb);
  if (p->enable_vorticity) {
    oracle_compute_vorticity(p, s, nb);
    oracle_vorticity_confinement(p, s, nb);
  }
  oracle_update_positions(s);
}

/* Warm-start features of every particle (no reference counterpart: they
 * are the inputs of the learned warm start of the constraint solve whose
 * plain iteration is particles.c:588-746).  Computed from the predicted
 * state (x*, v) and the neighbour buckets, in double:
 *   0 rho/rho0 - 1, 1 C = max(rho/rho0 - 1, 0), 2 lambda (particles.c:616-663),
 *   3 sum_q |grad_q C|^2 / rho0^2, 4 |sum_q grad_q C|^2 / rho0^2,
 *   5 neighbour count, 6-8 mean (x*_q - x*_p) / h,
 *   9-11 mean ((x* - x)_q - (x* - x)_p) / h (the mean relative velocity
 *   times dt / h away from the box walls), 12 SDF distance at x* / h clamped to
 *   [-4, 4] (4 without an obstacle or outside its box), 13 nearest-neighbour
 *   distance / h (1 without neighbours), 14 distance to the nearest box wall
 *   / h clamped to [0, 4], 15 (x* - x) along the gravity axis / h. */
void oracle_features(const OracleParams *p, const OracleState *s,
                     const OracleNeighbors *nb, double *feat) {
  const double h = p->h, m = p->rest_mass, rho0 = p->rest_density;
  const double W0 = m * p->W_norm * h * h * h * h * h * h;
  for (int i = 0; i < s->n; ++i) {
    const uint32_t *nbr = nb->nbr + (size_t)i * ORACLE_MAX_NEIGHBORS;
    const double xp = s->xs[i], yp = s->ys[i], zp = s->zs[i];
    double rho = W0, sgx = 0, sgy = 0, sgz = 0, sC = 0;
    double o[3] = {0, 0, 0}, u[3] = {0, 0, 0}, rmin2 = h * h;
    const int cnt = nb->count[i];
    for (int j = 0; j < cnt; ++j) {
      const int q = (int)nbr[j];
      const double dx = xp - s->xs[q], dy = yp - s->ys[q], dz = zp - s->zs[q];
      const double r2 = dx * dx + dy * dy + dz * dz;
      double r = sqrt(r2);
      rho += m * W(r, h, p->W_norm);
      if (r < h * 0.0001) r = h * 0.0001;
      const double g = m * DelW(r, h, p->DelW_norm);
      const double gx = g * dx / r, gy = g * dy / r, gz = g * dz / r;
      sgx += gx; sgy += gy; sgz += gz;
      sC += gx * gx + gy * gy + gz * gz;
      o[0] -= dx; o[1] -= dy; o[2] -= dz;
      u[0] += (s->xs[q] - s->x[q]) - (s->xs[i] - s->x[i]);
      u[1] += (s->ys[q] - s->y[q]) - (s->ys[i] - s->y[i]);
      u[2] += (s->zs[q] - s->z[q]) - (s->zs[i] - s->z[i]);
      if (r2 < rmin2) rmin2 = r2;
    }
    const double C0 = rho / rho0 - 1.0;
    const double C = C0 < 0.0 ? 0.0 : C0;
    const double s_pairs = sC / (rho0 * rho0);
    const double s_self = (sgx * sgx + sgy * sgy + sgz * sgz) / (rho0 * rho0);
    const double lam = -C / (s_pairs + s_self + p->lambda_epsilon);
    const double ic = cnt > 0 ? 1.0 / cnt : 0.0;
    double sdf = 4.0;
    if (p->sdf && xp > p->ob_min[0] && xp < p->ob_max[0] && yp > p->ob_min[1] &&
        yp < p->ob_max[1] && zp > p->ob_min[2] && zp < p->ob_max[2]) {
      const float L = (float)(p->ob_max[0] - p->ob_min[0]);
      const float H = (float)(p->ob_max[1] - p->ob_min[1]);
      const float D = (float)(p->ob_max[2] - p->ob_min[2]);
      const float d = oracle_sdf_sample(p, (float)((xp - p->ob_min[0]) / L),
                                        (float)((yp - p->ob_min[1]) / H),
                                        (float)((zp - p->ob_min[2]) / D));
      const double m2w = (double)(L / (float)(p->sdim[0] * p->sdf_spacing));
      sdf = d * m2w / h;
      if (sdf < -4.0) sdf = -4.0;
      if (sdf > 4.0) sdf = 4.0;
    }
    double wall = xp - p->bmin[0];
    const double wl[5] = {p->bmax[0] - xp, yp - p->bmin[1], p->bmax[1] - yp,
                          zp - p->bmin[2], p->bmax[2] - zp};
    for (int k = 0; k < 5; ++k) if (wl[k] < wall) wall = wl[k];
    wall /= h;
    if (wall < 0.0) wall = 0.0;
    if (wall > 4.0) wall = 4.0;
    const int ga = p->gravity_axis;
    const double dg = ga == 0 ? xp - s->x[i] : (ga == 1 ? yp - s->y[i] : zp - s->z[i]);
    double *f = feat + (size_t)i * 16;
    f[0] = C0; f[1] = C; f[2] = lam; f[3] = s_pairs; f[4] = s_self; f[5] = cnt;
    for (int k = 0; k < 3; ++k) {
      f[6 + k] = o[k] * ic / h;
      f[9 + k] = u[k] * ic / h;
    }
    f[12] = sdf;
    f[13] = sqrt(rmin2) / h;
    f[14] = wall;
    f[15] = dg / h;
  }
}

/* Training target of the warm start: one plain solve of `iterations`
 * substeps (ComputeDensities, ComputeLambda, UpdateDPs,
 * UpdatePositionStars; simulation.c:72-82) from the predicted state, with
 * target[i] = sum_k s_k lambda_k, s_k the stiffness of substep k
 * (particles.c:693-694).  Leaves s advanced by the solve. */
void oracle_lambda_target(const OracleParams *p, OracleState *s,
                          const OracleNeighbors *nb, int iterations, double *target) {
  for (int i = 0; i < s->n; ++i) target[i] = 0.0;
  for (int k = 0; k < iterations; ++k) {
    const double stiff = 1.0 - pow(1.0 - p->k_stiff, 1.0 / (double)k);
    oracle_compute_densities(p, s, nb);
    oracle_compute_lambda(p, s, nb);
    for (int i = 0; i < s->n; ++i) target[i] += stiff * s->lam[i];
    oracle_update_dps(p, s, nb, k);
    oracle_update_position_stars(p, s);
  }
}

void oracle_diagnostics(const OracleParams *p, const OracleState *s,
                        OracleDiag *d) {
  double mx = 0.0, sum = 0.0, ke = 0.0;
  double com[3] = {0, 0, 0}, mom[3] = {0, 0, 0};
  for (int i = 0; i < s->n; ++i) {
    double e = s->rho[i] / p->rest_density - 1.0;
    if (e < 0.0) e = 0.0;
    if (e > mx) mx = e;
    sum += e;
    ke += s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i];
    com[0] += s->x[i]; com[1] += s->y[i]; com[2] += s->z[i];
    mom[0] += s->vx[i]; mom[1] += s->vy[i]; mom[2] += s->vz[i];
  }
  d->max_density_error = mx;
  d->mean_density_error = s->n ? sum / s->n : 0.0;
  d->kinetic_energy = 0.5 * p->rest_mass * ke;
  for (int k = 0; k < 3; ++k) {
    d->com[k] = s->n ? com[k] / s->n : 0.0;
    d->momentum[k] = p->rest_mass * mom[k];
  }
}
