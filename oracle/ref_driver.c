/*
 * ref_driver.c -- a C harness around the reference's own step functions.
 *
 * TEST INFRASTRUCTURE ONLY: built into oracle/_ref/libsphpc_ref.so together
 * with the reference's particles.c and neighbors.c compiled in place.  It
 * sets up the reference structs (struct Params simulation.h:10-26, struct
 * Particles particles.h:11-42, struct Neighbors neighbors.h:13-28, struct
 * Obstacle obstacle.h:9-30) from an OracleParams and runs the loop body of
 * main (simulation.c:56-116) with the solve-iteration count as an argument
 * (hard-coded 10 at simulation.c:72).
 */
#include <stdlib.h>
#include <string.h>

#include "geometry.h"
#include "neighbors.h"
#include "obstacle.h"
#include "particles.h"
#include "pbf_oracle.h"
#include "simulation.h"

typedef struct RefSim {
  struct Params params;
  struct Particles particles;
  struct Neighbors neighbors;
  struct AABB boundary;
  struct Obstacle obstacle;
} RefSim;

static double *dalloc(int n) { return (double *)calloc((size_t)n, sizeof(double)); }

RefSim *ref_create(const OracleParams *op, int n) {
  RefSim *s = (RefSim *)calloc(1, sizeof(RefSim));
  s->params.smoothing_radius = op->h;
  s->params.W_norm = op->W_norm;
  s->params.DelW_norm = op->DelW_norm;
  s->params.DelW_poly_norm = op->DelW_poly_norm;
  s->params.g = op->g;
  s->params.time_step = op->dt;
  s->params.k = op->gamma;
  s->params.dq = op->dq;
  s->params.c = op->c;
  s->params.node_start_x = op->bmin[0];
  s->params.node_end_x = op->bmax[0];
  s->params.number_steps = 0;
  s->params.rank = 0;
  s->params.proc_count = 1;
  s->boundary.min_x = op->bmin[0];
  s->boundary.max_x = op->bmax[0];
  s->boundary.min_y = op->bmin[1];
  s->boundary.max_y = op->bmax[1];
  s->boundary.min_z = op->bmin[2];
  s->boundary.max_z = op->bmax[2];

  struct Particles *p = &s->particles;
  p->max_local = n;
  p->local_count = n;
  p->global_count = n;
  p->halo_count_left = 0;
  p->halo_count_right = 0;
  p->rest_density = op->rest_density;
  p->rest_mass = op->rest_mass;
  p->x_star = dalloc(n); p->y_star = dalloc(n); p->z_star = dalloc(n);
  p->x = dalloc(n); p->y = dalloc(n); p->z = dalloc(n);
  p->v_x = dalloc(n); p->v_y = dalloc(n); p->v_z = dalloc(n);
  p->dp_x = dalloc(n); p->dp_y = dalloc(n); p->dp_z = dalloc(n);
  p->w_x = dalloc(n); p->w_y = dalloc(n); p->w_z = dalloc(n);
  p->color_x = dalloc(n); p->color_y = dalloc(n); p->color_z = dalloc(n);
  p->density = dalloc(n);
  p->lambda = dalloc(n);
  p->id = (int *)calloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; ++i) p->id[i] = i;

  AllocInitNeighbors(&s->neighbors, p, &s->params, &s->boundary);

  memset(&s->obstacle, 0, sizeof(s->obstacle));
  if (op->sdf) {
    s->obstacle.SDF_dim_x = op->sdim[0];
    s->obstacle.SDF_dim_y = op->sdim[1];
    s->obstacle.SDF_dim_z = op->sdim[2];
    s->obstacle.SDF_spacing = op->sdf_spacing;
    s->obstacle.world_bounds.min_x = op->ob_min[0];
    s->obstacle.world_bounds.min_y = op->ob_min[1];
    s->obstacle.world_bounds.min_z = op->ob_min[2];
    s->obstacle.world_bounds.max_x = op->ob_max[0];
    s->obstacle.world_bounds.max_y = op->ob_max[1];
    s->obstacle.world_bounds.max_z = op->ob_max[2];
    s->obstacle.SDF_buffer = (float *)op->sdf; /* borrowed, host memory */
  }
  return s;
}

void ref_destroy(RefSim *s) {
  struct Particles *p = &s->particles;
  free(p->x_star); free(p->y_star); free(p->z_star);
  free(p->x); free(p->y); free(p->z);
  free(p->v_x); free(p->v_y); free(p->v_z);
  free(p->dp_x); free(p->dp_y); free(p->dp_z);
  free(p->w_x); free(p->w_y); free(p->w_z);
  free(p->color_x); free(p->color_y); free(p->color_z);
  free(p->density); free(p->lambda); free(p->id);
  FinalizeNeighbors(&s->neighbors);
  free(s);
}

/* Field order used by ref_set_field / ref_get_field. */
static double *field(RefSim *s, int f) {
  struct Particles *p = &s->particles;
  double *tab[20] = {p->x_star, p->y_star, p->z_star, p->x, p->y, p->z,
                     p->v_x, p->v_y, p->v_z, p->dp_x, p->dp_y, p->dp_z,
                     p->w_x, p->w_y, p->w_z, p->color_x, p->color_y,
                     p->color_z, p->density, p->lambda};
  return (f >= 0 && f < 20) ? tab[f] : NULL;
}

int ref_set_field(RefSim *s, int f, const double *src) {
  double *d = field(s, f);
  if (!d) return -1;
  memcpy(d, src, sizeof(double) * (size_t)s->particles.local_count);
  return 0;
}

int ref_get_field(RefSim *s, int f, double *dst) {
  double *d = field(s, f);
  if (!d) return -1;
  memcpy(dst, d, sizeof(double) * (size_t)s->particles.local_count);
  return 0;
}

void ref_get_neighbors(RefSim *s, unsigned int *keys, unsigned int *ids,
                       unsigned int *start, unsigned int *end,
                       unsigned int *nbr, int *count) {
  const int n = s->particles.local_count;
  const size_t C = (size_t)s->neighbors.hash_size_x * s->neighbors.hash_size_y *
                   s->neighbors.hash_size_z;
  if (keys) memcpy(keys, s->neighbors.hash_values, sizeof(unsigned) * (size_t)n);
  if (ids) memcpy(ids, s->neighbors.particle_ids, sizeof(unsigned) * (size_t)n);
  if (start) memcpy(start, s->neighbors.start_indices, sizeof(unsigned) * C);
  if (end) memcpy(end, s->neighbors.end_indices, sizeof(unsigned) * C);
  for (int i = 0; i < n; ++i) {
    const struct NeighborBucket *b = &s->neighbors.neighbor_buckets[i];
    if (count) count[i] = b->count;
    if (nbr)
      for (int j = 0; j < MAX_NEIGHBORS; ++j)
        nbr[(size_t)i * MAX_NEIGHBORS + j] = j < b->count ? b->neighbor_indices[j] : 0u;
  }
}

/* Individual reference functions, for per-kernel checks. */
void ref_apply_gravity(RefSim *s) { ApplyGravity(&s->particles, &s->params); }
void ref_predict_positions(RefSim *s) {
  PredictPositions(&s->particles, &s->params, &s->boundary);
}
void ref_find_all_neighbors(RefSim *s) {
  FindAllNeighbors(&s->particles, &s->params, &s->neighbors);
}
void ref_compute_densities(RefSim *s) {
  ComputeDensities(&s->particles, &s->params, &s->neighbors);
}
void ref_compute_lambda(RefSim *s) {
  ComputeLambda(&s->particles, &s->params, &s->neighbors);
}
void ref_update_dps(RefSim *s, int substep) {
  UpdateDPs(&s->particles, &s->params, &s->neighbors, substep);
}
void ref_update_position_stars(RefSim *s) {
  UpdatePositionStars(&s->particles, &s->boundary, &s->obstacle, &s->params);
}
void ref_update_velocities(RefSim *s) { UpdateVelocities(&s->particles, &s->params); }
void ref_surface_tension(RefSim *s) {
  ComputeSurfaceTension(&s->particles, &s->params, &s->neighbors);
}
void ref_apply_viscosity(RefSim *s) {
  ApplyViscosity(&s->particles, &s->params, &s->neighbors);
}
void ref_compute_vorticity(RefSim *s) {
  ComputeVorticity(&s->particles, &s->params, &s->neighbors);
}
void ref_vorticity_confinement(RefSim *s) {
  ApplyVorticityConfinement(&s->particles, &s->params, &s->neighbors);
}
void ref_update_positions(RefSim *s) { UpdatePositions(&s->particles); }

/* Loop body of main, simulation.c:56-116, repeated nsteps times. */
void ref_step(RefSim *s, int nsteps, int solve_iterations) {
  for (int n = 0; n < nsteps; ++n) {
    ApplyGravity(&s->particles, &s->params);
    PredictPositions(&s->particles, &s->params, &s->boundary);
    FindAllNeighbors(&s->particles, &s->params, &s->neighbors);
    for (int sub_i = 0; sub_i < solve_iterations; ++sub_i) {
      ComputeDensities(&s->particles, &s->params, &s->neighbors);
      ComputeLambda(&s->particles, &s->params, &s->neighbors);
      UpdateDPs(&s->particles, &s->params, &s->neighbors, sub_i);
      UpdatePositionStars(&s->particles, &s->boundary, &s->obstacle, &s->params);
    }
    UpdateVelocities(&s->particles, &s->params);
    ComputeSurfaceTension(&s->particles, &s->params, &s->neighbors);
    ApplyViscosity(&s->particles, &s->params, &s->neighbors);
    ComputeVorticity(&s->particles, &s->params, &s->neighbors);
    ApplyVorticityConfinement(&s->particles, &s->params, &s->neighbors);
    UpdatePositions(&s->particles);
  }
}
