/*
 * pbf_oracle.h -- CPU restatement of SPHPC's per-step PBF particle pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product library (sphpc_b200/libsphpc_cuda.so) never
 * links, loads or calls it.
 *
 * Parity pin: with the reference's own hard-coded constants ("reference-compat"
 * parameter set: 10 iterations, lambda epsilon 0.01, s_corr off, gravity -z,
 * vorticity eps 0.1h, in-place Gauss-Seidel XSPH) this restatement reproduces
 * the reference itself, compiled verbatim from Simulation/src/particles.c and
 * Simulation/src/neighbors.c by oracle/Makefile into oracle/_ref/, bit for bit
 * (tests/test_oracle_pin.py).  The reference ships no golden vectors or tests
 * of its own, so that comparison is the pin.
 *
 * Everything is in original particle-index order, like the reference: arrays
 * are never physically reordered; neighbour buckets hold original indices.
 *
 * Build: `real` is double by default (the FP64 oracle); -DORACLE_REAL_FLOAT
 * gives an FP32 build of the same code for tighter FP32-vs-FP32 checks.
 */
#ifndef SPHPC_ORACLE_H_
#define SPHPC_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_NEIGHBORS 60 /* neighbors.h:6 */

/* All physics parameters.  Fields that are hard-coded constants in the
 * reference carry the reference value as their "reference-compat" default
 * (see oracle_params_reference_compat). */
typedef struct OracleParams {
  /* struct Params (simulation.h:10-26) */
  double h;              /* smoothing_radius */
  double W_norm;         /* 315/(64 pi h^9)     simulation.c:175 */
  double DelW_norm;      /* -45/(pi h^6)        simulation.c:177 */
  double DelW_poly_norm; /* -6 W_norm           simulation.c:176 */
  double g;              /* gravity magnitude   PhysicalParameters.g */
  double dt;             /* time_step */
  double gamma;          /* surface tension k   PhysicalParameters.k */
  double dq;             /* params->dq (0.1h)   simulation.c:155 (unused by ref) */
  double c;              /* XSPH c              PhysicalParameters.c */
  /* struct AABB boundary_global (geometry.h:11-18); min must be 0 */
  double bmin[3];
  double bmax[3];
  /* struct Particles scalars (particles.h:34-36) */
  double rest_density;
  double rest_mass;
  /* Constants hard-coded in the reference, made parameters. */
  int solve_iterations;  /* simulation.c:72, 10 */
  int scorr_n;           /* exponent n of s_corr (particles.c:729-730) */
  double lambda_epsilon; /* particles.c:663, 0.01 */
  double scorr_k;        /* particles.c:730, 0 (disabled in reference) */
  double scorr_dq;       /* absolute delta-q of s_corr */
  double k_stiff;        /* particles.c:693, 0.95 */
  double vorticity_eps;  /* particles.c:289, 0.1h */
  double v_max;          /* particles.c:791, 100 */
  int gravity_axis;      /* particles.c:519-525 (axis 2 = z) */
  int xsph_mode;         /* 0: in-place Gauss-Seidel with the reference's r
                          *    expression (particles.c:439) -- verbatim CPU;
                          * 1: Jacobi (double-buffered) with the same r;
                          * 2: Jacobi with the Euclidean r. */
  int enable_tension;    /* run ComputeSurfaceTension (particles.c:67-205) */
  int enable_vorticity;  /* run ComputeVorticity + confinement */
  /* uniform grid (neighbors.c:23-28) */
  int nx, ny, nz;
  int pad0;
  /* obstacle SDF (obstacle.h:9-30); sdf == NULL means no obstacle */
  const float *sdf;      /* x fastest, dims sdim[0..2] */
  int sdim[3];
  int pad1;
  double sdf_spacing;
  double ob_min[3];      /* obstacle world bounds */
  double ob_max[3];
} OracleParams;

/* Particle state, SoA, original-index order (particles.h:11-42). */
typedef struct OracleState {
  int n;
  int pad;
  double *xs, *ys, *zs;     /* x_star */
  double *x, *y, *z;
  double *vx, *vy, *vz;
  double *dpx, *dpy, *dpz;
  double *wx, *wy, *wz;
  double *cx, *cy, *cz;     /* color */
  double *rho;
  double *lam;
} OracleState;

/* struct Neighbors (neighbors.h:13-28) */
typedef struct OracleNeighbors {
  uint32_t *keys;     /* hash_values[n], sorted after oracle_sort_hash */
  uint32_t *ids;      /* particle_ids[n] */
  uint32_t *start;    /* start_indices[C] */
  uint32_t *end;      /* end_indices[C] */
  uint32_t *nbr;      /* n * 60 neighbour indices */
  int32_t *count;     /* n */
} OracleNeighbors;

/* Diagnostics, FP64 reductions. */
typedef struct OracleDiag {
  double max_density_error; /* max_i max(rho_i/rho0 - 1, 0) */
  double mean_density_error;/* mean_i max(rho_i/rho0 - 1, 0) */
  double kinetic_energy;    /* 0.5 m sum |v|^2 */
  double com[3];            /* centre of mass of x */
  double momentum[3];       /* m sum v */
} OracleDiag;

/* ---- parameter helpers ---- */
/* SetParameters (simulation.c:130-178): h = 2*spacing, dq = 0.1h, norms. */
void oracle_set_kernel_norms(OracleParams *p, double h);
/* Reference-compat constants (the values hard-coded in particles.c etc.). */
void oracle_params_reference_compat(OracleParams *p);
/* Grid dims from the boundary (neighbors.c:23-28). */
void oracle_set_grid(OracleParams *p);

/* ---- scene generation ---- */
/* Counter-based uniform double in [0,1): SplitMix64 finaliser of
 * (seed, index, axis) (Steele, Lea, Flood, OOPSLA 2014). */
double oracle_uniform01(uint64_t seed, uint64_t index, uint32_t axis);
/* Cell-centred lattice (geometry.c:19-74) with +-jitter*spacing uniform
 * jitter; lattice index i = ix + nxl*(iy + nyl*iz). */
void oracle_lattice(int nxl, int nyl, int nzl, double spacing,
                    const double origin[3], double jitter, uint64_t seed,
                    double *x, double *y, double *z);
/* Sum of poly6 W over a perfect lattice (self included), used as rho0/m. */
double oracle_lattice_poly6_sum(const OracleParams *p, double spacing);

/* ---- neighbour search (neighbors.c) ---- */
uint32_t oracle_hash_val(const OracleParams *p, double x, double y, double z);
void oracle_hash_particles(const OracleParams *p, const OracleState *s,
                           OracleNeighbors *nb);
void oracle_sort_by_key(uint32_t *keys, uint32_t *vals, int n);
void oracle_lower_bounds(const uint32_t *keys, int n, int search_count,
                         uint32_t *out);
void oracle_upper_bounds(const uint32_t *keys, int n, int search_count,
                         uint32_t *out);
void oracle_fill_neighbors(const OracleParams *p, const OracleState *s,
                           OracleNeighbors *nb);
void oracle_find_all_neighbors(const OracleParams *p, const OracleState *s,
                               OracleNeighbors *nb);

/* ---- SDF obstacle (obstacle_cuda.cu) ---- */
/* tex3D-style sample, normalised coords, clamp addressing, exact FP32
 * trilinear weights. */
float oracle_sdf_sample(const OracleParams *p, float u, float v, float w);
void oracle_particle_collisions(const OracleParams *p, double *x, double *y,
                                double *z, int n);

/* ---- step functions (particles.c) ---- */
void oracle_apply_gravity(const OracleParams *p, OracleState *s);
void oracle_predict_positions(const OracleParams *p, OracleState *s);
void oracle_compute_densities(const OracleParams *p, OracleState *s,
                              const OracleNeighbors *nb);
void oracle_compute_lambda(const OracleParams *p, OracleState *s,
                           const OracleNeighbors *nb);
void oracle_update_dps(const OracleParams *p, OracleState *s,
                       const OracleNeighbors *nb, int substep);
void oracle_update_position_stars(const OracleParams *p, OracleState *s);
void oracle_update_velocities(const OracleParams *p, OracleState *s);
void oracle_surface_tension(const OracleParams *p, OracleState *s,
                            const OracleNeighbors *nb);
void oracle_apply_viscosity(const OracleParams *p, OracleState *s,
                            const OracleNeighbors *nb);
void oracle_compute_vorticity(const OracleParams *p, OracleState *s,
                              const OracleNeighbors *nb);
void oracle_vorticity_confinement(const OracleParams *p, OracleState *s,
                                  const OracleNeighbors *nb);
void oracle_update_positions(OracleState *s);

/* One full time step (simulation.c:56-116 loop body). */
void oracle_step(const OracleParams *p, OracleState *s, OracleNeighbors *nb);
/* warm-start features [n][16] and plain-solve multiplier-sum target */
void oracle_features(const OracleParams *p, const OracleState *s,
                     const OracleNeighbors *nb, double *feat);
void oracle_lambda_target(const OracleParams *p, OracleState *s,
                          const OracleNeighbors *nb, int iterations, double *target);
void oracle_diagnostics(const OracleParams *p, const OracleState *s,
                        OracleDiag *d);

/* Size of one element of `real` (8 for the FP64 build, 4 for FP32). */
int oracle_real_size(void);

#ifdef __cplusplus
}
#endif

#endif
