/*
 * sphpc_types.h -- the reference's host-visible structs, same field names,
 * order and types, so C host code written against SPHPC's headers compiles
 * and links against libsphpc_cuda.so unchanged:
 *
 *   struct Params          Simulation/src/simulation.h:10-26
 *   struct AABB            Simulation/src/geometry.h:11-18
 *   struct Particles       Simulation/src/particles.h:11-42
 *   struct NeighborBucket  Simulation/src/neighbors.h:25-28
 *   struct Neighbors       Simulation/src/neighbors.h:13-23
 *   struct Obstacle        Simulation/src/obstacle.h:9-30
 *
 * plus the settings the reference hard-codes in its sources (struct
 * SphpcSolver) and FP64 diagnostics (struct SphpcDiag).
 */
#ifndef SPHPC_TYPES_H_
#define SPHPC_TYPES_H_

#ifdef __cplusplus
#define SPHPC_RESTRICT __restrict
extern "C" {
#else
#define SPHPC_RESTRICT restrict
#endif

#define MAX_NEIGHBORS 60

struct Params {
  double smoothing_radius;
  double W_norm;
  double DelW_norm;
  double DelW_poly_norm;
  double g;
  double time_step;
  double k;
  double dq;
  double c;
  double node_start_x;
  double node_end_x;
  double fluid_volume;
  int number_steps;
  int rank;
  int proc_count;
};

struct AABB {
  double min_x;
  double max_x;
  double min_y;
  double max_y;
  double min_z;
  double max_z;
};

struct Particles {
  double *SPHPC_RESTRICT x_star;
  double *SPHPC_RESTRICT y_star;
  double *SPHPC_RESTRICT z_star;
  double *SPHPC_RESTRICT x;
  double *SPHPC_RESTRICT y;
  double *SPHPC_RESTRICT z;
  double *SPHPC_RESTRICT v_x;
  double *SPHPC_RESTRICT v_y;
  double *SPHPC_RESTRICT v_z;
  double *SPHPC_RESTRICT dp_x;
  double *SPHPC_RESTRICT dp_y;
  double *SPHPC_RESTRICT dp_z;
  double *SPHPC_RESTRICT w_x;
  double *SPHPC_RESTRICT w_y;
  double *SPHPC_RESTRICT w_z;
  double *SPHPC_RESTRICT color_x;
  double *SPHPC_RESTRICT color_y;
  double *SPHPC_RESTRICT color_z;
  double *SPHPC_RESTRICT density;
  double *SPHPC_RESTRICT lambda;
  int *SPHPC_RESTRICT id;

  double rest_density;
  double rest_mass;
  double rest_radius;
  int global_count;
  int local_count;
  int max_local;
  int halo_count_left;
  int halo_count_right;
};

struct NeighborBucket {
  unsigned int neighbor_indices[MAX_NEIGHBORS];
  int count;
};

struct Neighbors {
  unsigned int *SPHPC_RESTRICT start_indices;
  unsigned int *SPHPC_RESTRICT end_indices;
  unsigned int *SPHPC_RESTRICT hash_values;
  unsigned int *SPHPC_RESTRICT particle_ids;
  int hash_size_x;
  int hash_size_y;
  int hash_size_z;
  struct NeighborBucket *SPHPC_RESTRICT neighbor_buckets;
  double hash_spacing;
};

/* Opaque device side of an obstacle (the reference's struct Obstacle_CUDA,
 * obstacle_cuda.h:11-14, holds a cudaArray and a texture object; this one
 * holds a linear device copy of the SDF). */
struct Obstacle_CUDA;

/* Snapshot output state, fileio_MPI_IO.h:8-12 (same fields): write_buffer
 * holds 3 * max_local doubles (page-locked here), output_path the output
 * directory, file_num the number of the next file. */
struct FileIO {
  double *write_buffer;
  char *output_path;
  int file_num;
};

struct Obstacle {
  char SDF_file_name[128];
  double origin_x;
  double origin_y;
  double origin_z;
  double model_length;
  double model_width;
  double model_height;
  struct AABB world_bounds;
  double SDF_spacing;
  int SDF_dim_x;
  int SDF_dim_y;
  int SDF_dim_z;
  float *SDF_buffer;
  struct Obstacle_CUDA *obstacle_cuda;
};

/* Constants the reference hard-codes, as settings.  sphpc_default_solver()
 * fills the reference's values; the INI loader reads them from an optional
 * [Solver] section (and jitter/seed from [InitialFluidVolume]). */
struct SphpcSolver {
  int solve_iterations;       /* simulation.c:72: 10 */
  int scorr_n;                /* exponent of s_corr (particles.c:730): 4 */
  double lambda_epsilon;      /* particles.c:663: 0.01 (normalised units) */
  double scorr_k;             /* particles.c:730: 0 = s_corr off */
  double scorr_dq;            /* s_corr delta-q as a fraction of h: 0.1 */
  double stiffness_k;         /* particles.c:693: 0.95 */
  double vorticity_epsilon;   /* particles.c:289: 0.1 h (negative = 0.1 h) */
  double velocity_max;        /* particles.c:791: 100 */
  int gravity_axis;           /* particles.c:519-525: 2 (z) */
  int xsph_exact;             /* 0: distance as written at particles.c:439 */
  int surface_tension;        /* 1: ComputeSurfaceTension runs */
  int vorticity;              /* 1: ComputeVorticity + confinement run */
  double jitter;              /* initial lattice jitter, fraction of spacing */
  unsigned long long seed;    /* jitter seed */
  int rest_density_lattice;   /* 0: rho0 = 1000, m = 0.991 V rho0 / N
                                 (particles.c:1034-1037); 1: m = 1000 V / N,
                                 rho0 = m * lattice poly6 sum */
  int adaptive;               /* 1: iterate until max density error <=
                                 density_tolerance or max_iterations */
  double density_tolerance;
  int max_iterations;         /* cap on the position passes of a step, the
                                 warm-start pass included (solve_iterations
                                 likewise without adaptive) */
  int warm_start;             /* 1: MLP warm start of the first iteration */
  int lambda_epsilon_mass_units; /* 1: lambda_epsilon is added before the
                                    1/rho0^2 normalisation (particles.c:661),
                                    i.e. the effective value is eps/rho0^2 */
  int warm_start_gate;        /* 1: discard a warm pass that does not lower the
                                 FP64 max density error (default) */
  int warm_start_source;      /* 0: the MLP's multipliers (default); 1: the
                                 previous step's applied multipliers
                                 sum_k s_k lambda_k, carried through the
                                 sort permutation (no network) */
  double warm_start_scale;    /* multiplier on the network's Lambda (1) */
  double min_progress;        /* adaptive: also stop (not converged) when two
                                 iterations together lower the FP64 max density
                                 error by less than this fraction; 0 (default):
                                 off */
  double warm_start_min_error; /* warm start: run the network only when the
                                 feature pass's FP64 max density error is
                                 above this (0, the default: always); below
                                 it the step is a plain solve from the
                                 feature pass's lambda_0, and the next step
                                 (adaptive) is a plain solve without the
                                 feature pass */
};

/* FP64 reductions over the local particles. */
struct SphpcDiag {
  double max_density_error;   /* max_i max(rho_i / rho0 - 1, 0) */
  double mean_density_error;
  double kinetic_energy;      /* 0.5 m sum |v|^2 */
  double com[3];              /* centre of mass of x */
  double momentum[3];         /* m sum v */
  double iterations;          /* constraint iterations of the last step */
  double warm_start_used;     /* 1 if the last step used the MLP start */
};

/* Host-side record of the last sphpc_step (no device work to read it). */
struct SphpcStepInfo {
  int iterations;             /* constraint iterations run (warm start counts 1) */
  int converged;              /* adaptive: max density error reached tolerance */
  int warm_start_used;
  int warm_start_rejected;    /* the residual gate discarded the warm pass */
  double max_density_error;   /* FP64, at the last density evaluation */
  double mean_density_error;
  int trace_len;              /* density evaluations of the step (<= 16) */
  int pad;
  double trace[16];           /* FP64 max density error at each of them, in order */
};

/* Per-kernel device time collected with CUDA events (sphpc_profile). */
struct SphpcKernelTime {
  char name[32];
  int launches;
  int pad;
  double total_ms;
};

#ifdef __cplusplus
}
#endif

#endif
