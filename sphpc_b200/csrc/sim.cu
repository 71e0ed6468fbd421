// sim.cu -- device copy of a particle set and the C ABI of the pipeline.
//
// A DeviceSim is the device mirror of one struct Particles (the reference
// keeps the same arrays resident with OpenACC `enter data`,
// particles.c:1056-1078).  Its kernels run on one stream; the reference-named
// step functions launch one stage each, sphpc_step launches the fused step.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "host_internal.h"
#include "kernels.cuh"
#include "mlp.cuh"
#include "../../include/sphpc_device.h"

struct Obstacle_CUDA {
  float* sdf;
  size_t count;
};

namespace sphpc {

// Failure injection for the allocation error paths (sphpc_fail_device_alloc):
// the number of particle-set device allocations still to succeed before one
// fails with SPHPC_ENOMEM without calling cudaMalloc; -1: off.
static std::atomic<long long> g_alloc_fail_after{-1};

template <class T>
static int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  long long left = g_alloc_fail_after.load();
  while (left >= 0 && !g_alloc_fail_after.compare_exchange_weak(left, left - 1)) {
  }
  if (left == 0) {
    *p = nullptr;
    return set_error(SPHPC_ENOMEM, "cudaMalloc(%zu bytes): failure injected", n * sizeof(T));
  }
  const cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(SPHPC_ENOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T),
                     cudaGetErrorString(e));
  }
  return SPHPC_OK;
}

template <class T>
static void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

static int bits_for(uint32_t v) {  // bits needed to hold values 0..v
  int b = 0;
  while (b < 32 && (v >> b) != 0) ++b;
  return b > 0 ? b : 1;
}

class DeviceSim {
 public:
  int n = 0;    // active particles (struct Particles' local_count)
  int cap = 0;  // capacity of every per-particle array (max_local, as the
                // reference mirrors particles.c:1056-1078)
  SphpcSolver solver{};
  cudaStream_t stream = nullptr;
  double rho0 = 1000.0, mass = 1.0;
  int device = 0;

  // grid
  bool grid_ready = false;
  int nx = 0, ny = 0, nz = 0;
  uint32_t C = 0;
  int bx = 0, by = 0, passes = 1;

  // per-particle arrays, slot order
  PD *pd = nullptr, *pd_alt = nullptr;
  float4 *vel = nullptr, *vel_alt = nullptr, *color = nullptr, *omega = nullptr, *dp = nullptr;
  float *rho = nullptr, *lam = nullptr;
  // alternates for the full reorder of the per-function path
  float4 *color_alt = nullptr, *omega_alt = nullptr, *dp_alt = nullptr;
  float *rho_alt = nullptr, *lam_alt = nullptr;
  uint32_t *ids = nullptr, *ids_spare = nullptr, *keys_by_id = nullptr, *loc_by_id = nullptr;
  uint32_t* keys_sorted = nullptr;  // view into keys_by_id or sort.keys_alt
  uint32_t *cellp = nullptr, *nbr = nullptr, *cstart = nullptr;
  float4* xsa = nullptr;
  NV *nv_a = nullptr, *nv_b = nullptr;  // combined records of the post passes
  uint8_t* ncount = nullptr;
  uint4* gaps = nullptr;
  uint32_t* small = nullptr;  // [0] gap count, [1] explicit count, [2] error bits
  double* resid = nullptr;    // [0] max (bits), [1] sum, [2..] diagnostics
  SortScratch sort{};
  uint32_t* sort_aux = nullptr;
  double* stage = nullptr;  // 20 * n doubles for host transfers
  // host arrays of the particle set page-locked by enter_data (so that the
  // transfers run at full link speed); released in release()
  std::vector<void*> pinned;
  bool nbr_valid = false;

  MlpState mlp{};
  uint4 *nr = nullptr, *nr_alt = nullptr;  // 16-byte neighbour records (x* fixed point, payload)
  uint4* nr_w = nullptr;         // third record buffer (warm start, feature export)
  // carried warm start: the multiplier sum_k s_k lambda_k applied to each
  // particle over the last step (slot order of that step), and whether it
  // holds one
  float* lam_acc = nullptr;
  bool have_carry = false;
  // slab decomposition: global id and ownership of every particle (host
  // order), the records a pack keeps, and pack counters
  bool slab = false;
  uint32_t* gid = nullptr;
  uint8_t* owned = nullptr;
  SlabRecord* slab_keep = nullptr;
  uint32_t* slab_counters = nullptr;
  uint32_t slab_nkeep = 0;
  int last_warm_rejected = 0;
  double prev_err0 = -1.0;       // first residual of the previous step (< 0: none)
  std::vector<double> trace;     // max density error at each evaluation of the step
  // training-set collection of the current step (collect_iters > 0)
  int collect_iters = 0;
  long long collect_rows = 0;
  float* collect_feat = nullptr;
  float* collect_target = nullptr;

  unsigned long long launches = 0;  // kernels launched by this particle set
  double last_iterations = 0.0;
  double last_warm = 0.0;
  double last_max_err = 0.0, last_mean_err = 0.0;
  int last_converged = 0;

  // profiling
  bool prof = false;
  struct Pending {
    int name;
    cudaEvent_t a, b;
  };
  std::vector<std::string> prof_names;
  std::map<std::string, int> prof_index;
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<double> prof_ms;
  std::vector<int> prof_count;

  ~DeviceSim() { release(); }

  uint32_t* gap_count() { return small; }
  uint32_t* err() { return small + 2; }

  void release() {
    // a read-back in flight still writes the host arrays: finish it first
    if (copy_stream) {
      cudaStreamSynchronize(copy_stream);
      cudaStreamDestroy(copy_stream);
      cudaEventDestroy(gathered);
      cudaEventDestroy(copied);
      copy_stream = nullptr;
      copy_pending = false;
    }
    dfree(pd); dfree(pd_alt); dfree(vel); dfree(vel_alt);
    dfree(color); dfree(omega); dfree(dp); dfree(rho); dfree(lam);
    dfree(color_alt); dfree(omega_alt); dfree(dp_alt); dfree(rho_alt); dfree(lam_alt);
    dfree(ids); dfree(ids_spare); dfree(keys_by_id); dfree(loc_by_id); dfree(cellp);
    dfree(nbr); dfree(xsa); dfree(nv_a); dfree(nv_b);
    dfree(cstart); dfree(ncount); dfree(gaps); dfree(small);
    dfree(resid); dfree(sort.keys_alt); dfree(sort.vals_alt); dfree(sort_aux); dfree(stage);
    mlp_release(mlp);
    for (void* h : pinned) cudaHostUnregister(h);
    pinned.clear();
    dfree(nr); dfree(nr_alt); dfree(nr_w); dfree(lam_acc);
    dfree(gid); dfree(owned); dfree(slab_keep); dfree(slab_counters);
    for (auto& p : pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    pending.clear();
    for (auto e : ev_pool) cudaEventDestroy(e);
    ev_pool.clear();
  }

  int alloc(int n_, int cap_) {
    n = n_;
    cap = cap_ > n_ ? cap_ : n_;
    const int c = cap;
    SPHPC_RC(dalloc(&pd, c)); SPHPC_RC(dalloc(&pd_alt, c));
    SPHPC_RC(dalloc(&nr, c)); SPHPC_RC(dalloc(&nr_alt, c));
    SPHPC_RC(dalloc(&vel, c)); SPHPC_RC(dalloc(&vel_alt, c));
    SPHPC_RC(dalloc(&color, c)); SPHPC_RC(dalloc(&omega, c)); SPHPC_RC(dalloc(&dp, c));
    SPHPC_RC(dalloc(&rho, c)); SPHPC_RC(dalloc(&lam, c));
    SPHPC_RC(dalloc(&ids, c)); SPHPC_RC(dalloc(&ids_spare, c));
    SPHPC_RC(dalloc(&keys_by_id, c)); SPHPC_RC(dalloc(&loc_by_id, c));
    SPHPC_RC(dalloc(&cellp, c)); SPHPC_RC(dalloc(&ncount, c));
    SPHPC_RC(dalloc(&nbr, (size_t)kMaxNeighbors * c));
    SPHPC_RC(dalloc(&xsa, (size_t)c + 2));  // pair blocks: 32 bytes per slot pair
    SPHPC_RC(dalloc(&nv_a, c)); SPHPC_RC(dalloc(&nv_b, c));
    SPHPC_CK(cudaMemsetAsync(ncount, 0, c, stream));
    SPHPC_RC(dalloc(&small, 8));
    SPHPC_RC(dalloc(&resid, 16));
    SPHPC_RC(dalloc(&sort.keys_alt, c));
    SPHPC_RC(dalloc(&sort.vals_alt, c));
    const size_t aux = sort_aux_words(c) + 4;
    SPHPC_RC(dalloc(&sort_aux, aux));
    sort.hist = sort_aux;
    sort.counters = sort_aux + (size_t)kMaxPasses * kRadix;
    sort.err = sort_aux + (size_t)kMaxPasses * kRadix + kMaxPasses;
    sort.lookback = sort_aux + (size_t)kMaxPasses * kRadix + kMaxPasses + 4;
    SPHPC_CK(cudaMemsetAsync(small, 0, 8 * sizeof(uint32_t), stream));
    SPHPC_CK(cudaMemsetAsync(sort_aux, 0, aux * sizeof(uint32_t), stream));
    SPHPC_CK(cudaMemsetAsync(pd, 0, sizeof(PD) * c, stream));
    SPHPC_CK(cudaMemsetAsync(vel, 0, sizeof(float4) * c, stream));
    SPHPC_CK(cudaMemsetAsync(color, 0, sizeof(float4) * c, stream));
    SPHPC_CK(cudaMemsetAsync(omega, 0, sizeof(float4) * c, stream));
    SPHPC_CK(cudaMemsetAsync(dp, 0, sizeof(float4) * c, stream));
    SPHPC_CK(cudaMemsetAsync(lam, 0, sizeof(float) * c, stream));
    return SPHPC_OK;
  }

  int ensure_full_alts() {
    if (!color_alt) SPHPC_RC(dalloc(&color_alt, cap));
    if (!omega_alt) SPHPC_RC(dalloc(&omega_alt, cap));
    if (!dp_alt) SPHPC_RC(dalloc(&dp_alt, cap));
    if (!rho_alt) SPHPC_RC(dalloc(&rho_alt, cap));
    if (!lam_alt) SPHPC_RC(dalloc(&lam_alt, cap));
    return SPHPC_OK;
  }

  int ensure_stage() {
    if (!stage) SPHPC_RC(dalloc(&stage, (size_t)20 * cap));
    return SPHPC_OK;
  }

  // asynchronous read-back: copy stream and its events, created on first use
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t gathered = nullptr, copied = nullptr;
  bool copy_pending = false;

  int ensure_copy_stream() {
    if (copy_stream) return SPHPC_OK;
    SPHPC_CK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    SPHPC_CK(cudaEventCreateWithFlags(&gathered, cudaEventDisableTiming));
    SPHPC_CK(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
    return SPHPC_OK;
  }

  // Waits for an asynchronous read-back in flight (the staging buffer and
  // the host arrays are then free).
  int wait_copies() {
    if (!copy_pending) return SPHPC_OK;
    copy_pending = false;
    SPHPC_CK(cudaEventSynchronize(copied));
    return SPHPC_OK;
  }

  // Grid of the hash (neighbors.c:23-28).
  int init_grid(const AABB& b, double h) {
    const double nxd = ceil((b.max_x - b.min_x) / h) + 1;
    const double nyd = ceil((b.max_y - b.min_y) / h) + 1;
    const double nzd = ceil((b.max_z - b.min_z) / h) + 1;
    if (!(nxd >= 1 && nyd >= 1 && nzd >= 1) || nxd * nyd * nzd >= 4294967295.0)
      return set_error(SPHPC_EINVAL, "grid %.0f x %.0f x %.0f does not fit 32-bit keys", nxd,
                       nyd, nzd);
    const int nnx = (int)nxd, nny = (int)nyd, nnz = (int)nzd;
    const int bxx = bits_for((uint32_t)nnx - 1), byy = bits_for((uint32_t)nny - 1),
              bzz = bits_for((uint32_t)nnz - 1);
    if (bxx + byy + bzz > 31)
      return set_error(SPHPC_EINVAL, "grid %d x %d x %d needs %d bits of packed cell "
                                     "coordinates (31 available)", nnx, nny, nnz,
                       bxx + byy + bzz);
    const uint32_t CC = (uint32_t)nnx * (uint32_t)nny * (uint32_t)nnz;
    if (grid_ready && CC == C && nnx == nx && nny == ny && nnz == nz) return SPHPC_OK;
    dfree(cstart);
    nx = nnx; ny = nny; nz = nnz; C = CC; bx = bxx; by = byy;
    passes = (bits_for(C - 1) + kRadixBits - 1) / kRadixBits;
    if (passes > kMaxPasses) passes = kMaxPasses;
    SPHPC_RC(dalloc(&cstart, (size_t)C + 1));
    dfree(gaps);
    SPHPC_RC(dalloc(&gaps, (size_t)cap + 4 + C / 4096));
    SPHPC_CK(cudaMemsetAsync(cstart, 0, sizeof(uint32_t) * ((size_t)C + 1), stream));
    grid_ready = true;
    nbr_valid = false;
    return SPHPC_OK;
  }

  NbrView view() const {
    NbrView v;
    v.nbr = nbr;
    v.ncount = ncount;
    v.cstart = cstart;
    v.n = n;
    v.nx = nx; v.ny = ny; v.nz = nz;
    v.nxny = (uint32_t)nx * (uint32_t)ny;
    v.bx = bx; v.by = by;
    v.mx = (1u << bx) - 1u;
    v.my = (1u << by) - 1u;
    return v;
  }

  // ---- profiling ----
  cudaEvent_t take_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  int prof_begin(const char* name, cudaEvent_t* b) {
    if (!prof) return -1;
    auto it = prof_index.find(name);
    int id;
    if (it == prof_index.end()) {
      id = (int)prof_names.size();
      prof_names.push_back(name);
      prof_index[name] = id;
      prof_ms.push_back(0.0);
      prof_count.push_back(0);
    } else {
      id = it->second;
    }
    *b = take_event();
    cudaEventRecord(*b, stream);
    return id;
  }
  void prof_end(int id, cudaEvent_t b) {
    if (id < 0) return;
    cudaEvent_t e = take_event();
    cudaEventRecord(e, stream);
    pending.push_back({id, b, e});
  }
  // Folds the scopes whose end event has completed into the totals without
  // waiting (scopes complete in order on the one stream), so that a long
  // profiled run keeps a bounded pool of events.
  void prof_collect_ready() {
    const cudaError_t before = cudaPeekAtLastError();
    size_t k = 0;
    for (; k < pending.size(); ++k) {
      const Pending& p = pending[k];
      if (cudaEventQuery(p.b) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.a, p.b);
      prof_ms[p.name] += ms;
      prof_count[p.name] += 1;
      ev_pool.push_back(p.a);
      ev_pool.push_back(p.b);
    }
    // a not-ready answer is no error: clear it if the query left it behind,
    // and nothing else
    if (before != cudaErrorNotReady && cudaPeekAtLastError() == cudaErrorNotReady)
      cudaGetLastError();
    pending.erase(pending.begin(), pending.begin() + (std::ptrdiff_t)k);
  }

  void prof_collect() {
    if (pending.empty()) return;
    cudaStreamSynchronize(stream);
    for (auto& p : pending) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.a, p.b);
      prof_ms[p.name] += ms;
      prof_count[p.name] += 1;
      ev_pool.push_back(p.a);
      ev_pool.push_back(p.b);
    }
    pending.clear();
  }

  struct Scope {
    DeviceSim* s;
    int id;
    cudaEvent_t b;
    Scope(DeviceSim* s_, const char* name) : s(s_), id(-1), b(nullptr) {
      id = s->prof_begin(name, &b);
    }
    ~Scope() { s->prof_end(id, b); }
  };

  DevParams params(const Params& prm, const AABB* b, const Obstacle* ob) const;

  int slab_setup(uint32_t first_gid, double lo, double hi, bool has_left, bool has_right);
  int find_neighbors(const DevParams& P, bool predict, bool full, bool move_vel,
                     const float* carry_src = nullptr, uint4* carry_out = nullptr);
  int run_step(const DevParams& P, const Params& prm);

  int ensure_carry_buffers() {
    if (!nr_w) SPHPC_RC(dalloc(&nr_w, cap));
    if (!lam_acc) {
      SPHPC_RC(dalloc(&lam_acc, cap));
      have_carry = false;
    }
    return SPHPC_OK;
  }

  int ensure_warm_buffers() {
    if (!nr_w) SPHPC_RC(dalloc(&nr_w, cap));
    if (mlp.feat_cap < cap) {
      if (mlp.feat) cudaFree(mlp.feat);
      mlp.feat = nullptr;
      mlp.feat_cap = 0;
      SPHPC_RC(dalloc(&mlp.feat, (size_t)cap * kMlpIn));
      mlp.feat_cap = cap;
    }
    return SPHPC_OK;
  }
};

DevParams DeviceSim::params(const Params& prm, const AABB* b, const Obstacle* ob) const {
  DevParams P;
  memset(&P, 0, sizeof(P));
  const double h = prm.smoothing_radius;
  const double m = mass;
  P.n = n;
  P.nx = nx; P.ny = ny; P.nz = nz;
  P.nxny = (uint32_t)nx * (uint32_t)ny;
  P.ncells = C;
  P.bx = bx; P.by = by;
  P.mx = (1u << bx) - 1u;
  P.my = (1u << by) - 1u;
  P.hd = h;
  {
    // fixed-point records: 2^k units per length, as fine as keeps every
    // neighbour difference (< 8h, far more than a step moves a pair) below
    // 2^31 units, so the wrapping difference is the true one
    const int k = 28 - (int)ceil(log2(h));
    P.fx_scale = ldexp(1.0, k);
    P.fx_inv = (float)ldexp(1.0, -k);
    P.fx_inv2 = (float)ldexp(1.0, -2 * k);
    P.h_fx = (float)ldexp(h, k);
    P.rmin2_fx = (float)ldexp(h * 0.0001 * h * 0.0001, 2 * k);
  }
  P.h2d = h * h;
  {
    // coordinates that hash inside the grid lie below max(nx, ny, nz) h
    const int nmax = std::max(nx, std::max(ny, nz));
    if (sphpc_neighbor_pretest_fp32_safe((double)nmax * h, h)) {
      P.bld_h2lo = (float)(h * h) * (1.0f - 1.0f / 1024.0f);
      P.bld_h2hi = (float)(h * h) * (1.0f + 1.0f / 1024.0f);
    } else {
      P.bld_h2lo = -1.0f;
      P.bld_h2hi = INFINITY;
    }
  }
  P.h = (float)h;
  P.h2 = (float)(h * h);
  P.rmin = (float)(h * 0.0001);
  const double W0 = prm.W_norm * (h * h) * (h * h) * (h * h);
  P.W0m = (float)(m * W0);
  P.Wn = (float)prm.W_norm;
  P.Wn_m = (float)(m * prm.W_norm);
  P.DWn = (float)prm.DelW_norm;
  P.DWn_m = (float)(m * prm.DelW_norm);
  P.DWPn = (float)prm.DelW_poly_norm;
  P.m = (float)m;
  P.rho0 = (float)rho0;
  P.rho0_d = rho0;
  P.inv_rho0 = (float)(1.0 / rho0);
  P.inv_rho0_sq = (float)(1.0 / (rho0 * rho0));
  P.lambda_eps = (float)(solver.lambda_epsilon_mass_units
                             ? solver.lambda_epsilon / (rho0 * rho0)
                             : solver.lambda_epsilon);
  P.scorr_k = (float)solver.scorr_k;
  P.scorr_n = solver.scorr_n;
  {
    const double dq = solver.scorr_dq * h;
    const double t = h * h - dq * dq;
    const double Wdq = dq > h ? 0.0 : prm.W_norm * t * t * t;
    P.inv_Wdq = Wdq > 0.0 ? (float)(1.0 / Wdq) : 0.0f;
    P.scorr_u = Wdq > 0.0 ? (float)(1.0 / t) : 0.0f;
    P.scorr_u_fx = P.scorr_u * P.fx_inv2;  // a power of two: exact
    P.scorr_uh2 = P.scorr_u * P.h2;
    if (Wdq <= 0.0) P.scorr_k = 0.0f;
  }
  P.c_xsph = (float)prm.c;
  P.xsph_exact = solver.xsph_exact;
  P.gamma = (float)prm.k;
  P.C_norm = (float)(32.0 / (M_PI * pow(h, 9.0)));
  P.vort_eps = (float)(solver.vorticity_epsilon < 0.0 ? 0.1 * h : solver.vorticity_epsilon);
  P.dt = (float)prm.time_step;
  P.inv_dt = (float)(1.0 / prm.time_step);
  P.v_max = (float)solver.velocity_max;
  P.dt_d = prm.time_step;
  P.gdt_d = (-prm.g) * prm.time_step;
  P.gdt_f = (float)P.gdt_d;
  P.gaxis = solver.gravity_axis;
  if (b) {
    const double lo[3] = {b->min_x, b->min_y, b->min_z};
    const double hi[3] = {b->max_x, b->max_y, b->max_z};
    const double eps = h * 0.0001;
    for (int k = 0; k < 3; ++k) {
      P.bmin[k] = lo[k];
      P.bmax[k] = hi[k];
      P.bmax_eps[k] = hi[k] - eps;
    }
  }
  if (ob && ob->obstacle_cuda && ob->obstacle_cuda->sdf) {
    P.has_sdf = 1;
    P.sdf = ob->obstacle_cuda->sdf;
    P.sdim[0] = ob->SDF_dim_x;
    P.sdim[1] = ob->SDF_dim_y;
    P.sdim[2] = ob->SDF_dim_z;
    const double lo[3] = {ob->world_bounds.min_x, ob->world_bounds.min_y, ob->world_bounds.min_z};
    const double hi[3] = {ob->world_bounds.max_x, ob->world_bounds.max_y, ob->world_bounds.max_z};
    for (int k = 0; k < 3; ++k) {
      P.ob_min[k] = lo[k];
      P.ob_max[k] = hi[k];
      P.ob_len[k] = (float)(hi[k] - lo[k]);
      P.tex_sp[k] = (float)(1.0 / (float)P.sdim[k]);
    }
    const float len_model = (float)(ob->SDF_dim_x * ob->SDF_spacing);
    P.model_to_world = P.ob_len[0] / len_model;
  }
  return P;
}

int DeviceSim::slab_setup(uint32_t first_gid, double lo, double hi, bool has_left,
                          bool has_right) {
  if (!gid) SPHPC_RC(dalloc(&gid, cap));
  if (!owned) SPHPC_RC(dalloc(&owned, cap));
  if (!slab_keep) SPHPC_RC(dalloc(&slab_keep, cap));
  if (!slab_counters) SPHPC_RC(dalloc(&slab_counters, 4));
  launch_slab_init(n, ids, pd, first_gid, lo, hi, has_left, has_right, gid, owned, stream);
  SPHPC_CK(cudaGetLastError());
  slab = true;
  slab_nkeep = 0;
  return SPHPC_OK;
}

int DeviceSim::find_neighbors(const DevParams& P, bool predict, bool full, bool move_vel,
                              const float* carry_src, uint4* carry_out) {
  if (!grid_ready) return set_error(SPHPC_ENOTREADY, "neighbour grid not initialised");
  {
    Scope sc(this, "hash");
    SPHPC_CK(cudaMemsetAsync(sort.hist, 0, sizeof(uint32_t) * kMaxPasses * kRadix, stream));
    launch_hash(P, pd, vel, ids, keys_by_id, loc_by_id, sort.hist, passes, predict, err(),
                stream);
    launches += 1;
  }
  uint32_t *K = nullptr, *R = nullptr;
  {
    Scope sc(this, "radix_sort");
    const cudaError_t e = radix_sort_pairs(keys_by_id, ids_spare, n, passes, sort, stream, true,
                                           true, false, &K, &R);
    if (e != cudaSuccess)
      return set_error(SPHPC_ECUDA, "radix sort: %s", cudaGetErrorString(e));
    launches += 1 + (unsigned)passes;
  }
  keys_sorted = K;
  {
    Scope sc(this, "cell_starts");
    launch_cell_starts(K, n, C, cstart, gaps, gap_count(), err(), stream);
    launches += 2;
  }
  {
    Scope sc(this, "reorder");
    ReorderExtra ex{};
    if (full) {
      SPHPC_RC(ensure_full_alts());
      ex.in4[0] = color; ex.out4[0] = color_alt;
      ex.in4[1] = omega; ex.out4[1] = omega_alt;
      ex.in4[2] = dp; ex.out4[2] = dp_alt;
      ex.in1[0] = rho; ex.out1[0] = rho_alt;
      ex.in1[1] = lam; ex.out1[1] = lam_alt;
    }
    ex.carry_src = carry_src;
    ex.nr_carry = carry_src ? carry_out : nullptr;
    const bool mv = move_vel || full;
    launch_reorder(P, R, loc_by_id, pd, vel, pd_alt, vel_alt, xsa, nr, cellp, predict, mv, &ex,
                   stream);
    launches += 1;
    std::swap(pd, pd_alt);
    if (mv) std::swap(vel, vel_alt);
    if (full) {
      std::swap(color, color_alt);
      std::swap(omega, omega_alt);
      std::swap(dp, dp_alt);
      std::swap(rho, rho_alt);
      std::swap(lam, lam_alt);
    }
    // the carried multipliers follow this reorder only when it gathered them
    if (!carry_src) have_carry = false;
    uint32_t* old = ids;
    ids = R;
    if (R == ids_spare) ids_spare = old;
    else sort.vals_alt = old;
  }
  {
    Scope sc(this, "build_neighbors");
    launch_build_neighbors(P, view(), pd, xsa, cellp, nbr, ncount, stream);
    launches += 1;
  }
  SPHPC_CK(cudaGetLastError());
  nbr_valid = true;
  return SPHPC_OK;
}

static float stiffness_of(double k_stiff, int substep) {
  // particles.c:693-694 (substep 0 gives 1/0 = inf and stiffness 1)
  return (float)(1.0 - pow(1.0 - k_stiff, 1.0 / (double)substep));
}

int DeviceSim::run_step(const DevParams& P, const Params& prm) {
  if (prof) prof_collect_ready();
  const bool collect = collect_iters > 0;
  // A step whose predecessor started mildly compressed (first residual at or
  // below warm_start_min_error) is solved plainly, without the feature pass:
  // consecutive steps' first residuals are close, and such a step converges
  // in a pass or two that the network cannot beat.
  const bool mild = solver.warm_start_min_error > 0.0 && prev_err0 >= 0.0 &&
                    prev_err0 <= solver.warm_start_min_error;
  // warm start from the network (source 0) or from the multipliers the last
  // step applied, carried through this step's sort permutation (source 1)
  const bool carry_mode = !collect && solver.warm_start && solver.warm_start_source == 1;
  if (carry_mode) SPHPC_RC(ensure_carry_buffers());
  const bool warm_net = !collect && solver.warm_start && solver.warm_start_source != 1 &&
                        mlp.ready && !mild;
  const bool warm_carry = carry_mode && have_carry && !mild;
  const bool warm = warm_net || warm_carry;
  SPHPC_RC(find_neighbors(P, true, false, warm_net || collect,
                          warm_carry ? lam_acc : nullptr, warm_carry ? nr_w : nullptr));
  const NbrView V = view();
  PassArgs a{};
  a.rho = rho;
  a.vel = vel;
  a.vel_out = vel;
  a.resid = resid;
  const bool adaptive = solver.adaptive != 0 && !collect;
  const int plain_cap =
      collect ? collect_iters : (adaptive ? solver.max_iterations : solver.solve_iterations);
  const double tol = solver.density_tolerance;
  last_warm = 0.0;
  last_warm_rejected = 0;
  trace.clear();
  // The current positions are the particle records `pd` and the neighbour
  // records `nr` (same x*).  A density/lambda pass (A) reads nr and writes
  // records with lambda in the payload; a position pass (B) reads pd (own)
  // and such records, and writes the new positions into pd_alt (then
  // swapped into pd) and nr.
  auto pass_a = [&](uint4* out, bool with_resid) -> int {
    Scope sc(this, "density_lambda");
    if (with_resid) SPHPC_CK(cudaMemsetAsync(resid, 0, 2 * sizeof(double), stream));
    a.nr = nr;
    a.nr_out = out;
    a.lam = nullptr;
    launch_density_lambda(P, V, a, 0, with_resid, stream);
    launches += 1;
    return SPHPC_OK;
  };
  auto read_resid = [&](double& max_err) -> int {
    double h_res[2];
    SPHPC_CK(cudaMemcpyAsync(h_res, resid, sizeof(h_res), cudaMemcpyDeviceToHost, stream));
    SPHPC_CK(cudaStreamSynchronize(stream));
    last_max_err = max_err = h_res[0];
    last_mean_err = h_res[1] / (n > 0 ? n : 1);
    if (trace.size() < 16) trace.push_back(max_err);
    return SPHPC_OK;
  };
  // carried mode: lam_acc collects the multiplier the network stands for,
  // Lambda = sum over the first kCarrySubsteps substeps of stiffness *
  // lambda_p (a kept warm pass is those substeps); the first such pass of
  // the step (or the first after a discarded warm pass) starts it
  constexpr int kCarrySubsteps = 2;
  bool acc_restart = true;
  auto pass_b = [&](const uint4* in, float stiffness, bool last, bool acc) {
    Scope sc(this, "position");
    a.pd = pd;
    a.pd_out = pd_alt;
    a.nr = in;
    a.nr_out = nr;
    a.stiffness = stiffness;
    a.last = last ? 1 : 0;
    a.lam_acc = (carry_mode && acc) ? lam_acc : nullptr;
    a.acc_add = acc_restart ? 0 : 1;
    if (a.lam_acc) acc_restart = false;
    launch_position(P, V, a, 0, stream);
    a.lam_acc = nullptr;
    launches += 1;
    std::swap(pd, pd_alt);
  };
  int iters = 0, plain = 0;
  bool converged = false, stalled = false;
  bool carry_done = false;  // lam_acc holds the kept warm pass's Lambda
  const uint4* ready = nullptr;  // records with lambda for the next B (its A already run)
  if (collect) {
    // the first A also writes the features of the (predicted) state; the
    // target accumulates s_k * lambda_k over the fixed iterations
    Scope sc(this, "mlp_collect");
    SPHPC_CK(cudaMemsetAsync(collect_target, 0, sizeof(float) * (size_t)collect_rows, stream));
    SPHPC_CK(cudaMemsetAsync(resid, 0, 2 * sizeof(double), stream));
    a.pd = pd;
    a.nr_out = nr_alt;
    launch_features(P, V, a, collect_feat, (int)collect_rows, stream);
    launches += 1;
    ready = nr_alt;
  } else if (warm) {
    double err0 = 0.0, err1 = 0.0;
    if (warm_net) {
      SPHPC_RC(ensure_warm_buffers());
      Scope sc(this, "mlp_features");
      SPHPC_CK(cudaMemsetAsync(resid, 0, 2 * sizeof(double), stream));
      a.pd = pd;
      a.nr_out = nr_alt;
      launch_features_bf16(P, V, a, reinterpret_cast<__nv_bfloat16*>(mlp.feat), mlp.dev.norm,
                           stream);
      launches += 1;
    } else {
      // carried: the plain first density pass (lambda_0 into nr_alt for the
      // gate's fallback) gives the first residual; nr_w already holds the
      // records with the carried multipliers (written by the reorder)
      SPHPC_RC(pass_a(nr_alt, true));
    }
    SPHPC_RC(read_resid(err0));
    if (err0 <= tol && adaptive) {
      converged = true;
    } else if (err0 <= solver.warm_start_min_error) {
      // a mildly compressed step: the plain solve from the feature pass's
      // lambda_0 converges in a pass or two, which the network cannot beat
      ready = nr_alt;
    } else {
      if (warm_net) {
        Scope sc(this, "mlp_forward");
        launch_mlp_forward_bf16(mlp.dev, reinterpret_cast<const __nv_bfloat16*>(mlp.feat), n,
                                nr_alt, nr_w, err(), stream, (float)solver.warm_start_scale);
        launches += 1;
      }
      // the network's multipliers, applied at full stiffness in one pass;
      // pd_alt keeps the predicted positions until the gate has decided
      pass_b(nr_w, 1.0f, false, true);
      ++iters;
      last_warm = 1.0;
      SPHPC_RC(pass_a(nr_w, true));
      SPHPC_RC(read_resid(err1));
      if (adaptive && err1 <= tol) {
        converged = true;
      } else if (solver.warm_start_gate && !(err1 < err0)) {
        // FP64 residual gate: the warm pass did not lower the maximum density
        // error, so it is discarded and the plain solve restarts from the
        // predicted positions (pd_alt and nr_alt still hold them, the latter
        // with lambda_0)
        last_warm_rejected = 1;
        std::swap(pd, pd_alt);
        ready = nr_alt;
        acc_restart = true;
      } else {
        ready = nr_w;
        plain = 1;  // the warm pass takes the place of plain substep 0
        carry_done = true;
      }
    }
  }
  // The cap counts every position pass of the step, a warm pass (kept or
  // discarded) included, so that both arms of a comparison get the same work
  // budget.
  bool fused_velocity = false;
  while (!converged && iters < plain_cap) {
    const uint4* src = ready;
    ready = nullptr;
    if (!src) {
      SPHPC_RC(pass_a(nr_alt, adaptive));
      if (adaptive) {
        double e = 0.0;
        SPHPC_RC(read_resid(e));
        if (e <= tol) {
          converged = true;
          break;
        }
        // stall: the last two iterations together barely lowered the maximum
        // error (the relaxed constraint's fixed point lies above the
        // tolerance); one iteration alone may raise the maximum of a hard step
        const size_t nt = trace.size();
        if (solver.min_progress > 0.0 && nt >= 3 &&
            trace[nt - 1] > (1.0 - solver.min_progress) * trace[nt - 3]) {
          stalled = true;
          break;
        }
      }
      src = nr_alt;
    }
    const float stiff = stiffness_of(solver.stiffness_k, plain);
    if (collect) {
      launch_accum_lambda(src, stiff, collect_target, (int)collect_rows, stream);
      launches += 1;
    }
    const bool last = !adaptive && iters == plain_cap - 1;
    pass_b(src, stiff, last, !carry_done && plain < kCarrySubsteps);
    fused_velocity = last;
    ++plain;
    ++iters;
  }
  if (!fused_velocity) {
    // converged (or capped, or no plain pass): velocities from x* and the
    // freshest density
    Scope sc(this, "velocity");
    const bool pack = converged || stalled || iters == 0;
    launch_update_velocities(P, pd, vel, stream, pack ? rho : nullptr, pack ? nr : nullptr);
    launches += 1;
  }
  last_iterations = iters;
  last_converged = converged ? 1 : 0;
  // a step with no position pass applied no multiplier
  if (carry_mode) {
    if (acc_restart) SPHPC_CK(cudaMemsetAsync(lam_acc, 0, sizeof(float) * n, stream));
    have_carry = true;
  }
  prev_err0 = (adaptive && !trace.empty()) ? trace[0] : -1.0;
  // post-solve passes (simulation.c:93-106) on the records nr (payload: the
  // density); the last one writes x = x*, d = 0 (UpdatePositions) into pd_alt
  a.pd = pd;
  a.pd_out = pd_alt;
  a.nr = nr;
  a.nr_out = nullptr;
  // each pass that gathers the neighbours' velocities (or colours) with their
  // records reads them from combined 32-byte records {nr, v} written by the
  // pass before it
  if (solver.surface_tension) {
    Scope sc(this, "surface_tension");
    a.color = color;
    a.nv_out = nv_a;
    launch_color(P, V, a, stream);
    a.vel = vel;
    a.nv = nv_a;
    a.nv_out = nv_b;
    launch_tension(P, V, a, stream);
    launches += 2;
  }
  {
    Scope sc(this, "xsph");
    if (!solver.surface_tension) {
      launch_pack_nv(n, nr, vel, nv_b, stream);
      launches += 1;
    }
    a.nv = nv_b;
    a.nv_out = solver.vorticity ? nv_a : nullptr;
    a.vel_out = vel_alt;
    a.write_pos = solver.vorticity ? 0 : 1;
    launch_xsph(P, V, a, stream);
    launches += 1;
  }
  if (solver.vorticity) {
    Scope sc(this, "vorticity");
    // the vorticity pass also writes the records {X, |omega|} (into nr_alt)
    // that the confinement pass gathers
    a.nv = nv_a;
    a.nv_out = nullptr;
    a.vel = vel_alt;
    a.omega = omega;
    a.nr_out = nr_alt;
    a.write_pos = 0;
    launch_vorticity(P, V, a, stream);
    a.nr = nr_alt;
    a.nr_out = nullptr;
    a.write_pos = 1;
    launch_confinement(P, V, a, true, stream);
    launches += 2;
  }
  std::swap(vel, vel_alt);
  std::swap(pd, pd_alt);
  SPHPC_CK(cudaGetLastError());
  (void)prm;
  return SPHPC_OK;
}

// ---- registry of device copies (the "present" table) ----
static std::mutex g_mu;
static std::unordered_map<const Particles*, DeviceSim*> g_sims;

static DeviceSim* find_sim(const Particles* p) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_sims.find(p);
  return it == g_sims.end() ? nullptr : it->second;
}

#define SPHPC_SIM(var, particles)                                                        \
  DeviceSim* var = find_sim(particles);                                                  \
  if (!var)                                                                              \
    return set_error(SPHPC_ENOTREADY, "%s: particles have no device copy (call "         \
                                      "AllocInitParticles or sphpc_enter_data)",         \
                     __func__);

// ---- host <-> device transfers ----

// Gathers the requested fields (mask bit k: field k of struct Particles'
// FP64 arrays) into stage[k][id], id = original particle index.
__global__ void k_download(int n, const uint32_t* __restrict__ ids, const PD* __restrict__ pd,
                           const float4* __restrict__ vel,
                           const float4* __restrict__ dp, const float4* __restrict__ omega,
                           const float4* __restrict__ color, const float* __restrict__ rho,
                           const float* __restrict__ lam, unsigned mask,
                           double* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const size_t N = (size_t)n;
  const uint32_t id = ids[p];
  if (mask & 0x3Fu) {
    const float4 x = pd[p].x;
    const float4 d = pd[p].d;
    if (mask & 1u) out[0 * N + id] = xstar_d(x.x, d.x);
    if (mask & 2u) out[1 * N + id] = xstar_d(x.y, d.y);
    if (mask & 4u) out[2 * N + id] = xstar_d(x.z, d.z);
    if (mask & 8u) out[3 * N + id] = x.x;
    if (mask & 16u) out[4 * N + id] = x.y;
    if (mask & 32u) out[5 * N + id] = x.z;
  }
  if (mask & (7u << 6)) {
    const float4 v = vel[p];
    if (mask & (1u << 6)) out[6 * N + id] = v.x;
    if (mask & (1u << 7)) out[7 * N + id] = v.y;
    if (mask & (1u << 8)) out[8 * N + id] = v.z;
  }
  if (mask & (7u << 9)) {
    const float4 q = dp[p];
    if (mask & (1u << 9)) out[9 * N + id] = q.x;
    if (mask & (1u << 10)) out[10 * N + id] = q.y;
    if (mask & (1u << 11)) out[11 * N + id] = q.z;
  }
  if (mask & (7u << 12)) {
    const float4 w = omega[p];
    if (mask & (1u << 12)) out[12 * N + id] = w.x;
    if (mask & (1u << 13)) out[13 * N + id] = w.y;
    if (mask & (1u << 14)) out[14 * N + id] = w.z;
  }
  if (mask & (7u << 15)) {
    const float4 c = color[p];
    if (mask & (1u << 15)) out[15 * N + id] = c.x;
    if (mask & (1u << 16)) out[16 * N + id] = c.y;
    if (mask & (1u << 17)) out[17 * N + id] = c.z;
  }
  if (mask & (1u << 18)) out[18 * N + id] = rho[p];
  if (mask & (1u << 19)) out[19 * N + id] = lam[p];
}

__global__ void k_upload(int n, const uint32_t* __restrict__ ids, const double* __restrict__ in,
                         unsigned mask, PD* pd, float4* vel, float4* dp,
                         float4* omega, float4* color, float* rho, float* lam) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const size_t N = (size_t)n;
  const uint32_t id = ids[p];
  auto f = [&](int k) { return in[(size_t)k * N + id]; };
  if (mask & (1u << 3)) {
    const float x = (float)f(3), y = (float)f(4), z = (float)f(5);
    pd[p].x = make_float4(x, y, z, 0.f);
    float4 d = make_float4(0.f, 0.f, 0.f, pd[p].d.w);
    if (mask & (1u << 0)) {
      d.x = (float)(f(0) - (double)x);
      d.y = (float)(f(1) - (double)y);
      d.z = (float)(f(2) - (double)z);
    }
    pd[p].d = d;
  }
  if (mask & (1u << 6)) vel[p] = make_float4((float)f(6), (float)f(7), (float)f(8), 0.f);
  if (mask & (1u << 9)) dp[p] = make_float4((float)f(9), (float)f(10), (float)f(11), 0.f);
  if (mask & (1u << 12)) omega[p] = make_float4((float)f(12), (float)f(13), (float)f(14), 0.f);
  if (mask & (1u << 15)) color[p] = make_float4((float)f(15), (float)f(16), (float)f(17), 0.f);
  if (mask & (1u << 18)) rho[p] = (float)f(18);
  if (mask & (1u << 19)) lam[p] = (float)f(19);
}

__global__ void k_iota(uint32_t* a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = (uint32_t)i;
}

// FP64 diagnostics: [0] max err (u64 bits), [1] sum err, [2] sum |v|^2,
// [3..5] sum x, [6..8] sum v
__global__ void __launch_bounds__(kBlock)
    k_diag(int n, float rho0, const PD* __restrict__ pd, const float4* __restrict__ vel,
           const float* __restrict__ rho, double* __restrict__ out) {
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double e = fmax((double)rho[p] / (double)rho0 - 1.0, 0.0);
    v[0] = fmax(v[0], e);
    v[1] += e;
    const float4 u = vel[p], x = pd[p].x;
    v[2] += (double)u.x * u.x + (double)u.y * u.y + (double)u.z * u.z;
    v[3] += x.x; v[4] += x.y; v[5] += x.z;
    v[6] += u.x; v[7] += u.y; v[8] += u.z;
  }
  for (int o = 16; o > 0; o >>= 1) {
    v[0] = fmax(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
    for (int k = 1; k < 9; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(reinterpret_cast<unsigned long long*>(out),
              (unsigned long long)__double_as_longlong(v[0]));
    for (int k = 1; k < 9; ++k) atomicAdd(out + k, v[k]);
  }
}

static int enter_data(Particles* particles, const Params* params, DeviceSim** out) {
  if (!particles || !params) return set_error(SPHPC_EINVAL, "sphpc_enter_data: null argument");
  if (particles->local_count <= 0 || !particles->x || !particles->y || !particles->z)
    return set_error(SPHPC_EINVAL, "sphpc_enter_data: no particles");
  if (find_sim(particles))
    return set_error(SPHPC_EINVAL, "sphpc_enter_data: particles already have a device copy");
  int ndev = 0;
  const cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(SPHPC_ECUDA, "no CUDA device: %s", cudaGetErrorString(e));
  }
  DeviceSim* s = new DeviceSim();
  cudaGetDevice(&s->device);
  s->solver = current_solver();
  s->rho0 = particles->rest_density;
  s->mass = particles->rest_mass;
  int rc = s->alloc(particles->local_count, particles->max_local);
  if (!rc) {
    // Page-lock the large host arrays in place: the reference's calloc'd
    // arrays stay the caller's, only their transfers get faster.  Arrays
    // below 64 MB may share pages with other allocations and are left
    // pageable, as is any array the driver refuses to register.
    const size_t bytes = sizeof(double) * (size_t)particles->max_local;
    if (bytes >= ((size_t)64 << 20)) {
      double* fields[20] = {particles->x_star, particles->y_star, particles->z_star, particles->x,
                            particles->y, particles->z, particles->v_x, particles->v_y,
                            particles->v_z, particles->dp_x, particles->dp_y, particles->dp_z,
                            particles->w_x, particles->w_y, particles->w_z, particles->color_x,
                            particles->color_y, particles->color_z, particles->density,
                            particles->lambda};
      for (double* f : fields) {
        if (!f) continue;
        if (cudaHostRegister(f, bytes, cudaHostRegisterDefault) == cudaSuccess)
          s->pinned.push_back(f);
        else
          cudaGetLastError();
      }
    }
    k_iota<<<grid_for(s->n), kBlock, 0, s->stream>>>(s->ids, s->n);
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_sims[particles] = s;
    }
    rc = sphpc_update_device(particles);
    if (rc) {
      std::lock_guard<std::mutex> lk(g_mu);
      g_sims.erase(particles);
    }
  }
  if (rc) {
    delete s;
    return rc;
  }
  if (out) *out = s;
  return SPHPC_OK;
}

// Device scratch of the SortByKey seam, one cache per device.
struct SeamScratch {
  SortScratch s{};
  uint32_t* aux = nullptr;
  int cap = 0;
};
static std::mutex g_seam_mu;
static std::map<int, SeamScratch> g_seam;

// ---- snapshot gather (WriteParticles) ----

__global__ void k_interleave_xyz(int n, const uint32_t* __restrict__ ids,
                                 const PD* __restrict__ pd, double* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float4 x = pd[p].x;
  double* o = out + 3 * (size_t)__ldg(ids + p);
  o[0] = x.x;
  o[1] = x.y;
  o[2] = x.z;
}

int sim_interleave_positions(const struct Particles* particles, double* d_out, int* n,
                             void** stream) {
  SPHPC_SIM(s, particles);
  k_interleave_xyz<<<grid_for(s->n), kBlock, 0, s->stream>>>(s->n, s->ids, s->pd, d_out);
  SPHPC_CK(cudaGetLastError());
  *n = s->n;
  *stream = (void*)s->stream;
  return SPHPC_OK;
}

}  // namespace sphpc

using namespace sphpc;

extern "C" {

int sphpc_enter_data(struct Particles* particles, const struct Params* params) {
  clear_error();
  return enter_data(particles, params, nullptr);
}

int sphpc_exit_data(struct Particles* particles) {
  DeviceSim* s = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_sims.find(particles);
    if (it == g_sims.end()) return set_error(SPHPC_ENOTREADY, "sphpc_exit_data: no device copy");
    s = it->second;
    g_sims.erase(it);
  }
  cudaStreamSynchronize(s->stream);
  delete s;
  return SPHPC_OK;
}

int sphpc_set_solver(struct Particles* particles, const struct SphpcSolver* solver) {
  SPHPC_SIM(s, particles);
  if (!solver) return set_error(SPHPC_EINVAL, "sphpc_set_solver: null");
  s->solver = *solver;
  return SPHPC_OK;
}

int sphpc_get_solver(const struct Particles* particles, struct SphpcSolver* solver) {
  SPHPC_SIM(s, particles);
  if (!solver) return set_error(SPHPC_EINVAL, "sphpc_get_solver: null");
  *solver = s->solver;
  return SPHPC_OK;
}

int sphpc_set_stream(struct Particles* particles, void* cuda_stream) {
  SPHPC_SIM(s, particles);
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  s->stream = (cudaStream_t)cuda_stream;
  return SPHPC_OK;
}

int sphpc_update_host(struct Particles* p) { return sphpc_update_host_fields(p, 0xFFFFFFFFu); }

namespace {

// Gathers the fields of field_mask into the staging buffer (original particle
// order, doubles) and copies them to the host arrays: on the particle set's
// stream, or, with async, on its copy stream after the gather.
int download_fields(Particles* p, DeviceSim* s, unsigned int field_mask, bool async) {
  SPHPC_RC(s->wait_copies());
  SPHPC_RC(s->ensure_stage());
  if (async) SPHPC_RC(s->ensure_copy_stream());
  const int n = s->n;
  double* fields[20] = {p->x_star, p->y_star, p->z_star, p->x, p->y, p->z, p->v_x, p->v_y,
                        p->v_z, p->dp_x, p->dp_y, p->dp_z, p->w_x, p->w_y, p->w_z,
                        p->color_x, p->color_y, p->color_z, p->density, p->lambda};
  unsigned mask = 0;
  for (int k = 0; k < 20; ++k)
    if (fields[k] && (field_mask & (1u << k))) mask |= 1u << k;
  k_download<<<grid_for(n), kBlock, 0, s->stream>>>(n, s->ids, s->pd, s->vel, s->dp,
                                                    s->omega, s->color, s->rho, s->lam, mask,
                                                    s->stage);
  SPHPC_CK(cudaGetLastError());
  cudaStream_t cs = s->stream;
  if (async) {
    SPHPC_CK(cudaEventRecord(s->gathered, s->stream));
    SPHPC_CK(cudaStreamWaitEvent(s->copy_stream, s->gathered, 0));
    cs = s->copy_stream;
  }
  for (int k = 0; k < 20; ++k)
    if (mask & (1u << k))
      SPHPC_CK(cudaMemcpyAsync(fields[k], s->stage + (size_t)k * n, sizeof(double) * n,
                               cudaMemcpyDeviceToHost, cs));
  if (async) {
    SPHPC_CK(cudaEventRecord(s->copied, s->copy_stream));
    s->copy_pending = true;
  } else {
    SPHPC_CK(cudaStreamSynchronize(s->stream));
  }
  // the host arrays are in original order: ids are the identity (written on
  // full updates; a field subset leaves them as they are)
  if (p->id && field_mask == 0xFFFFFFFFu)
    for (int i = 0; i < n; ++i) p->id[i] = i;
  return SPHPC_OK;
}

}  // namespace

int sphpc_update_host_fields(struct Particles* p, unsigned int field_mask) {
  SPHPC_SIM(s, p);
  return download_fields(p, s, field_mask, false);
}

int sphpc_update_host_fields_async(struct Particles* p, unsigned int field_mask) {
  SPHPC_SIM(s, p);
  return download_fields(p, s, field_mask, true);
}

int sphpc_host_wait(struct Particles* p) {
  SPHPC_SIM(s, p);
  return s->wait_copies();
}

int sphpc_update_device(struct Particles* p) { return sphpc_update_device_fields(p, 0xFFFFFFFFu); }

int sphpc_update_device_fields(struct Particles* p, unsigned int field_mask) {
  SPHPC_SIM(s, p);
  SPHPC_RC(s->wait_copies());
  SPHPC_RC(s->ensure_stage());
  const int n = s->n;
  const double* fields[20] = {p->x_star, p->y_star, p->z_star, p->x, p->y, p->z, p->v_x,
                              p->v_y, p->v_z, p->dp_x, p->dp_y, p->dp_z, p->w_x, p->w_y,
                              p->w_z, p->color_x, p->color_y, p->color_z, p->density,
                              p->lambda};
  unsigned mask = 0;
  const int groups[8][2] = {{0, 3}, {3, 3}, {6, 3}, {9, 3}, {12, 3}, {15, 3}, {18, 1}, {19, 1}};
  for (auto& g : groups) {
    bool all = true;
    for (int k = g[0]; k < g[0] + g[1]; ++k)
      all = all && fields[k] != nullptr && (field_mask & (1u << k));
    if (!all) continue;
    mask |= 1u << g[0];
    for (int k = g[0]; k < g[0] + g[1]; ++k)
      SPHPC_CK(cudaMemcpyAsync(s->stage + (size_t)k * n, fields[k], sizeof(double) * n,
                               cudaMemcpyHostToDevice, s->stream));
  }
  if (!(mask & (1u << 3)))
    return set_error(SPHPC_EINVAL, "sphpc_update_device: x, y, z are required");
  k_upload<<<grid_for(n), kBlock, 0, s->stream>>>(n, s->ids, s->stage, mask, s->pd, s->vel,
                                                  s->dp, s->omega, s->color, s->rho, s->lam);
  SPHPC_CK(cudaGetLastError());
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  return SPHPC_OK;
}

int AllocInitParticles(struct Particles* particles, struct Params* params,
                       struct AABB* fluid_volume_initial) {
  clear_error();
  if (!particles || !params || !fluid_volume_initial)
    return set_error(SPHPC_EINVAL, "AllocInitParticles: null argument");
  if (particles->max_local <= 0)
    SPHPC_RC(SetParticleNumbers(fluid_volume_initial, particles, params, nullptr));
  const size_t n = (size_t)particles->max_local;
  double* SPHPC_RESTRICT* dfields[20] = {&particles->x_star, &particles->y_star, &particles->z_star,
                          &particles->x, &particles->y, &particles->z, &particles->v_x,
                          &particles->v_y, &particles->v_z, &particles->dp_x, &particles->dp_y,
                          &particles->dp_z, &particles->w_x, &particles->w_y, &particles->w_z,
                          &particles->color_x, &particles->color_y, &particles->color_z,
                          &particles->density, &particles->lambda};
  for (auto f : dfields) {
    *f = (double*)calloc(n, sizeof(double));
    if (!*f) return set_error(SPHPC_ENOMEM, "AllocInitParticles: calloc of %zu doubles", n);
  }
  particles->id = (int*)calloc(n, sizeof(int));
  if (!particles->id) return set_error(SPHPC_ENOMEM, "AllocInitParticles: calloc ids");
  SPHPC_RC(ConstructFluidVolume(particles, params, fluid_volume_initial));
  const SphpcSolver sv = current_solver();
  const double spacing = 2.0 * particles->rest_radius;
  if (sv.rest_density_lattice) {
    particles->rest_mass = params->fluid_volume * 1000.0 / (double)particles->global_count;
    particles->rest_density =
        particles->rest_mass *
        lattice_poly6_sum(params->smoothing_radius, params->W_norm, spacing);
  } else {
    // particles.c:1034-1037
    particles->rest_density = 1000.0;
    particles->rest_mass =
        params->fluid_volume * particles->rest_density / (double)particles->global_count;
    particles->rest_mass *= .991;
  }
  for (int i = 0; i < particles->local_count; ++i) {
    particles->v_x[i] = 0.0;
    particles->v_y[i] = 0.0;
    particles->v_z[i] = 0.0;
    particles->x_star[i] = particles->x[i];
    particles->y_star[i] = particles->y[i];
    particles->z_star[i] = particles->z[i];
    particles->density[i] = particles->rest_density;
  }
  particles->halo_count_left = 0;
  particles->halo_count_right = 0;
  return enter_data(particles, params, nullptr);
}

int FinalizeParticles(struct Particles* particles) {
  if (!particles) return set_error(SPHPC_EINVAL, "FinalizeParticles: null");
  if (find_sim(particles)) sphpc_exit_data(particles);
  double* SPHPC_RESTRICT* dfields[20] = {&particles->x_star, &particles->y_star, &particles->z_star,
                          &particles->x, &particles->y, &particles->z, &particles->v_x,
                          &particles->v_y, &particles->v_z, &particles->dp_x, &particles->dp_y,
                          &particles->dp_z, &particles->w_x, &particles->w_y, &particles->w_z,
                          &particles->color_x, &particles->color_y, &particles->color_z,
                          &particles->density, &particles->lambda};
  for (auto f : dfields) {
    free(*f);
    *f = nullptr;
  }
  free(particles->id);
  particles->id = nullptr;
  return SPHPC_OK;
}

// ---- neighbours ----

int AllocInitNeighbors(struct Neighbors* neighbors, const struct Particles* particles,
                       const struct Params* params, const struct AABB* boundary_global) {
  if (!neighbors || !params || !boundary_global)
    return set_error(SPHPC_EINVAL, "AllocInitNeighbors: null argument");
  memset(neighbors, 0, sizeof(*neighbors));
  const double h = params->smoothing_radius;
  neighbors->hash_size_x = (int)(ceil((boundary_global->max_x - boundary_global->min_x) / h) + 1);
  neighbors->hash_size_y = (int)(ceil((boundary_global->max_y - boundary_global->min_y) / h) + 1);
  neighbors->hash_size_z = (int)(ceil((boundary_global->max_z - boundary_global->min_z) / h) + 1);
  neighbors->hash_spacing = h;
  SPHPC_SIM(s, particles);
  return s->init_grid(*boundary_global, h);
}

int FinalizeNeighbors(struct Neighbors* neighbors) {
  if (neighbors) memset(neighbors, 0, sizeof(*neighbors));
  return SPHPC_OK;
}

int FindAllNeighbors(const struct Particles* particles, const struct Params* params,
                     struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_SIM(s, particles);
  if (!params) return set_error(SPHPC_EINVAL, "FindAllNeighbors: null params");
  const DevParams P = s->params(*params, nullptr, nullptr);
  return s->find_neighbors(P, false, true, true);
}

int sphpc_get_neighbor_buckets(const struct Particles* particles, unsigned int* indices,
                               int* counts) {
  SPHPC_SIM(s, particles);
  if (!s->nbr_valid) return set_error(SPHPC_ENOTREADY, "no neighbour lists built yet");
  uint32_t* d_nbr = nullptr;
  int32_t* d_cnt = nullptr;
  SPHPC_RC(dalloc(&d_nbr, (size_t)s->n * kMaxNeighbors));
  int rc = dalloc(&d_cnt, (size_t)s->n);
  if (rc) {
    dfree(d_nbr);
    return rc;
  }
  launch_export_buckets(s->view(), s->ids, d_nbr, d_cnt, s->err(), s->stream);
  cudaError_t e = cudaMemcpyAsync(indices, d_nbr, sizeof(uint32_t) * s->n * kMaxNeighbors,
                                  cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(counts, d_cnt, sizeof(int32_t) * s->n, cudaMemcpyDeviceToHost,
                        s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  dfree(d_nbr);
  dfree(d_cnt);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "bucket export: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

int sphpc_get_cell_data(const struct Particles* particles, unsigned int* hash_values,
                        unsigned int* particle_ids, unsigned int* start_indices) {
  SPHPC_SIM(s, particles);
  if (!s->nbr_valid || !s->keys_sorted) return set_error(SPHPC_ENOTREADY, "no cell data yet");
  if (hash_values)
    SPHPC_CK(cudaMemcpyAsync(hash_values, s->keys_sorted, sizeof(uint32_t) * s->n,
                             cudaMemcpyDeviceToHost, s->stream));
  if (particle_ids)
    SPHPC_CK(cudaMemcpyAsync(particle_ids, s->ids, sizeof(uint32_t) * s->n,
                             cudaMemcpyDeviceToHost, s->stream));
  if (start_indices)
    SPHPC_CK(cudaMemcpyAsync(start_indices, s->cstart, sizeof(uint32_t) * ((size_t)s->C + 1),
                             cudaMemcpyDeviceToHost, s->stream));
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  return SPHPC_OK;
}

// ---- step functions (one stage each) ----

#define SPHPC_STAGE_BEGIN(particles, params) \
  SPHPC_SIM(s, particles);                   \
  if (!(params)) return set_error(SPHPC_EINVAL, "%s: null params", __func__);

#define SPHPC_NEED_NBR()                                                                  \
  if (!s->nbr_valid)                                                                      \
    return set_error(SPHPC_ENOTREADY, "%s: call FindAllNeighbors first", __func__);

#define SPHPC_LAUNCH_DONE() SPHPC_CK(cudaGetLastError()); return SPHPC_OK;

int ApplyGravity(struct Particles* particles, const struct Params* params) {
  SPHPC_STAGE_BEGIN(particles, params);
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_gravity(P, s->vel, s->stream);
  SPHPC_LAUNCH_DONE();
}

int PredictPositions(struct Particles* particles, const struct Params* params,
                     const struct AABB* boundary_global) {
  SPHPC_STAGE_BEGIN(particles, params);
  if (!boundary_global) return set_error(SPHPC_EINVAL, "PredictPositions: null boundary");
  const DevParams P = s->params(*params, boundary_global, nullptr);
  launch_predict(P, s->pd, s->vel, s->stream);
  SPHPC_LAUNCH_DONE();
}

int ComputeDensities(struct Particles* particles, const struct Params* params,
                     const struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_make_nr(P, s->pd, nullptr, s->nr, s->stream);
  PassArgs a{};
  a.nr = s->nr;
  a.rho = s->rho;
  a.resid = s->resid;
  SPHPC_CK(cudaMemsetAsync(s->resid, 0, 2 * sizeof(double), s->stream));
  launch_density_lambda(P, s->view(), a, 1, true, s->stream);
  SPHPC_LAUNCH_DONE();
}

int ComputeLambda(struct Particles* particles, const struct Params* params,
                  const struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_make_nr(P, s->pd, nullptr, s->nr, s->stream);
  PassArgs a{};
  a.nr = s->nr;
  a.rho = s->rho;
  a.lam = s->lam;
  launch_density_lambda(P, s->view(), a, 2, false, s->stream);
  launch_pack_w(P, s->pd, nullptr, s->lam, s->stream);
  SPHPC_LAUNCH_DONE();
}

int UpdateDPs(struct Particles* particles, const struct Params* params,
              const struct Neighbors* neighbors, const int substep) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_pack_w(P, s->pd, nullptr, s->lam, s->stream);
  launch_make_nr(P, s->pd, s->lam, s->nr, s->stream);
  PassArgs a{};
  a.pd = s->pd;
  a.nr = s->nr;
  a.dp = s->dp;
  a.rho = s->rho;
  a.stiffness = stiffness_of(s->solver.stiffness_k, substep);
  launch_position(P, s->view(), a, 1, s->stream);
  SPHPC_LAUNCH_DONE();
}

int UpdatePositionStars(struct Particles* particles, const struct AABB* boundary_global,
                        const struct Obstacle* obstacle, const struct Params* params) {
  SPHPC_STAGE_BEGIN(particles, params);
  if (!boundary_global) return set_error(SPHPC_EINVAL, "UpdatePositionStars: null boundary");
  const DevParams P = s->params(*params, boundary_global, obstacle);
  PassArgs a{};
  a.pd_out = s->pd;
  a.dp = s->dp;
  launch_apply_dp(P, a, s->stream);
  SPHPC_LAUNCH_DONE();
}

int UpdateVelocities(struct Particles* particles, const struct Params* params) {
  SPHPC_STAGE_BEGIN(particles, params);
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_update_velocities(P, s->pd, s->vel, s->stream);
  SPHPC_LAUNCH_DONE();
}

int ComputeSurfaceTension(struct Particles* particles, const struct Params* params,
                          const struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_pack_w(P, s->pd, nullptr, s->rho, s->stream);
  launch_make_nr(P, s->pd, s->rho, s->nr, s->stream);
  PassArgs a{};
  a.pd = s->pd;
  a.nr = s->nr;
  a.color = s->color;
  a.vel = s->vel;
  a.nv_out = s->nv_a;
  launch_color(P, s->view(), a, s->stream);
  a.nv = s->nv_a;
  a.nv_out = nullptr;
  launch_tension(P, s->view(), a, s->stream);
  SPHPC_LAUNCH_DONE();
}

int ApplyViscosity(struct Particles* particles, const struct Params* params,
                   const struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_pack_w(P, s->pd, nullptr, s->rho, s->stream);
  launch_make_nr(P, s->pd, s->rho, s->nr, s->stream);
  launch_pack_nv(s->n, s->nr, s->vel, s->nv_a, s->stream);
  PassArgs a{};
  a.pd = s->pd;
  a.nr = s->nr;
  a.nv = s->nv_a;
  a.vel = s->vel;
  a.vel_out = s->vel_alt;
  launch_xsph(P, s->view(), a, s->stream);
  std::swap(s->vel, s->vel_alt);
  SPHPC_LAUNCH_DONE();
}

int ComputeVorticity(struct Particles* particles, const struct Params* params,
                     const struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_make_nr(P, s->pd, nullptr, s->nr, s->stream);
  launch_pack_nv(s->n, s->nr, s->vel, s->nv_a, s->stream);
  PassArgs a{};
  a.pd = s->pd;
  a.nr = s->nr;
  a.nv = s->nv_a;
  a.vel = s->vel;
  a.omega = s->omega;
  launch_vorticity(P, s->view(), a, s->stream);
  SPHPC_LAUNCH_DONE();
}

int ApplyVorticityConfinement(struct Particles* particles, const struct Params* params,
                              const struct Neighbors* neighbors) {
  (void)neighbors;
  SPHPC_STAGE_BEGIN(particles, params);
  SPHPC_NEED_NBR();
  const DevParams P = s->params(*params, nullptr, nullptr);
  launch_make_nr(P, s->pd, nullptr, s->nr, s->stream);
  PassArgs a{};
  a.pd = s->pd;
  a.nr = s->nr;
  a.vel = s->vel;
  a.omega = s->omega;
  launch_confinement(P, s->view(), a, false, s->stream);
  SPHPC_LAUNCH_DONE();
}

int UpdatePositions(struct Particles* particles) {
  SPHPC_SIM(s, particles);
  DevParams P{};
  P.n = s->n;
  launch_update_positions(P, s->pd, s->stream);
  SPHPC_LAUNCH_DONE();
}

// ---- whole step ----

int sphpc_step(struct Particles* particles, const struct Params* params,
               struct Neighbors* neighbors, const struct AABB* boundary_global,
               const struct Obstacle* obstacle, int steps) {
  (void)neighbors;
  SPHPC_SIM(s, particles);
  if (!params || !boundary_global) return set_error(SPHPC_EINVAL, "sphpc_step: null argument");
  if (steps < 0) return set_error(SPHPC_EINVAL, "sphpc_step: negative step count");
  if (!s->grid_ready) SPHPC_RC(s->init_grid(*boundary_global, params->smoothing_radius));
  if (s->slab && (s->solver.adaptive || s->solver.warm_start))
    return set_error(SPHPC_EINVAL, "sphpc_step: a slab of a decomposed domain steps with the "
                                   "fixed iteration count (adaptive and warm_start off): its "
                                   "residual would include the halo");
  const DevParams P = s->params(*params, boundary_global, obstacle);
  for (int k = 0; k < steps; ++k) SPHPC_RC(s->run_step(P, *params));
  return SPHPC_OK;
}

// ---- slab decomposition along x ----

int sphpc_slab_init(struct Particles* particles, unsigned int first_gid, double node_start_x,
                    double node_end_x, int has_left, int has_right) {
  SPHPC_SIM(s, particles);
  if (!(node_end_x > node_start_x))
    return set_error(SPHPC_EINVAL, "sphpc_slab_init: empty slab [%g, %g)", node_start_x, node_end_x);
  return s->slab_setup(first_gid, node_start_x, node_end_x, has_left != 0, has_right != 0);
}

int sphpc_slab_halo_width(const struct Params* params, const struct SphpcSolver* solver,
                          double* width) {
  if (!params || !solver || !width) return set_error(SPHPC_EINVAL, "sphpc_slab_halo_width: null");
  const int hops = 2 * solver->solve_iterations + (solver->surface_tension ? 2 : 0) + 1 +
                   (solver->vorticity ? 2 : 0);
  // one h per hop, one more for the list built at the predicted positions,
  // and the motion of the influencing and the influenced particle in a step
  // (velocities are clamped to velocity_max)
  *width = (hops + 1) * params->smoothing_radius +
           2.0 * solver->velocity_max * params->time_step;
  return SPHPC_OK;
}

int sphpc_slab_pack(struct Particles* particles, double node_start_x, double node_end_x,
                    double halo_width, int has_left, int has_right, void* send_left,
                    void* send_right, int send_capacity, int* count_left, int* count_right) {
  SPHPC_SIM(s, particles);
  if (!s->slab) return set_error(SPHPC_ENOTREADY, "sphpc_slab_pack: call sphpc_slab_init first");
  if (send_capacity < 0 || (send_capacity > 0 && (!send_left || !send_right)) || !count_left ||
      !count_right || !(node_end_x > node_start_x) || !(halo_width > 0.0))
    return set_error(SPHPC_EINVAL, "sphpc_slab_pack: bad arguments");
  SPHPC_CK(cudaMemsetAsync(s->slab_counters, 0, 4 * sizeof(uint32_t), s->stream));
  launch_slab_pack(s->n, s->ids, s->gid, s->owned, s->pd, s->vel, node_start_x, node_end_x,
                   halo_width, has_left != 0, has_right != 0, s->slab_keep,
                   static_cast<SlabRecord*>(send_left), static_cast<SlabRecord*>(send_right),
                   s->slab_counters, (uint32_t)s->cap, (uint32_t)send_capacity, s->stream);
  SPHPC_CK(cudaGetLastError());
  uint32_t h[3];
  SPHPC_CK(cudaMemcpyAsync(h, s->slab_counters, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  *count_left = (int)h[1];
  *count_right = (int)h[2];
  if (h[0] > (uint32_t)s->cap)
    return set_error(SPHPC_ENOMEM, "sphpc_slab_pack: %u kept particles exceed max_local %d", h[0],
                     s->cap);
  if (h[1] > (uint32_t)send_capacity || h[2] > (uint32_t)send_capacity)
    return set_error(SPHPC_ENOMEM, "sphpc_slab_pack: %u / %u records exceed the send capacity %d",
                     h[1], h[2], send_capacity);
  s->slab_nkeep = h[0];
  return SPHPC_OK;
}

int sphpc_slab_unpack(struct Particles* particles, const void* recv_left, int count_left,
                      const void* recv_right, int count_right) {
  SPHPC_SIM(s, particles);
  if (!s->slab) return set_error(SPHPC_ENOTREADY, "sphpc_slab_unpack: call sphpc_slab_init first");
  if (count_left < 0 || count_right < 0 || (count_left > 0 && !recv_left) ||
      (count_right > 0 && !recv_right))
    return set_error(SPHPC_EINVAL, "sphpc_slab_unpack: bad arguments");
  const long long m = (long long)s->slab_nkeep + count_left + count_right;
  if (m > s->cap)
    return set_error(SPHPC_ENOMEM, "sphpc_slab_unpack: %lld particles exceed max_local %d", m,
                     s->cap);
  if (m == 0) return set_error(SPHPC_EINVAL, "sphpc_slab_unpack: no particles left");
  SlabParts parts{s->slab_keep, static_cast<const SlabRecord*>(recv_left),
                  static_cast<const SlabRecord*>(recv_right), s->slab_nkeep,
                  (uint32_t)count_left, (uint32_t)count_right};
  // the new working set in gid order: sort (gid, record index)
  launch_slab_keys(parts, s->keys_by_id, s->stream);
  const cudaError_t e = radix_sort_pairs(s->keys_by_id, s->loc_by_id, (int)m, kMaxPasses, s->sort,
                                         s->stream, false, true, true, nullptr, nullptr);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "sphpc_slab_unpack: %s", cudaGetErrorString(e));
  launch_slab_load(parts, s->loc_by_id, s->pd, s->vel, s->gid, s->owned, s->ids, s->stream);
  SPHPC_CK(cudaGetLastError());
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  s->n = (int)m;
  particles->local_count = (int)m;
  s->slab_nkeep = 0;
  s->nbr_valid = false;
  s->have_carry = false;
  s->prev_err0 = -1.0;
  s->keys_sorted = nullptr;
  uint32_t herr = 0;
  SPHPC_CK(cudaMemcpy(&herr, s->sort.err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (herr) return set_error(SPHPC_EKERNEL, "sphpc_slab_unpack: sort error bits 0x%x", herr);
  return SPHPC_OK;
}

int sphpc_slab_owned(const struct Particles* particles, unsigned int* gids, double* xyz,
                     double* vel, int capacity, int* count) {
  SPHPC_SIM(s, particles);
  if (!s->slab) return set_error(SPHPC_ENOTREADY, "sphpc_slab_owned: call sphpc_slab_init first");
  if (!count || capacity < 0 || (capacity > 0 && (!gids || !xyz || !vel)))
    return set_error(SPHPC_EINVAL, "sphpc_slab_owned: bad arguments");
  SPHPC_CK(cudaMemsetAsync(s->slab_counters + 3, 0, sizeof(uint32_t), s->stream));
  // the keep buffer is free between an unpack and the next pack
  launch_slab_owned(s->n, s->ids, s->gid, s->owned, s->pd, s->vel, s->slab_keep,
                    s->slab_counters + 3, (uint32_t)s->cap, s->stream);
  SPHPC_CK(cudaGetLastError());
  uint32_t c = 0;
  SPHPC_CK(cudaMemcpyAsync(&c, s->slab_counters + 3, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  s->slab_nkeep = 0;
  *count = (int)c;
  if ((int)c > capacity)
    return set_error(SPHPC_EINVAL, "sphpc_slab_owned: %u owned particles exceed capacity %d", c,
                     capacity);
  std::vector<SlabRecord> h(c);
  if (c) SPHPC_CK(cudaMemcpy(h.data(), s->slab_keep, sizeof(SlabRecord) * c, cudaMemcpyDeviceToHost));
  for (uint32_t k = 0; k < c; ++k) {
    uint32_t g;
    memcpy(&g, &h[k].a.w, sizeof(g));
    gids[k] = g;
    xyz[3 * k] = h[k].a.x; xyz[3 * k + 1] = h[k].a.y; xyz[3 * k + 2] = h[k].a.z;
    vel[3 * k] = h[k].b.x; vel[3 * k + 1] = h[k].b.y; vel[3 * k + 2] = h[k].b.z;
  }
  return SPHPC_OK;
}

// BalanceNodes, geometry.c:102-166: with the particle counts and slab
// lengths of this rank and its neighbours (the reference trades them with
// MPI_Sendrecv), moves the slab's ends by h towards an even share.
int sphpc_balance_nodes(int rank, int proc_count, int num_rank, int num_right,
                        double length_left, double length_right, int global_count,
                        struct Params* params) {
  if (!params || proc_count < 1 || rank < 0 || rank >= proc_count)
    return set_error(SPHPC_EINVAL, "sphpc_balance_nodes: bad arguments");
  const double h = params->smoothing_radius;
  const double length = params->node_end_x - params->node_start_x;
  const int even_particles = (int)(global_count / (double)proc_count);
  const int max_diff = (int)(even_particles / 10.0f);
  const int diff_right = num_right - even_particles;
  const int diff_self = num_rank - even_particles;
  if (diff_self > max_diff && length > 2 * h && rank != 0)
    params->node_start_x += h;
  else if (diff_self < -max_diff && length_left > 2 * h && rank != 0)
    params->node_start_x -= h;
  if (diff_right > max_diff && length_right > 2 * h && rank != proc_count - 1)
    params->node_end_x += h;
  else if (diff_right < -max_diff && length > 2 * h && rank != proc_count - 1)
    params->node_end_x -= h;
  return SPHPC_OK;
}

// ---- learned warm start ----

int sphpc_mlp_load(struct Particles* particles, const float* params, const float* norm) {
  SPHPC_SIM(s, particles);
  if (!params || !norm) return set_error(SPHPC_EINVAL, "sphpc_mlp_load: null argument");
  SPHPC_RC(mlp_upload(s->mlp.dev, params, norm, s->stream));
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  s->mlp.ready = true;
  return SPHPC_OK;
}

int sphpc_mlp_unload(struct Particles* particles) {
  SPHPC_SIM(s, particles);
  mlp_release(s->mlp);
  return SPHPC_OK;
}

int sphpc_mlp_collect(struct Particles* particles, const struct Params* params,
                      struct Neighbors* neighbors, const struct AABB* boundary_global,
                      const struct Obstacle* obstacle, int iterations) {
  (void)neighbors;
  SPHPC_SIM(s, particles);
  if (!params || !boundary_global) return set_error(SPHPC_EINVAL, "sphpc_mlp_collect: null argument");
  if (iterations < 1 || iterations > 64)
    return set_error(SPHPC_EINVAL, "sphpc_mlp_collect: iterations %d outside [1, 64]", iterations);
  if (!s->grid_ready) SPHPC_RC(s->init_grid(*boundary_global, params->smoothing_radius));
  float *f = nullptr, *t = nullptr;
  long long got = 0;
  SPHPC_RC(mlp_dataset_claim(s->n, &f, &t, &got));
  const DevParams P = s->params(*params, boundary_global, obstacle);
  s->collect_iters = iterations;
  s->collect_rows = got;
  s->collect_feat = f;
  s->collect_target = t;
  const int rc = s->run_step(P, *params);
  s->collect_iters = 0;
  s->collect_rows = 0;
  s->collect_feat = s->collect_target = nullptr;
  if (rc) return rc;
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  return (int)got;
}

__global__ void k_scatter_rows16(int n, const uint32_t* __restrict__ ids,
                                 const float4* __restrict__ src, float4* __restrict__ dst) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t id = ids[p];
#pragma unroll
  for (int k = 0; k < 4; ++k) dst[(size_t)id * 4 + k] = src[(size_t)p * 4 + k];
}

int sphpc_mlp_features(struct Particles* particles, const struct Params* params,
                       const struct AABB* boundary_global, const struct Obstacle* obstacle,
                       float* features) {
  SPHPC_SIM(s, particles);
  if (!params || !boundary_global || !features)
    return set_error(SPHPC_EINVAL, "sphpc_mlp_features: null argument");
  if (!s->nbr_valid) return set_error(SPHPC_ENOTREADY, "sphpc_mlp_features: call FindAllNeighbors first");
  SPHPC_RC(s->ensure_warm_buffers());
  const DevParams P = s->params(*params, boundary_global, obstacle);
  PassArgs a{};
  a.pd = s->pd;
  a.nr_out = s->nr_w;
  a.rho = s->rho_alt ? s->rho_alt : s->rho;
  a.vel = s->vel;
  a.resid = s->resid;
  SPHPC_CK(cudaMemsetAsync(s->resid, 0, 2 * sizeof(double), s->stream));
  launch_features(P, s->view(), a, s->mlp.feat, s->n, s->stream);
  float4* out = nullptr;
  SPHPC_RC(dalloc(&out, (size_t)s->n * 4));
  k_scatter_rows16<<<(s->n + 255) / 256, 256, 0, s->stream>>>(
      s->n, s->ids, reinterpret_cast<const float4*>(s->mlp.feat), out);
  cudaError_t e = cudaMemcpyAsync(features, out, sizeof(float) * 16 * (size_t)s->n,
                                  cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  dfree(out);
  s->launches += 2;
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "sphpc_mlp_features: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

int sphpc_diagnostics(const struct Particles* particles, struct SphpcDiag* diag) {
  SPHPC_SIM(s, particles);
  if (!diag) return set_error(SPHPC_EINVAL, "sphpc_diagnostics: null");
  double* out = s->resid + 4;
  SPHPC_CK(cudaMemsetAsync(out, 0, 9 * sizeof(double), s->stream));
  k_diag<<<148 * 2, kBlock, 0, s->stream>>>(s->n, (float)s->rho0, s->pd, s->vel, s->rho, out);
  double h[9];
  SPHPC_CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  memset(diag, 0, sizeof(*diag));
  const double n = s->n > 0 ? s->n : 1;
  diag->max_density_error = h[0];
  diag->mean_density_error = h[1] / n;
  diag->kinetic_energy = 0.5 * s->mass * h[2];
  for (int k = 0; k < 3; ++k) {
    diag->com[k] = h[3 + k] / n;
    diag->momentum[k] = s->mass * h[6 + k];
  }
  diag->iterations = s->last_iterations;
  diag->warm_start_used = s->last_warm;
  return SPHPC_OK;
}

int sphpc_step_info(const struct Particles* particles, struct SphpcStepInfo* info) {
  SPHPC_SIM(s, particles);
  if (!info) return set_error(SPHPC_EINVAL, "sphpc_step_info: null");
  memset(info, 0, sizeof(*info));
  info->iterations = (int)s->last_iterations;
  info->converged = s->last_converged;
  info->warm_start_used = s->last_warm != 0.0;
  info->warm_start_rejected = s->last_warm_rejected;
  info->max_density_error = s->last_max_err;
  info->mean_density_error = s->last_mean_err;
  info->trace_len = (int)s->trace.size();
  for (size_t k = 0; k < s->trace.size() && k < 16; ++k) info->trace[k] = s->trace[k];
  return SPHPC_OK;
}

int sphpc_device_errors(const struct Particles* particles, unsigned int* bits) {
  SPHPC_SIM(s, particles);
  uint32_t h[2] = {0, 0};
  SPHPC_CK(cudaMemcpyAsync(&h[0], s->err(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  SPHPC_CK(cudaMemcpyAsync(&h[1], s->sort.err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           s->stream));
  SPHPC_CK(cudaStreamSynchronize(s->stream));
  SPHPC_CK(cudaMemsetAsync(s->err(), 0, sizeof(uint32_t), s->stream));
  SPHPC_CK(cudaMemsetAsync(s->sort.err, 0, sizeof(uint32_t), s->stream));
  if (bits) *bits = h[0] | h[1];
  return SPHPC_OK;
}

int sphpc_profile(struct Particles* particles, int enable) {
  SPHPC_SIM(s, particles);
  s->prof_collect();
  s->prof = enable != 0;
  for (auto& v : s->prof_ms) v = 0.0;
  for (auto& c : s->prof_count) c = 0;
  return SPHPC_OK;
}

int sphpc_profile_read(const struct Particles* particles, struct SphpcKernelTime* out,
                       int max_entries, int* n_entries) {
  SPHPC_SIM(s, particles);
  s->prof_collect();
  const int m = (int)s->prof_names.size();
  for (int i = 0; i < m && i < max_entries; ++i) {
    memset(&out[i], 0, sizeof(out[i]));
    strncpy(out[i].name, s->prof_names[i].c_str(), sizeof(out[i].name) - 1);
    out[i].launches = s->prof_count[i];
    out[i].total_ms = s->prof_ms[i];
  }
  if (m < max_entries) {
    memset(&out[m], 0, sizeof(out[m]));
    strncpy(out[m].name, "kernel_launches", sizeof(out[m].name) - 1);
    out[m].launches = (int)(s->launches & 0x7fffffff);
  }
  if (n_entries) *n_entries = m + 1;
  return SPHPC_OK;
}

// ---- obstacle ----

int AllocInitObstacle_CUDA(struct Obstacle* obstacle) {
  if (!obstacle || !obstacle->SDF_buffer)
    return set_error(SPHPC_EINVAL, "AllocInitObstacle_CUDA: no SDF buffer");
  const size_t count =
      (size_t)obstacle->SDF_dim_x * obstacle->SDF_dim_y * obstacle->SDF_dim_z;
  if (count == 0) return set_error(SPHPC_EINVAL, "AllocInitObstacle_CUDA: empty SDF");
  Obstacle_CUDA* oc = new Obstacle_CUDA{nullptr, count};
  int rc = dalloc(&oc->sdf, count);
  if (rc) {
    delete oc;
    return rc;
  }
  const cudaError_t e =
      cudaMemcpy(oc->sdf, obstacle->SDF_buffer, count * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    dfree(oc->sdf);
    delete oc;
    return set_error(SPHPC_ECUDA, "SDF upload: %s", cudaGetErrorString(e));
  }
  obstacle->obstacle_cuda = oc;
  return SPHPC_OK;
}

int FinalizeObstacle_CUDA(struct Obstacle_CUDA* obstacle_cuda) {
  if (!obstacle_cuda) return SPHPC_OK;
  dfree(obstacle_cuda->sdf);
  delete obstacle_cuda;
  return SPHPC_OK;
}

int AllocInitObstacle(struct Obstacle* obstacle) {
  clear_error();
  if (!obstacle) return set_error(SPHPC_EINVAL, "AllocInitObstacle: null");
  SPHPC_RC(sphpc_read_sdf(obstacle));
  return AllocInitObstacle_CUDA(obstacle);
}

int FinalizeObstacle(struct Obstacle* obstacle) {
  if (!obstacle) return SPHPC_OK;
  FinalizeObstacle_CUDA(obstacle->obstacle_cuda);
  obstacle->obstacle_cuda = nullptr;
  free(obstacle->SDF_buffer);
  obstacle->SDF_buffer = nullptr;
  return SPHPC_OK;
}

int CalculateParticleCollisions(double* x, double* y, double* z, const int particle_count,
                                const struct Obstacle obstacle) {
  if (particle_count <= 0) return SPHPC_OK;
  if (!obstacle.obstacle_cuda)
    return set_error(SPHPC_ENOTREADY, "CalculateParticleCollisions: obstacle not uploaded");
  DeviceSim tmp;
  tmp.n = particle_count;
  Params prm{};
  prm.smoothing_radius = 1.0;
  prm.time_step = 1.0;
  const DevParams P = tmp.params(prm, nullptr, &obstacle);
  tmp.n = 0;
  launch_collisions_double(P, x, y, z, particle_count, 0);
  SPHPC_CK(cudaGetLastError());
  return SPHPC_OK;
}

// ---- Thrust seam ----

static int seam_scratch(int count, SortScratch* out) {
  int dev = 0;
  SPHPC_CK(cudaGetDevice(&dev));
  SeamScratch& sc = g_seam[dev];
  if (sc.cap < count) {
    dfree(sc.s.keys_alt);
    dfree(sc.s.vals_alt);
    dfree(sc.aux);
    sc.cap = 0;
    SPHPC_RC(dalloc(&sc.s.keys_alt, (size_t)count));
    SPHPC_RC(dalloc(&sc.s.vals_alt, (size_t)count));
    const size_t aux = sort_aux_words(count) + 4;
    SPHPC_RC(dalloc(&sc.aux, aux));
    SPHPC_CK(cudaMemset(sc.aux, 0, aux * sizeof(uint32_t)));
    sc.s.hist = sc.aux;
    sc.s.counters = sc.aux + (size_t)kMaxPasses * kRadix;
    sc.s.err = sc.aux + (size_t)kMaxPasses * kRadix + kMaxPasses;
    sc.s.lookback = sc.aux + (size_t)kMaxPasses * kRadix + kMaxPasses + 4;
    sc.cap = count;
  }
  *out = sc.s;
  return SPHPC_OK;
}

int SortByKey(unsigned int* const keys, unsigned int* const values, const int count,
              const void* const cuda_stream) {
  if (count < 0 || (count > 0 && (!keys || !values)))
    return set_error(SPHPC_EINVAL, "SortByKey: bad arguments");
  if (count <= 1) return SPHPC_OK;
  std::lock_guard<std::mutex> lk(g_seam_mu);
  SortScratch sc;
  SPHPC_RC(seam_scratch(count, &sc));
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const cudaError_t e = radix_sort_pairs(keys, values, count, kMaxPasses, sc, st, false, false,
                                         true, nullptr, nullptr);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "SortByKey: %s", cudaGetErrorString(e));
  // the scratch is shared by every caller: finish before releasing it
  SPHPC_CK(cudaStreamSynchronize(st));
  uint32_t herr = 0;
  SPHPC_CK(cudaMemcpy(&herr, sc.err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (herr) {
    cudaMemset(sc.err, 0, sizeof(uint32_t));
    return set_error(SPHPC_EKERNEL, "SortByKey: look-back wait gave up (error bits 0x%x)", herr);
  }
  return SPHPC_OK;
}

// ---- failure detection of the bounded device waits ----

static int wait_check(const char* what, cudaError_t e, uint32_t bits, unsigned int* out) {
  if (out) *out = bits;
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  if (bits) return set_error(SPHPC_EKERNEL, "%s: the bounded wait gave up (error bits 0x%x)",
                             what, bits);
  return SPHPC_OK;
}

int sphpc_fail_device_alloc(int after) {
  if (after < -1) return set_error(SPHPC_EINVAL, "sphpc_fail_device_alloc: %d < -1", after);
  g_alloc_fail_after.store(after);
  return SPHPC_OK;
}

int sphpc_check_sort_wait(int spin_limit, unsigned int* error_bits) {
  if (spin_limit < 1 || spin_limit > kSpinLimit)
    return set_error(SPHPC_EINVAL, "sphpc_check_sort_wait: limit %d outside [1, %d]", spin_limit,
                     kSpinLimit);
  uint32_t bits = 0;
  const cudaError_t e = lookback_wait_probe(spin_limit, &bits);
  return wait_check("sphpc_check_sort_wait", e, bits, error_bits);
}

int sphpc_check_mbarrier_wait(int poll_limit, unsigned int* error_bits) {
  if (poll_limit < 1 || poll_limit > (1 << 20))
    return set_error(SPHPC_EINVAL, "sphpc_check_mbarrier_wait: limit %d outside [1, 2^20]",
                     poll_limit);
  uint32_t bits = 0;
  const cudaError_t e = mbar_wait_probe(poll_limit, &bits);
  return wait_check("sphpc_check_mbarrier_wait", e, bits, error_bits);
}

int FindLowerBounds(const unsigned int* const hash_values, const int value_count,
                    const int search_count, unsigned int* const start_indices,
                    const void* const cuda_stream) {
  if (value_count < 0 || search_count < 0)
    return set_error(SPHPC_EINVAL, "FindLowerBounds: negative count");
  const cudaError_t e = launch_bounds(hash_values, value_count, search_count, start_indices,
                                      false, (cudaStream_t)cuda_stream);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "FindLowerBounds: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

int FindUpperBounds(const unsigned int* const hash_values, const int value_count,
                    const int search_count, unsigned int* const end_indices,
                    const void* const cuda_stream) {
  if (value_count < 0 || search_count < 0)
    return set_error(SPHPC_EINVAL, "FindUpperBounds: negative count");
  const cudaError_t e = launch_bounds(hash_values, value_count, search_count, end_indices, true,
                                      (cudaStream_t)cuda_stream);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "FindUpperBounds: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

}  // extern "C"
