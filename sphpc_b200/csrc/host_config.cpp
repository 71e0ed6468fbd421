// host_config.cpp -- configuration, scene set-up and SDF file input.
//
// Restates the reference's host set-up on the C ABI with error codes:
//   ReadParameters        input_parser.cc:16-69 (Boost INI -> own parser)
//   SetParameters         simulation.c:130-178
//   SetParticleNumbers    geometry.c:77-99
//   ConstructFluidVolume  geometry.c:19-74 (+ seeded jitter)
//   AllocInitObstacle     obstacle.c:13-79 (SDFGen ASCII)
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "host_internal.h"

namespace sphpc {

namespace {
thread_local std::string g_error;
std::mutex g_solver_mu;
bool g_solver_set = false;
SphpcSolver g_solver;
}  // namespace

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

void clear_error() { g_error.clear(); }

void set_current_solver(const SphpcSolver& s) {
  std::lock_guard<std::mutex> lk(g_solver_mu);
  g_solver = s;
  g_solver_set = true;
}

SphpcSolver current_solver() {
  std::lock_guard<std::mutex> lk(g_solver_mu);
  if (!g_solver_set) {
    SphpcSolver s;
    sphpc_default_solver(&s);
    return s;
  }
  return g_solver;
}

double counter_uniform01(uint64_t seed, uint64_t index, uint32_t axis) {
  auto mix = [](uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  };
  const uint64_t k = mix(seed ^ mix(index * 4u + axis));
  return (double)(k >> 11) * (1.0 / 9007199254740992.0);
}

void set_kernel_norms(Params* p) {
  const double h = p->smoothing_radius;
  p->W_norm = 315.0 / (64.0 * M_PI * pow(h, 9.0));
  p->DelW_poly_norm = -3.0 * 2.0 * p->W_norm;
  p->DelW_norm = -45.0 / (M_PI * pow(h, 6.0));
}

double lattice_poly6_sum(double h, double W_norm, double spacing) {
  const int R = (int)ceil(h / spacing) + 1;
  double s = 0.0;
  for (int k = -R; k <= R; ++k)
    for (int j = -R; j <= R; ++j)
      for (int i = -R; i <= R; ++i) {
        const double r2 = (i * i + j * j + k * k) * spacing * spacing;
        if (r2 < h * h || (i == 0 && j == 0 && k == 0)) {
          const double r = sqrt(r2);
          if (r > h) continue;
          s += W_norm * (h * h - r * r) * (h * h - r * r) * (h * h - r * r);
        }
      }
  return s;
}

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) ++a;
  while (b > a && isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// Minimal INI reader with the subset Boost.PropertyTree's ini_parser accepts
// in the reference's files: [Section], key = value, ';'/'#' comments.
int read_ini(const char* path, std::map<std::string, std::string>& kv) {
  FILE* f = fopen(path, "r");
  if (!f) return set_error(SPHPC_EIO, "cannot open %s: %s", path, strerror(errno));
  char line[4096];
  std::string section;
  int lineno = 0;
  while (fgets(line, sizeof(line), f)) {
    ++lineno;
    std::string s(line);
    const size_t c = s.find_first_of("#;");
    if (c != std::string::npos) s = s.substr(0, c);
    s = trim(s);
    if (s.empty()) continue;
    if (s[0] == '[') {
      const size_t e = s.find(']');
      if (e == std::string::npos) {
        fclose(f);
        return set_error(SPHPC_EIO, "%s:%d: unterminated section header", path, lineno);
      }
      section = trim(s.substr(1, e - 1));
      continue;
    }
    const size_t eq = s.find('=');
    if (eq == std::string::npos) {
      fclose(f);
      return set_error(SPHPC_EIO, "%s:%d: expected key = value", path, lineno);
    }
    kv[section + "." + trim(s.substr(0, eq))] = trim(s.substr(eq + 1));
  }
  fclose(f);
  return SPHPC_OK;
}

struct Ini {
  std::map<std::string, std::string> kv;
  const char* path;
  int err = SPHPC_OK;

  bool has(const char* key) const { return kv.count(key) != 0; }

  double num(const char* key) {
    auto it = kv.find(key);
    if (it == kv.end()) {
      if (err == SPHPC_OK) err = set_error(SPHPC_EIO, "%s: missing key %s", path, key);
      return 0.0;
    }
    char* end = nullptr;
    const double v = strtod(it->second.c_str(), &end);
    if (end == it->second.c_str() || *end != '\0') {
      if (err == SPHPC_OK)
        err = set_error(SPHPC_EIO, "%s: key %s is not a number: '%s'", path, key,
                        it->second.c_str());
    }
    return v;
  }
  int integer(const char* key) {
    const double v = num(key);
    if (err == SPHPC_OK && v != floor(v))
      err = set_error(SPHPC_EIO, "%s: key %s is not an integer", path, key);
    return (int)v;
  }
  double num_or(const char* key, double d) { return has(key) ? num(key) : d; }
  std::string str_or(const char* key, const char* d) const {
    auto it = kv.find(key);
    return it == kv.end() ? std::string(d) : it->second;
  }
  bool flag_or(const char* key, bool d) {
    if (!has(key)) return d;
    std::string v = str_or(key, "");
    for (auto& ch : v) ch = (char)tolower((unsigned char)ch);
    if (v == "on" || v == "1" || v == "true" || v == "yes") return true;
    if (v == "off" || v == "0" || v == "false" || v == "no") return false;
    if (err == SPHPC_OK) err = set_error(SPHPC_EIO, "%s: key %s is not on/off", path, key);
    return d;
  }
};

}  // namespace
}  // namespace sphpc

using namespace sphpc;

extern "C" {

const char* sphpc_last_error(void) { return g_error.c_str(); }
const char* sphpc_version(void) { return "sphpc-b200 0.1"; }

void sphpc_default_solver(struct SphpcSolver* s) {
  memset(s, 0, sizeof(*s));
  s->solve_iterations = 10;
  s->scorr_n = 4;
  s->lambda_epsilon = 0.01;
  s->scorr_k = 0.0;
  s->scorr_dq = 0.1;
  s->stiffness_k = 0.95;
  s->vorticity_epsilon = -1.0;
  s->velocity_max = 100.0;
  s->gravity_axis = 2;
  s->xsph_exact = 0;
  s->surface_tension = 1;
  s->vorticity = 1;
  s->jitter = 0.0;
  s->seed = 0;
  s->rest_density_lattice = 0;
  s->adaptive = 0;
  s->density_tolerance = 0.01;
  s->max_iterations = 32;
  s->warm_start = 0;
  s->lambda_epsilon_mass_units = 0;
  s->warm_start_gate = 1;
  s->warm_start_source = 0;
  s->warm_start_scale = 1.0;
  s->min_progress = 0.0;
  s->warm_start_min_error = 0.0;
}

// The neighbour build decides r^2 < h^2 from FP32 copies of the absolute
// predicted positions, and leaves to the exact FP64 test of FillNeighbors
// (neighbors.c:278-285) only the pairs whose FP32 r^2 lies within
// +-2^-10 h^2 of h^2.  That is correct while the FP32 error of r^2 stays
// below the band.  A coordinate of magnitude up to max_coord is rounded to
// FP32 within u/2, u = 2^(floor(log2 max_coord) - 23); a pair difference
// (< 2h per axis between adjacent cells) is then off by at most
// e = u + 2^-24 (2h + u), and r^2 near h^2 by at most
// e (2 sqrt(3) h + 3e) plus the FP32 rounding of the sum of squares,
// 3 * 2^-24 h^2.  Safe when that total, with a 10% margin, is below
// 2^-10 h^2 (for h = 2: coordinates up to 2^13).
int sphpc_neighbor_pretest_fp32_safe(double max_coord, double h) {
  if (!(h > 0.0) || !(max_coord >= 0.0) || !std::isfinite(max_coord)) return 0;
  const double m = max_coord > h ? max_coord : h;
  const double u = std::ldexp(1.0, (int)std::floor(std::log2(m)) - 23);
  const double e = u + std::ldexp(2.0 * h + u, -24);
  const double err = e * (2.0 * std::sqrt(3.0) * h * 1.001 + 3.0 * e) +
                     3.0 * std::ldexp(1.0, -24) * 1.002 * h * h;
  return err < 0.9 * std::ldexp(h * h, -10) ? 1 : 0;
}

void sphpc_set_default_solver(const struct SphpcSolver* s) {
  if (s) set_current_solver(*s);
}

int sphpc_load_config(const char* path, struct Params* params, struct Particles* particles,
                      struct AABB* boundary, struct AABB* fluid, struct Obstacle* obstacle,
                      struct SphpcSolver* solver_out) {
  clear_error();
  if (!path || !params || !particles || !boundary || !fluid)
    return set_error(SPHPC_EINVAL, "sphpc_load_config: null argument");
  Ini ini;
  ini.path = path;
  int rc = read_ini(path, ini.kv);
  if (rc) return rc;
  // ReadParameters, input_parser.cc:27-62
  params->number_steps = ini.integer("SimParameters.number_steps");
  params->time_step = ini.num("SimParameters.time_step");
  particles->global_count = ini.integer("SimParameters.number_particles");
  params->g = ini.num("PhysicalParameters.g");
  params->c = ini.num("PhysicalParameters.c");
  params->k = ini.num("PhysicalParameters.k");
  boundary->min_x = ini.num("BoundaryVolume.min_x");
  boundary->min_y = ini.num("BoundaryVolume.min_y");
  boundary->min_z = ini.num("BoundaryVolume.min_z");
  boundary->max_x = ini.num("BoundaryVolume.max_x");
  boundary->max_y = ini.num("BoundaryVolume.max_y");
  boundary->max_z = ini.num("BoundaryVolume.max_z");
  fluid->min_x = ini.num("InitialFluidVolume.min_x");
  fluid->min_y = ini.num("InitialFluidVolume.min_y");
  fluid->min_z = ini.num("InitialFluidVolume.min_z");
  fluid->max_x = ini.num("InitialFluidVolume.max_x");
  fluid->max_y = ini.num("InitialFluidVolume.max_y");
  fluid->max_z = ini.num("InitialFluidVolume.max_z");
  if (obstacle) {
    memset(obstacle, 0, sizeof(*obstacle));
    if (ini.has("Obstacle.SDF_file_name")) {
      std::string fn = ini.str_or("Obstacle.SDF_file_name", "");
      if (!fn.empty() && fn[0] != '/') {
        // resolve next to the INI file when not found relative to the cwd
        FILE* probe = fopen(fn.c_str(), "r");
        if (probe) {
          fclose(probe);
        } else {
          std::string dir(path);
          const size_t sl = dir.find_last_of('/');
          if (sl != std::string::npos) fn = dir.substr(0, sl + 1) + fn;
        }
      }
      if (fn.size() >= sizeof(obstacle->SDF_file_name))
        return set_error(SPHPC_EINVAL, "%s: SDF_file_name longer than 127 characters", path);
      strcpy(obstacle->SDF_file_name, fn.c_str());
      obstacle->world_bounds.min_x = ini.num("Obstacle.min_x");
      obstacle->world_bounds.max_x = ini.num("Obstacle.max_x");
      obstacle->world_bounds.min_y = ini.num("Obstacle.min_y");
      obstacle->world_bounds.min_z = ini.num("Obstacle.min_z");
    }
  }
  // extension keys
  SphpcSolver s;
  sphpc_default_solver(&s);
  s.solve_iterations = (int)ini.num_or("Solver.solve_iterations", s.solve_iterations);
  s.lambda_epsilon = ini.num_or("Solver.lambda_epsilon", s.lambda_epsilon);
  {
    std::string u = ini.str_or("Solver.lambda_epsilon_units", "normalized");
    if (u == "mass_gradient") s.lambda_epsilon_mass_units = 1;
    else if (u != "normalized" && ini.err == SPHPC_OK)
      ini.err = set_error(SPHPC_EIO, "%s: lambda_epsilon_units must be normalized or "
                                     "mass_gradient", path);
  }
  s.scorr_k = ini.num_or("Solver.scorr_k", s.scorr_k);
  s.scorr_n = (int)ini.num_or("Solver.scorr_n", s.scorr_n);
  s.scorr_dq = ini.num_or("Solver.scorr_dq", s.scorr_dq);
  s.stiffness_k = ini.num_or("Solver.stiffness_k", s.stiffness_k);
  s.vorticity_epsilon = ini.num_or("Solver.vorticity_epsilon", s.vorticity_epsilon);
  s.velocity_max = ini.num_or("Solver.velocity_max", s.velocity_max);
  {
    std::string a = ini.str_or("Solver.gravity_axis", "z");
    if (a == "x" || a == "0") s.gravity_axis = 0;
    else if (a == "y" || a == "1") s.gravity_axis = 1;
    else if (a == "z" || a == "2") s.gravity_axis = 2;
    else if (ini.err == SPHPC_OK)
      ini.err = set_error(SPHPC_EIO, "%s: gravity_axis must be x, y or z", path);
  }
  {
    std::string x = ini.str_or("Solver.xsph", "jacobi");
    if (x == "jacobi") s.xsph_exact = 0;
    else if (x == "jacobi_exact") s.xsph_exact = 1;
    else if (ini.err == SPHPC_OK)
      ini.err = set_error(SPHPC_EIO, "%s: xsph must be jacobi or jacobi_exact (the in-place "
                                     "update of particles.c:455 is a data race on a GPU)", path);
  }
  s.surface_tension = ini.flag_or("Solver.surface_tension", true) ? 1 : 0;
  s.vorticity = ini.flag_or("Solver.vorticity", true) ? 1 : 0;
  s.adaptive = ini.flag_or("Solver.adaptive", false) ? 1 : 0;
  s.density_tolerance = ini.num_or("Solver.density_tolerance", s.density_tolerance);
  s.max_iterations = (int)ini.num_or("Solver.max_iterations", s.max_iterations);
  s.warm_start = ini.flag_or("Solver.warm_start", false) ? 1 : 0;
  s.jitter = ini.num_or("InitialFluidVolume.jitter", 0.0);
  s.seed = (unsigned long long)ini.num_or("InitialFluidVolume.seed", 0.0);
  {
    std::string r = ini.str_or("PhysicalParameters.rest_density", "reference");
    if (r == "lattice") s.rest_density_lattice = 1;
    else if (r != "reference" && ini.err == SPHPC_OK)
      ini.err = set_error(SPHPC_EIO, "%s: rest_density must be reference or lattice", path);
  }
  if (ini.err) return ini.err;
  if (s.solve_iterations < 0 || s.scorr_n < 0 || s.max_iterations < 1)
    return set_error(SPHPC_EINVAL, "%s: negative iteration count", path);
  if (particles->global_count <= 0)
    return set_error(SPHPC_EINVAL, "%s: number_particles must be positive", path);
  // SetParameters, simulation.c:130-178 (single rank)
  params->rank = 0;
  params->proc_count = 1;
  const double volume = (fluid->max_x - fluid->min_x) * (fluid->max_y - fluid->min_y) *
                        (fluid->max_z - fluid->min_z);
  if (!(volume > 0.0)) return set_error(SPHPC_EINVAL, "%s: empty InitialFluidVolume", path);
  const float spacing_particle = (float)pow(volume / particles->global_count, 1.0 / 3.0);
  particles->rest_radius = spacing_particle / 2.0;
  params->smoothing_radius = 2.0 * spacing_particle;
  params->dq = 0.1 * params->smoothing_radius;
  params->node_start_x = boundary->min_x;
  params->node_end_x = boundary->max_x;
  set_kernel_norms(params);
  if (boundary->min_x < 0.0 || boundary->min_y < 0.0 || boundary->min_z < 0.0)
    return set_error(SPHPC_EINVAL, "%s: BoundaryVolume minimum must be >= 0 (the hash of "
                                   "neighbors.c:86-88 has no offset)", path);
  set_current_solver(s);
  if (solver_out) *solver_out = s;
  return SPHPC_OK;
}

int ReadParameters(struct Params* parameters, struct Particles* particles,
                   struct AABB* boundary_volume, struct AABB* initial_fluid_volume,
                   struct Obstacle* obstacle) {
  return sphpc_load_config("./sim-config.ini", parameters, particles, boundary_volume,
                           initial_fluid_volume, obstacle, nullptr);
}

int SetParameters(struct Params* params, struct Particles* particles,
                  struct Neighbors* neighbors, struct AABB* boundary_global,
                  struct AABB* water_volume_global, struct Obstacle* obstacle) {
  (void)neighbors;
  return sphpc_load_config("./sim-config.ini", params, particles, boundary_global,
                           water_volume_global, obstacle, nullptr);
}

int SetParticleNumbers(const struct AABB* fluid_global, struct Particles* particles,
                       struct Params* params, void* communication) {
  (void)params;
  (void)communication;
  if (!fluid_global || !particles) return set_error(SPHPC_EINVAL, "SetParticleNumbers: null");
  const double spacing = 2.0 * particles->rest_radius;
  if (!(spacing > 0.0)) return set_error(SPHPC_EINVAL, "SetParticleNumbers: rest_radius unset");
  const int num_x = (int)floor((fluid_global->max_x - fluid_global->min_x) / spacing);
  const int num_y = (int)floor((fluid_global->max_y - fluid_global->min_y) / spacing);
  const int num_z = (int)floor((fluid_global->max_z - fluid_global->min_z) / spacing);
  const long long num_initial = (long long)num_x * num_y * num_z;
  if (num_initial <= 0 || num_initial > (1LL << 30))
    return set_error(SPHPC_EINVAL, "SetParticleNumbers: %lld particles out of range",
                     num_initial);
  const long long max_particles = num_initial / 5;
  particles->max_local = (int)(num_initial + 4 * max_particles);
  return SPHPC_OK;
}

int ConstructFluidVolume(struct Particles* particles, struct Params* params,
                         const struct AABB* fluid) {
  if (!particles || !params || !fluid || !particles->x)
    return set_error(SPHPC_EINVAL, "ConstructFluidVolume: null argument");
  const SphpcSolver s = current_solver();
  const double spacing = 2.0 * particles->rest_radius;
  const double min_x = fluid->min_x;
  const double max_x = fmin(fluid->max_x, params->node_end_x);
  const int num_x = (int)floor((max_x - min_x) / spacing);
  const int num_y = (int)floor((fluid->max_y - fluid->min_y) / spacing);
  const int num_z = (int)floor((fluid->max_z - fluid->min_z) / spacing);
  const long long total = (long long)num_x * num_y * num_z;
  if (total > particles->max_local)
    return set_error(SPHPC_EINVAL, "ConstructFluidVolume: %lld particles exceed max_local %d",
                     total, particles->max_local);
  long long i = 0;
  for (int nz = 0; nz < num_z; ++nz) {
    for (int ny = 0; ny < num_y; ++ny) {
      for (int nx = 0; nx < num_x; ++nx) {
        const double jx = s.jitter * spacing * (2.0 * counter_uniform01(s.seed, i, 0) - 1.0);
        const double jy = s.jitter * spacing * (2.0 * counter_uniform01(s.seed, i, 1) - 1.0);
        const double jz = s.jitter * spacing * (2.0 * counter_uniform01(s.seed, i, 2) - 1.0);
        particles->x[i] = min_x + nx * spacing + spacing / 2.0 + jx;
        particles->y[i] = fluid->min_y + ny * spacing + spacing / 2.0 + jy;
        particles->z[i] = fluid->min_z + nz * spacing + spacing / 2.0 + jz;
        if (particles->id) particles->id[i] = (int)i;
        ++i;
      }
    }
  }
  particles->local_count = (int)i;
  particles->global_count = (int)i;
  params->fluid_volume = (num_x * spacing) * (num_y * spacing) * (num_z * spacing);
  return SPHPC_OK;
}

// SDFGen ASCII reader, obstacle.c:13-79.
int sphpc_read_sdf(struct Obstacle* obstacle) {
  FILE* f = fopen(obstacle->SDF_file_name, "rb");
  if (!f) return set_error(SPHPC_EIO, "Can't open %s", obstacle->SDF_file_name);
  fseek(f, 0, SEEK_END);
  const long size = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<char> buf((size_t)size + 1);
  if (size > 0 && fread(buf.data(), 1, (size_t)size, f) != (size_t)size) {
    fclose(f);
    return set_error(SPHPC_EIO, "Error reading SDF file: %s", obstacle->SDF_file_name);
  }
  fclose(f);
  buf[(size_t)size] = '\0';
  char* p = buf.data();
  char* end = nullptr;
  auto next_long = [&](long& v) {
    v = strtol(p, &end, 10);
    if (end == p) return false;
    p = end;
    return true;
  };
  auto next_double = [&](double& v) {
    v = strtod(p, &end);
    if (end == p) return false;
    p = end;
    return true;
  };
  long dims[3];
  double org[3], dx;
  for (int k = 0; k < 3; ++k)
    if (!next_long(dims[k]))
      return set_error(SPHPC_EIO, "Error parsing SDF file: %s (dimensions)",
                       obstacle->SDF_file_name);
  for (int k = 0; k < 3; ++k)
    if (!next_double(org[k]))
      return set_error(SPHPC_EIO, "Error parsing SDF file: %s (origin)", obstacle->SDF_file_name);
  if (!next_double(dx))
    return set_error(SPHPC_EIO, "Error parsing SDF file: %s (spacing)", obstacle->SDF_file_name);
  if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || dims[0] * dims[1] * dims[2] > (1L << 28))
    return set_error(SPHPC_EIO, "SDF file %s: bad dimensions %ld %ld %ld",
                     obstacle->SDF_file_name, dims[0], dims[1], dims[2]);
  const size_t count = (size_t)dims[0] * dims[1] * dims[2];
  float* data = (float*)calloc(count, sizeof(float));
  if (!data) return set_error(SPHPC_ENOMEM, "SDF buffer of %zu floats", count);
  for (size_t i = 0; i < count; ++i) {
    const float v = strtof(p, &end);
    if (end == p) {
      free(data);
      return set_error(SPHPC_EIO, "Error parsing SDF file: %s (value %zu of %zu)",
                       obstacle->SDF_file_name, i, count);
    }
    p = end;
    data[i] = v;
  }
  obstacle->SDF_dim_x = (int)dims[0];
  obstacle->SDF_dim_y = (int)dims[1];
  obstacle->SDF_dim_z = (int)dims[2];
  obstacle->origin_x = org[0];
  obstacle->origin_y = org[1];
  obstacle->origin_z = org[2];
  obstacle->SDF_spacing = dx;
  if (obstacle->SDF_buffer) free(obstacle->SDF_buffer);
  obstacle->SDF_buffer = data;
  // obstacle.c:73-75
  const double obstacle_length = obstacle->world_bounds.max_x - obstacle->world_bounds.min_x;
  obstacle->world_bounds.max_y =
      obstacle_length * obstacle->SDF_dim_y / (float)obstacle->SDF_dim_x;
  obstacle->world_bounds.max_z =
      obstacle_length * obstacle->SDF_dim_z / (float)obstacle->SDF_dim_x;
  return SPHPC_OK;
}

}  // extern "C"
