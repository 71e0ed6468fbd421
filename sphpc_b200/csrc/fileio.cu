// fileio.cu -- particle snapshots in the reference's output format
// (fileio_MPI_IO.c:63-118): <cwd>/output/sim-N.bin holds the particles' x, y,
// z as interleaved doubles in original particle order (a single rank writes
// at offset 0), one file per WriteParticles call.
//
// The gather runs on the device (one kernel on the particle set's stream),
// the copy goes into the page-locked write_buffer asynchronously, and a host
// thread writes the file once the copy has landed, so WriteParticles returns
// without waiting for the disk.  The next WriteParticles, sphpc_fileio_wait
// and FinalizeFileIO wait for the previous file and report its errors.
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>

#include <cuda_runtime.h>

#include "host_internal.h"

namespace sphpc {
namespace {

struct Writer {
  double* d_buf = nullptr;   // device gather buffer, 3 * max_local doubles
  size_t cap = 0;            // doubles
  cudaEvent_t copied = nullptr;
  std::thread thread;
  int rc = SPHPC_OK;         // outcome of the last write
  std::string msg;
};

std::mutex g_fio_mu;
std::map<const FileIO*, Writer*> g_writers;

Writer* find_writer(const FileIO* f) {
  std::lock_guard<std::mutex> lk(g_fio_mu);
  auto it = g_writers.find(f);
  return it == g_writers.end() ? nullptr : it->second;
}

// Waits for the file in flight and returns its outcome.
int join_writer(Writer* w) {
  if (w->thread.joinable()) w->thread.join();
  const int rc = w->rc;
  if (rc) set_error(rc, "%s", w->msg.c_str());
  w->rc = SPHPC_OK;
  w->msg.clear();
  return rc;
}

}  // namespace
}  // namespace sphpc

using namespace sphpc;

extern "C" {

int AllocInitFileIO(struct FileIO* const file_io, const struct Particles* const particles,
                    const struct Params* params) {
  (void)params;
  if (!file_io || !particles) return set_error(SPHPC_EINVAL, "AllocInitFileIO: null argument");
  if (find_writer(file_io)) return set_error(SPHPC_EINVAL, "AllocInitFileIO: already initialised");
  const size_t cap = 3 * (size_t)(particles->max_local > 0 ? particles->max_local : 1);
  char cwd[1024];
  if (!getcwd(cwd, sizeof(cwd)))
    return set_error(SPHPC_EINVAL, "AllocInitFileIO: getcwd: %s", strerror(errno));
  const std::string out = std::string(cwd) + "/output";
  if (mkdir(out.c_str(), 0775) != 0 && errno != EEXIST)
    return set_error(SPHPC_EINVAL, "AllocInitFileIO: mkdir %s: %s", out.c_str(), strerror(errno));
  Writer* w = new Writer();
  w->cap = cap;
  double* host = nullptr;
  cudaError_t e = cudaMallocHost(&host, sizeof(double) * cap);
  if (e == cudaSuccess) e = cudaMalloc(&w->d_buf, sizeof(double) * cap);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->copied, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    if (host) cudaFreeHost(host);
    if (w->d_buf) cudaFree(w->d_buf);
    delete w;
    cudaGetLastError();
    return set_error(SPHPC_ENOMEM, "AllocInitFileIO: %s", cudaGetErrorString(e));
  }
  file_io->write_buffer = host;
  file_io->output_path = strdup(out.c_str());
  file_io->file_num = 0;
  std::lock_guard<std::mutex> lk(g_fio_mu);
  g_writers[file_io] = w;
  return SPHPC_OK;
}

int WriteParticles(const struct Particles* const particles, const struct Params* const params,
                   struct FileIO* const file_io) {
  (void)params;
  Writer* w = file_io ? find_writer(file_io) : nullptr;
  if (!w) return set_error(SPHPC_ENOTREADY, "WriteParticles: call AllocInitFileIO first");
  // the buffer is reused: the previous file must be on disk first
  SPHPC_RC(join_writer(w));
  int n = 0;
  void* stream = nullptr;
  SPHPC_RC(sim_interleave_positions(particles, w->d_buf, &n, &stream));
  const size_t count = 3 * (size_t)n;
  if (count > w->cap)
    return set_error(SPHPC_EINVAL, "WriteParticles: %d particles exceed max_local", n);
  cudaStream_t st = (cudaStream_t)stream;
  SPHPC_CK(cudaMemcpyAsync(file_io->write_buffer, w->d_buf, sizeof(double) * count,
                           cudaMemcpyDeviceToHost, st));
  SPHPC_CK(cudaEventRecord(w->copied, st));
  char name[1100];
  snprintf(name, sizeof(name), "%s/sim-%d.bin", file_io->output_path, file_io->file_num);
  ++file_io->file_num;
  const double* buf = file_io->write_buffer;
  const cudaEvent_t ev = w->copied;
  const std::string path = name;
  w->thread = std::thread([w, buf, count, ev, path]() {
    const cudaError_t e = cudaEventSynchronize(ev);
    if (e != cudaSuccess) {
      w->rc = SPHPC_ECUDA;
      w->msg = std::string("WriteParticles: ") + cudaGetErrorString(e);
      return;
    }
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) {
      w->rc = SPHPC_EINVAL;
      w->msg = "WriteParticles: cannot open " + path + ": " + strerror(errno);
      return;
    }
    const size_t wrote = fwrite(buf, sizeof(double), count, f);
    const int closed = fclose(f);
    if (wrote != count || closed != 0) {
      w->rc = SPHPC_EINVAL;
      w->msg = "WriteParticles: short write to " + path;
    }
  });
  return SPHPC_OK;
}

int sphpc_fileio_wait(struct FileIO* file_io) {
  Writer* w = file_io ? find_writer(file_io) : nullptr;
  if (!w) return set_error(SPHPC_ENOTREADY, "sphpc_fileio_wait: call AllocInitFileIO first");
  return join_writer(w);
}

int FinalizeFileIO(struct FileIO* const file_io) {
  if (!file_io) return set_error(SPHPC_EINVAL, "FinalizeFileIO: null");
  Writer* w = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_fio_mu);
    auto it = g_writers.find(file_io);
    if (it == g_writers.end()) return set_error(SPHPC_ENOTREADY, "FinalizeFileIO: not initialised");
    w = it->second;
    g_writers.erase(it);
  }
  const int rc = join_writer(w);
  if (w->d_buf) cudaFree(w->d_buf);
  if (w->copied) cudaEventDestroy(w->copied);
  delete w;
  if (file_io->write_buffer) cudaFreeHost(file_io->write_buffer);
  free(file_io->output_path);
  file_io->write_buffer = nullptr;
  file_io->output_path = nullptr;
  return rc;
}

}  // extern "C"
