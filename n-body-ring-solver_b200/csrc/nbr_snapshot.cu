// nbr_snapshot.cu -- checkpoints in the reference's binary snapshot format.
//
// NBody_system::save_particles (CPU/nbody_system.cpp:133-152) appends one
// record per call to "NBody_<N>.dat": the time time_step * delta_t, then the
// N masses, positions x, y, z, velocities x, y, z and forces x, y, z, all as
// native-endian doubles (8 + 80 N bytes per record); the call with
// time_step == 0 truncates the file.  The writer here produces the same bytes
// from caller arrays or from a context's device state; the reader turns any
// record back into arrays or into a context's system (resume).
#include "nbr.h"
#include "nbr_ctx.h"

#include <sys/stat.h>

#include <cstdio>
#include <string>
#include <vector>

using namespace nbr;

namespace {

constexpr size_t kFields = 10;  // m, x, y, z, vx, vy, vz, fx, fy, fz

size_t record_bytes(size_t n) { return sizeof(double) * (1 + kFields * n); }

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

}  // namespace

extern "C" int nbr_snapshot_write_arrays(const char* path, size_t n, size_t time_step,
                                         double delta_t, const double* m, const double* x,
                                         const double* y, const double* z, const double* vx,
                                         const double* vy, const double* vz, const double* fx,
                                         const double* fy, const double* fz) {
  if (!path || n == 0 || !m || !x || !y || !z)
    return fail(nullptr, NBR_ERR_INVALID_ARG, "snapshot: NULL path or array, or n = 0");
  File out;
  out.f = std::fopen(path, time_step == 0 ? "wb" : "ab");
  if (!out.f) return fail(nullptr, NBR_ERR_IO, std::string("snapshot: cannot open ") + path);
  const double t = time_step * delta_t;  // the reference's curr_time
  std::vector<double> zeros;
  bool ok = std::fwrite(&t, sizeof(double), 1, out.f) == 1;
  const double* fields[kFields] = {m, x, y, z, vx, vy, vz, fx, fy, fz};
  for (const double* a : fields) {
    if (!ok) break;
    if (!a) {
      if (zeros.empty()) zeros.assign(n, 0.0);
      a = zeros.data();
    }
    ok = std::fwrite(a, sizeof(double), n, out.f) == n;
  }
  if (std::fclose(out.f) != 0) ok = false;
  out.f = nullptr;
  return ok ? NBR_OK : fail(nullptr, NBR_ERR_IO, std::string("snapshot: write failed on ") + path);
}

extern "C" int nbr_snapshot_records(const char* path, size_t n, size_t* records) {
  if (!path || n == 0 || !records)
    return fail(nullptr, NBR_ERR_INVALID_ARG, "snapshot: NULL path or output, or n = 0");
  struct stat st;
  if (stat(path, &st) != 0) return fail(nullptr, NBR_ERR_IO, std::string("snapshot: no file ") + path);
  const size_t bytes = (size_t)st.st_size, rb = record_bytes(n);
  if (bytes % rb != 0)
    return fail(nullptr, NBR_ERR_INVALID_ARG,
                "snapshot: " + std::to_string(bytes) + " bytes is not a whole number of " +
                    std::to_string(n) + "-particle records");
  *records = bytes / rb;
  return NBR_OK;
}

extern "C" int nbr_snapshot_read_arrays(const char* path, size_t n, size_t record, double* time,
                                        double* m, double* x, double* y, double* z, double* vx,
                                        double* vy, double* vz, double* fx, double* fy,
                                        double* fz) {
  size_t count = 0;
  int rc = nbr_snapshot_records(path, n, &count);
  if (rc) return rc;
  if (record >= count)
    return fail(nullptr, NBR_ERR_INVALID_ARG,
                "snapshot: record " + std::to_string(record) + " of " + std::to_string(count));
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return fail(nullptr, NBR_ERR_IO, std::string("snapshot: cannot open ") + path);
  if (fseeko(in.f, (off_t)(record * record_bytes(n)), SEEK_SET) != 0)
    return fail(nullptr, NBR_ERR_IO, "snapshot: seek failed");
  double t = 0.0;
  bool ok = std::fread(&t, sizeof(double), 1, in.f) == 1;
  double* fields[kFields] = {m, x, y, z, vx, vy, vz, fx, fy, fz};
  for (double* a : fields) {
    if (!ok) break;
    if (a) ok = std::fread(a, sizeof(double), n, in.f) == n;
    else ok = fseeko(in.f, (off_t)(n * sizeof(double)), SEEK_CUR) == 0;
  }
  if (!ok) return fail(nullptr, NBR_ERR_IO, std::string("snapshot: short read on ") + path);
  if (time) *time = t;
  return NBR_OK;
}

extern "C" int nbr_snapshot_save(nbr_ctx* c, const char* path, size_t time_step, double delta_t) {
  TraceRange trace_range("nbr_snapshot_save");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  SysState& s = c->sys;
  if (s.n == 0) return fail(c, NBR_ERR_NO_SYSTEM, "no system uploaded");
  cudaSetDevice(c->device);
  const size_t n = s.n;
  std::vector<double> h(kFields * n, 0.0);
  double* H[kFields];
  for (size_t k = 0; k < kFields; ++k) H[k] = h.data() + k * n;
  const double* D[7] = {s.mass, s.pos[s.cur][0], s.pos[s.cur][1], s.pos[s.cur][2],
                        s.vel[0], s.vel[1], s.vel[2]};
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 7 && e == cudaSuccess; ++k)
    e = cudaMemcpyAsync(H[k], D[k], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  // Forces m_i a_i of the current positions when the context holds them
  // (after nbr_forces, nbr_forces_device or a KDK nbr_run), else zeros.
  const bool forces = c->acc_ok;
  for (int d = 0; d < 3 && forces && e == cudaSuccess; ++d)
    e = cudaMemcpyAsync(H[7 + d], s.acc[d], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "snapshot download");
  if (forces)
    for (int d = 0; d < 3; ++d)
      for (size_t i = 0; i < n; ++i) H[7 + d][i] *= H[0][i];
  const int rc = nbr_snapshot_write_arrays(path, n, time_step, delta_t, H[0], H[1], H[2], H[3],
                                           H[4], H[5], H[6], H[7], H[8], H[9]);
  if (rc) return fail(c, rc, nbr_last_error_string(nullptr));
  return NBR_OK;
}

extern "C" int nbr_snapshot_load(nbr_ctx* c, const char* path, size_t n, size_t record,
                                 double* time) {
  TraceRange trace_range("nbr_snapshot_load");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  std::vector<double> h(7 * n);
  double* H[7];
  for (size_t k = 0; k < 7; ++k) H[k] = h.data() + k * n;
  int rc = nbr_snapshot_read_arrays(path, n, record, time, H[0], H[1], H[2], H[3], H[4], H[5],
                                    H[6], nullptr, nullptr, nullptr);
  if (rc) return fail(c, rc, nbr_last_error_string(nullptr));
  return nbr_system_upload(c, n, H[1], H[2], H[3], H[4], H[5], H[6], H[0]);
}
