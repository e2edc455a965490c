// ref_glue.cpp -- C entry points over the reference's own CPU solver.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the UNMODIFIED reference sources CPU/nbody_system.cpp,
// CPU/force_calculation.cpp and CPU/omp_solver.cpp (read in place from the
// reference tree) into oracle/_ref/libnbr_ref_*.so.  Only tests/, the smoke
// check and bench.py's CPU-baseline / reference arm load that library, and only
// to check or to time against; the product never links it.
//
// Every function copies plain arrays into a reference NBody_system
// (CPU/nbody_system.h:41-74, alloc_particles at CPU/nbody_system.cpp:177-193),
// calls the reference routine exactly as the reference's own drivers do, and
// copies the result back out.  The reference prints progress to stdout from
// inside its solvers; the calls below silence file descriptor 1 around them so
// a caller that speaks JSON on stdout stays clean.

#include "nbody_system.h"
#include "force_calculation.h"
#include "omp_solver.h"

#include <omp.h>
#include <unistd.h>
#include <fcntl.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>

// CPU/omp_solver.h:11 declares a 7-argument reduced_solver_omp_lf that is never
// defined; the definition at CPU/omp_solver.cpp:257 takes a trailing Data_type.
void reduced_solver_omp_lf(NBody_system& nb_sys, size_t time_steps, double delta_t,
                           double* c, double* d, size_t lf_steps, bool blocked,
                           Data_type data_type);

namespace {

struct Quiet {
  int saved = -1;
  Quiet() {
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
  }
  ~Quiet() {
    fflush(stdout);
    if (saved >= 0) { dup2(saved, 1); close(saved); }
  }
};

void load(NBody_system& s, size_t n, const double* x, const double* y, const double* z,
          const double* vx, const double* vy, const double* vz, const double* m) {
  s.alloc_particles(n, n);
  for (size_t i = 0; i < n; ++i) {
    s.pos[X][i] = x[i]; s.pos[Y][i] = y[i]; s.pos[Z][i] = z[i];
    s.vel[X][i] = vx ? vx[i] : 0.0; s.vel[Y][i] = vy ? vy[i] : 0.0; s.vel[Z][i] = vz ? vz[i] : 0.0;
    s.force[X][i] = s.force[Y][i] = s.force[Z][i] = 0.0;
    s.mass[i] = m[i];
    s.mass_sp[i] = float(m[i]);
    s.pos_sp[X][i] = float(x[i]); s.pos_sp[Y][i] = float(y[i]); s.pos_sp[Z][i] = float(z[i]);
    s.vel_sp[X][i] = float(s.vel[X][i]); s.vel_sp[Y][i] = float(s.vel[Y][i]); s.vel_sp[Z][i] = float(s.vel[Z][i]);
    s.force_sp[X][i] = s.force_sp[Y][i] = s.force_sp[Z][i] = 0.0f;
  }
}

double* aalloc(size_t n) {
  size_t bytes = ((n * sizeof(double) + 63) / 64) * 64;
  if (bytes == 0) bytes = 64;
  return static_cast<double*>(aligned_alloc(64, bytes));
}

// Scratch exactly as reduced_solver_omp allocates it (CPU/omp_solver.cpp:20-57).
struct Scratch {
  size_t threads, n;
  double*** lf; double*** lrf;
  double* rp[DIM]; double* rf[DIM];
  Scratch(size_t n_, size_t threads_) : threads(threads_), n(n_) {
    lf = static_cast<double***>(malloc(threads * sizeof(double**)));
    lrf = static_cast<double***>(malloc(threads * sizeof(double**)));
    for (size_t t = 0; t < threads; ++t) {
      lf[t] = static_cast<double**>(malloc(DIM * sizeof(double*)));
      lrf[t] = static_cast<double**>(malloc(DIM * sizeof(double*)));
      for (int d = 0; d < DIM; ++d) { lf[t][d] = aalloc(n); lrf[t][d] = aalloc(n); }
    }
    for (int d = 0; d < DIM; ++d) { rp[d] = aalloc(n); rf[d] = aalloc(n); }
  }
  ~Scratch() {
    for (size_t t = 0; t < threads; ++t) {
      for (int d = 0; d < DIM; ++d) { free(lf[t][d]); free(lrf[t][d]); }
      free(lf[t]); free(lrf[t]);
    }
    free(lf); free(lrf);
    for (int d = 0; d < DIM; ++d) { free(rp[d]); free(rf[d]); }
  }
};

typedef void (*force_fn)(NBody_system&, double**, double**, double***, double***,
                         size_t, size_t, size_t, size_t, size_t);

force_fn pick(int variant) {
  switch (variant) {
    case 0: return compute_forces_simple;                    // CPU/force_calculation.cpp:34
    case 1: return compute_forces_avx2;                      // :109
    case 2: return compute_forces_avx2_blocked;              // :477
#ifdef __AVX512F__
    case 3: return compute_forces_avx512_rsqrt_blocked;      // :894
    case 4: return compute_forces_avx512_rsqrt_4i_blocked;   // :1137
#endif
    default: return nullptr;
  }
}

// Yoshida weights -> DKD c/d tables, the construction of CPU/omp_solver.cpp:677-726.
size_t yoshida(int order, double* c, double* d) {
  double w2[] = {1.0};
  double w4[] = {-std::cbrt(2.0) / (2.0 - std::cbrt(2.0)), 1.0 / (2.0 - std::cbrt(2.0))};
  double w6[] = {1.0, -1.17767998417887, 0.235573213359357, 0.78451361047756};
  for (size_t i = 1; i < 4; ++i) w6[0] -= 2.0 * w6[i];
  double w8[] = {1.0, -0.161582374150097e1, -0.244699182370524e1, -0.716989419708120e-2,
                 0.244002732616735e1, 0.157739928123617, 0.182020630970714e1, 0.104242620869991e1};
  for (size_t i = 1; i < 8; ++i) w8[0] -= 2.0 * w8[i];
  double* w = w2; size_t ws = 1;
  if (order == 4) { w = w4; ws = 2; }
  else if (order == 6) { w = w6; ws = 4; }
  else if (order == 8) { w = w8; ws = 8; }
  for (size_t i = 0; i < ws; ++i) {
    if (i == 0) c[i] = c[2 * ws - 1 - i] = w[ws - 1] / 2.0;
    else c[i] = c[2 * ws - 1 - i] = (w[ws - i] + w[ws - 1 - i]) / 2.0;
    d[i] = d[2 * ws - 2 - i] = w[ws - 1 - i];
  }
  return 2 * ws;
}

}  // namespace

extern "C" {

int ref_has_avx512(void) {
#ifdef __AVX512F__
  return 1;
#else
  return 0;
#endif
}

int ref_max_threads(void) { return omp_get_max_threads(); }
void ref_set_threads(int t) { if (t > 0) omp_set_num_threads(t); }

// Full force F_k = m_k a_k on every particle (eps = 0), through one of the
// reference kernels, called the way reduced_solver_omp calls it
// (CPU/omp_solver.cpp:60-103): zero force and recv_force, recv_pos = pos,
// then force += recv_force (:124-126).
int ref_forces(int variant, size_t n, const double* x, const double* y, const double* z,
               const double* m, double* fx, double* fy, double* fz) {
  force_fn f = pick(variant);
  if (!f || n == 0) return -1;
  Quiet q;
  NBody_system s;
  load(s, n, x, y, z, nullptr, nullptr, nullptr, m);
  size_t threads = omp_get_max_threads();
  Scratch sc(n, threads);
  for (size_t i = 0; i < n; ++i)
    for (int d = 0; d < DIM; ++d) { sc.rp[d][i] = s.pos[d][i]; sc.rf[d][i] = 0.0; s.force[d][i] = 0.0; }
  f(s, sc.rp, sc.rf, sc.lf, sc.lrf, n, 0, 1, 0, threads);
  for (size_t i = 0; i < n; ++i) {
    fx[i] = s.force[X][i] + sc.rf[X][i];
    fy[i] = s.force[Y][i] + sc.rf[Y][i];
    fz[i] = s.force[Z][i] + sc.rf[Z][i];
  }
  return 0;
}

// Symplectic DKD leapfrog of the given order through reduced_solver_omp_lf
// (CPU/omp_solver.cpp:257-456), AVX2-blocked FP64 forces, eps = 0.  Updates
// the state arrays in place.  Returns the seconds the solver took.
double ref_lf(size_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
              const double* m, size_t steps, double dt, int order) {
  Quiet q;
  NBody_system s;
  load(s, n, x, y, z, vx, vy, vz, m);
  double c[16], d[16];
  size_t lf_steps = yoshida(order, c, d);
  double t0 = omp_get_wtime();
  reduced_solver_omp_lf(s, steps, dt, c, d, lf_steps, true, Data_type::DOUBLE_PRECISION);
  double t1 = omp_get_wtime();
  for (size_t i = 0; i < n; ++i) {
    x[i] = s.pos[X][i]; y[i] = s.pos[Y][i]; z[i] = s.pos[Z][i];
    vx[i] = s.vel[X][i]; vy[i] = s.vel[Y][i]; vz[i] = s.vel[Z][i];
  }
  return t1 - t0;
}

// Euler steps through reduced_solver_omp (CPU/omp_solver.cpp:16-178) with the
// given kernel (2 = AVX2 blocked, 4 = AVX-512 rsqrt 4i).  Returns seconds.
double ref_euler(size_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                 const double* m, size_t steps, double dt, int variant) {
  Vectorization_type vt = Vectorization_type::AVX2;
#ifdef __AVX512F__
  if (variant == 4) vt = Vectorization_type::AVX512RSQRT4I;
  if (variant == 3) vt = Vectorization_type::AVX512RSQRT;
#endif
  Quiet q;
  NBody_system s;
  load(s, n, x, y, z, vx, vy, vz, m);
  double t0 = omp_get_wtime();
  reduced_solver_omp(s, steps, dt, true, vt, Data_type::DOUBLE_PRECISION);
  double t1 = omp_get_wtime();
  for (size_t i = 0; i < n; ++i) {
    x[i] = s.pos[X][i]; y[i] = s.pos[Y][i]; z[i] = s.pos[Z][i];
    vx[i] = s.vel[X][i]; vy[i] = s.vel[Y][i]; vz[i] = s.vel[Z][i];
  }
  return t1 - t0;
}

// Rank 0's share of one force evaluation of the reference's ring
// decomposition (hybrid_ring_solver, CPU/hybrid_solver.cpp:14-107): the
// system is cut into comm_sz blocks, block 0 is "this rank", and for every
// recv_round the block (0 + recv_round) % comm_sz is the received message.
// The message passing itself is replaced by pointing recv_pos at that block.
// That share is N(N-1)/comm_sz effective pairs.  Returns seconds of compute.
double ref_ring_share(size_t n, const double* x, const double* y, const double* z,
                      const double* m, size_t comm_sz, int variant) {
  force_fn f = pick(variant);
  if (!f || comm_sz == 0 || n % comm_sz != 0) return -1.0;
  size_t local_n = n / comm_sz;
  Quiet q;
  NBody_system s;
  s.alloc_particles(n, n);
  for (size_t i = 0; i < n; ++i) {
    s.pos[X][i] = x[i]; s.pos[Y][i] = y[i]; s.pos[Z][i] = z[i];
    s.mass[i] = m[i];
    s.force[X][i] = s.force[Y][i] = s.force[Z][i] = 0.0;
  }
  size_t threads = omp_get_max_threads();
  Scratch sc(local_n, threads);
  double secs = 0.0;
  for (size_t round = 0; round < comm_sz; ++round) {
    size_t src = round % comm_sz;
    for (size_t i = 0; i < local_n; ++i)
      for (int d = 0; d < DIM; ++d) { sc.rp[d][i] = s.pos[d][src * local_n + i]; sc.rf[d][i] = 0.0; }
    double t0 = omp_get_wtime();
    f(s, sc.rp, sc.rf, sc.lf, sc.lrf, local_n, 0, comm_sz, round, threads);
    secs += omp_get_wtime() - t0;
  }
  return secs;
}

double ref_kinetic(size_t n, const double* vx, const double* vy, const double* vz, const double* m) {
  NBody_system s;
  std::vector<double> zero(n, 0.0);
  load(s, n, zero.data(), zero.data(), zero.data(), vx, vy, vz, m);
  return compute_kinetic_energy(s);  // CPU/force_calculation.cpp:1740-1748
}

// variant 0: calculate_potential_energy (scalar, :1880-1904);
// variant 1: compute_potential_energy_avx2 (:1749-1879).
double ref_potential(size_t n, const double* x, const double* y, const double* z, const double* m,
                     int variant) {
  Quiet q;
  NBody_system s;
  load(s, n, x, y, z, nullptr, nullptr, nullptr, m);
  return variant == 0 ? calculate_potential_energy(s) : compute_potential_energy_avx2(s);
}

// Ring initial condition with analytic forces
// (init_stable_orbiting_particles, CPU/nbody_system.cpp:319-384).
int ref_ring_init(size_t n, double R, double omega, double ratio, double* x, double* y, double* z,
                  double* vx, double* vy, double* vz, double* m, double* fx, double* fy, double* fz) {
  if (n < 2) return -1;
  NBody_system s;
  s.init_stable_orbiting_particles(n, R, omega, ratio);
  for (size_t i = 0; i < n; ++i) {
    x[i] = s.pos[X][i]; y[i] = s.pos[Y][i]; z[i] = s.pos[Z][i];
    vx[i] = s.vel[X][i]; vy[i] = s.vel[Y][i]; vz[i] = s.vel[Z][i];
    m[i] = s.mass[i];
    fx[i] = s.force[X][i]; fy[i] = s.force[Y][i]; fz[i] = s.force[Z][i];
  }
  return 0;
}

// Analytic rigid rotation after `step` of `steps_per_rev` steps
// (predict_stable_orbiting_particles, CPU/nbody_system.cpp:386-408).
int ref_ring_predict(size_t n, double R, double omega, size_t step, size_t steps_per_rev,
                     double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  if (n < 2) return -1;
  NBody_system s;
  s.init_stable_orbiting_particles(n, R, omega, 1.0);
  s.predict_stable_orbiting_particles(R, omega, step, steps_per_rev);
  for (size_t i = 0; i < n; ++i) {
    x[i] = s.pos[X][i]; y[i] = s.pos[Y][i]; z[i] = s.pos[Z][i];
    vx[i] = s.vel[X][i]; vy[i] = s.vel[Y][i]; vz[i] = s.vel[Z][i];
  }
  return 0;
}

int ref_yoshida(int order, double* c, double* d) { return int(yoshida(order, c, d)); }

// `records` snapshot records of one state through NBody_system::save_particles
// (CPU/nbody_system.cpp:133-152), time steps 0 .. records-1: the reference
// writes "NBody_<n>.dat" in the working directory, so the call runs with
// `dir` as the working directory.  Returns 0, or -1 if dir is unusable.
int ref_save_snapshot(const char* dir, size_t n, const double* m, const double* x, const double* y,
                      const double* z, const double* vx, const double* vy, const double* vz,
                      const double* fx, const double* fy, const double* fz, size_t records,
                      double delta_t) {
  char old[4096];
  if (!getcwd(old, sizeof(old)) || chdir(dir) != 0) return -1;
  {
    NBody_system s;
    load(s, n, x, y, z, vx, vy, vz, m);
    for (size_t i = 0; i < n; ++i) {
      s.force[X][i] = fx[i]; s.force[Y][i] = fy[i]; s.force[Z][i] = fz[i];
    }
    for (size_t t = 0; t < records; ++t) s.save_particles(t, delta_t);
  }  // the destructor closes (flushes) the file
  return chdir(old) == 0 ? 0 : -1;
}

}  // extern "C"
