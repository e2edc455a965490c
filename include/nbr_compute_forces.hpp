// nbr_compute_forces.hpp -- the reference-signature drop-in for the force call.
//
// compute_forces_gpu has the signature of the reference's force kernels
// (compute_forces_simple / _avx2 / _avx2_blocked / _avx512_rsqrt_blocked /
// _avx512_rsqrt_4i_blocked, CPU/force_calculation.h:7-14), so a caller such as
// reduced_solver_omp_lf (CPU/omp_solver.cpp:364) or hybrid_ring_solver
// (CPU/hybrid_solver.cpp:84-95) can call it in their place.  It is a template
// over the state type so it binds to the reference's NBody_system
// (CPU/nbody_system.h:41-74: N, mass, pos[3], force[3], static G) without this
// header depending on that one.
//
// Contract, matched to the reference's:
//   * the callee ACCUMULATES into nb_sys.force (the caller zeroes it first,
//     CPU/omp_solver.cpp:343-355) -- here the full force of the received block
//     on the local block is added;
//   * recv_force is left untouched: the GPU evaluates every ordered pair
//     instead of the Newton-3 half, so the reaction forces the reference would
//     send back in recv_force are already included on their owner's side, and
//     the caller's force += recv_force (CPU/omp_solver.cpp:381-383) adds zero;
//   * local_force / local_recv_force / num_threads (per-thread CPU scratch)
//     are not used;
//   * no softening (eps = 0): pairs at zero distance are skipped, as the
//     reference skips q == k.
// The reference has no error channel; a failing call leaves nb_sys.force
// unchanged, prints the reason to stderr and is visible through
// nbr_dropin::last_status().  Environment: NBR_DEVICE (default 0),
// NBR_PRECISION=fp32c selects the FP32-compensated kernel (default fp64).
#pragma once

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nbr.h"

namespace nbr_dropin {

inline int& status_ref() {
  static int st = NBR_OK;
  return st;
}
inline int last_status() { return status_ref(); }

// Process-wide context, created on first use.
inline nbr_ctx* default_ctx() {
  static nbr_ctx* ctx = [] {
    nbr_ctx* c = nullptr;
    const char* dev = std::getenv("NBR_DEVICE");
    int rc = nbr_ctx_create(dev ? std::atoi(dev) : 0, &c);
    if (rc != NBR_OK) {
      std::fprintf(stderr, "nbr: no GPU context (%s)\n", nbr_last_error_string(nullptr));
      status_ref() = rc;
      return static_cast<nbr_ctx*>(nullptr);
    }
    return c;
  }();
  return ctx;
}

inline int precision_from_env() {
  const char* p = std::getenv("NBR_PRECISION");
  return (p && std::strcmp(p, "fp32c") == 0) ? NBR_FP32C : NBR_FP64;
}

}  // namespace nbr_dropin

template <class System>
void compute_forces_gpu(System& nb_sys, double* recv_pos[3], double* recv_force[3],
                        double*** local_force, double*** local_recv_force, size_t local_N,
                        size_t rank, size_t comm_sz, size_t recv_round, size_t num_threads) {
  (void)recv_force; (void)local_force; (void)local_recv_force; (void)num_threads;
  nbr_ctx* ctx = nbr_dropin::default_ctx();
  if (!ctx) return;
  if (comm_sz == 0) comm_sz = 1;
  // Local block: nb_sys.pos[*][0 .. local_N) with masses mass[rank * local_N ..];
  // received block: recv_pos with masses mass[((rank + recv_round) % comm_sz) * local_N ..]
  // (the offsets of CPU/force_calculation.cpp:62-69).
  const double* m_local = nb_sys.mass + rank * local_N;
  const double* m_recv = nb_sys.mass + ((rank + recv_round) % comm_sz) * local_N;
  std::vector<double> f(3 * local_N);
  const int rc = nbr_accel_ij(ctx, nbr_dropin::precision_from_env(), local_N, nb_sys.pos[0],
                              nb_sys.pos[1], nb_sys.pos[2], m_local, local_N, recv_pos[0],
                              recv_pos[1], recv_pos[2], m_recv, System::G, 0.0, 1, f.data(),
                              f.data() + local_N, f.data() + 2 * local_N);
  nbr_dropin::status_ref() = rc;
  if (rc != NBR_OK) {
    std::fprintf(stderr, "nbr: compute_forces_gpu failed: %s\n", nbr_last_error_string(ctx));
    return;
  }
  for (size_t i = 0; i < local_N; ++i) {
    nb_sys.force[0][i] += f[i];
    nb_sys.force[1][i] += f[local_N + i];
    nb_sys.force[2][i] += f[2 * local_N + i];
  }
}
