// nbr_main.cpp -- command-line driver with the reference's flag surface.
//
// Mirrors CPU/main.cpp: the same flags, defaults and validation
// (get_arguments, :11-289), dispatch on -t (:291-356), and the reference's
// experiment drivers re-targeted to the GPU through the C ABI:
//   -t gpu           omp_main (CPU/omp_solver.cpp:635-797): ring system by
//                    default, Euler or leapfrog of -order, MPairs/s and the
//                    deviation from the initial state;
//   -t gpu-bench     the scaling benchmark's CSV row (CPU/hybrid_solver.cpp:623-645);
//   -t gpu-accuracy  omp_accuracy (CPU/omp_solver.cpp:899-993);
//   -t gpu-ratio     omp_ratio_accuracy (CPU/omp_solver.cpp:995-1243);
//   -t gpu-batch     many independent systems in one persistent launch;
//   -t gpu-multi     one system over -ngpu GPUs from this one process: the
//                    Newton-3 slices of each GPU, an NCCL all-to-all of the
//                    partial forces and an NCCL all-gather of the positions
//                    per force evaluation (hybrid_ring_solver's partition of
//                    the pair work, CPU/hybrid_solver.cpp:14-224, on NVLink).
// Added flags: -eps (softening length), -dt (overrides T/s), -ic
// ring|plummer|ball|twocomp|random, -seed, -scheme dkd|kdk, -G, -nsys, -nmin,
// -nmax, -autotune, -save K (a record of the reference's snapshot format,
// NBody_<N>.dat as save_particles names it, at step 0 and every K steps) and
// -resume PATH (start from the last record of a snapshot file of N particles).
// -p accepts dp|sp (reference names) and fp64|fp32c; sp selects the
// FP32-compensated kernel.
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nccl.h>

#include "nbr.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Args {
  size_t N = 1000, start_N = 1000, step_N = 1000, num_steps = 1, time_steps = 1000;
  double T = 1.0, ratio = 100000.0, ratio_start = 1e6, ratio_stop = 1e9;
  size_t ratio_steps = 3, rev_steps = 1000;
  double max_error = 1.0;
  bool verbose = false;
  std::string output = "output.csv";
  bool output_given = false;
  std::string exec = "gpu";
  std::string integ = "euler";
  int order = 1;
  int precision = NBR_FP64;
  // added
  double eps = 0.0, dt = 0.0, G = 1.0;
  std::string ic = "ring";
  uint64_t seed = 0;
  int scheme = NBR_DKD;
  size_t nsys = 4096, nmin = 64, nmax = 4096;
  bool autotune = false;
  int device = 0;
  size_t save_every = 0;  // -save K: snapshot every K steps (NBody_<N>.dat)
  std::string resume;     // -resume PATH: start from the file's last record
  int ngpu = 1;           // -ngpu W: GPUs of -t gpu-multi
  int slices = 0;         // -slices V: Newton-3 slices (0: max(8, W))
  std::string final_snapshot;  // -final PATH: the end state as one snapshot record
};

bool parse(int argc, char** argv, Args& a) {
  for (int i = 1; i < argc; ++i) {
    auto is = [&](const char* f) { return std::strcmp(argv[i], f) == 0 && i + 1 < argc; };
    if (is("-N")) a.N = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-start")) a.start_N = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-step")) a.step_N = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-n")) a.num_steps = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-ratio-start")) a.ratio_start = std::atof(argv[++i]);
    else if (is("-ratio-stop")) a.ratio_stop = std::atof(argv[++i]);
    else if (is("-ratio-steps")) a.ratio_steps = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-rev-steps")) a.rev_steps = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-max-error")) a.max_error = std::atof(argv[++i]);
    else if (is("-s")) a.time_steps = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-T")) a.T = std::atof(argv[++i]);
    else if (is("-r")) a.ratio = std::atof(argv[++i]);
    else if (std::strcmp(argv[i], "-v") == 0) a.verbose = true;
    else if (std::strcmp(argv[i], "-autotune") == 0) a.autotune = true;
    else if (is("-o")) { a.output = argv[++i]; a.output_given = true; }
    else if (is("-t")) {
      std::string t = argv[++i];
      static const char* known[] = {"gpu", "gpu-bench", "gpu-accuracy", "gpu-ratio", "gpu-batch",
                                    "gpu-multi"};
      bool ok = false;
      for (auto k : known) ok |= (t == k);
      if (!ok) {
        std::printf("Unknown Execution type: %s\n Defaulting to gpu\n", t.c_str());
        t = "gpu";
      }
      a.exec = t;
    } else if (is("-i")) {
      std::string k = argv[++i];
      if (k != "euler" && k != "lf") {
        std::printf("Unknown or unsupported Integration kind: %s\n Defaulting to euler\n", k.c_str());
        k = "euler";
      }
      a.integ = k;
    } else if (is("-V") || is("-S")) {
      ++i;  // CPU vectorisation / Newton-3 choices have no GPU meaning
    } else if (is("-p")) {
      std::string k = argv[++i];
      if (k == "dp" || k == "fp64") a.precision = NBR_FP64;
      else if (k == "sp" || k == "fp32c") a.precision = NBR_FP32C;
      else std::printf("Unknown Data type: %s\n Defaulting to double precision\n", k.c_str());
    } else if (is("-order")) a.order = (int)std::strtoull(argv[++i], nullptr, 10);
    else if (is("-eps")) a.eps = std::atof(argv[++i]);
    else if (is("-dt")) a.dt = std::atof(argv[++i]);
    else if (is("-G")) a.G = std::atof(argv[++i]);
    else if (is("-ic")) a.ic = argv[++i];
    else if (is("-seed")) a.seed = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-scheme")) a.scheme = std::strcmp(argv[++i], "kdk") == 0 ? NBR_KDK : NBR_DKD;
    else if (is("-nsys")) a.nsys = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-nmin")) a.nmin = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-nmax")) a.nmax = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-device")) a.device = std::atoi(argv[++i]);
    else if (is("-save")) a.save_every = std::strtoull(argv[++i], nullptr, 10);
    else if (is("-resume")) a.resume = argv[++i];
    else if (is("-ngpu")) a.ngpu = std::atoi(argv[++i]);
    else if (is("-slices")) a.slices = std::atoi(argv[++i]);
    else if (is("-final")) a.final_snapshot = argv[++i];
  }
  // Validation and resets of CPU/main.cpp:271-288.
  if (a.N >= 100000000 || a.start_N >= 100000000 ||
      a.start_N + a.step_N * a.num_steps >= 100000000) {
    std::printf("Input problem size might be too large!\nMake sure to stay below 10^8 particles.\nResetting to defaults");
    a.N = 1000; a.start_N = 1000; a.step_N = 1000; a.num_steps = 1;
  }
  if (a.T <= 0.0) { std::printf("T has to be >= 0!\n Resetting to 1.0\n"); a.T = 1.0; }
  if (a.ratio < 0.0) { std::printf("ratio has to be >= 0!\n Resetting to 1e6\n"); a.ratio = 1e6; }
  return true;
}

struct State {
  size_t n = 0;
  std::vector<double> x, y, z, vx, vy, vz, m, fx, fy, fz;
  void resize(size_t k) {
    n = k;
    for (auto* v : {&x, &y, &z, &vx, &vy, &vz, &m, &fx, &fy, &fz}) v->assign(k, 0.0);
  }
};

int make_ic(const Args& a, size_t n, double ratio, State& s) {
  s.resize(n);
  if (a.ic == "ring")
    return nbr_ic_ring(n, 1.0, 2.0 * kPi, ratio, s.x.data(), s.y.data(), s.z.data(), s.vx.data(),
                       s.vy.data(), s.vz.data(), s.m.data(), s.fx.data(), s.fy.data(), s.fz.data());
  if (a.ic == "plummer")
    return nbr_ic_plummer(n, a.seed, s.x.data(), s.y.data(), s.z.data(), s.vx.data(), s.vy.data(),
                          s.vz.data(), s.m.data());
  if (a.ic == "ball")
    return nbr_ic_uniform_ball(n, a.seed, s.x.data(), s.y.data(), s.z.data(), s.vx.data(),
                               s.vy.data(), s.vz.data(), s.m.data());
  if (a.ic == "twocomp")
    return nbr_ic_two_component(n, (size_t)std::llround(0.01 * double(n)), 1000.0, a.seed,
                                s.x.data(), s.y.data(), s.z.data(), s.vx.data(), s.vy.data(),
                                s.vz.data(), s.m.data());
  if (a.ic == "random") {
    // The reference's init_particles (CPU/nbody_system.cpp:238-274) with a seed:
    // masses U(0, 1e6), positions U(-1, 1), velocities U(-0.01, 0.01).
    std::mt19937_64 g(a.seed);
    auto u = [&](double lo, double hi) { return lo + (hi - lo) * (double(g() >> 11) * 0x1.0p-53); };
    for (size_t i = 0; i < n; ++i) {
      s.m[i] = u(0.0, 1e6);
      s.x[i] = u(-1, 1); s.y[i] = u(-1, 1); s.z[i] = u(-1, 1);
      s.vx[i] = u(-0.01, 0.01); s.vy[i] = u(-0.01, 0.01); s.vz[i] = u(-0.01, 0.01);
    }
    return NBR_OK;
  }
  std::printf("Unknown initial condition %s\n", a.ic.c_str());
  return NBR_ERR_INVALID_ARG;
}

// print_deviation (CPU/nbody_system.cpp:500-519): mean |calc - ref|.
void print_deviation(const std::vector<double>& cx, const std::vector<double>& cy,
                     const std::vector<double>& cz, const State& r, bool vel, const char* kind) {
  const auto& rx = vel ? r.vx : r.x;
  const auto& ry = vel ? r.vy : r.y;
  const auto& rz = vel ? r.vz : r.z;
  double mean = 0.0;
  for (size_t i = 0; i < cx.size(); ++i)
    mean += std::sqrt((cx[i] - rx[i]) * (cx[i] - rx[i]) + (cy[i] - ry[i]) * (cy[i] - ry[i]) +
                      (cz[i] - rz[i]) * (cz[i] - rz[i]));
  mean /= double(cx.size());
  std::printf("Average %s deviation from reference: %.13f\n", kind, mean);
}

// calculate_deviation (CPU/nbody_system.cpp:521-540): mean distance and the
// largest relative length error.
void deviation(const double* cx, const double* cy, const double* cz, const double* rx,
               const double* ry, const double* rz, size_t n, double& mean, double& maxlen) {
  mean = 0.0;
  maxlen = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double dx = cx[i] - rx[i], dy = cy[i] - ry[i], dz = cz[i] - rz[i];
    mean += std::sqrt(dx * dx + dy * dy + dz * dz);
    const double lc = std::sqrt(cx[i] * cx[i] + cy[i] * cy[i] + cz[i] * cz[i]);
    const double lr = std::sqrt(rx[i] * rx[i] + ry[i] * ry[i] + rz[i] * rz[i]);
    if (lr > 0.0 && std::fabs(lc - lr) / lr > maxlen) maxlen = std::fabs(lc - lr) / lr;
  }
  mean /= double(n);
}

bool file_exists(const std::string& p) { return access(p.c_str(), F_OK) != -1; }

int run_gpu(nbr_ctx* ctx, const Args& a, bool bench) {
  State s;
  const double dt = a.dt > 0.0 ? a.dt : a.T / double(a.time_steps);
  const double eps2 = a.eps * a.eps;
  size_t step0 = 0;
  std::printf("N = %zu, s = %zu\n", a.N, a.time_steps);
  if (!a.resume.empty()) {
    size_t records = 0;
    double t = 0.0;
    if (nbr_snapshot_records(a.resume.c_str(), a.N, &records) != NBR_OK || records == 0 ||
        nbr_snapshot_load(ctx, a.resume.c_str(), a.N, records - 1, &t) != NBR_OK) {
      std::printf("resume failed: %s\n", nbr_last_error_string(ctx));
      return 1;
    }
    step0 = dt > 0.0 ? (size_t)std::llround(t / dt) : 0;
    std::printf("Resumed from %s, record %zu (t = %f, step %zu)\n", a.resume.c_str(), records - 1, t,
                step0);
    s.resize(a.N);
    nbr_system_download(ctx, s.x.data(), s.y.data(), s.z.data(), s.vx.data(), s.vy.data(),
                        s.vz.data());
  } else {
    if (make_ic(a, a.N, a.ratio, s) != NBR_OK) return 1;
    if (nbr_system_upload(ctx, s.n, s.x.data(), s.y.data(), s.z.data(), s.vx.data(), s.vy.data(),
                          s.vz.data(), s.m.data()) != NBR_OK) {
      std::printf("upload failed: %s\n", nbr_last_error_string(ctx));
      return 1;
    }
  }
  State ref = s;
  if (a.autotune) nbr_autotune(ctx, a.precision, eps2);
  nbr_diag d[2];
  nbr_run_stats st{};
  int rc = NBR_OK;
  double evals_per_step = 1.0;
  int scheme = NBR_EULER, use_order = 1;
  if (a.integ == "lf") {
    const int order = a.order < 2 ? 2 : a.order;
    double c[16], dd[16];
    const int lf = nbr_yoshida_coefficients(order, c, dd);
    use_order = lf ? order : 2;
    if (!lf) std::printf("Order %d not supported! Defaulting to 2nd order\n", order);
    if (a.scheme == NBR_KDK && use_order != 2) {
      std::printf("KDK is second order; using DKD for order %d\n", use_order);
    }
    scheme = use_order == 2 ? a.scheme : NBR_DKD;
    evals_per_step = scheme == NBR_DKD ? double((lf ? lf : 2) - 1) : 1.0;
  }
  auto t0 = std::chrono::steady_clock::now();
  if (a.save_every == 0) {
    rc = nbr_run(ctx, a.precision, scheme, use_order, dt, a.time_steps, a.G, eps2, d, &st);
  } else {
    // Chunks of save_every steps and a snapshot record after each.  A fresh
    // run first writes the initial state as record 0 (truncating the file); a
    // resumed run appends, its starting state being the record it came from.
    const std::string snap = "NBody_" + std::to_string(a.N) + ".dat";
    if (a.resume.empty()) rc = nbr_snapshot_save(ctx, snap.c_str(), 0, dt);
    size_t done = 0;
    while (rc == NBR_OK && done < a.time_steps) {
      const size_t k = std::min(a.save_every, a.time_steps - done);
      nbr_diag dk[2];
      nbr_run_stats sk{};
      rc = nbr_run(ctx, a.precision, scheme, use_order, dt, k, a.G, eps2, dk, &sk);
      if (rc != NBR_OK) break;
      if (done == 0) d[0] = dk[0];
      d[1] = dk[1];
      st.gpu_ms += sk.gpu_ms;
      st.force_evals += sk.force_evals;
      st.pairs += sk.pairs;
      st.kernels += sk.kernels;
      done += k;
      rc = nbr_snapshot_save(ctx, snap.c_str(), step0 + done, dt);
    }
    if (rc == NBR_OK) std::printf("Snapshots written to %s\n", snap.c_str());
  }
  auto t1 = std::chrono::steady_clock::now();
  if (rc != NBR_OK) {
    std::printf("run failed: %s\n", nbr_last_error_string(ctx));
    return 1;
  }
  const double wall = std::chrono::duration<double>(t1 - t0).count();
  const double t_gpu = st.gpu_ms * 1e-3;
  const double pairs = double(a.time_steps) * evals_per_step * double(a.N) * double(a.N - 1);
  const double mpairs = t_gpu > 0 ? pairs / (1e6 * t_gpu) : 0.0;
  std::printf("GPU %s solver took %fs (wall %fs)\n", a.integ == "lf" ? "symplectic" : "Euler", t_gpu, wall);
  std::printf("Performance: %fMPairs/s\n", mpairs);
  std::printf("Energy: E0 = %.12e  E1 = %.12e  |dE/E0| = %.3e\n", d[0].E, d[1].E,
              d[0].E != 0.0 ? std::fabs((d[1].E - d[0].E) / d[0].E) : 0.0);
  std::vector<double> x(a.N), y(a.N), z(a.N), vx(a.N), vy(a.N), vz(a.N);
  nbr_system_download(ctx, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data());
  print_deviation(x, y, z, ref, false, "position");
  print_deviation(vx, vy, vz, ref, true, "velocity");
  if (bench || a.output_given) {
    const bool exists = file_exists(a.output);
    FILE* f = std::fopen(a.output.c_str(), exists ? "a" : "w");
    if (!f) {
      std::perror("Failed to open output file: ");
      return 1;
    }
    if (!exists)
      std::fprintf(f, "#Nodes, Cores, N, t_total[s], performance[Mpairs/s], time_steps/s, ms/time_step\n");
    std::fprintf(f, "%d,%d,%zu,%f,%f,%f,%f\n", 1, nbr_device_count() > 0 ? 148 : 0, a.N, t_gpu,
                 mpairs, double(a.time_steps) / t_gpu, t_gpu * 1000.0 / double(a.time_steps));
    std::fclose(f);
  }
  return 0;
}

// omp_accuracy on the GPU: one force evaluation of the permuted ring against
// the analytic ring forces, averaged length and angle errors in percent.
int run_accuracy(nbr_ctx* ctx, const Args& a) {
  const bool exists = file_exists(a.output);
  FILE* f = std::fopen(a.output.c_str(), exists ? "a" : "w");
  if (!f) { std::perror("Failed to open output file: "); return 1; }
  if (!exists)
    std::fprintf(f, "N, precision, ratio, average_force_length_error[%%], average_force_angle_error[%%]\n");
  const double root = std::pow(a.ratio_stop / a.ratio_start, 1.0 / double(a.ratio_steps));
  for (size_t rs = 0; rs <= a.ratio_steps; ++rs) {
    const double ratio = a.ratio_start * std::pow(root, double(rs));
    for (size_t k = 0; k < a.num_steps; ++k) {
      const size_t n = a.start_N * size_t(std::llround(std::pow(double(a.step_N), double(k))));
      Args ring = a;
      ring.ic = "ring";
      State s;
      make_ic(ring, n, ratio, s);
      std::vector<size_t> perm(n);
      std::iota(perm.begin(), perm.end(), 0);
      std::mt19937_64 g(a.seed);
      std::shuffle(perm.begin(), perm.end(), g);
      State p = s;
      for (size_t i = 0; i < n; ++i) {
        p.x[i] = s.x[perm[i]]; p.y[i] = s.y[perm[i]]; p.z[i] = s.z[perm[i]];
        p.m[i] = s.m[perm[i]];
        p.fx[i] = s.fx[perm[i]]; p.fy[i] = s.fy[perm[i]]; p.fz[i] = s.fz[perm[i]];
      }
      if (nbr_system_upload(ctx, n, p.x.data(), p.y.data(), p.z.data(), nullptr, nullptr, nullptr,
                            p.m.data()) != NBR_OK) {
        std::printf("upload failed: %s\n", nbr_last_error_string(ctx));
        std::fclose(f);
        return 1;
      }
      std::vector<double> fx(n), fy(n), fz(n);
      if (nbr_forces(ctx, a.precision, 1.0, 0.0, 1, fx.data(), fy.data(), fz.data()) != NBR_OK) {
        std::printf("forces failed: %s\n", nbr_last_error_string(ctx));
        std::fclose(f);
        return 1;
      }
      // calculate_force_error (CPU/nbody_system.cpp:542-652): angle in the
      // x-y plane, normalised by 2 pi; length error normalised by the length
      // of particle 0's reference force.
      double ang = 0.0, len = 0.0;
      for (size_t i = 0; i < n; ++i) {
        const double sl = std::sqrt(fx[i] * fx[i] + fy[i] * fy[i] + fz[i] * fz[i]);
        const double rl = std::sqrt(p.fx[i] * p.fx[i] + p.fy[i] * p.fy[i] + p.fz[i] * p.fz[i]);
        const double dot = fx[i] * p.fx[i] + fy[i] * p.fy[i];
        const double det = fx[i] * p.fy[i] - fy[i] * p.fx[i];
        if (p.fx[i] != 0.0 && p.fy[i] != 0.0) ang += std::fabs(std::atan2(det, dot));
        len += std::fabs(sl - rl);
      }
      const double r0 = std::sqrt(p.fx[0] * p.fx[0] + p.fy[0] * p.fy[0] + p.fz[0] * p.fz[0]);
      const double len_err = r0 > 0 ? len / (r0 * double(n)) : 0.0;
      const double ang_err = ang / (2.0 * kPi * double(n));
      std::printf("N = %zu ratio = %.3e: length error %.6e, angle error %.6e\n", n, ratio, len_err, ang_err);
      std::fprintf(f, "%zu, %s, %.5e, %.5e, %.6e\n", n, a.precision == NBR_FP64 ? "dp" : "sp", ratio,
                   len_err * 100.0, ang_err * 100.0);
    }
  }
  std::fclose(f);
  return 0;
}

// omp_ratio_accuracy on the GPU: DKD order 2 with dt = 1 / rev_steps, each
// step compared with the analytic rigid rotation and the initial energy;
// stops at the collapse criterion of CPU/omp_solver.cpp:1215.
int run_ratio(nbr_ctx* ctx, const Args& a) {
  const bool exists = file_exists(a.output);
  FILE* f = std::fopen(a.output.c_str(), exists ? "a" : "w");
  if (!f) { std::perror("Failed to open output file: "); return 1; }
  if (!exists)
    std::fprintf(f, "N, precision, s, s_collapse, ratio, max_error, last_E_dev, last_avg_pos_dev, last_avg_vel_dev, max_pos_dev, max_vel_dev\n");
  const double dt = 1.0 / double(a.rev_steps);
  for (size_t k = 0; k < a.num_steps; ++k) {
    const size_t n = a.start_N + k * a.step_N;
    const double root = std::pow(a.ratio_stop / a.ratio_start, 1.0 / double(a.ratio_steps));
    for (size_t rs = 0; rs <= a.ratio_steps; ++rs) {
      const double ratio = a.ratio_start * std::pow(root, double(rs));
      Args ring = a;
      ring.ic = "ring";
      State s;
      make_ic(ring, n, ratio, s);
      if (nbr_system_upload(ctx, n, s.x.data(), s.y.data(), s.z.data(), s.vx.data(), s.vy.data(),
                            s.vz.data(), s.m.data()) != NBR_OK) {
        std::fclose(f);
        return 1;
      }
      nbr_diag d0;
      nbr_diagnostics(ctx, 1.0, 0.0, &d0);
      size_t s_collapse = a.time_steps;
      double e_sol = 0, ap = 0, av = 0, mp = 0, mv = 0;
      std::vector<double> x(n), y(n), z(n), vx(n), vy(n), vz(n);
      std::vector<double> px(n), py(n), pz(n), pvx(n), pvy(n), pvz(n);
      for (size_t t = 1; t <= a.time_steps; ++t) {
        nbr_diag d[2];
        if (nbr_run(ctx, a.precision, NBR_DKD, 2, dt, 1, 1.0, 0.0, d, nullptr) != NBR_OK) {
          std::printf("run failed: %s\n", nbr_last_error_string(ctx));
          std::fclose(f);
          return 1;
        }
        nbr_system_download(ctx, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data());
        nbr_ic_ring_predict(n, 1.0, 2.0 * kPi, t, a.rev_steps, px.data(), py.data(), pz.data(),
                            pvx.data(), pvy.data(), pvz.data());
        double pmean, pmax, vmean, vmax;
        deviation(x.data(), y.data(), z.data(), px.data(), py.data(), pz.data(), n, pmean, pmax);
        deviation(vx.data(), vy.data(), vz.data(), pvx.data(), pvy.data(), pvz.data(), n, vmean, vmax);
        const double edev = std::fabs((d0.E - d[1].E) / d0.E);
        if (edev >= 1.0 || pmax >= a.max_error || vmax >= a.max_error) {
          s_collapse = t;
          break;
        }
        e_sol = edev; ap = pmean; av = vmean; mp = pmax; mv = vmax;
      }
      std::printf("true solution = %zu\n", s_collapse);
      std::fprintf(f, "%zu, %s, %zu, %zu, %f, %f, %f, %f, %f, %f, %f\n", n,
                   a.precision == NBR_FP64 ? "dp" : "sp", a.time_steps, s_collapse, ratio,
                   a.max_error, e_sol, ap, av, mp, mv);
    }
  }
  std::fclose(f);
  return 0;
}

int run_batch(nbr_ctx* ctx, const Args& a) {
  std::vector<size_t> sizes(a.nsys), off(a.nsys + 1, 0);
  nbr_ic_batch_sizes(a.nsys, a.seed, a.nmin, a.nmax, sizes.data());
  for (size_t s = 0; s < a.nsys; ++s) off[s + 1] = off[s] + sizes[s];
  const size_t n = off[a.nsys];
  State st;
  st.resize(n);
  for (size_t s = 0; s < a.nsys; ++s) {
    const size_t o = off[s];
    nbr_ic_plummer(sizes[s], nbr_ic_system_seed(a.seed, s), st.x.data() + o, st.y.data() + o,
                   st.z.data() + o, st.vx.data() + o, st.vy.data() + o, st.vz.data() + o,
                   st.m.data() + o);
  }
  if (nbr_batch_upload(ctx, a.nsys, off.data(), st.x.data(), st.y.data(), st.z.data(), st.vx.data(),
                       st.vy.data(), st.vz.data(), st.m.data()) != NBR_OK) {
    std::printf("batch upload failed: %s\n", nbr_last_error_string(ctx));
    return 1;
  }
  const double dt = a.dt > 0.0 ? a.dt : a.T / double(a.time_steps);
  nbr_run_stats rs{};
  if (nbr_batch_run(ctx, a.precision, dt, a.time_steps, a.G, a.eps * a.eps, &rs) != NBR_OK) {
    std::printf("batch run failed: %s\n", nbr_last_error_string(ctx));
    return 1;
  }
  const double secs = rs.gpu_ms * 1e-3;
  std::printf("systems = %zu, particles = %zu, steps = %zu\n", a.nsys, n, a.time_steps);
  std::printf("GPU batched solver took %fs: %.1f systems*steps/s, %.3f GPairs/s\n", secs,
              double(a.nsys) * double(a.time_steps) / secs, rs.pairs / secs * 1e-9);
  return 0;
}

// ------------------------------------------------------------ multi-GPU ----
// One process drives W GPUs (one libnbr context each, one NCCL communicator
// per GPU from ncclCommInitAll).  Rank r owns the receivers [r c, (r + 1) c),
// c = n / W rounded up to 128, and computes Newton-3 slices [r V / W,
// (r + 1) V / W) for every particle; per force evaluation:
//   1. nbr_n3_slice_accel for its slices (on its context's stream);
//   2. one NCCL group of point-to-point transfers: the columns of every
//      rank's receivers of each of its slices go to that rank (its own by a
//      device copy); rank r receives slice v's columns into recv[v];
//   3. nbr_step_range_sum: its receivers' V partials added in slice order,
//      then the fused kick/drift;
//   4. an in-place NCCL all-gather of x, y, z (MPI_Allgather of
//      hybrid_full_solver, CPU/hybrid_solver.cpp:310).
// The sum order depends on V only: any W <= V gives the same bits.
struct MultiRank {
  int dev = 0;
  nbr_ctx* ctx = nullptr;
  ncclComm_t comm = nullptr;
  cudaStream_t st = nullptr;
  size_t i0 = 0, owned = 0;
  int v0 = 0, v1 = 0;
  double* mine = nullptr;  // [v1 - v0][3][ld]
  double* recv = nullptr;  // [V][3][c]
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

int multi_fail(const char* what, const char* msg) {
  std::printf("gpu-multi: %s: %s\n", what, msg);
  return 1;
}

int run_multi(const Args& a) {
  const int W = a.ngpu;
  if (W < 1 || W > nbr_device_count())
    return multi_fail("-ngpu", "needs 1 <= W <= the number of visible GPUs");
  const int V = a.slices > 0 ? a.slices : std::max(8, W);
  if (V < W) return multi_fail("-slices", "needs at least one slice per GPU");
  const int scheme = a.integ == "lf" ? NBR_KDK : NBR_EULER;
  State s;
  if (make_ic(a, a.N, a.ratio, s) != NBR_OK) return 1;
  const size_t n = a.N;
  const size_t c = ((n + W - 1) / W + 127) / 128 * 128;
  const size_t n_pad = (n + 1023) / 1024 * 1024;
  const size_t ld = std::max(n_pad, (size_t)W * c);
  const double dt = a.dt > 0.0 ? a.dt : a.T / double(a.time_steps);
  const double eps2 = a.eps * a.eps;
  std::vector<MultiRank> R(W);
  std::vector<ncclComm_t> comms(W);
  std::vector<int> devs(W);
  for (int r = 0; r < W; ++r) devs[r] = r;
  if (ncclCommInitAll(comms.data(), W, devs.data()) != ncclSuccess)
    return multi_fail("ncclCommInitAll", "failed");
  int rc = 0;
  for (int r = 0; r < W && rc == 0; ++r) {
    MultiRank& k = R[r];
    k.dev = r;
    k.comm = comms[r];
    if (nbr_ctx_create(r, &k.ctx) != NBR_OK) {
      rc = multi_fail("context", nbr_last_error_string(nullptr));
      break;
    }
    k.st = static_cast<cudaStream_t>(nbr_ctx_stream(k.ctx));
    if (nbr_system_upload(k.ctx, n, s.x.data(), s.y.data(), s.z.data(), s.vx.data(), s.vy.data(),
                          s.vz.data(), s.m.data()) != NBR_OK) {
      rc = multi_fail("upload", nbr_last_error_string(k.ctx));
      break;
    }
    size_t len = 0;
    nbr_state_pointers(k.ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &len);
    if ((size_t)W * c > len) {
      rc = multi_fail("-ngpu", "the shards of the in-place all-gather exceed the state arrays");
      break;
    }
    k.i0 = (size_t)r * c;
    k.owned = k.i0 < n ? std::min(c, n - k.i0) : 0;
    k.v0 = r * V / W;
    k.v1 = (r + 1) * V / W;
    cudaSetDevice(r);
    const size_t bm = (size_t)(k.v1 - k.v0) * 3 * ld * sizeof(double);
    const size_t br = (size_t)V * 3 * c * sizeof(double);
    if (cudaMalloc((void**)&k.mine, bm) != cudaSuccess || cudaMalloc((void**)&k.recv, br) != cudaSuccess ||
        cudaMemset(k.mine, 0, bm) != cudaSuccess || cudaMemset(k.recv, 0, br) != cudaSuccess ||
        cudaEventCreate(&k.e0) != cudaSuccess || cudaEventCreate(&k.e1) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess)
      rc = multi_fail("buffers", "device allocation failed");
  }
  auto nccl_ok = [&](ncclResult_t e, const char* what) {
    if (e != ncclSuccess && rc == 0) rc = multi_fail(what, ncclGetErrorString(e));
    return e == ncclSuccess;
  };
  auto evaluate = [&](double kick, double drift) {
    for (int r = 0; r < W && rc == 0; ++r)
      if (nbr_n3_slice_accel(R[r].ctx, a.precision, eps2, R[r].v0, R[r].v1, V, R[r].mine, ld) !=
          NBR_OK)
        rc = multi_fail("slice", nbr_last_error_string(R[r].ctx));
    if (rc) return;
    nccl_ok(ncclGroupStart(), "group");
    for (int r = 0; r < W; ++r) {
      MultiRank& k = R[r];
      cudaSetDevice(k.dev);
      for (int q = 0; q < W; ++q) {
        for (int v = k.v0; v < k.v1; ++v)
          for (int d = 0; d < 3; ++d) {
            const double* src = k.mine + ((size_t)(v - k.v0) * 3 + d) * ld + (size_t)q * c;
            if (q == r)
              cudaMemcpyAsync(k.recv + ((size_t)v * 3 + d) * c, src, c * sizeof(double),
                              cudaMemcpyDeviceToDevice, k.st);
            else
              nccl_ok(ncclSend(src, c, ncclDouble, q, k.comm, k.st), "send");
          }
        if (q == r) continue;
        for (int v = R[q].v0; v < R[q].v1; ++v)
          for (int d = 0; d < 3; ++d)
            nccl_ok(ncclRecv(k.recv + ((size_t)v * 3 + d) * c, c, ncclDouble, q, k.comm, k.st), "recv");
      }
    }
    nccl_ok(ncclGroupEnd(), "group");
    for (int r = 0; r < W && rc == 0; ++r)
      if (R[r].owned &&
          nbr_step_range_sum(R[r].ctx, a.precision, scheme, R[r].i0, R[r].owned, kick, drift, a.G,
                             R[r].recv, V, 3 * c, c) != NBR_OK)
        rc = multi_fail("update", nbr_last_error_string(R[r].ctx));
    if (rc) return;
    std::vector<double*> px(W), py(W), pz(W);
    for (int r = 0; r < W; ++r)
      nbr_state_pointers(R[r].ctx, &px[r], &py[r], &pz[r], nullptr, nullptr, nullptr, nullptr);
    nccl_ok(ncclGroupStart(), "group");
    for (int r = 0; r < W; ++r)
      for (double* p : {px[r], py[r], pz[r]})
        nccl_ok(ncclAllGather(p + R[r].i0, p, c, ncclDouble, R[r].comm, R[r].st), "all-gather");
    nccl_ok(ncclGroupEnd(), "group");
    for (int r = 0; r < W; ++r) nbr_state_changed(R[r].ctx);
  };
  std::vector<std::pair<double, double>> sched;
  if (scheme == NBR_KDK) {
    sched.push_back({0.5 * dt, dt});
    for (size_t t = 1; t < a.time_steps; ++t) sched.push_back({dt, dt});
    sched.push_back({0.5 * dt, 0.0});
  } else {
    for (size_t t = 0; t < a.time_steps; ++t) sched.push_back({dt, dt});
  }
  for (int r = 0; r < W && rc == 0; ++r) cudaEventRecord(R[r].e0, R[r].st);
  for (auto& kd : sched) {
    if (rc) break;
    evaluate(kd.first, kd.second);
  }
  float ms_max = 0.f;
  for (int r = 0; r < W && rc == 0; ++r) {
    cudaEventRecord(R[r].e1, R[r].st);
    if (nbr_ctx_synchronize(R[r].ctx) != NBR_OK) {
      rc = multi_fail("run", nbr_last_error_string(R[r].ctx));
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, R[r].e0, R[r].e1);
    ms_max = std::max(ms_max, ms);
  }
  if (rc == 0) {
    // velocities of every rank's receivers to every rank, then the state out of rank 0
    std::vector<double*> vx(W), vy(W), vz(W);
    for (int r = 0; r < W; ++r)
      nbr_state_pointers(R[r].ctx, nullptr, nullptr, nullptr, &vx[r], &vy[r], &vz[r], nullptr);
    nccl_ok(ncclGroupStart(), "group");
    for (int r = 0; r < W; ++r)
      for (double* p : {vx[r], vy[r], vz[r]})
        nccl_ok(ncclAllGather(p + R[r].i0, p, c, ncclDouble, R[r].comm, R[r].st), "all-gather");
    nccl_ok(ncclGroupEnd(), "group");
    for (int r = 0; r < W; ++r) nbr_ctx_synchronize(R[r].ctx);
  }
  if (rc == 0) {
    const double secs = ms_max * 1e-3;
    const double pairs = double(sched.size()) * double(n) * double(n - 1);
    std::printf("GPUs = %d, slices = %d, N = %zu, evaluations = %zu\n", W, V, n, sched.size());
    std::printf("GPU multi solver took %fs (max over GPUs): %.3f GPairs/s\n", secs, pairs / secs * 1e-9);
    if (!a.final_snapshot.empty() &&
        nbr_snapshot_save(R[0].ctx, a.final_snapshot.c_str(), a.time_steps, dt) != NBR_OK)
      rc = multi_fail("snapshot", nbr_last_error_string(R[0].ctx));
    if (a.output_given && rc == 0) {
      const bool exists = file_exists(a.output);
      FILE* f = std::fopen(a.output.c_str(), exists ? "a" : "w");
      if (f) {
        if (!exists)
          std::fprintf(f, "#Nodes, Cores, N, t_total[s], performance[Mpairs/s], time_steps/s, ms/time_step\n");
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
        std::fprintf(f, "%d,%d,%zu,%f,%f,%f,%f\n", W, W * sms, n, secs, pairs / secs * 1e-6,
                     double(a.time_steps) / secs, secs * 1000.0 / double(a.time_steps));
        std::fclose(f);
      }
    }
  }
  for (auto& k : R) {
    if (k.ctx) nbr_ctx_synchronize(k.ctx);
    cudaSetDevice(k.dev);
    if (k.mine) cudaFree(k.mine);
    if (k.recv) cudaFree(k.recv);
    if (k.e0) cudaEventDestroy(k.e0);
    if (k.e1) cudaEventDestroy(k.e1);
    if (k.ctx) nbr_ctx_destroy(k.ctx);
  }
  for (auto cm : comms)
    if (cm) ncclCommDestroy(cm);
  return rc;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  parse(argc, argv, a);
  if (a.exec == "gpu-multi") return run_multi(a);
  nbr_ctx* ctx = nullptr;
  if (nbr_ctx_create(a.device, &ctx) != NBR_OK) {
    std::printf("No GPU context: %s\n", nbr_last_error_string(nullptr));
    return 1;
  }
  int rc = 0;
  if (a.exec == "gpu") rc = run_gpu(ctx, a, false);
  else if (a.exec == "gpu-bench") rc = run_gpu(ctx, a, true);
  else if (a.exec == "gpu-accuracy") rc = run_accuracy(ctx, a);
  else if (a.exec == "gpu-ratio") rc = run_ratio(ctx, a);
  else if (a.exec == "gpu-batch") rc = run_batch(ctx, a);
  nbr_ctx_destroy(ctx);
  return rc;
}
