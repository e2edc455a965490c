// nbr_persist.cu -- the whole leapfrog loop of a small system in one launch.
//
// For a few thousand particles one force evaluation is a few microseconds of
// work, comparable to the gap between two kernel launches even inside a CUDA
// graph.  This file runs every step of nbr_run (KDK, Yoshida DKD or Euler,
// the schedules of reduced_solver_omp_lf / reduced_solver_omp,
// CPU/omp_solver.cpp:16-178, 257-456) inside ONE cooperative launch:
//
//  * each CTA owns fixed receiver chunks (about n / SMs particles, at most RPC
//    lane slots) for the whole run;
//  * per force evaluation every CTA stages all N positions (masses once) in
//    shared memory with L2 loads, its 8 warps split the sources 8 ways and the
//    F lane groups of each warp split them again (k_force_small's layout), and
//    the partial sums are combined in a fixed order (xor shuffles, then the
//    warps in order): deterministic;
//  * the CTA applies the fused kick/drift to its receivers, writing the next
//    position buffer, and all CTAs meet at one grid barrier before the next
//    evaluation reads it.
//
// The barrier is a 64-bit arrival counter that only grows; its wait is bounded by
// %globaltimer (the context's wait limit) and gives up, with an error code
// for the host, if the limit passes or another CTA has already recorded an
// error.  The cooperative launch guarantees that all CTAs are resident, so no
// CTA waits on one that cannot run.  Pair arithmetic is k_force_f64's (CUDA's
// rsqrt(double)): results equal the other FP64 kernels' up to summation order.
#include "nbr.h"
#include "nbr_ctx.h"
#include "nbr_device.cuh"
#include "nbr_kernels.cuh"

#include <algorithm>
#include <vector>

namespace nbr {

namespace {

constexpr int kPNIDefault = 4;  // receivers per lane

struct PersistArgs {
  int n;                   // particles (<= kPersistMaxN)
  int chunks;              // receiver chunks of cs particles
  int cs;                  // receivers per chunk (<= RPC slots of the lane layout)
  int evals;               // force evaluations
  const double2* sched;    // (kick, drift) of every evaluation
  int mode;                // 1: leapfrog (drift with the kicked velocity); 2: Euler
  int pre;                 // a standalone kick/drift before the first evaluation
  int pre_use_acc;         // its kick uses the accelerations left by the last run
  double pre_kick, pre_drift;
  double G, eps2;
  double* px[2];
  double* py[2];
  double* pz[2];
  int cur0;                // buffer the first phase reads
  double* vx; double* vy; double* vz;
  double* ax; double* ay; double* az;
  const double* m;
  unsigned long long* bar; // arrivals at grid barriers (only grows; zero at launch)
  int* err;
  unsigned long long wait_ns;
  int skip_barrier;        // test hook: CTA 0 leaves before this barrier (-1: off)
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid-wide barrier number `k` (0, 1, ...) of the launch, with a bounded
// wait.  The arrival counter only grows (zeroed by the host before the
// launch): barrier k is complete when it reaches (k + 1) x gridDim.x, so an
// arrival is one release add and nothing is reset.  Returns false in every
// thread of the CTA if the barrier did not complete within the limit or an
// error was already recorded (the CTA then leaves the kernel).
__device__ bool grid_barrier(unsigned long long* bar, int* err, unsigned long long limit_ns,
                             unsigned long long k) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned long long target = (k + 1) * gridDim.x;
    __threadfence();
    red_release_add_u64(bar, 1ull);
    if (ld_acquire_u64(bar) < target) {
      const unsigned long long t0 = global_ns();
      while (ld_acquire_u64(bar) < target) {
        if (*reinterpret_cast<volatile int*>(err) != 0 || global_ns() - t0 > limit_ns) {
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    if (!ok) record_error(err, kErrGridWait);
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// W warps per CTA (8 or 16), F lane groups per warp, kPNI receivers per lane.
template <int F, int W, int kPNI, bool EXCL>
__global__ void __launch_bounds__(W * 32, 1) k_run_small_f64(const PersistArgs A) {
  constexpr int kPWarps = W;
  constexpr int kPThreads = W * 32;
  constexpr int G = 32 / F;        // receiver columns per warp
  constexpr int RPC = G * kPNI;    // receivers per chunk
  constexpr int S = kPWarps * F;   // ways the sources are split
  extern __shared__ __align__(16) double smem_d[];
  const int n = A.n;
  const int ns = (n + 1) & ~1;
  double* sx = smem_d;
  double* sy = sx + ns;
  double* sz = sy + ns;
  double* sm = sz + ns;
  double* red = sm + ns;  // [kPWarps][RPC][3]
  // velocities of this CTA's receivers for the whole run: [round][RPC][3]
  double* svel = red + (size_t)kPWarps * RPC * 3;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gl = lane % G, grp = lane / G;

  for (int j = threadIdx.x; j < n; j += kPThreads) sm[j] = A.m[j];
  int cur = A.cur0;
  unsigned long long nbar = 0;  // grid barriers passed

  if (A.pre) {
    for (int c = blockIdx.x; c < A.chunks; c += gridDim.x) {
      for (int t = threadIdx.x; t < A.cs; t += kPThreads) {
        const int i = c * A.cs + t;
        if (i >= n) continue;
        double ux = A.vx[i], uy = A.vy[i], uz = A.vz[i];
        if (A.pre_use_acc) {
          ux += A.pre_kick * A.ax[i]; uy += A.pre_kick * A.ay[i]; uz += A.pre_kick * A.az[i];
          A.vx[i] = ux; A.vy[i] = uy; A.vz[i] = uz;
        }
        A.px[1 - cur][i] = __ldcg(A.px[cur] + i) + A.pre_drift * ux;
        A.py[1 - cur][i] = __ldcg(A.py[cur] + i) + A.pre_drift * uy;
        A.pz[1 - cur][i] = __ldcg(A.pz[cur] + i) + A.pre_drift * uz;
      }
    }
    if (!grid_barrier(A.bar, A.err, A.wait_ns, nbar++)) return;
    cur ^= 1;
  }
  // the CTA owns its receivers for the whole run: their velocities stay in
  // shared memory until the end
  for (int c = blockIdx.x, r = 0; c < A.chunks; c += gridDim.x, ++r)
    for (int t = threadIdx.x; t < RPC; t += kPThreads) {
      const int i = c * A.cs + t;
      const bool own = t < A.cs && i < n;
      double* v = svel + ((size_t)r * RPC + t) * 3;
      v[0] = own ? A.vx[i] : 0.0;
      v[1] = own ? A.vy[i] : 0.0;
      v[2] = own ? A.vz[i] : 0.0;
    }

  for (int e = 0; e < A.evals; ++e) {
    // all positions of this evaluation, from L2 (other CTAs wrote them)
    const double* X = A.px[cur];
    const double* Y = A.py[cur];
    const double* Z = A.pz[cur];
    // 16-byte L2 loads, several in flight per thread before the stores (the
    // arrays hold at least ns entries: n_pad is a multiple of 1024)
    {
      const double2* X2 = reinterpret_cast<const double2*>(X);
      const double2* Y2 = reinterpret_cast<const double2*>(Y);
      const double2* Z2 = reinterpret_cast<const double2*>(Z);
      double2* sx2 = reinterpret_cast<double2*>(sx);
      double2* sy2 = reinterpret_cast<double2*>(sy);
      double2* sz2 = reinterpret_cast<double2*>(sz);
#pragma unroll 4
      for (int j = threadIdx.x; j < ns / 2; j += kPThreads) {
        const double2 a = __ldcg(X2 + j), b = __ldcg(Y2 + j), c = __ldcg(Z2 + j);
        sx2[j] = a;
        sy2[j] = b;
        sz2[j] = c;
      }
    }
    __syncthreads();
    const double2 kd = A.sched[e];
    for (int c = blockIdx.x, round = 0; c < A.chunks; c += gridDim.x, ++round) {
      const int base = c * A.cs;
      double xi[kPNI], yi[kPNI], zi[kPNI], ax[kPNI], ay[kPNI], az[kPNI];
#pragma unroll
      for (int k = 0; k < kPNI; ++k) {
        const int slot = gl + G * k, i = base + slot;
        const bool real = slot < A.cs && i < n;
        xi[k] = real ? sx[i] : 0.0;
        yi[k] = real ? sy[i] : 0.0;
        zi[k] = real ? sz[i] : 0.0;
        ax[k] = ay[k] = az[k] = 0.0;
      }
#pragma unroll 2
      for (int j = warp * F + grp; j < n; j += S) {
        const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
        for (int k = 0; k < kPNI; ++k) {
          const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
          double r2 = fma(dx, dx, A.eps2);
          r2 = fma(dy, dy, r2);
          r2 = fma(dz, dz, r2);
          double y = rsqrt(r2);
          if (EXCL) y = r2 > 0.0 ? y : 0.0;
          const double s = mj * (y * y * y);
          ax[k] = fma(s, dx, ax[k]);
          ay[k] = fma(s, dy, ay[k]);
          az[k] = fma(s, dz, az[k]);
        }
      }
      // lane groups of the warp, then the warps in order
#pragma unroll
      for (int off = G; off < 32; off <<= 1) {
#pragma unroll
        for (int k = 0; k < kPNI; ++k) {
          ax[k] += __shfl_xor_sync(0xffffffffu, ax[k], off);
          ay[k] += __shfl_xor_sync(0xffffffffu, ay[k], off);
          az[k] += __shfl_xor_sync(0xffffffffu, az[k], off);
        }
      }
      if (grp == 0) {
#pragma unroll
        for (int k = 0; k < kPNI; ++k) {
          double* r = red + ((size_t)warp * RPC + gl + G * k) * 3;
          r[0] = ax[k]; r[1] = ay[k]; r[2] = az[k];
        }
      }
      __syncthreads();
      if (threadIdx.x < RPC) {
        const int t = threadIdx.x, i = base + t;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
        for (int w = 0; w < kPWarps; ++w) {
          const double* r = red + ((size_t)w * RPC + t) * 3;
          a0 += r[0]; a1 += r[1]; a2 += r[2];
        }
        if (t < A.cs && i < n) {
          // the epilogue of the large kernels: a -> acc, v += kick a, x' = x + drift v
          // (Euler: drift with the old velocity)
          const double gx = A.G * a0, gy = A.G * a1, gz = A.G * a2;
          A.ax[i] = gx; A.ay[i] = gy; A.az[i] = gz;
          double* v = svel + ((size_t)round * RPC + t) * 3;
          const double ux = v[0], uy = v[1], uz = v[2];
          const double vx = ux + kd.x * gx, vy = uy + kd.x * gy, vz = uz + kd.x * gz;
          v[0] = vx; v[1] = vy; v[2] = vz;
          const bool euler = A.mode == 2;
          A.px[1 - cur][i] = sx[i] + kd.y * (euler ? ux : vx);
          A.py[1 - cur][i] = sy[i] + kd.y * (euler ? uy : vy);
          A.pz[1 - cur][i] = sz[i] + kd.y * (euler ? uz : vz);
        }
      }
      __syncthreads();  // red is reused by the next chunk
    }
    if (e + 1 < A.evals) {
      if (e == A.skip_barrier && blockIdx.x == 0) return;  // test hook: never arrives
      if (!grid_barrier(A.bar, A.err, A.wait_ns, nbar++)) return;
    }
    cur ^= 1;
  }
  for (int c = blockIdx.x, r = 0; c < A.chunks; c += gridDim.x, ++r)
    for (int t = threadIdx.x; t < A.cs; t += kPThreads) {
      const int i = c * A.cs + t;
      if (i >= n) continue;
      const double* v = svel + ((size_t)r * RPC + t) * 3;
      A.vx[i] = v[0]; A.vy[i] = v[1]; A.vz[i] = v[2];
    }
}

template <int F, int NI>
const void* persist_fn_f(int W, bool excl) {
  if (W == 8) return excl ? (const void*)k_run_small_f64<F, 8, NI, true> : (const void*)k_run_small_f64<F, 8, NI, false>;
  if (W == 16) return excl ? (const void*)k_run_small_f64<F, 16, NI, true> : (const void*)k_run_small_f64<F, 16, NI, false>;
  return nullptr;
}

const void* persist_fn(int F, int W, int NI, bool excl) {
  if (NI == 4) {
    switch (F) {
      case 4: return persist_fn_f<4, 4>(W, excl);
      case 8: return persist_fn_f<8, 4>(W, excl);
      case 16: return persist_fn_f<16, 4>(W, excl);
      default: return nullptr;
    }
  }
  if (NI == 8) {
    switch (F) {
      case 8: return persist_fn_f<8, 8>(W, excl);
      case 16: return persist_fn_f<16, 8>(W, excl);
      default: return nullptr;
    }
  }
  return nullptr;
}

// Shared memory of a launch: positions and masses, the warps' partial sums, and
// the velocities of up to `rounds` receiver chunks per CTA.
size_t persist_smem(int n, int F, int W, int NI, int rounds) {
  const int ns = (n + 1) & ~1;
  const size_t rpc = (size_t)(32 / F) * NI;
  return (size_t)4 * ns * sizeof(double) + ((size_t)W + rounds) * rpc * 3 * sizeof(double);
}

// Lane groups per warp: the most (the finest split of the sources) whose
// chunk of (32 / F) x 4 receiver slots still holds n / SMs receivers, so that
// one round of chunks covers the system.
int persist_groups(int n, int sms) {
  const int need = (n + sms - 1) / sms;
  for (int F : {16, 8, 4})
    if ((32 / F) * kPNIDefault >= need) return F;
  return 4;
}

}  // namespace

bool persistent_run_applies(nbr_ctx* c, int precision, size_t n) {
  const ForceConfig& o = c->override_cfg[precision];
  if (o.ni != 0 && o.ni != kPersistNI) return false;
  return precision == kFP64 && c->coop && n >= 2 && n <= (size_t)kPersistMaxN;
}

int run_persistent(nbr_ctx* c, int precision, int scheme, double dt, size_t steps, double G,
                   double eps2, bool fsal, const double* cc, const double* dd, int lf,
                   nbr_run_stats* st) {
  (void)precision;
  SysState& s = c->sys;
  const int n = (int)s.n;
  // the schedule: the launch sequence of nbr_run's graph, one entry per evaluation
  std::vector<double2> sched;
  PersistArgs A{};
  A.mode = scheme == NBR_EULER ? 2 : 1;
  if (scheme == NBR_KDK) {
    if (fsal) {
      A.pre = 1; A.pre_use_acc = 1; A.pre_kick = 0.5 * dt; A.pre_drift = dt;
    } else {
      sched.push_back(make_double2(0.5 * dt, dt));
    }
    for (size_t k = 1; k < steps; ++k) sched.push_back(make_double2(dt, dt));
    sched.push_back(make_double2(0.5 * dt, 0.0));
  } else if (scheme == NBR_EULER) {
    for (size_t k = 0; k < steps; ++k) sched.push_back(make_double2(dt, dt));
  } else {
    A.pre = 1; A.pre_use_acc = 0; A.pre_kick = 0.0; A.pre_drift = cc[0] * dt;
    for (size_t k = 0; k < steps; ++k)
      for (int sub = 0; sub < lf - 1; ++sub) {
        const double drift = sub < lf - 2 ? cc[sub + 1]
                                          : ((k + 1 < steps) ? cc[lf - 1] + cc[0] : cc[lf - 1]);
        sched.push_back(make_double2(dd[sub] * dt, drift * dt));
      }
  }
  const int E = (int)sched.size();
  cudaError_t e = c->scr.need_red((size_t)2 * E + 16);
  if (e != cudaSuccess) return cuda_fail(c, e, "persistent schedule");
  e = cudaMemcpyAsync(c->scr.red, sched.data(), sched.size() * sizeof(double2),
                      cudaMemcpyHostToDevice, c->stream);
  // the arrival counter: the context's error block words 2-3 (8-byte aligned)
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(c->d_err + 2);
  if (e == cudaSuccess) e = cudaMemsetAsync(bar, 0, sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "persistent setup");

  const ForceConfig& o = c->override_cfg[kFP64];
  int F = persist_groups(n, c->sms), W = kPersistDefaultWarps, NI = kPNIDefault;
  if (o.ni == kPersistNI) {
    F = o.warps;
    if (o.split > 1) W = o.split;
    if (o.tile > 0) NI = o.tile;
  }
  const bool excl = eps2 == 0.0;
  const void* fn = persist_fn(F, W, NI, excl);
  if (!fn)
    return fail(c, NBR_ERR_INVALID_ARG,
                "persistent run: (lane groups, receivers per lane) must be (4|8|16, 4) or "
                "(8|16, 8) and warps per CTA 8 or 16");
  const int kPThreads = W * 32;
  const int rpc = (32 / F) * NI;
  // receivers per chunk: n / SMs (one chunk per SM) when the slots allow it
  const int cs = std::max(1, std::min(rpc, (n + c->sms - 1) / c->sms));
  const int chunks = (n + cs - 1) / cs;
  // the grid is at least min(chunks, SMs) CTAs, so no CTA gets more rounds than this
  const int rounds = (chunks + std::min(chunks, c->sms) - 1) / std::min(chunks, c->sms);
  const size_t smem = persist_smem(n, F, W, NI, rounds);
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPThreads, smem);
  if (e != cudaSuccess) return cuda_fail(c, e, "persistent kernel setup");
  if (per_sm < 1) return fail(c, NBR_ERR_UNSUPPORTED, "persistent kernel does not fit an SM");
  A.n = n;
  A.chunks = chunks;
  A.cs = cs;
  A.evals = E;
  A.sched = reinterpret_cast<const double2*>(c->scr.red);
  A.G = G;
  A.eps2 = eps2;
  for (int b = 0; b < 2; ++b) {
    A.px[b] = s.pos[b][0]; A.py[b] = s.pos[b][1]; A.pz[b] = s.pos[b][2];
  }
  A.cur0 = s.cur;
  A.vx = s.vel[0]; A.vy = s.vel[1]; A.vz = s.vel[2];
  A.ax = s.acc[0]; A.ay = s.acc[1]; A.az = s.acc[2];
  A.m = s.mass;
  A.bar = bar;
  A.err = c->d_err;
  JStream probe{};
  pipeline_params(probe);
  A.wait_ns = probe.wait_ns;
  A.skip_barrier = probe.skip_tile;
  const int grid = std::min(A.chunks, per_sm * c->sms);
  void* args[] = {&A};
  e = cudaEventRecord(c->ev0, c->stream);
  if (e == cudaSuccess)
    e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kPThreads), args, smem, c->stream);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    c->acc_ok = false;
    return cuda_fail(c, e, "persistent run launch");
  }
  s.cur = (s.cur + A.pre + E) & 1;
  s.rec_ok[0] = s.rec_ok[1] = false;
  const int rc = check_device_error(c);
  if (rc) return rc;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  st->gpu_ms = ms;
  st->kernels = 1;
  st->force_evals = E;
  st->pairs = double(E) * double(n) * double(n - 1);
  return NBR_OK;
}

}  // namespace nbr
