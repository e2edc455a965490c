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
//    shared memory with L2 loads, its W warps (8 or 16) split the sources W
//    ways and the F lane groups of each warp split them again
//    (k_force_small's layout), and the partial sums are combined in a fixed
//    order (xor shuffles, then the warps in order): deterministic;
//  * the CTA applies the fused kick/drift to its receivers, whose velocities
//    (and, FP32C, positions) stay in shared memory for the run, writes their
//    positions to the next buffer, and all CTAs meet at one grid barrier
//    before the next evaluation reads it.
//
// The barrier is a 64-bit arrival counter that only grows; its wait is bounded
// by %globaltimer (the context's wait limit) and gives up, with an error code
// for the host, if the limit passes or another CTA has already recorded an
// error.  The cooperative launch guarantees that all CTAs are resident, so no
// CTA waits on one that cannot run.  FP64 pair arithmetic is k_force_f64's
// (CUDA's rsqrt(double)): results equal the other FP64 kernels' up to
// summation order; the FP32C form (k_run_small_f32c) is described there.
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
// Ordering: the CTA's writes precede thread 0's release add through the
// bar.sync (a CTA-scope synchronization), and the acquire load that sees the
// last arrival precedes the other threads' reads through the second bar.sync;
// causality order is transitive, so no separate fence is needed (two
// __threadfence() here cost 0.45 us per barrier).  The error word and the
// timer are checked every 32 polls.
__device__ bool grid_barrier(unsigned long long* bar, int* err, unsigned long long limit_ns,
                             unsigned long long k) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned long long target = (k + 1) * gridDim.x;
    red_release_add_u64(bar, 1ull);
    if (ld_acquire_u64(bar) < target) {
      const unsigned long long t0 = global_ns();
      unsigned polls = 0;
      while (ld_acquire_u64(bar) < target) {
        if ((++polls & 31u) == 0 &&
            (*reinterpret_cast<volatile int*>(err) != 0 || global_ns() - t0 > limit_ns)) {
          ok = 0;
          break;
        }
      }
    }
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
#pragma unroll 4
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

// The FP32C form, with the pair arithmetic of k_force_small / k_force_f32c
// (f32x2 differences, rsqrt.approx with the first-order Newton correction of
// y^3 folded into the mass terms).  16 warps per CTA, 4 receivers per lane.
// Per force evaluation every CTA reads all N positions from L2 into registers,
// takes their FP64 mean as the origin (summed in a fixed order), and writes
// FP32 source records relative to it into shared memory: (x, x, y, y),
// (z, z, -1.5 m, -1.5 m), (2.5 m, 2.5 m), the mass terms once per run.  The
// CTA's own receivers keep their FP64 positions and velocities in shared
// memory for the whole run.  A thread's FP32 sums cover N / (16 F) sources;
// lane groups and warps are then added in FP64 in a fixed order.
constexpr int kPW32 = 16;
constexpr int kPLoads32 = (int)((kPersistMaxN / 2 + kPW32 * 32 - 1) / (kPW32 * 32));

template <int F, bool EXCL>
__global__ void __launch_bounds__(kPW32 * 32, 1) k_run_small_f32c(const PersistArgs A) {
  constexpr int W = kPW32, NT = W * 32, NI = 4, IPAIR = 2;
  constexpr int G = 32 / F, RPC = G * NI, S = W * F;
  extern __shared__ __align__(16) unsigned char smem_b[];
  __shared__ double s_org[W][3];
  __shared__ double s_o[3];
  const int n = A.n, ns = (n + 1) & ~1;
  ulonglong2* rxy = reinterpret_cast<ulonglong2*>(smem_b);  // [ns] (x, x, y, y)
  ulonglong2* rzm = rxy + ns;                               // [ns] (z, z, -1.5 m, -1.5 m)
  u64* rb = reinterpret_cast<u64*>(rzm + ns);               // [ns] (2.5 m, 2.5 m)
  double* red = reinterpret_cast<double*>(rb + ns);         // [W][RPC][3]
  const int rounds = (A.chunks + gridDim.x - 1) / gridDim.x;
  double* svel = red + (size_t)W * RPC * 3;                 // [rounds][RPC][3]
  double* spos = svel + (size_t)rounds * RPC * 3;           // [rounds][RPC][3]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gl = lane % G, grp = lane / G;
  const float e2f = (float)A.eps2;
  const u64 EPS2 = pack2(e2f, e2f);

  for (int j = threadIdx.x; j < ns; j += NT) {
    const double m = j < n ? A.m[j] : 0.0;
    const float fa = __double2float_rn(-1.5 * m), fb = __double2float_rn(2.5 * m);
    rzm[j] = make_ulonglong2(0ull, pack2(fa, fa));
    rb[j] = pack2(fb, fb);
  }
  int cur = A.cur0;
  unsigned long long nbar = 0;

  if (A.pre) {
    for (int c = blockIdx.x; c < A.chunks; c += gridDim.x) {
      for (int t = threadIdx.x; t < A.cs; t += NT) {
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
  // the CTA's receivers: positions and velocities in shared memory for the run
  for (int c = blockIdx.x, r = 0; c < A.chunks; c += gridDim.x, ++r)
    for (int t = threadIdx.x; t < RPC; t += NT) {
      const int i = c * A.cs + t;
      const bool own = t < A.cs && i < n;
      double* v = svel + ((size_t)r * RPC + t) * 3;
      double* x = spos + ((size_t)r * RPC + t) * 3;
      v[0] = own ? A.vx[i] : 0.0; v[1] = own ? A.vy[i] : 0.0; v[2] = own ? A.vz[i] : 0.0;
      x[0] = own ? __ldcg(A.px[cur] + i) : 0.0;
      x[1] = own ? __ldcg(A.py[cur] + i) : 0.0;
      x[2] = own ? __ldcg(A.pz[cur] + i) : 0.0;
    }

  for (int e = 0; e < A.evals; ++e) {
    // all positions from L2 into registers, and their sum for the origin
    const double2* X2 = reinterpret_cast<const double2*>(A.px[cur]);
    const double2* Y2 = reinterpret_cast<const double2*>(A.py[cur]);
    const double2* Z2 = reinterpret_cast<const double2*>(A.pz[cur]);
    double2 qx[kPLoads32], qy[kPLoads32], qz[kPLoads32];
    double ox = 0.0, oy = 0.0, oz = 0.0;
#pragma unroll
    for (int k = 0; k < kPLoads32; ++k) {
      const int j2 = threadIdx.x + k * NT;
      qx[k] = qy[k] = qz[k] = make_double2(0.0, 0.0);
      if (j2 < ns / 2) {
        qx[k] = __ldcg(X2 + j2); qy[k] = __ldcg(Y2 + j2); qz[k] = __ldcg(Z2 + j2);
        ox += qx[k].x; oy += qy[k].x; oz += qz[k].x;
        if (2 * j2 + 1 < n) { ox += qx[k].y; oy += qy[k].y; oz += qz[k].y; }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ox += __shfl_xor_sync(0xffffffffu, ox, off);
      oy += __shfl_xor_sync(0xffffffffu, oy, off);
      oz += __shfl_xor_sync(0xffffffffu, oz, off);
    }
    if (lane == 0) { s_org[warp][0] = ox; s_org[warp][1] = oy; s_org[warp][2] = oz; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0, cc = 0.0;
      for (int w = 0; w < W; ++w) { a += s_org[w][0]; b += s_org[w][1]; cc += s_org[w][2]; }
      s_o[0] = a / n; s_o[1] = b / n; s_o[2] = cc / n;
    }
    __syncthreads();
    const double o0 = s_o[0], o1 = s_o[1], o2 = s_o[2];
#pragma unroll
    for (int k = 0; k < kPLoads32; ++k) {
      const int j2 = threadIdx.x + k * NT;
      if (j2 < ns / 2) {
        const float x0 = __double2float_rn(qx[k].x - o0), x1 = __double2float_rn(qx[k].y - o0);
        const float y0 = __double2float_rn(qy[k].x - o1), y1 = __double2float_rn(qy[k].y - o1);
        const float z0 = __double2float_rn(qz[k].x - o2), z1 = __double2float_rn(qz[k].y - o2);
        rxy[2 * j2] = make_ulonglong2(pack2(x0, x0), pack2(y0, y0));
        rxy[2 * j2 + 1] = make_ulonglong2(pack2(x1, x1), pack2(y1, y1));
        reinterpret_cast<u64*>(rzm + 2 * j2)[0] = pack2(z0, z0);
        reinterpret_cast<u64*>(rzm + 2 * j2 + 1)[0] = pack2(z1, z1);
      }
    }
    __syncthreads();
    const double2 kd = A.sched[e];
    for (int c = blockIdx.x, round = 0; c < A.chunks; c += gridDim.x, ++round) {
      const int base = c * A.cs;
      double* sp = spos + (size_t)round * RPC * 3;
      u64 XI[IPAIR], YI[IPAIR], ZI[IPAIR], AX[IPAIR], AY[IPAIR], AZ[IPAIR];
#pragma unroll
      for (int p = 0; p < IPAIR; ++p) {
        const double* r0 = sp + (gl + G * (2 * p)) * 3;
        const double* r1 = sp + (gl + G * (2 * p + 1)) * 3;
        XI[p] = pack2(__double2float_rn(r0[0] - o0), __double2float_rn(r1[0] - o0));
        YI[p] = pack2(__double2float_rn(r0[1] - o1), __double2float_rn(r1[1] - o1));
        ZI[p] = pack2(__double2float_rn(r0[2] - o2), __double2float_rn(r1[2] - o2));
        AX[p] = AY[p] = AZ[p] = 0ull;
      }
#pragma unroll 2
      for (int j = warp * F + grp; j < n; j += S) {
        const ulonglong2 q0 = rxy[j];
        const ulonglong2 q1 = rzm[j];
        const u64 bj = rb[j];
#pragma unroll
        for (int p = 0; p < IPAIR; ++p) {
          const u64 dx = sub2(q0.x, XI[p]);
          const u64 dy = sub2(q0.y, YI[p]);
          const u64 dz = sub2(q1.x, ZI[p]);
          u64 r2 = fma2(dx, dx, EPS2);
          r2 = fma2(dy, dy, r2);
          r2 = fma2(dz, dz, r2);
          u64 y;
          if (EXCL) {
            float rl, rh;
            unpack2(r2, rl, rh);
            y = pack2(rl > 0.f ? rsqrt_mufu(rl) : 0.f, rh > 0.f ? rsqrt_mufu(rh) : 0.f);
          } else {
            y = rsqrt2(r2);
          }
          const u64 y2 = mul2(y, y);
          const u64 pr = mul2(r2, y2);
          const u64 mg = fma2(q1.y, pr, bj);
          const u64 y3 = mul2(y2, y);
          const u64 sv = mul2(y3, mg);
          AX[p] = fma2(sv, dx, AX[p]);
          AY[p] = fma2(sv, dy, AY[p]);
          AZ[p] = fma2(sv, dz, AZ[p]);
        }
      }
      double ax[NI], ay[NI], az[NI];
#pragma unroll
      for (int p = 0; p < IPAIR; ++p) {
        float l, h;
        unpack2(AX[p], l, h); ax[2 * p] = l; ax[2 * p + 1] = h;
        unpack2(AY[p], l, h); ay[2 * p] = l; ay[2 * p + 1] = h;
        unpack2(AZ[p], l, h); az[2 * p] = l; az[2 * p + 1] = h;
      }
#pragma unroll
      for (int off = G; off < 32; off <<= 1) {
#pragma unroll
        for (int k = 0; k < NI; ++k) {
          ax[k] += __shfl_xor_sync(0xffffffffu, ax[k], off);
          ay[k] += __shfl_xor_sync(0xffffffffu, ay[k], off);
          az[k] += __shfl_xor_sync(0xffffffffu, az[k], off);
        }
      }
      if (grp == 0) {
#pragma unroll
        for (int k = 0; k < NI; ++k) {
          double* r = red + ((size_t)warp * RPC + gl + G * k) * 3;
          r[0] = ax[k]; r[1] = ay[k]; r[2] = az[k];
        }
      }
      __syncthreads();
      if (threadIdx.x < RPC) {
        const int t = threadIdx.x, i = base + t;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const double* r = red + ((size_t)w * RPC + t) * 3;
          a0 += r[0]; a1 += r[1]; a2 += r[2];
        }
        if (t < A.cs && i < n) {
          const double gx = A.G * a0, gy = A.G * a1, gz = A.G * a2;
          A.ax[i] = gx; A.ay[i] = gy; A.az[i] = gz;
          double* v = svel + ((size_t)round * RPC + t) * 3;
          double* x = sp + (size_t)t * 3;
          const double ux = v[0], uy = v[1], uz = v[2];
          const double vx = ux + kd.x * gx, vy = uy + kd.x * gy, vz = uz + kd.x * gz;
          v[0] = vx; v[1] = vy; v[2] = vz;
          const bool euler = A.mode == 2;
          const double nx = x[0] + kd.y * (euler ? ux : vx);
          const double ny = x[1] + kd.y * (euler ? uy : vy);
          const double nz = x[2] + kd.y * (euler ? uz : vz);
          x[0] = nx; x[1] = ny; x[2] = nz;
          A.px[1 - cur][i] = nx; A.py[1 - cur][i] = ny; A.pz[1 - cur][i] = nz;
        }
      }
      __syncthreads();  // red and the receivers' positions are read again
    }
    if (e + 1 < A.evals) {
      if (e == A.skip_barrier && blockIdx.x == 0) return;  // test hook: never arrives
      if (!grid_barrier(A.bar, A.err, A.wait_ns, nbar++)) return;
    }
    cur ^= 1;
  }
  for (int c = blockIdx.x, r = 0; c < A.chunks; c += gridDim.x, ++r)
    for (int t = threadIdx.x; t < A.cs; t += NT) {
      const int i = c * A.cs + t;
      if (i >= n) continue;
      const double* v = svel + ((size_t)r * RPC + t) * 3;
      A.vx[i] = v[0]; A.vy[i] = v[1]; A.vz[i] = v[2];
    }
}

const void* persist_fn32(int F, bool excl) {
  switch (F) {
    case 4: return excl ? (const void*)k_run_small_f32c<4, true> : (const void*)k_run_small_f32c<4, false>;
    case 8: return excl ? (const void*)k_run_small_f32c<8, true> : (const void*)k_run_small_f32c<8, false>;
    case 16: return excl ? (const void*)k_run_small_f32c<16, true> : (const void*)k_run_small_f32c<16, false>;
    default: return nullptr;
  }
}

size_t persist_smem32(int n, int F, int rounds) {
  const int ns = (n + 1) & ~1;
  const size_t rpc = (size_t)(32 / F) * 4;
  return (size_t)40 * ns + ((size_t)kPW32 + 2 * (size_t)rounds) * rpc * 3 * sizeof(double);
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
  return c->coop && n >= 2 && n <= (size_t)kPersistMaxN;
}

int run_persistent(nbr_ctx* c, int precision, int scheme, double dt, size_t steps, double G,
                   double eps2, bool fsal, const double* cc, const double* dd, int lf,
                   nbr_run_stats* st) {
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

  const ForceConfig& o = c->override_cfg[precision];
  int F = persist_groups(n, c->sms), W = kPersistDefaultWarps, NI = kPNIDefault;
  if (o.ni == kPersistNI) {
    F = o.warps;
    if (o.split > 1) W = o.split;
    if (o.tile > 0) NI = o.tile;
  }
  const bool excl = eps2 == 0.0;
  const bool fp32 = precision == kFP32C;
  if (fp32) {
    W = kPW32;
    NI = kPNIDefault;
  }
  const void* fn = fp32 ? persist_fn32(F, excl) : persist_fn(F, W, NI, excl);
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
  const size_t smem = fp32 ? persist_smem32(n, F, rounds) : persist_smem(n, F, W, NI, rounds);
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
