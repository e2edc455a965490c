// nbr_kernels.cu -- all-pairs softened gravity on sm_100a.
//
// The hot path replaces the reference's force kernels (compute_forces_* in
// CPU/force_calculation.cpp, e.g. compute_forces_avx2_blocked :477-690) and the
// kick/drift loops of reduced_solver_omp_lf (CPU/omp_solver.cpp:320-420).
//
// Structure of a force launch (both precisions):
//  * Each warp owns 32 * NI consecutive receivers ("i-block"); lane l keeps
//    receivers ibase + l + 32k, k < NI, in registers.  A CTA of W warps shares
//    one stream of source tiles ("j-tiles", kTile particles each).
//  * j-tiles stream through a 4-stage shared-memory ring filled by 1-D TMA
//    bulk copies (cp.async.bulk, mbarrier completion, one elected producer
//    thread).  This is the single-GPU image of the reference's ring pass, where
//    blocks of particles travel past every rank (CPU/hybrid_solver.cpp:79-107).
//  * The j range can be split over gridDim.y CTAs; each writes its partial
//    sums and the last CTA to finish a receiver chunk adds them in split order
//    (deterministic) and runs the epilogue.
//  * Epilogue: either write a (or m a), or the fused leapfrog update
//    v += kick a; x' = x + drift v into the other position buffer, plus the
//    FP32 records of x' for the next FP32C evaluation.
//
// FP32C pair arithmetic (per ordered pair; f32x2 instructions work on two
// receivers at once):
//     d  = x_j - x_i           3 sub      (relative to the tile's FP64 origin)
//     r2 = d.d + eps^2         3 fma
//     y  = rsqrt.approx(r2)    1 MUFU
//     y2 = y*y; p = r2*y2      2 mul      (p = 1 - e, e the rsqrt error)
//     mg = (-1.5 m) p + 2.5 m  1 fma      (m (1 + 3e/2): first-order Newton
//     y3 = y2*y; s = y3*mg     2 mul       correction of y^3 with the mass folded in)
//     acc += s d               3 fma
// = 14 FP32-pipe operations + 1 MUFU per pair.  One Newton-Raphson step on
// y followed by cubing gives y^3 (1 + 3e/2 + O(e^2)) as well; the form above
// applies the same first-order correction to y^3 directly.  Tile partial sums
// (kTile sources) are FP32; across tiles they are combined with Knuth
// TwoSum into a (hi, lo) FP32 pair per component, and hi + lo is formed in
// FP64 at the end.
#include "nbr_device.cuh"
#include "nbr_kernels.cuh"

#include <algorithm>
#include <cstdio>
#include <functional>
#include <map>
#include <mutex>
#include <queue>
#include <tuple>
#include <vector>

namespace nbr {

namespace {

constexpr int kStages = 4;
constexpr int kRecBytes = kTile * 48;          // 3 x float4 per source
constexpr int kStage32 = kRecBytes + 32;       // + FP64 tile origin (double4)
constexpr int kStage64 = 4 * kTile * 8;        // x, y, z, m tiles
constexpr int kSmemHead = 128;                 // mbarriers

// ------------------------------------------------------------ pipeline ----
// Runs body(stage) for the ntl tiles of this CTA's j range.  Thread 0 is the
// producer: it issues the bulk copies of a tile once every thread has finished
// with the stage it reuses.  Returns false if a tile wait timed out; the abort
// is CTA-uniform (decided by __syncthreads_or), the error word is set, and the
// copies that were issued but not consumed are drained (bounded wait) so that
// none lands after the CTA exits.  js.skip_tile >= 0 makes the producer never
// issue that tile: a test hook that lets a bounded wait expire on purpose.
template <class Issue, class Body>
__device__ __forceinline__ bool tile_pipeline(uint64_t* bars, int ntl, const JStream& js, int* err,
                                              Issue issue, Body body) {
  const int tid = threadIdx.x;
  uint32_t pending = 0;  // producer only: stages with an issued, unconsumed copy
  auto produce = [&](int st, int t) {
    if (t == js.skip_tile) return;
    issue(st, t);
    pending |= 1u << st;
  };
  if (tid == 0) {
    for (int st = 0; st < kStages; ++st) mbar_init(smem_u32(&bars[st]), 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int st = 0; st < kStages && st < ntl; ++st) produce(st, st);
  int t = 0;
  bool aborted = false;
  for (; t < ntl; ++t) {
    const int st = t % kStages;
    const uint32_t par = (uint32_t)(t / kStages) & 1u;
    const bool ok = mbar_wait_bounded(smem_u32(&bars[st]), par, js.wait_ns);
    body(st);
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    if (tid == 0) {
      pending &= ~(1u << st);
      if (t + kStages < ntl) produce(st, t + kStages);
    }
  }
  if (aborted && tid == 0) {
    record_error(err, kErrTileWait);
    for (int u = t; u < ntl && u < t + kStages; ++u) {
      const int st = u % kStages;
      if (!(pending & (1u << st))) continue;
      if (!mbar_wait_bounded(smem_u32(&bars[st]), (uint32_t)(u / kStages) & 1u, js.wait_ns)) {
        record_error(err, kErrDrainWait);
        break;
      }
    }
  }
  return !aborted;
}

// --------------------------------------------------------- FP32C pack ----
// Writes the FP32 source records of one warp's 32 * NI receivers (NI / 4 tiles
// of kTile).  The tile origin is the FP64 mean of the tile's real particles;
// each record holds (x-o, x-o, y-o, y-o), (z-o, z-o, -1.5 m, -1.5 m),
// (2.5 m, 2.5 m, 0, 0) in FP32.  Padding entries get zeros (zero mass).
template <int NI>
__device__ __forceinline__ void pack_warp(long long n, long long ibase, int lane, const double* xn,
                                          const double* yn, const double* zn, const double* m,
                                          float4* rec, double4* org) {
  static_assert(NI % 4 == 0, "a warp must cover whole tiles");
#pragma unroll
  for (int q = 0; q < NI / 4; ++q) {
    double sx = 0.0, sy = 0.0, sz = 0.0, cnt = 0.0;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const int k = 4 * q + kk;
      if (ibase + 32 * k < n) {
        sx += xn[k]; sy += yn[k]; sz += zn[k]; cnt += 1.0;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, off);
      sy += __shfl_xor_sync(0xffffffffu, sy, off);
      sz += __shfl_xor_sync(0xffffffffu, sz, off);
      cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    }
    const double ox = cnt > 0.0 ? sx / cnt : 0.0;
    const double oy = cnt > 0.0 ? sy / cnt : 0.0;
    const double oz = cnt > 0.0 ? sz / cnt : 0.0;
    const long long tile = (ibase - lane + (long long)kTile * q) / kTile;
    if (lane == 0) org[tile] = make_double4(ox, oy, oz, 0.0);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const int k = 4 * q + kk;
      const long long i = ibase + 32 * k;
      float fx = 0.f, fy = 0.f, fz = 0.f, fa = 0.f, fb = 0.f;
      if (i < n) {
        fx = __double2float_rn(xn[k] - ox);
        fy = __double2float_rn(yn[k] - oy);
        fz = __double2float_rn(zn[k] - oz);
        fa = __double2float_rn(-1.5 * m[i]);
        fb = __double2float_rn(2.5 * m[i]);
      }
      rec[3 * i + 0] = make_float4(fx, fx, fy, fy);
      rec[3 * i + 1] = make_float4(fz, fz, fa, fa);
      rec[3 * i + 2] = make_float4(fb, fb, 0.f, 0.f);
    }
  }
}

// ------------------------------------------------------------ epilogue ----
template <int NI>
__device__ __forceinline__ void epilogue(const IParticles& ip, const Epilogue& ep, long long ibase,
                                         int lane, const double* xi, const double* yi,
                                         const double* zi, const double* ax, const double* ay,
                                         const double* az) {
  if (ep.mode == 0) {
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      const long long i = ibase + 32 * k;
      if (i < ip.n) {
        const double sc = ep.want_force ? ep.G * ip.m[i] : ep.G;
        ep.ax[i] = sc * ax[k];
        ep.ay[i] = sc * ay[k];
        ep.az[i] = sc * az[k];
      }
    }
    return;
  }
  double xn[NI], yn[NI], zn[NI];
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = ibase + 32 * k;
    xn[k] = yn[k] = zn[k] = 0.0;
    if (i < ip.n) {
      const double gx = ep.G * ax[k], gy = ep.G * ay[k], gz = ep.G * az[k];
      ep.ax[i] = gx; ep.ay[i] = gy; ep.az[i] = gz;
      const double ux = ep.vx[i], uy = ep.vy[i], uz = ep.vz[i];
      const double vx = ux + ep.kick * gx;
      const double vy = uy + ep.kick * gy;
      const double vz = uz + ep.kick * gz;
      ep.vx[i] = vx; ep.vy[i] = vy; ep.vz[i] = vz;
      // mode 1: drift with the kicked velocity (leapfrog); mode 2: with the
      // old one (explicit Euler, reduced_solver_omp, CPU/omp_solver.cpp:121-135).
      const bool euler = ep.mode == 2;
      xn[k] = xi[k] + ep.drift * (euler ? ux : vx);
      yn[k] = yi[k] + ep.drift * (euler ? uy : vy);
      zn[k] = zi[k] + ep.drift * (euler ? uz : vz);
      ep.xn[i] = xn[k]; ep.yn[i] = yn[k]; ep.zn[i] = zn[k];
    }
  }
  if (ep.rec_next && NBR_IN(ibase - lane + 32 * NI - 1, ep.rec_len, ep.err))
    pack_warp<NI>(ip.n, ibase, lane, xn, yn, zn, ip.m, ep.rec_next, ep.origin_next);
}

// Split reduction (if any) followed by the epilogue.
template <int NI>
__device__ __forceinline__ void finish(const IParticles& ip, const Epilogue& ep, long long ibase,
                                       int lane, const double* xi, const double* yi,
                                       const double* zi, double* ax, double* ay, double* az) {
  if (gridDim.y > 1) {
    __shared__ int s_last;
    const long long np = ep.n_pad;
    double* P = ep.part + (size_t)blockIdx.y * 3 * (size_t)np;
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      const long long i = ibase + 32 * k;
      if (!NBR_IN((long long)blockIdx.y * 3 * np + 2 * np + i, ep.part_len, ep.err)) continue;
      P[i] = ax[k];
      P[np + i] = ay[k];
      P[2 * np + i] = az[k];
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned prev =
          NBR_IN(blockIdx.x, ep.cnt_len, ep.err) ? atomicAdd(&ep.counters[blockIdx.x], 1u) : 0u;
      s_last = (prev == gridDim.y - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      const long long i = ibase + 32 * k;
      double sx = 0.0, sy = 0.0, sz = 0.0;
      for (int s = 0; s < (int)gridDim.y; ++s) {
        const double* Q = ep.part + (size_t)s * 3 * (size_t)np;
        if (!NBR_IN((long long)s * 3 * np + 2 * np + i, ep.part_len, ep.err)) continue;
        sx += __ldcg(Q + i);
        sy += __ldcg(Q + np + i);
        sz += __ldcg(Q + 2 * np + i);
      }
      ax[k] = sx; ay[k] = sy; az[k] = sz;
    }
    if (threadIdx.x == 0 && NBR_IN(blockIdx.x, ep.cnt_len, ep.err)) ep.counters[blockIdx.x] = 0u;
  }
  epilogue<NI>(ip, ep, ibase, lane, xi, yi, zi, ax, ay, az);
}

// ------------------------------------------------------ FP32C kernel ----
// Stage bytes of the large FP32C kernel with TJ sources per stage: the
// records plus the FP64 origins of the 128-particle tiles the stage spans (one
// for TJ = 64, the origin of the tile it lies in).
template <int TJ>
__host__ __device__ constexpr int stage32_bytes() { return TJ * 48 + 32 * (TJ >= kTile ? TJ / kTile : 1); }

// TJ: sources per ring stage (64, 128, 256); UNR: unroll depth of the source
// loop.  The compensated sum works per 128-source tile (per 64 for TJ = 64),
// whatever TJ is.
template <int NI, int WARPS, bool EXCL, int TJ, int UNR>
__global__ void __launch_bounds__(WARPS * 32)
    k_force_f32c(const IParticles ip, const JStream js, const Epilogue ep, const float eps2f) {
  constexpr int IPAIR = NI / 2;
  constexpr int SUB = TJ >= kTile ? kTile : TJ;  // sources per origin
  constexpr int NSUB = TJ / SUB;
  constexpr int SB = stage32_bytes<TJ>();
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long ibase = ((long long)blockIdx.x * WARPS + warp) * (32 * NI) + lane;
  const int S = gridDim.y, sp = blockIdx.y;
  const int nch = (int)(((long long)js.ntiles * kTile + TJ - 1) / TJ);  // stages of sources
  const int t0 = (int)((long long)nch * sp / S);
  const int t1 = (int)((long long)nch * (sp + 1) / S);

  double xi[NI], yi[NI], zi[NI];
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = ibase + 32 * k;
    xi[k] = yi[k] = zi[k] = 0.0;
    if (NBR_IN(i, ip.len, ep.err)) { xi[k] = ip.x[i]; yi[k] = ip.y[i]; zi[k] = ip.z[i]; }
  }
  u64 hx[IPAIR], hy[IPAIR], hz[IPAIR], lx[IPAIR], ly[IPAIR], lz[IPAIR];
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) hx[p] = hy[p] = hz[p] = lx[p] = ly[p] = lz[p] = 0ull;
  const u64 EPS2 = pack2(eps2f, eps2f);

  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * SB;
    const uint32_t bar = smem_u32(&bars[st]);
    const long long first = (long long)(t0 + t) * TJ;  // first source of the stage
    if (!NBR_IN(first + TJ - 1, js.len, ep.err)) return;  // the wait expires
    mbar_expect_tx(bar, SB);
    bulk_g2s(dst, js.rec + (size_t)first * 3, TJ * 48, bar);
    bulk_g2s(dst + TJ * 48, js.origin + first / kTile, 32 * NSUB, bar);
  };
  int tcur = t0;
  auto body = [&](int st) {
    const unsigned char* base = stages + st * SB;
    const long long first = (long long)(tcur++) * TJ;
#pragma unroll
    for (int sb = 0; sb < NSUB; ++sb) {
      // a 128-tile past the system's last one holds no records of it
      if (NSUB > 1 && (first + sb * SUB) / kTile >= js.ntiles) break;
      const double4 o = *reinterpret_cast<const double4*>(base + TJ * 48 + 32 * sb);
      u64 XI[IPAIR], YI[IPAIR], ZI[IPAIR], AX[IPAIR], AY[IPAIR], AZ[IPAIR];
#pragma unroll
      for (int p = 0; p < IPAIR; ++p) {
        XI[p] = pack2(__double2float_rn(xi[2 * p] - o.x), __double2float_rn(xi[2 * p + 1] - o.x));
        YI[p] = pack2(__double2float_rn(yi[2 * p] - o.y), __double2float_rn(yi[2 * p + 1] - o.y));
        ZI[p] = pack2(__double2float_rn(zi[2 * p] - o.z), __double2float_rn(zi[2 * p + 1] - o.z));
        AX[p] = AY[p] = AZ[p] = 0ull;
      }
      const ulonglong2* R = reinterpret_cast<const ulonglong2*>(base) + 3 * SUB * sb;
#pragma unroll UNR
      for (int j = 0; j < SUB; ++j) {
        const ulonglong2 q0 = R[3 * j];
        const ulonglong2 q1 = R[3 * j + 1];
        const u64 bj = R[3 * j + 2].x;
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
          const u64 s = mul2(y3, mg);
          AX[p] = fma2(s, dx, AX[p]);
          AY[p] = fma2(s, dy, AY[p]);
          AZ[p] = fma2(s, dz, AZ[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < IPAIR; ++p) {
        two_sum2(hx[p], lx[p], AX[p]);
        two_sum2(hy[p], ly[p], AY[p]);
        two_sum2(hz[p], lz[p], AZ[p]);
      }
    }
  };
  if (!tile_pipeline(bars, t1 - t0, js, ep.err, issue, body)) return;

  double ax[NI], ay[NI], az[NI];
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) {
    float h0, h1, l0, l1;
    unpack2(hx[p], h0, h1); unpack2(lx[p], l0, l1);
    ax[2 * p] = (double)h0 + (double)l0; ax[2 * p + 1] = (double)h1 + (double)l1;
    unpack2(hy[p], h0, h1); unpack2(ly[p], l0, l1);
    ay[2 * p] = (double)h0 + (double)l0; ay[2 * p + 1] = (double)h1 + (double)l1;
    unpack2(hz[p], h0, h1); unpack2(lz[p], l0, l1);
    az[2 * p] = (double)h0 + (double)l0; az[2 * p + 1] = (double)h1 + (double)l1;
  }
  finish<NI>(ip, ep, ibase, lane, xi, yi, zi, ax, ay, az);
}

// ------------------------------------------------------- FP64 kernel ----
// The drop-in form: every operation in FP64, the reciprocal square root from
// CUDA's rsqrt(double).  Matches the reference's double-precision forces up to
// summation order.  TJ sources per ring stage (x, y, z, m: 32 TJ bytes), UNR
// the unroll depth of the source loop.
template <int NI, int WARPS, bool EXCL, int TJ, int UNR>
__global__ void __launch_bounds__(WARPS * 32)
    k_force_f64(const IParticles ip, const JStream js, const Epilogue ep, const double eps2) {
  constexpr int SB = 32 * TJ;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long ibase = ((long long)blockIdx.x * WARPS + warp) * (32 * NI) + lane;
  const int S = gridDim.y, sp = blockIdx.y;
  const int nch = (int)(((long long)js.ntiles * kTile + TJ - 1) / TJ);
  const int t0 = (int)((long long)nch * sp / S);
  const int t1 = (int)((long long)nch * (sp + 1) / S);

  double xi[NI], yi[NI], zi[NI], ax[NI], ay[NI], az[NI];
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = ibase + 32 * k;
    xi[k] = yi[k] = zi[k] = 0.0;
    if (NBR_IN(i, ip.len, ep.err)) { xi[k] = ip.x[i]; yi[k] = ip.y[i]; zi[k] = ip.z[i]; }
    ax[k] = ay[k] = az[k] = 0.0;
  }

  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * SB;
    const uint32_t bar = smem_u32(&bars[st]);
    const size_t off = (size_t)(t0 + t) * TJ;
    if (!NBR_IN((long long)off + TJ - 1, js.len, ep.err)) return;  // the wait expires
    mbar_expect_tx(bar, SB);
    bulk_g2s(dst, js.x + off, TJ * 8, bar);
    bulk_g2s(dst + TJ * 8, js.y + off, TJ * 8, bar);
    bulk_g2s(dst + 2 * TJ * 8, js.z + off, TJ * 8, bar);
    bulk_g2s(dst + 3 * TJ * 8, js.m + off, TJ * 8, bar);
  };
  auto body = [&](int st) {
    const double* sx = reinterpret_cast<const double*>(stages + st * SB);
    const double* sy = sx + TJ;
    const double* sz = sy + TJ;
    const double* sm = sz + TJ;
#pragma unroll UNR
    for (int j = 0; j < TJ; ++j) {
      const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
        double r2 = fma(dx, dx, eps2);
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
  };
  if (!tile_pipeline(bars, t1 - t0, js, ep.err, issue, body)) return;
  finish<NI>(ip, ep, ibase, lane, xi, yi, zi, ax, ay, az);
}

// ------------------------------------------------- small-N force kernel ----
// Warp-shuffle splitting for systems too small to fill the GPU with 32 * NI
// receivers per warp: each warp splits into F lane groups of G = 32 / F
// lanes; every group holds the same G * kSmallNI receivers (lane gl:
// receivers base + gl + G k) and takes every F-th source of each tile.  The
// groups' sums are combined with xor shuffles in a fixed order
// (deterministic).  A CTA of kSmallWarps warps covers
// kSmallWarps * G * kSmallNI receivers and, as in the large kernels, one range
// of the split source tiles.  Pair arithmetic is that of k_force_f32c /
// k_force_f64.  The fused FP32C record pack is left to the next evaluation's
// pack kernel.
template <int PREC, int F, bool EXCL>
__global__ void __launch_bounds__(kSmallWarps * 32)
    k_force_small(const IParticles ip, const JStream js, const Epilogue ep, const double eps2) {
  constexpr int G = 32 / F;
  constexpr int NI = kSmallNI;
  constexpr int IPAIR = NI / 2;
  constexpr int SB = PREC == kFP32C ? kStage32 : kStage64;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_last;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gl = lane % G, phase = lane / G;
  const long long rbase = ((long long)blockIdx.x * kSmallWarps + warp) * (G * NI) + gl;
  const int S = gridDim.y, sp = blockIdx.y;
  const int t0 = (int)((long long)js.ntiles * sp / S);
  const int t1 = (int)((long long)js.ntiles * (sp + 1) / S);

  double xi[NI], yi[NI], zi[NI], ax[NI], ay[NI], az[NI];
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = rbase + G * k;
    xi[k] = yi[k] = zi[k] = 0.0;
    if (NBR_IN(i, ip.len, ep.err)) { xi[k] = ip.x[i]; yi[k] = ip.y[i]; zi[k] = ip.z[i]; }
    ax[k] = ay[k] = az[k] = 0.0;
  }
  u64 hx[IPAIR], hy[IPAIR], hz[IPAIR], lx[IPAIR], ly[IPAIR], lz[IPAIR];
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) hx[p] = hy[p] = hz[p] = lx[p] = ly[p] = lz[p] = 0ull;
  const float e2f = (float)eps2;
  const u64 EPS2 = pack2(e2f, e2f);

  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * SB;
    const uint32_t bar = smem_u32(&bars[st]);
    const size_t tile = (size_t)(t0 + t);
    if (!NBR_IN((long long)(tile + 1) * kTile - 1, js.len, ep.err)) return;  // the wait expires
    mbar_expect_tx(bar, SB);
    if (PREC == kFP32C) {
      bulk_g2s(dst, js.rec + tile * kTile * 3, kRecBytes, bar);
      bulk_g2s(dst + kRecBytes, js.origin + tile, 32, bar);
    } else {
      const size_t off = tile * kTile;
      bulk_g2s(dst, js.x + off, kTile * 8, bar);
      bulk_g2s(dst + kTile * 8, js.y + off, kTile * 8, bar);
      bulk_g2s(dst + 2 * kTile * 8, js.z + off, kTile * 8, bar);
      bulk_g2s(dst + 3 * kTile * 8, js.m + off, kTile * 8, bar);
    }
  };
  auto body = [&](int st) {
    const unsigned char* base = stages + st * SB;
    if (PREC == kFP32C) {
      const double4 o = *reinterpret_cast<const double4*>(base + kRecBytes);
      u64 XI[IPAIR], YI[IPAIR], ZI[IPAIR], AX[IPAIR], AY[IPAIR], AZ[IPAIR];
#pragma unroll
      for (int p = 0; p < IPAIR; ++p) {
        XI[p] = pack2(__double2float_rn(xi[2 * p] - o.x), __double2float_rn(xi[2 * p + 1] - o.x));
        YI[p] = pack2(__double2float_rn(yi[2 * p] - o.y), __double2float_rn(yi[2 * p + 1] - o.y));
        ZI[p] = pack2(__double2float_rn(zi[2 * p] - o.z), __double2float_rn(zi[2 * p + 1] - o.z));
        AX[p] = AY[p] = AZ[p] = 0ull;
      }
      const ulonglong2* R = reinterpret_cast<const ulonglong2*>(base);
#pragma unroll 4
      for (int j = phase; j < kTile; j += F) {
        const ulonglong2 q0 = R[3 * j];
        const ulonglong2 q1 = R[3 * j + 1];
        const u64 bj = R[3 * j + 2].x;
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
          const u64 s = mul2(y3, mg);
          AX[p] = fma2(s, dx, AX[p]);
          AY[p] = fma2(s, dy, AY[p]);
          AZ[p] = fma2(s, dz, AZ[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < IPAIR; ++p) {
        two_sum2(hx[p], lx[p], AX[p]);
        two_sum2(hy[p], ly[p], AY[p]);
        two_sum2(hz[p], lz[p], AZ[p]);
      }
    } else {
      const double* sx = reinterpret_cast<const double*>(base);
      const double* sy = sx + kTile;
      const double* sz = sy + kTile;
      const double* sm = sz + kTile;
#pragma unroll 2
      for (int j = phase; j < kTile; j += F) {
        const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
        for (int k = 0; k < NI; ++k) {
          const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
          double r2 = fma(dx, dx, eps2);
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
    }
  };
  if (!tile_pipeline(bars, t1 - t0, js, ep.err, issue, body)) return;

  if (PREC == kFP32C) {
#pragma unroll
    for (int p = 0; p < IPAIR; ++p) {
      float h0, h1, l0, l1;
      unpack2(hx[p], h0, h1); unpack2(lx[p], l0, l1);
      ax[2 * p] = (double)h0 + (double)l0; ax[2 * p + 1] = (double)h1 + (double)l1;
      unpack2(hy[p], h0, h1); unpack2(ly[p], l0, l1);
      ay[2 * p] = (double)h0 + (double)l0; ay[2 * p + 1] = (double)h1 + (double)l1;
      unpack2(hz[p], h0, h1); unpack2(lz[p], l0, l1);
      az[2 * p] = (double)h0 + (double)l0; az[2 * p + 1] = (double)h1 + (double)l1;
    }
  }
  // Lane groups -> one sum per receiver (every lane of a gl ends with it).
#pragma unroll
  for (int off = G; off < 32; off <<= 1) {
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      ax[k] += __shfl_xor_sync(0xffffffffu, ax[k], off);
      ay[k] += __shfl_xor_sync(0xffffffffu, ay[k], off);
      az[k] += __shfl_xor_sync(0xffffffffu, az[k], off);
    }
  }
  if (S > 1) {
    const long long np = ep.n_pad;
    double* P = ep.part + (size_t)sp * 3 * (size_t)np;
    if (phase == 0) {
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const long long i = rbase + G * k;
        if (!NBR_IN((long long)sp * 3 * np + 2 * np + i, ep.part_len, ep.err)) continue;
        P[i] = ax[k];
        P[np + i] = ay[k];
        P[2 * np + i] = az[k];
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned prev =
          NBR_IN(blockIdx.x, ep.cnt_len, ep.err) ? atomicAdd(&ep.counters[blockIdx.x], 1u) : 0u;
      s_last = (prev == gridDim.y - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (phase == 0) {
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const long long i = rbase + G * k;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int q = 0; q < S; ++q) {
          if (!NBR_IN((long long)q * 3 * np + 2 * np + i, ep.part_len, ep.err)) continue;
          const double* Q = ep.part + (size_t)q * 3 * (size_t)np;
          sx += __ldcg(Q + i);
          sy += __ldcg(Q + np + i);
          sz += __ldcg(Q + 2 * np + i);
        }
        ax[k] = sx; ay[k] = sy; az[k] = sz;
      }
    }
    if (threadIdx.x == 0 && NBR_IN(blockIdx.x, ep.cnt_len, ep.err)) ep.counters[blockIdx.x] = 0u;
  }
  if (phase != 0) return;
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = rbase + G * k;
    if (i >= ip.n) continue;
    if (ep.mode == 0) {
      const double sc = ep.want_force ? ep.G * ip.m[i] : ep.G;
      ep.ax[i] = sc * ax[k]; ep.ay[i] = sc * ay[k]; ep.az[i] = sc * az[k];
      continue;
    }
    const double gx = ep.G * ax[k], gy = ep.G * ay[k], gz = ep.G * az[k];
    ep.ax[i] = gx; ep.ay[i] = gy; ep.az[i] = gz;
    const double ux = ep.vx[i], uy = ep.vy[i], uz = ep.vz[i];
    const double vx = ux + ep.kick * gx, vy = uy + ep.kick * gy, vz = uz + ep.kick * gz;
    ep.vx[i] = vx; ep.vy[i] = vy; ep.vz[i] = vz;
    const bool euler = ep.mode == 2;
    ep.xn[i] = xi[k] + ep.drift * (euler ? ux : vx);
    ep.yn[i] = yi[k] + ep.drift * (euler ? uy : vy);
    ep.zn[i] = zi[k] + ep.drift * (euler ? uz : vz);
  }
}

// ------------------------------------------ Newton-3 FP32C force kernel ----
// Every unordered pair is evaluated once and acts on both particles, as the
// reference's blocked kernels do (compute_forces_avx512_rsqrt_4i_blocked
// applies +f to the receiver and -f to the source, CPU/force_calculation.cpp:
// 1137-1561).  Particles form blocks of kN3Block = 256 (2 tiles).  A CTA of
// kN3Warps warps owns row group g (row blocks 8g .. 8g+7, one per warp, 8
// receivers per lane as in k_force_f32c) and a chunk of up to p3.cols column
// blocks (group g's chunks tile its column blocks 8g .. nb - 1; the width from
// the grid model of n3_cols / n3_slice_cols); the column tiles stream through
// the bulk-copy ring.  Warp a and column block c:
//   c < a   nothing (the pair of blocks belongs to warp c);
//   c == a  every ordered pair of the block, action only (the k_force_f32c body);
//   c > a   each unordered pair once: the 32 sources of a batch sit one per
//           lane and rotate through the warp with shuffles, carrying their
//           reaction sums, so after 32 steps every source has met all 256
//           receivers of the warp and holds its reaction from them.
// Per unordered pair: the 14 FMA-pipe operations of k_force_f32c plus 5 for
// the reaction (receiver-mass correction, its product, 3 accumulations), and
// one MUFU rsqrt: 9.5 operations per ordered pair instead of 14.
// Results leave as FP64 partial sums: per (CTA, row block) the action, per
// (CTA, column block) the reaction (summed over the CTA's warps in warp
// order); k_n3_reduce adds them per particle in a fixed order and runs the
// epilogue.  Deterministic.  RANGED: the launch covers the row groups
// [p3.g0, p3.g1) (a slice); otherwise all of them (a separate instantiation,
// the whole-system launch keeps its own code).
template <bool EXCL, bool RANGED>
__global__ void __launch_bounds__(kN3Warps * 32)
    k_force_n3_f32c(const IParticles ip, const JStream js, const N3Params p3, const float eps2f,
                    int* err) {
  constexpr int NI = 8, IPAIR = 4;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;
  float* red = reinterpret_cast<float*>(stages + kStages * kStage32);  // [warp][3][256]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // (row group, chunk) from the CTA's group-major number (whole-system
  // launches run in the longest-first order of p3.order); the partial sums are
  // indexed by blockIdx.x (a register-free index in the hot loop)
  int g = RANGED ? p3.g0 : 0, k = RANGED ? (int)blockIdx.x : p3.order[blockIdx.x];
  // row groups [g0, g1) of this launch
  const int groups = RANGED ? p3.g1 : (int)((p3.nb + kN3Warps - 1) / kN3Warps);
  while (g < groups) {  // the grid has exactly sum_g n3_chunks(nb, cols, g) CTAs
    const int K = n3_chunks(p3.nb, p3.cols, g);
    if (k < K) break;
    k -= K;
    ++g;
  }
  if (g >= groups) return;
  const long long r0 = (long long)g * kN3Warps;
  const long long a = r0 + warp;
  const long long cs = r0 + (long long)k * p3.cols;
  const long long ce = min(cs + (long long)p3.cols, p3.nb);
  const int ntl = (int)(2 * (ce - cs));
  const bool row_ok = a < p3.nb;
  const long long ibase = a * kN3Block + lane;

  double xi[NI], yi[NI], zi[NI];
  u64 AI[IPAIR], BI[IPAIR];
#pragma unroll
  for (int q = 0; q < NI; ++q) xi[q] = yi[q] = zi[q] = 0.0;
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) {
    float m0 = 0.f, m1 = 0.f;
    if (row_ok) {
      const long long i0 = ibase + 64 * p, i1 = i0 + 32;
      if (NBR_IN(i1, ip.len, err)) {
        xi[2 * p] = ip.x[i0]; yi[2 * p] = ip.y[i0]; zi[2 * p] = ip.z[i0];
        xi[2 * p + 1] = ip.x[i1]; yi[2 * p + 1] = ip.y[i1]; zi[2 * p + 1] = ip.z[i1];
        m0 = (float)ip.m[i0];
        m1 = (float)ip.m[i1];
      }
    }
    AI[p] = pack2(-1.5f * m0, -1.5f * m1);
    BI[p] = pack2(2.5f * m0, 2.5f * m1);
  }
  u64 hx[IPAIR], hy[IPAIR], hz[IPAIR], lx[IPAIR], ly[IPAIR], lz[IPAIR];
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) hx[p] = hy[p] = hz[p] = lx[p] = ly[p] = lz[p] = 0ull;
  const u64 EPS2 = pack2(eps2f, eps2f);

  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * kStage32;
    const uint32_t bar = smem_u32(&bars[st]);
    const long long tile = 2 * cs + t;
    if (!NBR_IN((tile + 1) * kTile - 1, js.len, err)) return;  // the wait expires
    mbar_expect_tx(bar, kStage32);
    bulk_g2s(dst, js.rec + (size_t)tile * kTile * 3, kRecBytes, bar);
    bulk_g2s(dst + kRecBytes, js.origin + tile, 32, bar);
  };
  int tcur = 0;
  auto body = [&](int st) {
    const int t = tcur++;
    const long long c = cs + t / 2;
    const int half = t & 1;
    const unsigned char* base = stages + st * kStage32;
    const double4 o = *reinterpret_cast<const double4*>(base + kRecBytes);
    u64 XI[IPAIR], YI[IPAIR], ZI[IPAIR], AX[IPAIR], AY[IPAIR], AZ[IPAIR];
#pragma unroll
    for (int p = 0; p < IPAIR; ++p) {
      // pair p: receivers 2p (lane + 64p) and 2p + 1 (lane + 64p + 32)
      XI[p] = pack2(__double2float_rn(xi[2 * p] - o.x), __double2float_rn(xi[2 * p + 1] - o.x));
      YI[p] = pack2(__double2float_rn(yi[2 * p] - o.y), __double2float_rn(yi[2 * p + 1] - o.y));
      ZI[p] = pack2(__double2float_rn(zi[2 * p] - o.z), __double2float_rn(zi[2 * p + 1] - o.z));
      AX[p] = AY[p] = AZ[p] = 0ull;
    }
    float* myred = red + warp * 3 * kN3Block + half * kTile;
    if (row_ok && c == a) {
      const ulonglong2* R = reinterpret_cast<const ulonglong2*>(base);
#pragma unroll 4
      for (int j = 0; j < kTile; ++j) {
        const ulonglong2 q0 = R[3 * j];
        const ulonglong2 q1 = R[3 * j + 1];
        const u64 bj = R[3 * j + 2].x;
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
          const u64 s = mul2(y3, mg);
          AX[p] = fma2(s, dx, AX[p]);
          AY[p] = fma2(s, dy, AY[p]);
          AZ[p] = fma2(s, dz, AZ[p]);
        }
      }
#pragma unroll
      for (int bt = 0; bt < 4; ++bt)
        myred[bt * 32 + lane] = myred[kN3Block + bt * 32 + lane] = myred[2 * kN3Block + bt * 32 + lane] = 0.f;
    } else if (row_ok && c > a) {
      const float4* R4 = reinterpret_cast<const float4*>(base);
      const int from = (lane + 31) & 31;
#pragma unroll 1
      for (int bt = 0; bt < 4; ++bt) {
        const int j = bt * 32 + lane;
        const float4 q0 = R4[3 * j], q1 = R4[3 * j + 1], q2 = R4[3 * j + 2];
        float sx = q0.x, sy = q0.z, sz = q1.x, sa = q1.z, sb = q2.x;
        u64 RX = 0ull, RY = 0ull, RZ = 0ull;
#pragma unroll 2
        for (int step = 0; step < 32; ++step) {
          const u64 SX = pack2(sx, sx), SY = pack2(sy, sy), SZ = pack2(sz, sz);
          const u64 SA = pack2(sa, sa), SB = pack2(sb, sb);
#pragma unroll
          for (int p = 0; p < IPAIR; ++p) {
            const u64 dx = sub2(SX, XI[p]);
            const u64 dy = sub2(SY, YI[p]);
            const u64 dz = sub2(SZ, ZI[p]);
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
            const u64 y3 = mul2(y2, y);
            const u64 sj = mul2(y3, fma2(SA, pr, SB));  // m_j (1 + 3e/2) y^3
            const u64 si = mul2(y3, fma2(AI[p], pr, BI[p]));  // m_i (1 + 3e/2) y^3
            // the reaction sums first: this order schedules 2.4 % faster than
            // the action first (same instructions; measured at N = 262144)
            RX = fma2(si, dx, RX);
            RY = fma2(si, dy, RY);
            RZ = fma2(si, dz, RZ);
            AX[p] = fma2(sj, dx, AX[p]);
            AY[p] = fma2(sj, dy, AY[p]);
            AZ[p] = fma2(sj, dz, AZ[p]);
          }
          // (the reaction sums' shuffles first: 0.25 % faster than after the sources')
          RX = __shfl_sync(0xffffffffu, RX, from);
          RY = __shfl_sync(0xffffffffu, RY, from);
          RZ = __shfl_sync(0xffffffffu, RZ, from);
          sx = __shfl_sync(0xffffffffu, sx, from);
          sy = __shfl_sync(0xffffffffu, sy, from);
          sz = __shfl_sync(0xffffffffu, sz, from);
          sa = __shfl_sync(0xffffffffu, sa, from);
          sb = __shfl_sync(0xffffffffu, sb, from);
        }
        // back at its own lane: the force on source j is -sum s_i d
        float u0, u1;
        unpack2(RX, u0, u1); myred[bt * 32 + lane] = -(u0 + u1);
        unpack2(RY, u0, u1); myred[kN3Block + bt * 32 + lane] = -(u0 + u1);
        unpack2(RZ, u0, u1); myred[2 * kN3Block + bt * 32 + lane] = -(u0 + u1);
      }
    } else {
#pragma unroll
      for (int bt = 0; bt < 4; ++bt)
        myred[bt * 32 + lane] = myred[kN3Block + bt * 32 + lane] = myred[2 * kN3Block + bt * 32 + lane] = 0.f;
    }
#pragma unroll
    for (int p = 0; p < IPAIR; ++p) {
      two_sum2(hx[p], lx[p], AX[p]);
      two_sum2(hy[p], ly[p], AY[p]);
      two_sum2(hz[p], lz[p], AZ[p]);
    }
    if (half == 1) {
      // end of column block c: its reaction from this CTA's rows, summed in
      // warp order in FP64, to the block's partial slot
      __syncthreads();
      const int tid = threadIdx.x;  // one source of the block per thread
      const long long off = ((long long)blockIdx.x * p3.cols + (c - cs)) * 3 * kN3Block;
      double* out = p3.rea + off;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int w = 0; w < kN3Warps; ++w) s += (double)red[(w * 3 + d) * kN3Block + tid];
        if (NBR_IN((p3.rea - p3.act) + off + d * kN3Block + tid, p3.act_len, err))
          out[d * kN3Block + tid] = s;
      }
      __syncthreads();
    }
  };
  if (!tile_pipeline(bars, ntl, js, err, issue, body)) return;
  double* act = p3.act + ((size_t)blockIdx.x * kN3Warps + warp) * 3 * kN3Block;
  if (!NBR_IN(((long long)blockIdx.x * kN3Warps + warp + 1) * 3 * kN3Block - 1, p3.act_len, err))
    return;
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) {
    float h0, h1, l0, l1;
    unpack2(hx[p], h0, h1); unpack2(lx[p], l0, l1);
    act[lane + 64 * p] = (double)h0 + (double)l0;
    act[lane + 64 * p + 32] = (double)h1 + (double)l1;
    unpack2(hy[p], h0, h1); unpack2(ly[p], l0, l1);
    act[kN3Block + lane + 64 * p] = (double)h0 + (double)l0;
    act[kN3Block + lane + 64 * p + 32] = (double)h1 + (double)l1;
    unpack2(hz[p], h0, h1); unpack2(lz[p], l0, l1);
    act[2 * kN3Block + lane + 64 * p] = (double)h0 + (double)l0;
    act[2 * kN3Block + lane + 64 * p + 32] = (double)h1 + (double)l1;
  }
}

// Two warps per row block (ForceConfig {3, 16} for FP32C): the blocks, CTA
// map, source rotation and partial-sum layout of k_force_n3_f32c, with 16
// warps per CTA: warp w takes row block a = r0 + w / 2 and, in lane L, its
// receivers a * kN3Block + 128 (w % 2) + L + 32 q, q < 4 (two packed pairs).
// Half the receivers per lane keeps a thread under 128 registers, so twice
// the warps share an SM and hide the latency of the rotation's dependent
// shuffles, at 11 shuffles per 4 unordered pairs instead of per 8.  The
// reaction staging sums the two warps' halves in warp order; the results
// equal k_force_n3_f32c's to FP32 rounding of the per-warp reaction sums.
template <bool EXCL>
__global__ void __launch_bounds__(kN3F64Warps * 32, 1)
    k_force_n3_f32c_w2(const IParticles ip, const JStream js, const N3Params p3, const float eps2f,
                       int* err) {
  constexpr int NI = 4, IPAIR = 2, WARPS = kN3F64Warps;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;
  float* red = reinterpret_cast<float*>(stages + kStages * kStage32);  // [warp][3][256]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rb = warp >> 1, hf = warp & 1;  // row block in the group, its receiver half
  int g = p3.g0, k = p3.order ? p3.order[blockIdx.x] : (int)blockIdx.x;  // group-major number
  const int groups = p3.g1;  // row groups [g0, g1) of this launch
  while (g < groups) {  // the grid has exactly sum_g n3_chunks(nb, cols, g) CTAs
    const int K = n3_chunks(p3.nb, p3.cols, g);
    if (k < K) break;
    k -= K;
    ++g;
  }
  if (g >= groups) return;
  const long long r0 = (long long)g * kN3Warps;
  const long long a = r0 + rb;
  const long long cs = r0 + (long long)k * p3.cols;
  const long long ce = min(cs + (long long)p3.cols, p3.nb);
  const int ntl = (int)(2 * (ce - cs));
  const bool row_ok = a < p3.nb;
  const long long ibase = a * kN3Block + hf * (kN3Block / 2) + lane;

  double xi[NI], yi[NI], zi[NI];
  u64 AI[IPAIR], BI[IPAIR];
#pragma unroll
  for (int q = 0; q < NI; ++q) xi[q] = yi[q] = zi[q] = 0.0;
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) {
    float m0 = 0.f, m1 = 0.f;
    if (row_ok) {
      const long long i0 = ibase + 64 * p, i1 = i0 + 32;
      if (NBR_IN(i1, ip.len, err)) {
        xi[2 * p] = ip.x[i0]; yi[2 * p] = ip.y[i0]; zi[2 * p] = ip.z[i0];
        xi[2 * p + 1] = ip.x[i1]; yi[2 * p + 1] = ip.y[i1]; zi[2 * p + 1] = ip.z[i1];
        m0 = (float)ip.m[i0];
        m1 = (float)ip.m[i1];
      }
    }
    AI[p] = pack2(-1.5f * m0, -1.5f * m1);
    BI[p] = pack2(2.5f * m0, 2.5f * m1);
  }
  u64 hx[IPAIR], hy[IPAIR], hz[IPAIR], lx[IPAIR], ly[IPAIR], lz[IPAIR];
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) hx[p] = hy[p] = hz[p] = lx[p] = ly[p] = lz[p] = 0ull;
  const u64 EPS2 = pack2(eps2f, eps2f);

  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * kStage32;
    const uint32_t bar = smem_u32(&bars[st]);
    const long long tile = 2 * cs + t;
    if (!NBR_IN((tile + 1) * kTile - 1, js.len, err)) return;  // the wait expires
    mbar_expect_tx(bar, kStage32);
    bulk_g2s(dst, js.rec + (size_t)tile * kTile * 3, kRecBytes, bar);
    bulk_g2s(dst + kRecBytes, js.origin + tile, 32, bar);
  };
  int tcur = 0;
  auto body = [&](int st) {
    const int t = tcur++;
    const long long c = cs + t / 2;
    const int half = t & 1;
    const unsigned char* base = stages + st * kStage32;
    const double4 o = *reinterpret_cast<const double4*>(base + kRecBytes);
    u64 XI[IPAIR], YI[IPAIR], ZI[IPAIR], AX[IPAIR], AY[IPAIR], AZ[IPAIR];
#pragma unroll
    for (int p = 0; p < IPAIR; ++p) {
      XI[p] = pack2(__double2float_rn(xi[2 * p] - o.x), __double2float_rn(xi[2 * p + 1] - o.x));
      YI[p] = pack2(__double2float_rn(yi[2 * p] - o.y), __double2float_rn(yi[2 * p + 1] - o.y));
      ZI[p] = pack2(__double2float_rn(zi[2 * p] - o.z), __double2float_rn(zi[2 * p + 1] - o.z));
      AX[p] = AY[p] = AZ[p] = 0ull;
    }
    float* myred = red + warp * 3 * kN3Block + half * kTile;
    if (row_ok && c == a) {
      const ulonglong2* R = reinterpret_cast<const ulonglong2*>(base);
#pragma unroll 4
      for (int j = 0; j < kTile; ++j) {
        const ulonglong2 q0 = R[3 * j];
        const ulonglong2 q1 = R[3 * j + 1];
        const u64 bj = R[3 * j + 2].x;
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
          const u64 s = mul2(y3, mg);
          AX[p] = fma2(s, dx, AX[p]);
          AY[p] = fma2(s, dy, AY[p]);
          AZ[p] = fma2(s, dz, AZ[p]);
        }
      }
#pragma unroll
      for (int bt = 0; bt < 4; ++bt)
        myred[bt * 32 + lane] = myred[kN3Block + bt * 32 + lane] = myred[2 * kN3Block + bt * 32 + lane] = 0.f;
    } else if (row_ok && c > a) {
      const float4* R4 = reinterpret_cast<const float4*>(base);
      const int from = (lane + 31) & 31;
#pragma unroll 1
      for (int bt = 0; bt < 4; ++bt) {
        const int j = bt * 32 + lane;
        const float4 q0 = R4[3 * j], q1 = R4[3 * j + 1], q2 = R4[3 * j + 2];
        float sx = q0.x, sy = q0.z, sz = q1.x, sa = q1.z, sb = q2.x;
        u64 RX = 0ull, RY = 0ull, RZ = 0ull;
#pragma unroll 2
        for (int step = 0; step < 32; ++step) {
          const u64 SX = pack2(sx, sx), SY = pack2(sy, sy), SZ = pack2(sz, sz);
          const u64 SA = pack2(sa, sa), SB = pack2(sb, sb);
#pragma unroll
          for (int p = 0; p < IPAIR; ++p) {
            const u64 dx = sub2(SX, XI[p]);
            const u64 dy = sub2(SY, YI[p]);
            const u64 dz = sub2(SZ, ZI[p]);
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
            const u64 y3 = mul2(y2, y);
            const u64 sj = mul2(y3, fma2(SA, pr, SB));  // m_j (1 + 3e/2) y^3
            const u64 si = mul2(y3, fma2(AI[p], pr, BI[p]));  // m_i (1 + 3e/2) y^3
            AX[p] = fma2(sj, dx, AX[p]);
            AY[p] = fma2(sj, dy, AY[p]);
            AZ[p] = fma2(sj, dz, AZ[p]);
            RX = fma2(si, dx, RX);
            RY = fma2(si, dy, RY);
            RZ = fma2(si, dz, RZ);
          }
          sx = __shfl_sync(0xffffffffu, sx, from);
          sy = __shfl_sync(0xffffffffu, sy, from);
          sz = __shfl_sync(0xffffffffu, sz, from);
          sa = __shfl_sync(0xffffffffu, sa, from);
          sb = __shfl_sync(0xffffffffu, sb, from);
          RX = __shfl_sync(0xffffffffu, RX, from);
          RY = __shfl_sync(0xffffffffu, RY, from);
          RZ = __shfl_sync(0xffffffffu, RZ, from);
        }
        // back at its own lane: the force on source j is -sum s_i d
        float u0, u1;
        unpack2(RX, u0, u1); myred[bt * 32 + lane] = -(u0 + u1);
        unpack2(RY, u0, u1); myred[kN3Block + bt * 32 + lane] = -(u0 + u1);
        unpack2(RZ, u0, u1); myred[2 * kN3Block + bt * 32 + lane] = -(u0 + u1);
      }
    } else {
#pragma unroll
      for (int bt = 0; bt < 4; ++bt)
        myred[bt * 32 + lane] = myred[kN3Block + bt * 32 + lane] = myred[2 * kN3Block + bt * 32 + lane] = 0.f;
    }
#pragma unroll
    for (int p = 0; p < IPAIR; ++p) {
      two_sum2(hx[p], lx[p], AX[p]);
      two_sum2(hy[p], ly[p], AY[p]);
      two_sum2(hz[p], lz[p], AZ[p]);
    }
    if (half == 1) {
      // end of column block c: its reaction from this CTA's rows, summed in
      // warp order in FP64, to the block's partial slot
      __syncthreads();
      const int tid = threadIdx.x;  // one source of the block per thread
      if (tid < kN3Block) {
        const long long off = ((long long)blockIdx.x * p3.cols + (c - cs)) * 3 * kN3Block;
        double* out = p3.rea + off;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double s = 0.0;
          for (int w = 0; w < WARPS; ++w) s += (double)red[(w * 3 + d) * kN3Block + tid];
          if (NBR_IN((p3.rea - p3.act) + off + d * kN3Block + tid, p3.act_len, err))
            out[d * kN3Block + tid] = s;
        }
      }
      __syncthreads();
    }
  };
  if (!tile_pipeline(bars, ntl, js, err, issue, body)) return;
  double* act = p3.act + ((size_t)blockIdx.x * kN3Warps + rb) * 3 * kN3Block + hf * (kN3Block / 2);
  if (!NBR_IN(((long long)blockIdx.x * kN3Warps + rb + 1) * 3 * kN3Block - 1, p3.act_len, err))
    return;
#pragma unroll
  for (int p = 0; p < IPAIR; ++p) {
    float h0, h1, l0, l1;
    unpack2(hx[p], h0, h1); unpack2(lx[p], l0, l1);
    act[lane + 64 * p] = (double)h0 + (double)l0;
    act[lane + 64 * p + 32] = (double)h1 + (double)l1;
    unpack2(hy[p], h0, h1); unpack2(ly[p], l0, l1);
    act[kN3Block + lane + 64 * p] = (double)h0 + (double)l0;
    act[kN3Block + lane + 64 * p + 32] = (double)h1 + (double)l1;
    unpack2(hz[p], h0, h1); unpack2(lz[p], l0, l1);
    act[2 * kN3Block + lane + 64 * p] = (double)h0 + (double)l0;
    act[2 * kN3Block + lane + 64 * p + 32] = (double)h1 + (double)l1;
  }
}

// FP64 form of the Newton-3 kernel (ForceConfig ni = 3 with NBR_FP64): the
// blocks, CTA map, source rotation and partial-sum layout of k_force_n3_f32c,
// with every operation in FP64 and the reciprocal square root from CUDA's
// rsqrt(double), as in k_force_f64; the source tiles are the FP64 x, y, z, m
// arrays.  Two warps share each row block: warp w of the CTA takes row block
// a = r0 + w / 2 and, in lane L, its receivers a * kN3Block + 128 (w % 2) +
// L + 32 q, q < 4 (16 warps, under 128 registers: twice the warps per SM of
// a one-warp-per-block layout, for the long FP64 rsqrt chain).  Per
// unordered pair: 3 sub, 3 fma, rsqrt, 2 mul (y^3), 2 mul (m_j y^3, m_i y^3)
// and 6 fma, against 12 operations and one rsqrt per ordered pair in
// k_force_f64.  Equal to k_force_f64 up to summation order; deterministic.
template <bool EXCL>
__global__ void __launch_bounds__(kN3F64Warps * 32)
    k_force_n3_f64(const IParticles ip, const JStream js, const N3Params p3, const double eps2,
                   int* err) {
  constexpr int NI = kN3Block / 64;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;
  double* red = reinterpret_cast<double*>(stages + kStages * kStage64);  // [warp][3][256]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rb = warp >> 1, hf = warp & 1;  // row block in the group, its receiver half
  int g = p3.g0, k = p3.order ? p3.order[blockIdx.x] : (int)blockIdx.x;  // group-major number
  const int groups = p3.g1;  // row groups [g0, g1) of this launch
  while (g < groups) {  // the grid has exactly sum_g n3_chunks(nb, cols, g) CTAs
    const int K = n3_chunks(p3.nb, p3.cols, g);
    if (k < K) break;
    k -= K;
    ++g;
  }
  if (g >= groups) return;
  const long long r0 = (long long)g * kN3Warps;
  const long long a = r0 + rb;
  const long long cs = r0 + (long long)k * p3.cols;
  const long long ce = min(cs + (long long)p3.cols, p3.nb);
  const int ntl = (int)(2 * (ce - cs));
  const bool row_ok = a < p3.nb;
  const long long ibase = a * kN3Block + hf * (kN3Block / 2) + lane;

  double xi[NI], yi[NI], zi[NI], mi[NI], AX[NI], AY[NI], AZ[NI];
#pragma unroll
  for (int q = 0; q < NI; ++q) {
    xi[q] = yi[q] = zi[q] = mi[q] = 0.0;
    AX[q] = AY[q] = AZ[q] = 0.0;
    const long long i = ibase + 32 * q;
    if (row_ok && NBR_IN(i, ip.len, err)) {
      xi[q] = ip.x[i]; yi[q] = ip.y[i]; zi[q] = ip.z[i]; mi[q] = ip.m[i];
    }
  }

  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * kStage64;
    const uint32_t bar = smem_u32(&bars[st]);
    const size_t off = (size_t)(2 * cs + t) * kTile;
    if (!NBR_IN((long long)off + kTile - 1, js.len, err)) return;  // the wait expires
    mbar_expect_tx(bar, kStage64);
    bulk_g2s(dst, js.x + off, kTile * 8, bar);
    bulk_g2s(dst + kTile * 8, js.y + off, kTile * 8, bar);
    bulk_g2s(dst + 2 * kTile * 8, js.z + off, kTile * 8, bar);
    bulk_g2s(dst + 3 * kTile * 8, js.m + off, kTile * 8, bar);
  };
  int tcur = 0;
  auto body = [&](int st) {
    const int t = tcur++;
    const long long c = cs + t / 2;
    const int half = t & 1;
    const double* sx = reinterpret_cast<const double*>(stages + st * kStage64);
    const double* sy = sx + kTile;
    const double* sz = sy + kTile;
    const double* sm = sz + kTile;
    double* myred = red + warp * 3 * kN3Block + half * kTile;
    if (row_ok && c == a) {
      // every ordered pair of the block, action only (the k_force_f64 body)
#pragma unroll 2
      for (int j = 0; j < kTile; ++j) {
        const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
        for (int q = 0; q < NI; ++q) {
          const double dx = xj - xi[q], dy = yj - yi[q], dz = zj - zi[q];
          double r2 = fma(dx, dx, eps2);
          r2 = fma(dy, dy, r2);
          r2 = fma(dz, dz, r2);
          double y = rsqrt(r2);
          if (EXCL) y = r2 > 0.0 ? y : 0.0;
          const double s = mj * (y * y * y);
          AX[q] = fma(s, dx, AX[q]);
          AY[q] = fma(s, dy, AY[q]);
          AZ[q] = fma(s, dz, AZ[q]);
        }
      }
#pragma unroll
      for (int bt = 0; bt < 4; ++bt)
        myred[bt * 32 + lane] = myred[kN3Block + bt * 32 + lane] = myred[2 * kN3Block + bt * 32 + lane] = 0.0;
    } else if (row_ok && c > a) {
      const int from = (lane + 31) & 31;
#pragma unroll 1
      for (int bt = 0; bt < 4; ++bt) {
        const int j = bt * 32 + lane;
        double xs = sx[j], ys = sy[j], zs = sz[j], ms = sm[j];
        double RX = 0.0, RY = 0.0, RZ = 0.0;
#pragma unroll 1  // 3 % faster than unrolled by 2 or 4 (N = 262144)
        for (int step = 0; step < 32; ++step) {
#pragma unroll
          for (int q = 0; q < NI; ++q) {
            const double dx = xs - xi[q], dy = ys - yi[q], dz = zs - zi[q];
            double r2 = fma(dx, dx, eps2);
            r2 = fma(dy, dy, r2);
            r2 = fma(dz, dz, r2);
            double y = rsqrt(r2);
            if (EXCL) y = r2 > 0.0 ? y : 0.0;
            const double y3 = y * y * y;
            const double sj = ms * y3, si = mi[q] * y3;
            // reaction first, and its shuffles before the sources': the faster
            // schedule (+1.7 % at N = 262144), as in k_force_n3_f32c
            RX = fma(si, dx, RX);
            RY = fma(si, dy, RY);
            RZ = fma(si, dz, RZ);
            AX[q] = fma(sj, dx, AX[q]);
            AY[q] = fma(sj, dy, AY[q]);
            AZ[q] = fma(sj, dz, AZ[q]);
          }
          RX = __shfl_sync(0xffffffffu, RX, from);
          RY = __shfl_sync(0xffffffffu, RY, from);
          RZ = __shfl_sync(0xffffffffu, RZ, from);
          xs = __shfl_sync(0xffffffffu, xs, from);
          ys = __shfl_sync(0xffffffffu, ys, from);
          zs = __shfl_sync(0xffffffffu, zs, from);
          ms = __shfl_sync(0xffffffffu, ms, from);
        }
        // back at its own lane: the force on source j is -sum m_i y^3 d
        myred[bt * 32 + lane] = -RX;
        myred[kN3Block + bt * 32 + lane] = -RY;
        myred[2 * kN3Block + bt * 32 + lane] = -RZ;
      }
    } else {
#pragma unroll
      for (int bt = 0; bt < 4; ++bt)
        myred[bt * 32 + lane] = myred[kN3Block + bt * 32 + lane] = myred[2 * kN3Block + bt * 32 + lane] = 0.0;
    }
    if (half == 1) {
      // end of column block c: its reaction from this CTA's rows, summed in
      // warp order, to the block's partial slot
      __syncthreads();
      const int tid = threadIdx.x;  // one source of the block per thread
      if (tid < kN3Block) {
        const long long off = ((long long)blockIdx.x * p3.cols + (c - cs)) * 3 * kN3Block;
        double* out = p3.rea + off;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double s = 0.0;
          for (int w = 0; w < kN3F64Warps; ++w) s += red[(w * 3 + d) * kN3Block + tid];
          if (NBR_IN((p3.rea - p3.act) + off + d * kN3Block + tid, p3.act_len, err))
            out[d * kN3Block + tid] = s;
        }
      }
      __syncthreads();
    }
  };
  if (!tile_pipeline(bars, ntl, js, err, issue, body)) return;
  double* act = p3.act + ((size_t)blockIdx.x * kN3Warps + rb) * 3 * kN3Block + hf * (kN3Block / 2);
  if (!NBR_IN(((long long)blockIdx.x * kN3Warps + rb + 1) * 3 * kN3Block - 1, p3.act_len, err))
    return;
#pragma unroll
  for (int q = 0; q < NI; ++q) {
    act[lane + 32 * q] = AX[q];
    act[kN3Block + lane + 32 * q] = AY[q];
    act[2 * kN3Block + lane + 32 * q] = AZ[q];
  }
}

// Adds the Newton-3 partial sums of each particle in a fixed order (its row
// group's chunks, then the reactions from the launch's row groups g0 .. its
// own) and then, by mode: 0 runs the epilogue of the large kernels; 1 stores
// the sums into dst[d * ld + i] (zero for particles the row groups do not
// reach); 2 adds them to dst.  One warp per 128-particle tile.
__global__ void __launch_bounds__(128)
    k_n3_reduce(const IParticles ip, const Epilogue ep, const N3Params p3, int mode, double* dst,
                long long ld) {
  const int lane = threadIdx.x & 31;
  const long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (tile * kTile >= p3.nb * kN3Block) return;
  const long long b = tile / 2;                   // block of the tile
  const int g = (int)(b / kN3Warps), w = (int)(b % kN3Warps);
  const int jb0 = (int)(tile & 1) * kTile + lane;  // particle index inside the block (k = 0)
  double ax[4] = {0, 0, 0, 0}, ay[4] = {0, 0, 0, 0}, az[4] = {0, 0, 0, 0};
  long long prefix = 0;  // CTAs of the launch's row groups before g'
  const int glast = min(g, p3.g1 - 1);
  for (int gp = p3.g0; gp <= glast; ++gp) {
    const int K = n3_chunks(p3.nb, p3.cols, gp);
    if (gp == g) {
      for (int k = 0; k < K; ++k) {
        const long long sk = p3.slot ? p3.slot[prefix + k] : prefix + k;  // partial-sum index
        const double* A = p3.act + ((size_t)sk * kN3Warps + w) * 3 * kN3Block;
        if (!NBR_IN((A - p3.act) + 3 * kN3Block - 1, p3.act_len, ep.err)) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int jb = jb0 + 32 * q;
          ax[q] += A[jb]; ay[q] += A[kN3Block + jb]; az[q] += A[2 * kN3Block + jb];
        }
      }
    }
    const long long cs0 = (long long)gp * kN3Warps;
    const int kk = (int)((b - cs0) / p3.cols);
    const int col = (int)(b - (cs0 + (long long)kk * p3.cols));
    const long long skk = p3.slot ? p3.slot[prefix + kk] : prefix + kk;
    const double* Rr = p3.rea + ((size_t)skk * p3.cols + col) * 3 * kN3Block;
    if (!NBR_IN((Rr - p3.act) + 3 * kN3Block - 1, p3.act_len, ep.err)) {
      prefix += K;
      continue;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int jb = jb0 + 32 * q;
      ax[q] += Rr[jb]; ay[q] += Rr[kN3Block + jb]; az[q] += Rr[2 * kN3Block + jb];
    }
    prefix += K;
  }
  const long long ibase = tile * kTile + lane;
  if (mode != 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long i = ibase + 32 * q;
      if (!NBR_IN(2 * ld + i, p3.dst_len, ep.err)) continue;
      if (mode == 1) {
        dst[i] = ax[q]; dst[ld + i] = ay[q]; dst[2 * ld + i] = az[q];
      } else {
        dst[i] += ax[q]; dst[ld + i] += ay[q]; dst[2 * ld + i] += az[q];
      }
    }
    return;
  }
  double xi[4], yi[4], zi[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long i = ibase + 32 * q;
    xi[q] = ip.x[i]; yi[q] = ip.y[i]; zi[q] = ip.z[i];
  }
  epilogue<4>(ip, ep, ibase, lane, xi, yi, zi, ax, ay, az);
}

// Sums V partial accelerations per particle in slice order, src[v * vstride
// + d * ld + i] (i < ip.n, rounded up to whole tiles), and runs the epilogue
// of the large kernels on the receivers ip.  One warp per 128-particle tile.
__global__ void __launch_bounds__(128)
    k_sum_finish(const IParticles ip, const Epilogue ep, const double* src, int V, long long vstride,
                 long long ld, long long src_len) {
  const int lane = threadIdx.x & 31;
  const long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (tile * kTile >= ip.n) return;
  const long long ibase = tile * kTile + lane;
  double ax[4] = {0, 0, 0, 0}, ay[4] = {0, 0, 0, 0}, az[4] = {0, 0, 0, 0};
  double xi[4], yi[4], zi[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long i = ibase + 32 * q;
    for (int v = 0; v < V; ++v) {
      const double* S = src + (size_t)v * vstride;
      if (!NBR_IN((long long)v * vstride + 2 * ld + i, src_len, ep.err)) continue;
      ax[q] += S[i]; ay[q] += S[ld + i]; az[q] += S[2 * ld + i];
    }
    xi[q] = yi[q] = zi[q] = 0.0;
    if (NBR_IN(i, ip.len, ep.err)) { xi[q] = ip.x[i]; yi[q] = ip.y[i]; zi[q] = ip.z[i]; }
  }
  epilogue<4>(ip, ep, ibase, lane, xi, yi, zi, ax, ay, az);
}

// --------------------------------------------------- kick / drift / pack ----
// One warp per kTile particles (4 per lane).  ax == nullptr: no kick;
// xn == nullptr: positions are not written (pack of x itself, drift ignored).
__global__ void __launch_bounds__(128)
    k_kick_drift(long long n, long long n_pad, const double* __restrict__ x,
                 const double* __restrict__ y, const double* __restrict__ z,
                 const double* __restrict__ m, const double* __restrict__ ax,
                 const double* __restrict__ ay, const double* __restrict__ az, double kick,
                 double drift, double* vx, double* vy, double* vz, double* xn, double* yn,
                 double* zn, float4* rec, double4* org) {
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long ibase = w * kTile + lane;
  if (ibase - lane >= n_pad) return;
  double px[4], py[4], pz[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long i = ibase + 32 * k;
    px[k] = py[k] = pz[k] = 0.0;
    if (i < n) {
      px[k] = x[i]; py[k] = y[i]; pz[k] = z[i];
      if (vx) {
        double ux = vx[i], uy = vy[i], uz = vz[i];
        if (ax) {
          ux += kick * ax[i]; uy += kick * ay[i]; uz += kick * az[i];
          vx[i] = ux; vy[i] = uy; vz[i] = uz;
        }
        if (xn) {
          px[k] += drift * ux; py[k] += drift * uy; pz[k] += drift * uz;
        }
      }
      if (xn) { xn[i] = px[k]; yn[i] = py[k]; zn[i] = pz[k]; }
    }
  }
  if (rec) pack_warp<4>(n, ibase, lane, px, py, pz, m, rec, org);
}

// ----------------------------------------------------------- diagnostics ----
// Fixed-order block tree reduction of `W` values per thread (blockDim 128).
template <int W>
__device__ __forceinline__ void block_reduce_store(double (&v)[W], double* out) {
  __shared__ double red[W][128];
#pragma unroll
  for (int c = 0; c < W; ++c) red[c][threadIdx.x] = v[c];
  __syncthreads();
  for (int h = 64; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
#pragma unroll
      for (int c = 0; c < W; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < W; ++c) out[(size_t)blockIdx.x * W + c] = red[c][0];
  }
}

// Softened potential phi_i = -G sum_{j != i} m_j / sqrt(r^2 + eps2), FP64, with
// the structure of the FP64 force kernel (receivers in registers, source tiles
// through the bulk-copy ring, j range split over gridDim.y with a
// deterministic last-CTA reduction).  Per pair: 3 sub, 3 fma, CUDA's
// rsqrt(double), 1 fma; the self pair is skipped by index (with eps2 > 0 it
// would add m_i / eps).  The last CTA of each receiver chunk writes phi and
// the chunk's sum of 1/2 m_i phi_i (fixed-order tree: deterministic).
template <int NI, int WARPS, bool EXCL>
__global__ void __launch_bounds__(WARPS * 32)
    k_potential_f64(const IParticles ip, const JStream js, const PotentialOut po,
                    const double eps2) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double red[WARPS * 32];
  __shared__ int s_last;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + kSmemHead;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long ibase = ((long long)blockIdx.x * WARPS + warp) * (32 * NI) + lane;
  const int S = gridDim.y, sp = blockIdx.y;
  const int t0 = (int)((long long)js.ntiles * sp / S);
  const int t1 = (int)((long long)js.ntiles * (sp + 1) / S);

  double xi[NI], yi[NI], zi[NI], ph[NI];
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = ibase + 32 * k;
    xi[k] = yi[k] = zi[k] = 0.0;
    if (NBR_IN(i, ip.len, po.err)) { xi[k] = ip.x[i]; yi[k] = ip.y[i]; zi[k] = ip.z[i]; }
    ph[k] = 0.0;
  }
  const int i0 = (int)ibase;  // n < 2^31
  auto issue = [&](int st, int t) {
    unsigned char* dst = stages + st * kStage64;
    const uint32_t bar = smem_u32(&bars[st]);
    const size_t off = (size_t)(t0 + t) * kTile;
    if (!NBR_IN((long long)off + kTile - 1, js.len, po.err)) return;  // the wait expires
    mbar_expect_tx(bar, kStage64);
    bulk_g2s(dst, js.x + off, kTile * 8, bar);
    bulk_g2s(dst + kTile * 8, js.y + off, kTile * 8, bar);
    bulk_g2s(dst + 2 * kTile * 8, js.z + off, kTile * 8, bar);
    bulk_g2s(dst + 3 * kTile * 8, js.m + off, kTile * 8, bar);
  };
  int tcur = t0;  // the body runs once per tile, in order
  auto body = [&](int st) {
    const double* sx = reinterpret_cast<const double*>(stages + st * kStage64);
    const double* sy = sx + kTile;
    const double* sz = sy + kTile;
    const double* sm = sz + kTile;
    const int jself = i0 - tcur * kTile;  // receiver k's own index in this tile is jself + 32 k
    ++tcur;
#pragma unroll 2
    for (int j = 0; j < kTile; ++j) {
      const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
        double r2 = fma(dx, dx, eps2);
        r2 = fma(dy, dy, r2);
        r2 = fma(dz, dz, r2);
        double y = rsqrt(r2);
        if (EXCL) y = r2 > 0.0 ? y : 0.0;
        y = (j == jself + 32 * k) ? 0.0 : y;
        ph[k] = fma(mj, y, ph[k]);
      }
    }
  };
  if (!tile_pipeline(bars, t1 - t0, js, po.err, issue, body)) return;

  if (S > 1) {
    const long long np = po.n_pad;
    double* P = po.part + (size_t)sp * (size_t)np;
#pragma unroll
    for (int k = 0; k < NI; ++k)
      if (NBR_IN((long long)sp * np + ibase + 32 * k, po.part_len, po.err)) P[ibase + 32 * k] = ph[k];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned prev =
          NBR_IN(blockIdx.x, po.cnt_len, po.err) ? atomicAdd(&po.counters[blockIdx.x], 1u) : 0u;
      s_last = (prev == gridDim.y - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      double v = 0.0;
      for (int q = 0; q < S; ++q)
        if (NBR_IN((long long)q * np + ibase + 32 * k, po.part_len, po.err))
          v += __ldcg(po.part + (size_t)q * (size_t)np + ibase + 32 * k);
      ph[k] = v;
    }
    if (threadIdx.x == 0 && NBR_IN(blockIdx.x, po.cnt_len, po.err)) po.counters[blockIdx.x] = 0u;
  }
  double half = 0.0;
#pragma unroll
  for (int k = 0; k < NI; ++k) {
    const long long i = ibase + 32 * k;
    if (i < ip.n) {
      const double p = -po.G * ph[k];
      if (po.phi) po.phi[i] = p;
      half += 0.5 * ip.m[i] * p;
    }
  }
  red[threadIdx.x] = half;
  __syncthreads();
  for (int h = WARPS * 16; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0 && NBR_IN(blockIdx.x, po.blocksum_len, po.err)) po.blocksum[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(128)
    k_moments(long long n, const double* __restrict__ x, const double* __restrict__ y,
              const double* __restrict__ z, const double* __restrict__ vx,
              const double* __restrict__ vy, const double* __restrict__ vz,
              const double* __restrict__ m, double* __restrict__ part) {
  const long long i = (long long)blockIdx.x * 128 + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double mi = m[i];
    v[0] = 0.5 * mi * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
    v[1] = mi * vx[i]; v[2] = mi * vy[i]; v[3] = mi * vz[i];
    v[4] = mi * (y[i] * vz[i] - z[i] * vy[i]);
    v[5] = mi * (z[i] * vx[i] - x[i] * vz[i]);
    v[6] = mi * (x[i] * vy[i] - y[i] * vx[i]);
    v[7] = mi;
  }
  block_reduce_store<8>(v, part);
}

__global__ void __launch_bounds__(256) k_rowsum(const double* __restrict__ part, int nblocks,
                                                int width, double* __restrict__ out) {
  __shared__ double red[256];
  for (int c = 0; c < width; ++c) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 256) s += part[(size_t)b * width + c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = red[0];
    __syncthreads();
  }
}

// Input validation of an uploaded system, on the device after the copy:
// sets bit 0 of *flags if a coordinate, velocity or mass is NaN or Inf and
// bit 1 if a mass is negative.  Velocities may be null.
__global__ void __launch_bounds__(256) k_validate(long long n, const double* __restrict__ x,
                                                  const double* __restrict__ y,
                                                  const double* __restrict__ z,
                                                  const double* __restrict__ vx,
                                                  const double* __restrict__ vy,
                                                  const double* __restrict__ vz,
                                                  const double* __restrict__ m, int* flags) {
  int f = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double mm = m[i];
    bool bad = !isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i]) || !isfinite(mm);
    if (vx) bad = bad || !isfinite(vx[i]) || !isfinite(vy[i]) || !isfinite(vz[i]);
    f |= (bad ? 1 : 0) | (mm < 0.0 ? 2 : 0);
  }
  f = __reduce_or_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

// -------------------------------------------------------------- dispatch ----
#define NBR_CFG_LIST(X) X(4, 2) X(4, 4) X(4, 8) X(8, 2) X(8, 4)
#define NBR_SMALL_LIST(X) X(2) X(4) X(8)
// (j-tile, unroll) variants built for the default large configurations
#define NBR_TU_LIST(X) X(64, 2) X(64, 4) X(64, 8) X(128, 2) X(128, 4) X(128, 8) \
                       X(256, 2) X(256, 4) X(256, 8)

int norm_tile(const ForceConfig& c) { return c.tile > 0 ? c.tile : kDefaultTileJ; }
int norm_unroll(int precision, const ForceConfig& c) {
  return c.unroll > 0 ? c.unroll : default_unroll(precision);
}

// The large kernel of a configuration, or nullptr if that variant is not built.
const void* large_fn(int precision, int ni, int w, int tj, int u, bool ex) {
  if (precision == kFP32C) {
#define NBR_F32(a, b)                                                                        \
  if (ni == a && w == b && tj == kDefaultTileJ && u == 4)                                    \
    return ex ? (const void*)k_force_f32c<a, b, true, kDefaultTileJ, 4>                      \
              : (const void*)k_force_f32c<a, b, false, kDefaultTileJ, 4>;
    NBR_CFG_LIST(NBR_F32)
#undef NBR_F32
#define NBR_F32TU(t, v)                                                                      \
  if (ni == 8 && w == 2 && tj == t && u == v)                                                \
    return ex ? (const void*)k_force_f32c<8, 2, true, t, v> : (const void*)k_force_f32c<8, 2, false, t, v>;
    NBR_TU_LIST(NBR_F32TU)
#undef NBR_F32TU
  } else {
#define NBR_F64(a, b)                                                                        \
  if (ni == a && w == b && tj == kDefaultTileJ && u == 2)                                    \
    return ex ? (const void*)k_force_f64<a, b, true, kDefaultTileJ, 2>                       \
              : (const void*)k_force_f64<a, b, false, kDefaultTileJ, 2>;
    NBR_CFG_LIST(NBR_F64)
#undef NBR_F64
#define NBR_F64TU(t, v)                                                                      \
  if (ni == 4 && w == 4 && tj == t && u == v)                                                \
    return ex ? (const void*)k_force_f64<4, 4, true, t, v> : (const void*)k_force_f64<4, 4, false, t, v>;
    NBR_TU_LIST(NBR_F64TU)
#undef NBR_F64TU
  }
  return nullptr;
}

size_t large_smem(int precision, int tj) {
  size_t stage = 0;
  if (precision == kFP32C)
    stage = tj == 64 ? stage32_bytes<64>() : tj == 256 ? stage32_bytes<256>() : stage32_bytes<128>();
  else
    stage = 32 * (size_t)tj;
  return kSmemHead + (size_t)kStages * stage;
}

cudaError_t launch_large(int precision, double eps2, const ForceConfig& c, const IParticles& ip,
                         const JStream& js, const Epilogue& ep, cudaStream_t st) {
  const int tj = norm_tile(c), u = norm_unroll(precision, c);
  const void* fn = large_fn(precision, c.ni, c.warps, tj, u, eps2 == 0.0);
  if (!fn) return cudaErrorInvalidValue;
  const long long chunk = 32LL * c.ni * c.warps;
  const dim3 grid((unsigned)((ip.n + chunk - 1) / chunk), (unsigned)c.split);
  IParticles a0 = ip;
  JStream a1 = js;
  Epilogue a2 = ep;
  float e32 = (float)eps2;
  double e64 = eps2;
  void* args[] = {&a0, &a1, &a2, precision == kFP32C ? (void*)&e32 : (void*)&e64};
  return cudaLaunchKernel(fn, grid, dim3(c.warps * 32), args, large_smem(precision, tj), st);
}

template <int PREC, int F>
const void* small_fn(bool ex) {
  return ex ? (const void*)k_force_small<PREC, F, true> : (const void*)k_force_small<PREC, F, false>;
}

template <int PREC, int F>
cudaError_t launch_small_t(double eps2, int split, const IParticles& ip, const JStream& js,
                           const Epilogue& ep, cudaStream_t st) {
  const size_t smem = kSmemHead + (size_t)kStages * (PREC == kFP32C ? kStage32 : kStage64);
  const long long chunk = 32LL * kSmallWarps * kSmallNI / F;
  const dim3 grid((unsigned)((ip.n + chunk - 1) / chunk), (unsigned)split);
  if (eps2 == 0.0)
    k_force_small<PREC, F, true><<<grid, kSmallWarps * 32, smem, st>>>(ip, js, ep, eps2);
  else
    k_force_small<PREC, F, false><<<grid, kSmallWarps * 32, smem, st>>>(ip, js, ep, eps2);
  return cudaGetLastError();
}

}  // namespace

size_t n3_smem_bytes(int precision, int warps);

bool force_config_supported(int precision, const ForceConfig& c) {
  if (c.ni == kPersistNI) {  // warps = lane groups, split = warps per CTA, tile = receivers
    const bool f4 = c.warps == 4 || c.warps == 8 || c.warps == 16;
    if (precision == kFP32C)  // 16 warps, 4 receivers per lane
      return f4 && (c.split <= 1 || c.split == 16) && (c.tile == 0 || c.tile == 4);
    return (c.split <= 1 || c.split == 8 || c.split == 16) &&
           (((c.tile == 0 || c.tile == 4) && f4) || (c.tile == 8 && (c.warps == 8 || c.warps == 16)));
  }
  if (c.ni == 3)  // Newton-3: FP32C one or two warps per row block; FP64 (two)
    return c.warps == kN3Warps || (precision == kFP32C && c.warps == kN3F64Warps);
  if (c.ni == 1) return (c.warps == 2 || c.warps == 4 || c.warps == 8) && c.split >= 1;
  if (c.split < 1) return false;
  return large_fn(precision, c.ni, c.warps, norm_tile(c), norm_unroll(precision, c), false) != nullptr;
}

int force_blocks_per_sm(int precision, double eps2, const ForceConfig& c) {
  int nb = 0;
  if (c.ni == 3) {
    const bool ex = eps2 == 0.0;
    const bool w2 = precision == kFP32C && c.warps == kN3F64Warps;
    const void* fn = precision == kFP32C
                         ? (w2 ? (ex ? (const void*)k_force_n3_f32c_w2<true> : (const void*)k_force_n3_f32c_w2<false>)
                               : (ex ? (const void*)k_force_n3_f32c<true, false> : (const void*)k_force_n3_f32c<false, false>))
                         : (ex ? (const void*)k_force_n3_f64<true> : (const void*)k_force_n3_f64<false>);
    const int threads = (precision == kFP32C && !w2 ? kN3Warps : kN3F64Warps) * 32;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, n3_smem_bytes(precision, c.warps)) !=
        cudaSuccess)
      nb = 0;
    return nb;
  }
  const size_t smem = force_smem_bytes(precision, c);
  const bool ex = (eps2 == 0.0);
  if (c.ni == 1) {
    const void* fn = nullptr;
#define NBR_SOCC(f)                                                                        \
  if (c.warps == f) fn = precision == kFP32C ? small_fn<kFP32C, f>(ex) : small_fn<kFP64, f>(ex);
    NBR_SMALL_LIST(NBR_SOCC)
#undef NBR_SOCC
    if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kSmallWarps * 32, smem) !=
                   cudaSuccess)
      nb = 0;
    return nb;
  }
  const void* fn = large_fn(precision, c.ni, c.warps, norm_tile(c), norm_unroll(precision, c), ex);
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, c.warps * 32, smem) != cudaSuccess)
    nb = 0;
  return nb;
}

size_t force_smem_bytes(int precision, const ForceConfig& c) {
  if (c.ni == 1) return kSmemHead + (size_t)kStages * (precision == kFP32C ? kStage32 : kStage64);
  return large_smem(precision, norm_tile(c));
}

cudaError_t launch_force(int precision, double eps2, const ForceConfig& c, const IParticles& ip,
                         const JStream& js, const Epilogue& ep, cudaStream_t st) {
  if (ip.n <= 0 || js.ntiles <= 0) return cudaSuccess;
  const bool ex = (eps2 == 0.0);
  if (c.ni == 1) {
#define NBR_SGO(f)                                                                         \
  if (c.warps == f)                                                                        \
    return precision == kFP32C ? launch_small_t<kFP32C, f>(eps2, c.split, ip, js, ep, st)  \
                               : launch_small_t<kFP64, f>(eps2, c.split, ip, js, ep, st);
    NBR_SMALL_LIST(NBR_SGO)
#undef NBR_SGO
    return cudaErrorInvalidValue;
  }
  return launch_large(precision, eps2, c, ip, js, ep, st);
}

// Tile ring plus the per-warp reaction staging (floats for FP32C, doubles for
// FP64); `warps` per CTA.
size_t n3_smem_bytes(int precision, int warps) {
  return precision == kFP32C
             ? kSmemHead + (size_t)kStages * kStage32 + (size_t)warps * 3 * kN3Block * sizeof(float)
             : kSmemHead + (size_t)kStages * kStage64 + (size_t)kN3F64Warps * 3 * kN3Block * sizeof(double);
}

// The column-chunk width and launch order of the Newton-3 grid.  A CTA (row
// group g, chunk k) costs a fixed 0.15 plus, per column block of its chunk, 1
// (0.8 for the group's first 8 blocks, where the diagonal leaves warps idle),
// in units of one column block's pair work; the CTAs are handed to the SMs in
// launch order as SMs free up (list scheduling, one CTA per SM).  Both
// constants were fitted on B200 to 27 timed (N, width) pairs from N = 32768 to
// 2^20 in group-major order, which the model reproduces to 1 % (0.2 % on
// average).  Narrow chunks cut the last wave's idle time, wide ones the
// per-CTA cost; launching the longest CTAs first (the diagonal and partial
// chunks last) leaves the short ones for the last wave.
namespace {
// SM count of the current device (148 if it cannot be read).
int device_sms() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
    sms = 148;
  return sms;
}

// Modeled cost of every CTA of row groups [g0, g1), group-major.
void n3_cta_costs_range(long long nb, int cols, long long g0, long long g1,
                        std::vector<double>& cost) {
  constexpr double kCtaCost = 0.15, kDiagBlock = 0.8;
  cost.clear();
  for (long long g = g0; g < g1; ++g) {
    const long long r0 = g * kN3Warps;
    for (long long cs = r0; cs < nb; cs += cols) {
      const long long ce = std::min(cs + (long long)cols, nb);
      const long long diag = std::max(0LL, std::min(ce, r0 + kN3Warps) - cs);  // blocks < r0 + 8
      cost.push_back(kCtaCost + kDiagBlock * (double)diag + (double)(ce - cs - diag));
    }
  }
}

// Finishing time of CTAs of the given costs handed in that order to `sms`
// SMs, each to the first SM free (list scheduling, one CTA per SM).
double list_schedule(const std::vector<double>& cost, int sms) {
  std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
  for (int i = 0; i < sms; ++i) free_at.push(0.0);
  double end = 0.0;
  for (const double t : cost) {
    const double start = free_at.top();
    free_at.pop();
    free_at.push(start + t);
    end = std::max(end, start + t);
  }
  return end;
}

// Modeled finishing time of the group-major grid of row groups [g0, g1).
double n3_range_makespan(long long nb, int cols, int g0, int g1, int sms) {
  std::vector<double> cost;
  n3_cta_costs_range(nb, cols, g0, g1, cost);
  return list_schedule(cost, sms);
}
}  // namespace

void n3_cta_costs(long long nb, int cols, std::vector<double>& cost) {
  n3_cta_costs_range(nb, cols, 0, (nb + kN3Warps - 1) / kN3Warps, cost);
}

void n3_launch_order(long long nb, int cols, std::vector<int>& order) {
  std::vector<double> cost;
  n3_cta_costs(nb, cols, cost);
  order.resize(cost.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
}

double n3_makespan(long long nb, int cols, int sms) {
  std::vector<double> cost;
  n3_cta_costs(nb, cols, cost);
  std::stable_sort(cost.begin(), cost.end(), std::greater<double>());
  return list_schedule(cost, sms);
}

int n3_cols(long long nb) { return n3_cols_for(nb, device_sms()); }
int n3_slice_cols(long long nb, int V) { return n3_slice_cols_for(nb, V, device_sms()); }
double n3_grid_efficiency(long long nb) { return n3_grid_efficiency_for(nb, device_sms()); }

int n3_cols_for(long long nb, int sms) {
  if (nb <= 1) return 1;
  if (sms < 1) sms = 1;
  static std::mutex mu;
  static std::map<std::pair<long long, int>, int> memo;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(nb, sms);
  const auto it = memo.find(key);
  if (it != memo.end()) return it->second;
  int best = kN3MaxCols;
  // many waves at the widest chunk: the last wave's idle time is negligible
  if (n3_ctas(nb, kN3MaxCols) < 64LL * sms) {
    double best_t = n3_makespan(nb, kN3MaxCols, sms);
    for (int c = kN3MaxCols - 1; c >= 1; --c) {
      if (n3_ctas(nb, c) > 128LL * sms) break;  // narrower still: only more CTA cost
      const double t = n3_makespan(nb, c, sms);
      if (t < best_t * (1.0 - 1e-3)) {  // ties keep the wider chunk (fewer partial sums)
        best_t = t;
        best = c;
      }
    }
  }
  memo[key] = best;
  return best;
}


int n3_slice_cols_for(long long nb, int V, int sms) {
  if (nb <= 1 || V < 1) return 1;
  if (sms < 1) sms = 1;
  static std::mutex mu;
  static std::map<std::tuple<long long, int, int>, int> memo;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_tuple(nb, V, sms);
  const auto it = memo.find(key);
  if (it != memo.end()) return it->second;
  // 32 waves or more per slice at the widest chunk: the last wave's idle time
  // is negligible (and the model would simulate millions of CTAs)
  if (n3_ctas(nb, kN3MaxCols) >= 32LL * sms * V) {
    memo[key] = kN3MaxCols;
    return kN3MaxCols;
  }
  std::vector<int> worlds;
  for (int W : {2, 4, 8})
    if (W <= V) worlds.push_back(W);
  if (V != 2 && V != 4 && V != 8) worlds.push_back(V);
  // the ideal time per rank: the widest chunks' total cost (the least per-CTA
  // cost) spread evenly over all SMs of the W ranks
  double total = 0.0;
  {
    std::vector<double> cost;
    n3_cta_costs(nb, kN3MaxCols, cost);
    for (const double t : cost) total += t;
  }
  int best = kN3MaxCols;
  double best_eff = -1.0;
  for (int c = kN3MaxCols; c >= 1; --c) {
    if (c < kN3MaxCols && n3_ctas(nb, c) > 64LL * sms * V) break;  // only more CTA cost
    // worst-case efficiency over the world sizes: ideal time / slowest rank
    double eff = 1e30;
    for (const int W : worlds) {
      double worst = 0.0;
      for (int r = 0; r < W; ++r) {
        const int v0 = (int)((long long)V * r / W), v1 = (int)((long long)V * (r + 1) / W);
        if (v1 <= v0) continue;
        int g0 = 0, g1 = 0, g = 0;
        n3_slice_groups(nb, c, v0, V, &g0, &g);
        n3_slice_groups(nb, c, v1 - 1, V, &g, &g1);
        worst = std::max(worst, n3_range_makespan(nb, c, g0, g1, sms));
      }
      if (worst > 0.0) eff = std::min(eff, total / ((double)sms * W) / worst);
    }
    if (eff > best_eff * (1.0 + 1e-3)) {  // ties keep the wider chunk
      best_eff = eff;
      best = c;
    }
  }
  memo[key] = best;
  return best;
}

double n3_grid_efficiency_for(long long nb, int sms) {
  if (nb < 1) return 0.0;
  if (sms < 1) sms = 1;
  const int cols = n3_cols_for(nb, sms);  // before taking the lock (it has its own)
  static std::mutex mu;
  static std::map<std::pair<long long, int>, double> memo;  // the choice runs per evaluation
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(nb, sms);
  const auto it = memo.find(key);
  if (it != memo.end()) return it->second;
  // one unit: a CTA's 8 warps against one column block; (row block, column
  // block >= it) pairs / 8 units in all
  const double units = (double)nb * (double)(nb + 1) / 2.0 / kN3Warps;
  const double eff = units / (double)sms / n3_makespan(nb, cols, sms);
  memo[key] = eff;
  return eff;
}

cudaError_t configure_kernels() {
  // The Newton-3 kernels need more than the default 48 KB of dynamic shared
  // memory; set once per device, outside any stream capture.
  const int s32 = (int)n3_smem_bytes(kFP32C, kN3Warps), s64 = (int)n3_smem_bytes(kFP64, kN3F64Warps);
  const int s32w = (int)n3_smem_bytes(kFP32C, kN3F64Warps);
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute((const void*)k_force_n3_f32c<true, false>, at, s32);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f32c<false, false>, at, s32);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f32c<true, true>, at, s32);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f32c<false, true>, at, s32);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f32c_w2<true>, at, s32w);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f32c_w2<false>, at, s32w);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f64<true>, at, s64);
  if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_force_n3_f64<false>, at, s64);
  // large kernels: the 256-source FP32C stages need more than the default 48 KB
  for (int prec = 0; prec < 2 && e == cudaSuccess; ++prec)
    for (int ni : {4, 8})
      for (int w : {2, 4, 8})
        for (int tj : {64, 128, 256})
          for (int u : {2, 4, 8})
            for (int ex = 0; ex < 2 && e == cudaSuccess; ++ex)
              if (const void* fn = large_fn(prec, ni, w, tj, u, ex != 0))
                e = cudaFuncSetAttribute(fn, at, (int)large_smem(prec, tj));
  return e;
}

cudaError_t launch_force_n3(int precision, int warps, double eps2, const IParticles& ip,
                            const JStream& js, const Epilogue& ep, double* scratch,
                            long long scratch_len, const int* order, cudaStream_t st) {
  (void)scratch_len;
  if (ip.n <= 0 || js.ntiles <= 0) return cudaSuccess;
  N3Params p3;
  p3.nb = (ip.n + kN3Block - 1) / kN3Block;
  p3.cols = n3_cols(p3.nb);
  const long long ctas = n3_ctas(p3.nb, p3.cols);
  if (ctas > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  p3.g0 = 0;
  p3.g1 = (int)((p3.nb + kN3Warps - 1) / kN3Warps);
  p3.act = scratch;
  p3.rea = scratch + (size_t)ctas * kN3Warps * 3 * kN3Block;
  p3.order = order;
  p3.slot = order ? order + ctas : nullptr;
  NBR_CHECKED_ONLY(p3.act_len = scratch_len;)
  const bool w2 = precision == kFP32C && warps == kN3F64Warps;
  const size_t smem = n3_smem_bytes(precision, precision == kFP32C ? warps : kN3F64Warps);
  const unsigned grid = (unsigned)ctas,
                 block = (precision == kFP32C && !w2 ? kN3Warps : kN3F64Warps) * 32;
  if (w2) {
    if (eps2 == 0.0)
      k_force_n3_f32c_w2<true><<<grid, block, smem, st>>>(ip, js, p3, 0.f, ep.err);
    else
      k_force_n3_f32c_w2<false><<<grid, block, smem, st>>>(ip, js, p3, (float)eps2, ep.err);
  } else if (precision == kFP32C && !order) {
    // no launch order: the range form over all row groups (group-major order)
    if (eps2 == 0.0)
      k_force_n3_f32c<true, true><<<grid, block, smem, st>>>(ip, js, p3, 0.f, ep.err);
    else
      k_force_n3_f32c<false, true><<<grid, block, smem, st>>>(ip, js, p3, (float)eps2, ep.err);
  } else if (precision == kFP32C) {
    if (eps2 == 0.0)
      k_force_n3_f32c<true, false><<<grid, block, smem, st>>>(ip, js, p3, 0.f, ep.err);
    else
      k_force_n3_f32c<false, false><<<grid, block, smem, st>>>(ip, js, p3, (float)eps2, ep.err);
  } else {
    if (eps2 == 0.0)
      k_force_n3_f64<true><<<grid, block, smem, st>>>(ip, js, p3, 0.0, ep.err);
    else
      k_force_n3_f64<false><<<grid, block, smem, st>>>(ip, js, p3, eps2, ep.err);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long threads = p3.nb * 2 * 32;  // a warp per tile
  k_n3_reduce<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(ip, ep, p3, 0, nullptr, 0);
  return cudaGetLastError();
}

// The pair kernel of a Newton-3 launch over row groups [g0, g1).
cudaError_t launch_n3_pairs(int precision, int warps, double eps2, const IParticles& ip,
                            const JStream& js, int* err, N3Params& p3, cudaStream_t st) {
  const long long ctas = n3_ctas_range(p3.nb, p3.cols, p3.g0, p3.g1);
  if (ctas <= 0) return cudaSuccess;
  if (ctas > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  const bool w2 = precision == kFP32C && warps == kN3F64Warps;
  const size_t smem = n3_smem_bytes(precision, precision == kFP32C ? warps : kN3F64Warps);
  const unsigned grid = (unsigned)ctas,
                 block = (precision == kFP32C && !w2 ? kN3Warps : kN3F64Warps) * 32;
  const float e32 = (float)eps2;
  if (w2) {
    if (eps2 == 0.0) k_force_n3_f32c_w2<true><<<grid, block, smem, st>>>(ip, js, p3, 0.f, err);
    else k_force_n3_f32c_w2<false><<<grid, block, smem, st>>>(ip, js, p3, e32, err);
  } else if (precision == kFP32C) {
    if (eps2 == 0.0) k_force_n3_f32c<true, true><<<grid, block, smem, st>>>(ip, js, p3, 0.f, err);
    else k_force_n3_f32c<false, true><<<grid, block, smem, st>>>(ip, js, p3, e32, err);
  } else {
    if (eps2 == 0.0) k_force_n3_f64<true><<<grid, block, smem, st>>>(ip, js, p3, 0.0, err);
    else k_force_n3_f64<false><<<grid, block, smem, st>>>(ip, js, p3, eps2, err);
  }
  return cudaGetLastError();
}

cudaError_t launch_n3_slices(int precision, int warps, double eps2, const IParticles& ip,
                             const JStream& js, int* err, int v0, int v1, int nslices,
                             double* scratch, long long scratch_len, double* dst, long long ld,
                             long long dst_len, bool accumulate, cudaStream_t st) {
  if (ip.n <= 0 || js.ntiles <= 0 || v1 <= v0) return cudaSuccess;
  N3Params p3{};
  p3.nb = (ip.n + kN3Block - 1) / kN3Block;
  p3.cols = n3_slice_cols(p3.nb, nslices);
  // one pair launch over the slices' consecutive row groups: a CTA's partial
  // sums depend on its (row group, chunk) only, so they equal those of
  // per-slice launches, with fewer partly filled waves
  int g_last = 0;
  n3_slice_groups(p3.nb, p3.cols, v0, nslices, &p3.g0, &g_last);
  n3_slice_groups(p3.nb, p3.cols, v1 - 1, nslices, &g_last, &p3.g1);
  const long long ctas = n3_ctas_range(p3.nb, p3.cols, p3.g0, p3.g1);
  p3.act = scratch;
  p3.rea = scratch + (size_t)ctas * kN3Warps * 3 * kN3Block;
  NBR_CHECKED_ONLY(p3.act_len = scratch_len; p3.dst_len = dst_len;)
  (void)scratch_len;
  (void)dst_len;
  cudaError_t e = launch_n3_pairs(precision, warps, eps2, ip, js, err, p3, st);
  if (e != cudaSuccess) return e;
  Epilogue ep{};
  ep.err = err;
  const long long threads = p3.nb * 2 * 32;  // a warp per tile
  for (int v = v0; v < v1; ++v) {
    // slice v's row groups and the offset of their CTAs inside the launch
    N3Params pv = p3;
    n3_slice_groups(p3.nb, p3.cols, v, nslices, &pv.g0, &pv.g1);
    const long long before = n3_ctas_range(p3.nb, p3.cols, p3.g0, pv.g0);
    pv.act = p3.act + (size_t)before * kN3Warps * 3 * kN3Block;
    pv.rea = p3.rea + (size_t)before * p3.cols * 3 * kN3Block;
    NBR_CHECKED_ONLY(pv.act_len = scratch_len - (pv.act - scratch);
                     pv.dst_len = dst_len - (long long)(v - v0) * 3 * ld;)
    k_n3_reduce<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(
        ip, ep, pv, accumulate ? 2 : 1, dst + (size_t)(v - v0) * 3 * ld, ld);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_n3_slice(int precision, int warps, double eps2, const IParticles& ip,
                            const JStream& js, int* err, int slice, int nslices, double* scratch,
                            long long scratch_len, double* dst, long long ld, long long dst_len,
                            bool accumulate, cudaStream_t st) {
  return launch_n3_slices(precision, warps, eps2, ip, js, err, slice, slice + 1, nslices, scratch,
                          scratch_len, dst, ld, dst_len, accumulate, st);
}

cudaError_t launch_sum_finish(const IParticles& ip, const Epilogue& ep, const double* src, int V,
                              long long vstride, long long ld, long long src_len, cudaStream_t st) {
  if (ip.n <= 0) return cudaSuccess;
  const long long threads = ((ip.n + kTile - 1) / kTile) * 32;
  k_sum_finish<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(ip, ep, src, V, vstride, ld,
                                                                  src_len);
  return cudaGetLastError();
}

cudaError_t launch_kick_drift(long long n, long long n_pad, const double* x, const double* y,
                              const double* z, const double* m, const double* ax,
                              const double* ay, const double* az, double kick, double drift,
                              double* vx, double* vy, double* vz, double* xn, double* yn,
                              double* zn, float4* rec, double4* org, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const long long warps = (n + kTile - 1) / kTile;
  const unsigned blocks = (unsigned)((warps + 3) / 4);
  k_kick_drift<<<blocks, 128, 0, st>>>(n, n_pad, x, y, z, m, ax, ay, az, kick, drift, vx, vy, vz,
                                       xn, yn, zn, rec, org);
  return cudaGetLastError();
}

cudaError_t launch_potential(int split, const IParticles& ip, const JStream& js,
                             const PotentialOut& po, double eps2, cudaStream_t st) {
  if (ip.n <= 0 || js.ntiles <= 0) return cudaSuccess;
  const size_t smem = kSmemHead + (size_t)kStages * kStage64;
  const long long chunk = 32LL * kPotNI * kPotWarps;
  const dim3 grid((unsigned)((ip.n + chunk - 1) / chunk), (unsigned)(split < 1 ? 1 : split));
  if (eps2 == 0.0)
    k_potential_f64<kPotNI, kPotWarps, true><<<grid, kPotWarps * 32, smem, st>>>(ip, js, po, eps2);
  else
    k_potential_f64<kPotNI, kPotWarps, false><<<grid, kPotWarps * 32, smem, st>>>(ip, js, po, eps2);
  return cudaGetLastError();
}

cudaError_t launch_moments(long long n, long long n_pad, const double* x, const double* y,
                           const double* z, const double* vx, const double* vy, const double* vz,
                           const double* m, double* part, cudaStream_t st) {
  (void)n_pad;
  if (n <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n + 127) / 128);
  k_moments<<<blocks, 128, 0, st>>>(n, x, y, z, vx, vy, vz, m, part);
  return cudaGetLastError();
}

cudaError_t launch_rowsum(const double* part, int nblocks, int width, double* out,
                          cudaStream_t st) {
  k_rowsum<<<1, 256, 0, st>>>(part, nblocks, width, out);
  return cudaGetLastError();
}

cudaError_t launch_validate(long long n, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz,
                            const double* m, int* flags, int sms, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const long long want = (n + 255) / 256;
  const unsigned blocks = (unsigned)std::min<long long>(want, 8LL * (sms > 0 ? sms : 148));
  k_validate<<<blocks, 256, 0, st>>>(n, x, y, z, vx, vy, vz, m, flags);
  return cudaGetLastError();
}

}  // namespace nbr
