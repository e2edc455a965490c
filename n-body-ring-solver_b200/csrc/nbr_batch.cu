// nbr_batch.cu -- thousands of independent systems in one persistent launch.
//
// Layout: the systems are stored back to back, each padded to whole
// 128-particle tiles (padding: zero mass at the origin), so a tile never mixes
// systems.  A force evaluation is one launch of k_batch_force: a persistent
// grid whose warps pull work items (system, 128-receiver tile) from a device
// queue with atomicAdd.  Items are ordered by cost (receivers x system size,
// largest first) so the tail of the queue holds the cheapest items.  Each warp
// streams its system's source tiles through its own 3-stage shared-memory ring
// (1-D bulk copies, one mbarrier per stage, lane 0 produces).
//
// Wide items: a system's receiver tiles can be paired into two-tile items
// (256 receivers, 8 per lane): every source read from shared memory then
// feeds 8 receivers and each lane runs four independent f32x2 chains.  A
// system's odd last tile stays a one-tile item.
//
// Small items: when an item has R <= 64 real receivers (a system of <= 64
// particles, or the last tile of a system), the warp splits into F = 2, 4 or
// 8 lane groups that take every F-th source; the partial sums are combined
// with warp shuffles (xor over the group bits).  Padded sources of a system's
// last tile are skipped (the loop stops at the tile's real count rounded up to
// 4), so padding costs ~1 % of the pair work on the log-uniform workload.
//
// Newton-3 row blocks (the default work list): a system large enough is
// split into row blocks of R receiver tiles (FP32C R = 2, 8 receivers per
// lane; FP64 R = 1, 4 per lane), each an item that walks the column tiles
// from its own: its own tiles with every ordered pair, every later tile with
// each pair once, the sources rotating through the warp by shuffles with
// their reaction sums.  The action goes to a per-particle array, each
// (row block, later tile) reaction to its own slot; k_batch_n3_reduce then
// adds every particle's action and reactions in a fixed order and runs the
// epilogue: deterministic, no atomics.
//
// Pair arithmetic and accumulation are those of the single-system kernels
// (nbr_kernels.cu): FP32C f32x2 pairs with TwoSum-compensated tile sums, or
// FP64.  The epilogue applies the KDK kick/drift and packs the FP32C records of
// the item's tile for the next evaluation.
#include "nbr.h"
#include "nbr_ctx.h"
#include "nbr_device.cuh"
#include "nbr_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

using namespace nbr;

namespace {

constexpr int kBWarps = 4;                    // warps per CTA
constexpr int kBStages = 3;                   // tile stages per warp
constexpr int kRec32 = kTile * 48;            // FP32C records of one tile
constexpr int kStageB32 = kRec32 + 32;        // + origin
constexpr int kStageB64 = 4 * kTile * 8;      // FP64 x, y, z, m
constexpr int kBHead = 128;                   // barriers: kBWarps * kBStages * 8 <= 128
constexpr int kWideItem = 1 << 30;            // item flag: two receiver tiles
constexpr int kN3Item = 1 << 29;              // item flag: a Newton-3 row block

struct BatchParams {
  const double* x; const double* y; const double* z; const double* m;  // current buffer
  const float4* rec; const double4* org;
  const long long* poff;     // padded offset of each system (multiple of kTile)
  const int* nreal;          // real size of each system
  const int2* items;         // (system, global tile index of the receivers)
  int n_items;
  unsigned* head;            // queue head, zero at launch
  int mode;                  // 0: write a; 1: leapfrog kick + drift
  double G, kick, drift;
  double* ax; double* ay; double* az;
  double* vx; double* vy; double* vz;
  double* xn; double* yn; double* zn;
  float4* rec_next; double4* org_next;
  int* err;
  unsigned long long wait_ns;
  int skip_tile;
  // Newton-3 items: the action of every particle [3][n_pad], the reaction
  // partials (one 3 x 128 slot per (row block, later column tile) of a
  // system), each system's first slot (-1: the system has no N3 items), and
  // the tiles per row block (FP32C 2, FP64 1)
  double* act;
  double* rea;
  const long long* rea_off;
  long long n_pad;
  int n3_rows;
  NBR_CHECKED_FIELD(long long len)  // entries allocated in the particle arrays
  NBR_CHECKED_FIELD(int nsys)
  NBR_CHECKED_FIELD(long long rea_len)  // doubles allocated in rea
};

// Reaction slots before row block b of a system of T tiles, with `rows` tiles
// per row block: row block b' has T - rows (b' + 1) later column tiles (every
// b' < b has at least one).
__host__ __device__ inline long long n3b_prefix(int T, int b, int rows) {
  return (long long)b * (T - rows) - (long long)rows * b * (b - 1) / 2;
}

template <int P>
struct Stage;
template <>
struct Stage<kFP32C> {
  static constexpr int bytes = kStageB32;
};
template <>
struct Stage<kFP64> {
  static constexpr int bytes = kStageB64;
};

// One source tile of FP32C records against the lane's NP receiver pairs.
// Sources j = j0, j0 + step, ... < jend.
template <bool EXCL, bool FULL, int NP>
__device__ __forceinline__ void tile_f32c(const unsigned char* base, int j0, int step, int jend,
                                          const double* xi, const double* yi, const double* zi,
                                          u64 EPS2, u64* hx, u64* hy, u64* hz, u64* lx, u64* ly,
                                          u64* lz) {
  const double4 o = *reinterpret_cast<const double4*>(base + kRec32);
  u64 XI[NP], YI[NP], ZI[NP], AX[NP], AY[NP], AZ[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    XI[p] = pack2(__double2float_rn(xi[2 * p] - o.x), __double2float_rn(xi[2 * p + 1] - o.x));
    YI[p] = pack2(__double2float_rn(yi[2 * p] - o.y), __double2float_rn(yi[2 * p + 1] - o.y));
    ZI[p] = pack2(__double2float_rn(zi[2 * p] - o.z), __double2float_rn(zi[2 * p + 1] - o.z));
    AX[p] = AY[p] = AZ[p] = 0ull;
  }
  const ulonglong2* R = reinterpret_cast<const ulonglong2*>(base);
  auto pair = [&](int j) {
    const ulonglong2 q0 = R[3 * j];
    const ulonglong2 q1 = R[3 * j + 1];
    const u64 bj = R[3 * j + 2].x;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
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
  };
  if (FULL) {
#pragma unroll 4
    for (int j = 0; j < kTile; ++j) pair(j);
  } else {
#pragma unroll 4
    for (int j = j0; j < jend; j += step) pair(j);
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    two_sum2(hx[p], lx[p], AX[p]);
    two_sum2(hy[p], ly[p], AY[p]);
    two_sum2(hz[p], lz[p], AZ[p]);
  }
}

// One FP64 source tile against the lane's NR receivers.
template <bool EXCL, bool FULL, int NR>
__device__ __forceinline__ void tile_f64(const unsigned char* base, int j0, int step, int jend,
                                         const double* xi, const double* yi, const double* zi,
                                         double eps2, double* ax, double* ay, double* az) {
  const double* sx = reinterpret_cast<const double*>(base);
  const double* sy = sx + kTile;
  const double* sz = sy + kTile;
  const double* sm = sz + kTile;
  auto pair = [&](int j) {
    const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
      double r2 = fma(dx, dx, eps2);
      r2 = fma(dy, dy, r2);
      r2 = fma(dz, dz, r2);
      double yv = rsqrt(r2);
      if (EXCL) yv = r2 > 0.0 ? yv : 0.0;
      const double s = mj * (yv * yv * yv);
      ax[k] = fma(s, dx, ax[k]);
      ay[k] = fma(s, dy, ay[k]);
      az[k] = fma(s, dz, az[k]);
    }
  };
  if (FULL) {
#pragma unroll 2
    for (int j = 0; j < kTile; ++j) pair(j);
  } else {
#pragma unroll 2
    for (int j = j0; j < jend; j += step) pair(j);
  }
}

// The per-warp state that persists across items: the tile ring.
struct Ring {
  uint64_t* bars;
  unsigned char* stages;
  unsigned tcount;  // tiles this warp has consumed (ring position)
};

// One work item: NR / 4 receiver tiles (4 receivers per lane per tile)
// starting at global tile `tile0` of system `s`, against all of the system's
// source tiles.  Narrow items (NR = 4) split the warp into lane groups when
// they hold <= 64 real receivers.  Returns false if a tile wait gave up.
template <int PREC, bool EXCL, int NR>
__device__ __forceinline__ bool run_item(const BatchParams& p, double eps2, u64 EPS2, Ring& ring,
                                         int lane, int s, int tile0) {
  constexpr int SB = Stage<PREC>::bytes;
  constexpr int NP = NR / 2;
  const long long poff = p.poff[s];
  const int ns = p.nreal[s];
  const long long rbase = (long long)tile0 * kTile;             // first receiver (padded index)
  const int rfirst = (int)(rbase - poff);                       // its index inside the system
  const int R = min(32 * NR, ns - rfirst);                      // real receivers in this item
  const int F = NR > 4 ? 1 : R > 64 ? 1 : R > 32 ? 2 : R > 16 ? 4 : 8;  // lane groups
  const int G = 32 / F;
  const int gl = lane % G, phase = lane / G;
  const int t_first = (int)(poff / kTile);
  const int ntl = (ns + kTile - 1) / kTile;
  const int last_cnt = ((ns - (ntl - 1) * kTile) + 3) & ~3;  // real sources of the last tile, to 4

  double xi[NR], yi[NR], zi[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const long long i = rbase + gl + G * k;  // inside the item's tiles for every F
    xi[k] = yi[k] = zi[k] = 0.0;
    if (NBR_IN(i, p.len, p.err)) { xi[k] = p.x[i]; yi[k] = p.y[i]; zi[k] = p.z[i]; }
  }
  u64 hx[NP], hy[NP], hz[NP], lx[NP], ly[NP], lz[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) hx[q] = hy[q] = hz[q] = lx[q] = ly[q] = lz[q] = 0ull;
  double ax[NR], ay[NR], az[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) ax[k] = ay[k] = az[k] = 0.0;

  uint32_t pending = 0;
  auto issue = [&](int t) {  // lane 0 only
    if (t == p.skip_tile) return;
    const unsigned pos = ring.tcount + t;
    const int st = pos % kBStages;
    unsigned char* dst = ring.stages + st * SB;
    const uint32_t bar = smem_u32(&ring.bars[st]);
    const size_t tile = (size_t)(t_first + t);
    if (!NBR_IN((long long)(tile + 1) * kTile - 1, p.len, p.err)) return;  // the wait expires
    if (PREC == kFP32C) {
      mbar_expect_tx(bar, kStageB32);
      bulk_g2s(dst, p.rec + tile * kTile * 3, kRec32, bar);
      bulk_g2s(dst + kRec32, p.org + tile, 32, bar);
    } else {
      mbar_expect_tx(bar, kStageB64);
      const size_t off = tile * kTile;
      bulk_g2s(dst, p.x + off, kTile * 8, bar);
      bulk_g2s(dst + kTile * 8, p.y + off, kTile * 8, bar);
      bulk_g2s(dst + 2 * kTile * 8, p.z + off, kTile * 8, bar);
      bulk_g2s(dst + 3 * kTile * 8, p.m + off, kTile * 8, bar);
    }
    pending |= 1u << st;
  };
  if (lane == 0)
    for (int t = 0; t < kBStages && t < ntl; ++t) issue(t);
  bool aborted = false;
  int t = 0;
  for (; t < ntl; ++t) {
    const unsigned pos = ring.tcount + t;
    const int st = pos % kBStages;
    const bool ok = mbar_wait_bounded(smem_u32(&ring.bars[st]), (pos / kBStages) & 1u, p.wait_ns);
    const unsigned char* base = ring.stages + st * SB;
    const int jend = (t == ntl - 1) ? last_cnt : kTile;
    const bool full = (F == 1) && (jend == kTile);
    if (PREC == kFP32C) {
      if (full) tile_f32c<EXCL, true, NP>(base, 0, 1, kTile, xi, yi, zi, EPS2, hx, hy, hz, lx, ly, lz);
      else tile_f32c<EXCL, false, NP>(base, phase, F, jend, xi, yi, zi, EPS2, hx, hy, hz, lx, ly, lz);
    } else {
      if (full) tile_f64<EXCL, true, NR>(base, 0, 1, kTile, xi, yi, zi, eps2, ax, ay, az);
      else tile_f64<EXCL, false, NR>(base, phase, F, jend, xi, yi, zi, eps2, ax, ay, az);
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, !ok)) {
      aborted = true;
      break;
    }
    if (lane == 0) {
      pending &= ~(1u << st);
      if (t + kBStages < ntl) issue(t + kBStages);
    }
  }
  if (aborted) {
    if (lane == 0) {
      record_error(p.err, kErrTileWait);
      for (int u = t; u < ntl && u < t + kBStages; ++u) {
        const unsigned pos = ring.tcount + u;
        const int st = pos % kBStages;
        if (!(pending & (1u << st))) continue;
        if (!mbar_wait_bounded(smem_u32(&ring.bars[st]), (pos / kBStages) & 1u, p.wait_ns)) {
          record_error(p.err, kErrDrainWait);
          break;
        }
      }
    }
    return false;  // this warp takes no more items; the host reports the error
  }
  ring.tcount += ntl;

  if (PREC == kFP32C) {
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      float h0, h1, l0, l1;
      unpack2(hx[q], h0, h1); unpack2(lx[q], l0, l1);
      ax[2 * q] = (double)h0 + (double)l0; ax[2 * q + 1] = (double)h1 + (double)l1;
      unpack2(hy[q], h0, h1); unpack2(ly[q], l0, l1);
      ay[2 * q] = (double)h0 + (double)l0; ay[2 * q + 1] = (double)h1 + (double)l1;
      unpack2(hz[q], h0, h1); unpack2(lz[q], l0, l1);
      az[2 * q] = (double)h0 + (double)l0; az[2 * q + 1] = (double)h1 + (double)l1;
    }
  }
  // Combine the lane groups' partial sums (fixed xor order: deterministic).
  for (int off = G; off < 32; off <<= 1) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      ax[k] += __shfl_xor_sync(0xffffffffu, ax[k], off);
      ay[k] += __shfl_xor_sync(0xffffffffu, ay[k], off);
      az[k] += __shfl_xor_sync(0xffffffffu, az[k], off);
    }
  }
  // Epilogue: lane group 0 owns receivers gl + G k of the item.
  if (phase == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const int loc = gl + G * k;
      if (loc >= R) continue;
      const long long i = rbase + loc;
      if (!NBR_IN(i, p.len, p.err)) continue;
      const double gx = p.G * ax[k], gy = p.G * ay[k], gz = p.G * az[k];
      p.ax[i] = gx; p.ay[i] = gy; p.az[i] = gz;
      if (p.mode == 1) {
        const double vx = p.vx[i] + p.kick * gx;
        const double vy = p.vy[i] + p.kick * gy;
        const double vz = p.vz[i] + p.kick * gz;
        p.vx[i] = vx; p.vy[i] = vy; p.vz[i] = vz;
        p.xn[i] = xi[k] + p.drift * vx;
        p.yn[i] = yi[k] + p.drift * vy;
        p.zn[i] = zi[k] + p.drift * vz;
      }
    }
  }
  if (p.mode == 1 && p.rec_next && NBR_IN(rbase + 32 * NR - 1, p.len, p.err)) {
    // Pack each of the item's tiles of the new positions (layout lane + 32k);
    // every tile of an item holds at least one real receiver.
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NR / 4; ++q) {
      double px[4], py[4], pz[4];
      double sx = 0.0, sy = 0.0, sz = 0.0, cnt = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int loc = kTile * q + lane + 32 * k;
        const long long i = rbase + loc;
        px[k] = py[k] = pz[k] = 0.0;
        if (loc < R) {
          px[k] = p.xn[i]; py[k] = p.yn[i]; pz[k] = p.zn[i];
          sx += px[k]; sy += py[k]; sz += pz[k]; cnt += 1.0;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, off);
        sy += __shfl_xor_sync(0xffffffffu, sy, off);
        sz += __shfl_xor_sync(0xffffffffu, sz, off);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
      }
      const double ox = sx / cnt, oy = sy / cnt, oz = sz / cnt;  // cnt >= 1
      if (lane == 0) p.org_next[tile0 + q] = make_double4(ox, oy, oz, 0.0);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int loc = kTile * q + lane + 32 * k;
        const long long i = rbase + loc;
        float fx = 0.f, fy = 0.f, fz = 0.f, fa = 0.f, fb = 0.f;
        if (loc < R) {
          fx = __double2float_rn(px[k] - ox);
          fy = __double2float_rn(py[k] - oy);
          fz = __double2float_rn(pz[k] - oz);
          fa = __double2float_rn(-1.5 * p.m[i]);
          fb = __double2float_rn(2.5 * p.m[i]);
        }
        p.rec_next[3 * i + 0] = make_float4(fx, fx, fy, fy);
        p.rec_next[3 * i + 1] = make_float4(fz, fz, fa, fa);
        p.rec_next[3 * i + 2] = make_float4(fb, fb, 0.f, 0.f);
      }
    }
  }
  __syncwarp();
  return true;
}

// One Newton-3 item (FP32C): row block `blk` of system s -- its tiles 2 blk and
// 2 blk + 1, 256 receivers, 8 per lane (lane + 32 q) -- against the system's
// column tiles c >= 2 blk.  Its own two tiles: every ordered pair, action only.
// Each later tile c: every pair once, the tile's 128 sources in 4 batches of
// 32, one per lane, rotating through the warp by shuffles with their reaction
// sums (the scheme of k_force_n3_f32c); the reaction of tile c from this block
// goes to its slot, the action of the block's receivers to p.act.  The epilogue
// runs later, in k_batch_n3_reduce.  Returns false if a tile wait gave up.
template <bool EXCL>
__device__ __forceinline__ bool run_item_n3(const BatchParams& p, u64 EPS2, Ring& ring, int lane,
                                            int s, int blk) {
  constexpr int SB = kStageB32;
  const long long poff = p.poff[s];
  const int ns = p.nreal[s];
  const int T = (ns + kTile - 1) / kTile;
  const int t_first = (int)(poff / kTile);
  const int c0 = 2 * blk;
  const int ntl = T - c0;                          // column tiles c0 .. T - 1
  const int rloc = c0 * kTile + lane;              // receiver q = 0 inside the system
  const long long slot0 = p.rea_off[s] + n3b_prefix(T, blk, 2);

  double xi[8], yi[8], zi[8];
  u64 AI[4], BI[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float m0 = 0.f, m1 = 0.f;
    const int l0 = rloc + 64 * q, l1 = l0 + 32;  // receivers 2q and 2q + 1 of the lane
    xi[2 * q] = yi[2 * q] = zi[2 * q] = xi[2 * q + 1] = yi[2 * q + 1] = zi[2 * q + 1] = 0.0;
    if (l0 < ns && NBR_IN(poff + l0, p.len, p.err)) {
      xi[2 * q] = p.x[poff + l0]; yi[2 * q] = p.y[poff + l0]; zi[2 * q] = p.z[poff + l0];
      m0 = (float)p.m[poff + l0];
    }
    if (l1 < ns && NBR_IN(poff + l1, p.len, p.err)) {
      xi[2 * q + 1] = p.x[poff + l1]; yi[2 * q + 1] = p.y[poff + l1]; zi[2 * q + 1] = p.z[poff + l1];
      m1 = (float)p.m[poff + l1];
    }
    AI[q] = pack2(-1.5f * m0, -1.5f * m1);
    BI[q] = pack2(2.5f * m0, 2.5f * m1);
  }
  u64 hx[4], hy[4], hz[4], lx[4], ly[4], lz[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) hx[q] = hy[q] = hz[q] = lx[q] = ly[q] = lz[q] = 0ull;

  uint32_t pending = 0;
  auto issue = [&](int t) {  // lane 0 only
    if (t == p.skip_tile) return;
    const unsigned pos = ring.tcount + t;
    const int st = pos % kBStages;
    unsigned char* dst = ring.stages + st * SB;
    const uint32_t bar = smem_u32(&ring.bars[st]);
    const size_t tile = (size_t)(t_first + c0 + t);
    if (!NBR_IN((long long)(tile + 1) * kTile - 1, p.len, p.err)) return;  // the wait expires
    mbar_expect_tx(bar, kStageB32);
    bulk_g2s(dst, p.rec + tile * kTile * 3, kRec32, bar);
    bulk_g2s(dst + kRec32, p.org + tile, 32, bar);
    pending |= 1u << st;
  };
  if (lane == 0)
    for (int t = 0; t < kBStages && t < ntl; ++t) issue(t);
  bool aborted = false;
  int t = 0;
  for (; t < ntl; ++t) {
    const unsigned pos = ring.tcount + t;
    const int st = pos % kBStages;
    const bool ok = mbar_wait_bounded(smem_u32(&ring.bars[st]), (pos / kBStages) & 1u, p.wait_ns);
    const unsigned char* base = ring.stages + st * SB;
    const double4 o = *reinterpret_cast<const double4*>(base + kRec32);
    u64 XI[4], YI[4], ZI[4], AX[4], AY[4], AZ[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      XI[q] = pack2(__double2float_rn(xi[2 * q] - o.x), __double2float_rn(xi[2 * q + 1] - o.x));
      YI[q] = pack2(__double2float_rn(yi[2 * q] - o.y), __double2float_rn(yi[2 * q + 1] - o.y));
      ZI[q] = pack2(__double2float_rn(zi[2 * q] - o.z), __double2float_rn(zi[2 * q + 1] - o.z));
      AX[q] = AY[q] = AZ[q] = 0ull;
    }
    if (t < 2) {
      // the block's own tiles: every ordered pair, action only
      const ulonglong2* R = reinterpret_cast<const ulonglong2*>(base);
#pragma unroll 4
      for (int j = 0; j < kTile; ++j) {
        const ulonglong2 q0 = R[3 * j];
        const ulonglong2 q1 = R[3 * j + 1];
        const u64 bj = R[3 * j + 2].x;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const u64 dx = sub2(q0.x, XI[q]);
          const u64 dy = sub2(q0.y, YI[q]);
          const u64 dz = sub2(q1.x, ZI[q]);
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
          AX[q] = fma2(sv, dx, AX[q]);
          AY[q] = fma2(sv, dy, AY[q]);
          AZ[q] = fma2(sv, dz, AZ[q]);
        }
      }
    } else {
      // a later tile: every pair once; reaction of source j (bt 32 + lane)
      const float4* R4 = reinterpret_cast<const float4*>(base);
      const int from = (lane + 31) & 31;
      double* slot = p.rea + (size_t)(slot0 + (t - 2)) * 3 * kTile;
      const int nsrc = min(kTile, ns - (c0 + t) * kTile);  // real sources of the tile
#pragma unroll 1
      for (int bt = 0; bt < 4; ++bt) {
        const int j = bt * 32 + lane;
        if (bt * 32 >= nsrc) {  // a batch of padding: no pairs, zero reactions
          if (NBR_IN((slot - p.rea) + 2 * kTile + j, p.rea_len, p.err))
            slot[j] = slot[kTile + j] = slot[2 * kTile + j] = 0.0;
          continue;
        }
        const float4 q0 = R4[3 * j], q1 = R4[3 * j + 1], q2 = R4[3 * j + 2];
        float sx = q0.x, sy = q0.z, sz = q1.x, sa = q1.z, sb = q2.x;
        u64 RX = 0ull, RY = 0ull, RZ = 0ull;
#pragma unroll 2
        for (int step = 0; step < 32; ++step) {
          const u64 SX = pack2(sx, sx), SY = pack2(sy, sy), SZ = pack2(sz, sz);
          const u64 SA = pack2(sa, sa), SBv = pack2(sb, sb);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const u64 dx = sub2(SX, XI[q]);
            const u64 dy = sub2(SY, YI[q]);
            const u64 dz = sub2(SZ, ZI[q]);
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
            const u64 sj = mul2(y3, fma2(SA, pr, SBv));       // m_j (1 + 3e/2) y^3
            const u64 si = mul2(y3, fma2(AI[q], pr, BI[q]));  // m_i (1 + 3e/2) y^3
            // reaction first, and its shuffles before the sources' (as in
            // k_force_n3_f32c: the faster schedule, +0.6 % here)
            RX = fma2(si, dx, RX);
            RY = fma2(si, dy, RY);
            RZ = fma2(si, dz, RZ);
            AX[q] = fma2(sj, dx, AX[q]);
            AY[q] = fma2(sj, dy, AY[q]);
            AZ[q] = fma2(sj, dz, AZ[q]);
          }
          RX = __shfl_sync(0xffffffffu, RX, from);
          RY = __shfl_sync(0xffffffffu, RY, from);
          RZ = __shfl_sync(0xffffffffu, RZ, from);
          sx = __shfl_sync(0xffffffffu, sx, from);
          sy = __shfl_sync(0xffffffffu, sy, from);
          sz = __shfl_sync(0xffffffffu, sz, from);
          sa = __shfl_sync(0xffffffffu, sa, from);
          sb = __shfl_sync(0xffffffffu, sb, from);
        }
        // back at its own lane: the acceleration of source j is -sum m_i y^3 d
        if (NBR_IN((slot - p.rea) + 2 * kTile + j, p.rea_len, p.err)) {
          float u0, u1;
          unpack2(RX, u0, u1); slot[j] = -((double)u0 + (double)u1);
          unpack2(RY, u0, u1); slot[kTile + j] = -((double)u0 + (double)u1);
          unpack2(RZ, u0, u1); slot[2 * kTile + j] = -((double)u0 + (double)u1);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      two_sum2(hx[q], lx[q], AX[q]);
      two_sum2(hy[q], ly[q], AY[q]);
      two_sum2(hz[q], lz[q], AZ[q]);
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, !ok)) {
      aborted = true;
      break;
    }
    if (lane == 0) {
      pending &= ~(1u << st);
      if (t + kBStages < ntl) issue(t + kBStages);
    }
  }
  if (aborted) {
    if (lane == 0) {
      record_error(p.err, kErrTileWait);
      for (int u = t; u < ntl && u < t + kBStages; ++u) {
        const unsigned pos = ring.tcount + u;
        const int st = pos % kBStages;
        if (!(pending & (1u << st))) continue;
        if (!mbar_wait_bounded(smem_u32(&ring.bars[st]), (pos / kBStages) & 1u, p.wait_ns)) {
          record_error(p.err, kErrDrainWait);
          break;
        }
      }
    }
    return false;
  }
  ring.tcount += ntl;
  // the block's action, compensated sum hi + lo formed in FP64
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float h0, h1, l0, l1;
    const long long i0 = poff + rloc + 64 * q, i1 = i0 + 32;
    double a0[3], a1[3];
    unpack2(hx[q], h0, h1); unpack2(lx[q], l0, l1);
    a0[0] = (double)h0 + (double)l0; a1[0] = (double)h1 + (double)l1;
    unpack2(hy[q], h0, h1); unpack2(ly[q], l0, l1);
    a0[1] = (double)h0 + (double)l0; a1[1] = (double)h1 + (double)l1;
    unpack2(hz[q], h0, h1); unpack2(lz[q], l0, l1);
    a0[2] = (double)h0 + (double)l0; a1[2] = (double)h1 + (double)l1;
    if (rloc + 64 * q < ns && NBR_IN(i0, p.len, p.err))
      for (int d = 0; d < 3; ++d) p.act[(size_t)d * p.n_pad + i0] = a0[d];
    if (rloc + 64 * q + 32 < ns && NBR_IN(i1, p.len, p.err))
      for (int d = 0; d < 3; ++d) p.act[(size_t)d * p.n_pad + i1] = a1[d];
  }
  __syncwarp();
  return true;
}
// One Newton-3 item (FP64): row tile r of system s -- 128 receivers, 4 per
// lane (lane + 32 k) -- against the system's column tiles c >= r.  Its own
// tile: every ordered pair, action only (tile_f64).  Each later tile c: every
// pair once, the tile's sources in batches of 32, one per lane, rotating
// through the warp by shuffles with their reaction sums (the scheme of
// k_force_n3_f64); batches of padding are skipped.  The reaction of tile c
// goes to its slot, the action to p.act; the epilogue runs in
// k_batch_n3_reduce.  Returns false if a tile wait gave up.
template <bool EXCL>
__device__ __forceinline__ bool run_item_n3_f64(const BatchParams& p, double eps2, Ring& ring,
                                                int lane, int s, int r) {
  constexpr int SB = kStageB64;
  const long long poff = p.poff[s];
  const int ns = p.nreal[s];
  const int T = (ns + kTile - 1) / kTile;
  const int t_first = (int)(poff / kTile);
  const int ntl = T - r;                 // column tiles r .. T - 1
  const int rloc = r * kTile + lane;     // receiver k = 0 inside the system
  const long long slot0 = p.rea_off[s] + n3b_prefix(T, r, 1);
  const int last_cnt = ((ns - (T - 1) * kTile) + 3) & ~3;  // real sources of the last tile, to 4

  double xi[4], yi[4], zi[4], mi[4], ax[4], ay[4], az[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int l = rloc + 32 * k;
    xi[k] = yi[k] = zi[k] = mi[k] = ax[k] = ay[k] = az[k] = 0.0;
    if (l < ns && NBR_IN(poff + l, p.len, p.err)) {
      xi[k] = p.x[poff + l]; yi[k] = p.y[poff + l]; zi[k] = p.z[poff + l]; mi[k] = p.m[poff + l];
    }
  }

  uint32_t pending = 0;
  auto issue = [&](int t) {  // lane 0 only
    if (t == p.skip_tile) return;
    const unsigned pos = ring.tcount + t;
    const int st = pos % kBStages;
    unsigned char* dst = ring.stages + st * SB;
    const uint32_t bar = smem_u32(&ring.bars[st]);
    const size_t tile = (size_t)(t_first + r + t);
    if (!NBR_IN((long long)(tile + 1) * kTile - 1, p.len, p.err)) return;  // the wait expires
    mbar_expect_tx(bar, kStageB64);
    const size_t off = tile * kTile;
    bulk_g2s(dst, p.x + off, kTile * 8, bar);
    bulk_g2s(dst + kTile * 8, p.y + off, kTile * 8, bar);
    bulk_g2s(dst + 2 * kTile * 8, p.z + off, kTile * 8, bar);
    bulk_g2s(dst + 3 * kTile * 8, p.m + off, kTile * 8, bar);
    pending |= 1u << st;
  };
  if (lane == 0)
    for (int t = 0; t < kBStages && t < ntl; ++t) issue(t);
  bool aborted = false;
  int t = 0;
  for (; t < ntl; ++t) {
    const unsigned pos = ring.tcount + t;
    const int st = pos % kBStages;
    const bool ok = mbar_wait_bounded(smem_u32(&ring.bars[st]), (pos / kBStages) & 1u, p.wait_ns);
    const unsigned char* base = ring.stages + st * SB;
    const int c = r + t;
    if (t == 0) {
      // the own tile: every ordered pair, action only
      const int jend = (c == T - 1) ? last_cnt : kTile;
      if (jend == kTile) tile_f64<EXCL, true, 4>(base, 0, 1, kTile, xi, yi, zi, eps2, ax, ay, az);
      else tile_f64<EXCL, false, 4>(base, 0, 1, jend, xi, yi, zi, eps2, ax, ay, az);
    } else {
      const double* SX = reinterpret_cast<const double*>(base);
      const double* SY = SX + kTile;
      const double* SZ = SY + kTile;
      const double* SM = SZ + kTile;
      const int from = (lane + 31) & 31;
      double* slot = p.rea + (size_t)(slot0 + (t - 1)) * 3 * kTile;
      const int nsrc = min(kTile, ns - c * kTile);  // real sources of the tile
#pragma unroll 1
      for (int bt = 0; bt < 4; ++bt) {
        const int j = bt * 32 + lane;
        const bool in = NBR_IN((slot - p.rea) + 2 * kTile + j, p.rea_len, p.err);
        if (bt * 32 >= nsrc) {  // a batch of padding: no pairs, zero reactions
          if (in) slot[j] = slot[kTile + j] = slot[2 * kTile + j] = 0.0;
          continue;
        }
        double sx = SX[j], sy = SY[j], sz = SZ[j], sm = SM[j];
        double RX = 0.0, RY = 0.0, RZ = 0.0;
#pragma unroll 2
        for (int step = 0; step < 32; ++step) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double dx = sx - xi[k], dy = sy - yi[k], dz = sz - zi[k];
            double r2 = fma(dx, dx, eps2);
            r2 = fma(dy, dy, r2);
            r2 = fma(dz, dz, r2);
            double y = rsqrt(r2);
            if (EXCL) y = r2 > 0.0 ? y : 0.0;
            const double y3 = y * y * y;
            const double sj = sm * y3, si = mi[k] * y3;
            ax[k] = fma(sj, dx, ax[k]);
            ay[k] = fma(sj, dy, ay[k]);
            az[k] = fma(sj, dz, az[k]);
            RX = fma(si, dx, RX);
            RY = fma(si, dy, RY);
            RZ = fma(si, dz, RZ);
          }
          sx = __shfl_sync(0xffffffffu, sx, from);
          sy = __shfl_sync(0xffffffffu, sy, from);
          sz = __shfl_sync(0xffffffffu, sz, from);
          sm = __shfl_sync(0xffffffffu, sm, from);
          RX = __shfl_sync(0xffffffffu, RX, from);
          RY = __shfl_sync(0xffffffffu, RY, from);
          RZ = __shfl_sync(0xffffffffu, RZ, from);
        }
        // back at its own lane: the acceleration of source j is -sum m_i y^3 d
        if (in) {
          slot[j] = -RX;
          slot[kTile + j] = -RY;
          slot[2 * kTile + j] = -RZ;
        }
      }
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, !ok)) {
      aborted = true;
      break;
    }
    if (lane == 0) {
      pending &= ~(1u << st);
      if (t + kBStages < ntl) issue(t + kBStages);
    }
  }
  if (aborted) {
    if (lane == 0) {
      record_error(p.err, kErrTileWait);
      for (int u = t; u < ntl && u < t + kBStages; ++u) {
        const unsigned pos = ring.tcount + u;
        const int st = pos % kBStages;
        if (!(pending & (1u << st))) continue;
        if (!mbar_wait_bounded(smem_u32(&ring.bars[st]), (pos / kBStages) & 1u, p.wait_ns)) {
          record_error(p.err, kErrDrainWait);
          break;
        }
      }
    }
    return false;
  }
  ring.tcount += ntl;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long i = poff + rloc + 32 * k;
    if (rloc + 32 * k < ns && NBR_IN(i, p.len, p.err)) {
      p.act[i] = ax[k];
      p.act[p.n_pad + i] = ay[k];
      p.act[2 * p.n_pad + i] = az[k];
    }
  }
  __syncwarp();
  return true;
}

// The persistent kernel.  WIDE = 0: every item is narrow (4 receivers per
// lane); WIDE = 1: items flagged kWideItem cover two tiles (8 receivers per
// lane: twice the pair work per source read, four independent f32x2 chains);
// WIDE = 2: items flagged kN3Item are Newton-3 row blocks (FP32C: two tiles,
// systems of three tiles or more; FP64: one tile, systems of two tiles or
// more; their epilogue runs in k_batch_n3_reduce), the other systems' items
// as for WIDE = 1 (FP32C) or 0 (FP64).
template <int PREC, bool EXCL, int WIDE>
__global__ void __launch_bounds__(kBWarps * 32) k_batch_force(const BatchParams p, const double eps2) {
  constexpr int SB = Stage<PREC>::bytes;
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Ring ring;
  ring.bars = reinterpret_cast<uint64_t*>(smem) + warp * kBStages;
  ring.stages = smem + kBHead + (size_t)warp * kBStages * SB;
  ring.tcount = 0;
  if (lane == 0) {
    for (int st = 0; st < kBStages; ++st) mbar_init(smem_u32(&ring.bars[st]), 1);
    mbar_fence_init();
  }
  __syncwarp();
  const float e2f = (float)eps2;
  const u64 EPS2 = pack2(e2f, e2f);
  while (true) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(p.head, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= p.n_items) break;
    const int2 it = p.items[item];
    const int s = it.x & ~(kWideItem | kN3Item);
    if (!NBR_IN(s, p.nsys, p.err)) return;
    bool ok;
    if (WIDE == 2 && (it.x & kN3Item)) {
      if constexpr (PREC == kFP32C) ok = run_item_n3<EXCL>(p, EPS2, ring, lane, s, it.y);
      else ok = run_item_n3_f64<EXCL>(p, eps2, ring, lane, s, it.y);
    } else if (WIDE == 1 && (it.x & kWideItem)) {
      ok = run_item<PREC, EXCL, 8>(p, eps2, EPS2, ring, lane, s, it.y);
    } else if (WIDE == 2 && PREC == kFP32C && (it.x & kWideItem)) {
      // (the FP64 Newton-3 list has no two-tile items: not compiled in)
      if constexpr (PREC == kFP32C) ok = run_item<PREC, EXCL, 8>(p, eps2, EPS2, ring, lane, s, it.y);
    } else {
      ok = run_item<PREC, EXCL, 4>(p, eps2, EPS2, ring, lane, s, it.y);
    }
    if (!ok) return;
  }
}

// The epilogue of the Newton-3 systems: one warp per tile (system, local tile
// c); each particle's acceleration is its action plus the reactions from the
// system's row blocks before its own (b = 0 .. c / rows - 1, rows = tiles per
// row block) in that order: deterministic.  Then the kick/drift and, FP32C, the tile's record pack, as
// in run_item.
__global__ void __launch_bounds__(128) k_batch_n3_reduce(const BatchParams p, const int2* tiles,
                                                         int ntiles) {
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= ntiles) return;
  const int2 tc = tiles[w];
  const int s = tc.x, c = tc.y;
  const long long poff = p.poff[s];
  const int ns = p.nreal[s];
  const int T = (ns + kTile - 1) / kTile;
  const int rows = p.n3_rows;
  const int B = c / rows;
  const long long rbase = poff + (long long)c * kTile;
  const int R = min(kTile, ns - c * kTile);  // real particles of the tile
  double ax[4], ay[4], az[4], xi[4], yi[4], zi[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int loc = lane + 32 * k;
    const long long i = rbase + loc;
    ax[k] = ay[k] = az[k] = xi[k] = yi[k] = zi[k] = 0.0;
    if (loc >= R || !NBR_IN(i, p.len, p.err)) continue;
    ax[k] = p.act[i]; ay[k] = p.act[p.n_pad + i]; az[k] = p.act[2 * p.n_pad + i];
    xi[k] = p.x[i]; yi[k] = p.y[i]; zi[k] = p.z[i];
  }
  // The reaction slots in block order; the 12 loads of a slot (every slot
  // entry is written, padding included) are issued before its adds.
  const long long slot_b0 = p.rea_off[s] + (c - rows);
#pragma unroll 2
  for (int b = 0; b < B; ++b) {
    const long long sl = slot_b0 + n3b_prefix(T, b, rows) - (long long)rows * b;
    if (!NBR_IN((sl + 1) * 3 * kTile - 1, p.rea_len, p.err)) break;
    const double* r = p.rea + (size_t)sl * 3 * kTile + lane;
    double tx[4], ty[4], tz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      tx[k] = r[32 * k]; ty[k] = r[kTile + 32 * k]; tz[k] = r[2 * kTile + 32 * k];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ax[k] += tx[k]; ay[k] += ty[k]; az[k] += tz[k];
    }
  }
  double px[4], py[4], pz[4];
  double sx = 0.0, sy = 0.0, sz = 0.0, cnt = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int loc = lane + 32 * k;
    const long long i = rbase + loc;
    px[k] = py[k] = pz[k] = 0.0;
    if (loc >= R || !NBR_IN(i, p.len, p.err)) continue;
    const double gx = p.G * ax[k], gy = p.G * ay[k], gz = p.G * az[k];
    p.ax[i] = gx; p.ay[i] = gy; p.az[i] = gz;
    if (p.mode == 1) {
      const double vx = p.vx[i] + p.kick * gx;
      const double vy = p.vy[i] + p.kick * gy;
      const double vz = p.vz[i] + p.kick * gz;
      p.vx[i] = vx; p.vy[i] = vy; p.vz[i] = vz;
      px[k] = xi[k] + p.drift * vx;
      py[k] = yi[k] + p.drift * vy;
      pz[k] = zi[k] + p.drift * vz;
      p.xn[i] = px[k]; p.yn[i] = py[k]; p.zn[i] = pz[k];
      sx += px[k]; sy += py[k]; sz += pz[k]; cnt += 1.0;
    }
  }
  if (p.mode != 1 || !p.rec_next || !NBR_IN(rbase + kTile - 1, p.len, p.err)) return;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, off);
    sy += __shfl_xor_sync(0xffffffffu, sy, off);
    sz += __shfl_xor_sync(0xffffffffu, sz, off);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
  }
  const double ox = sx / cnt, oy = sy / cnt, oz = sz / cnt;  // cnt >= 1
  if (lane == 0) p.org_next[rbase / kTile] = make_double4(ox, oy, oz, 0.0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int loc = lane + 32 * k;
    const long long i = rbase + loc;
    float fx = 0.f, fy = 0.f, fz = 0.f, fa = 0.f, fb = 0.f;
    if (loc < R) {
      fx = __double2float_rn(px[k] - ox);
      fy = __double2float_rn(py[k] - oy);
      fz = __double2float_rn(pz[k] - oz);
      fa = __double2float_rn(-1.5 * p.m[i]);
      fb = __double2float_rn(2.5 * p.m[i]);
    }
    p.rec_next[3 * i + 0] = make_float4(fx, fx, fy, fy);
    p.rec_next[3 * i + 1] = make_float4(fz, fz, fa, fa);
    p.rec_next[3 * i + 2] = make_float4(fb, fb, 0.f, 0.f);
  }
}

// Per-system diagnostics: one CTA per system.  out[s * 9 + c] =
// T, Px, Py, Pz, Lx, Ly, Lz, M, U (softened, FP64, fixed-order reductions).
__global__ void __launch_bounds__(256)
    k_batch_diag(const double* __restrict__ x, const double* __restrict__ y,
                 const double* __restrict__ z, const double* __restrict__ vx,
                 const double* __restrict__ vy, const double* __restrict__ vz,
                 const double* __restrict__ m, const long long* __restrict__ poff,
                 const int* __restrict__ nreal, double G, double eps2, double* __restrict__ out) {
  __shared__ double red[9][256];
  __shared__ double sx[256], sy[256], sz[256], sm[256];
  const int s = blockIdx.x;
  const long long o = poff[s];
  const int n = nreal[s];
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i0 = 0; i0 < n; i0 += 256) {
    const int i = i0 + threadIdx.x;
    const bool valid = i < n;
    const double xi = valid ? x[o + i] : 0.0, yi = valid ? y[o + i] : 0.0, zi = valid ? z[o + i] : 0.0;
    const double mi = valid ? m[o + i] : 0.0;
    if (valid) {
      const double ux = vx[o + i], uy = vy[o + i], uz = vz[o + i];
      v[0] += 0.5 * mi * (ux * ux + uy * uy + uz * uz);
      v[1] += mi * ux; v[2] += mi * uy; v[3] += mi * uz;
      v[4] += mi * (yi * uz - zi * uy);
      v[5] += mi * (zi * ux - xi * uz);
      v[6] += mi * (xi * uy - yi * ux);
      v[7] += mi;
    }
    double phi = 0.0;
    for (int j0 = 0; j0 < n; j0 += 256) {
      const int jl = j0 + threadIdx.x;
      __syncthreads();
      sx[threadIdx.x] = jl < n ? x[o + jl] : 0.0;
      sy[threadIdx.x] = jl < n ? y[o + jl] : 0.0;
      sz[threadIdx.x] = jl < n ? z[o + jl] : 0.0;
      sm[threadIdx.x] = jl < n ? m[o + jl] : 0.0;
      __syncthreads();
      const int cnt = min(256, n - j0);
      for (int jj = 0; jj < cnt; ++jj) {
        if (j0 + jj == i) continue;
        const double dx = sx[jj] - xi, dy = sy[jj] - yi, dz = sz[jj] - zi;
        phi += sm[jj] / sqrt(dx * dx + dy * dy + dz * dz + eps2);
      }
    }
    if (valid) v[8] += -0.5 * G * mi * phi;
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) red[c][threadIdx.x] = v[c];
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int c = 0; c < 9; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 9; ++c) out[(size_t)s * 9 + c] = red[c][0];
}

template <int PREC, bool EXCL, int WIDE>
const void* batch_fn() {
  return (const void*)k_batch_force<PREC, EXCL, WIDE>;
}

// wide: 0, 1 or 2 -- the work list the kernel variant takes.
const void* batch_kernel(int prec, bool excl, int wide) {
  if (prec == kFP32C) {
    if (excl)
      return wide == 2 ? batch_fn<kFP32C, true, 2>()
             : wide   ? batch_fn<kFP32C, true, 1>()
                      : batch_fn<kFP32C, true, 0>();
    return wide == 2 ? batch_fn<kFP32C, false, 2>()
           : wide   ? batch_fn<kFP32C, false, 1>()
                    : batch_fn<kFP32C, false, 0>();
  }
  if (excl)
    return wide == 2 ? batch_fn<kFP64, true, 2>()
           : wide   ? batch_fn<kFP64, true, 1>()
                    : batch_fn<kFP64, true, 0>();
  return wide == 2 ? batch_fn<kFP64, false, 2>()
         : wide   ? batch_fn<kFP64, false, 1>()
                  : batch_fn<kFP64, false, 0>();
}

size_t batch_smem(int prec) {
  return kBHead + (size_t)kBWarps * kBStages * (prec == kFP32C ? kStageB32 : kStageB64);
}

cudaError_t launch_batch(int prec, int wide, const BatchParams& p, double eps2, int grid,
                         cudaStream_t st) {
  const void* fn = batch_kernel(prec, eps2 == 0.0, wide);
  const size_t smem = batch_smem(prec);
  void* args[] = {(void*)&p, (void*)&eps2};
  return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(kBWarps * 32), args, smem, st);
}

// Autotune-cache key of a batch: precision, log2 of the system count and of
// the largest system, eps == 0.
std::string batch_key(int prec, size_t nsys, int max_ns, bool excl) {
  int sb = 0, nb = 0;
  while (((size_t)1 << (sb + 1)) <= nsys) ++sb;
  while ((1 << (nb + 1)) <= max_ns) ++nb;
  return std::string("batch:") + (prec == kFP32C ? "fp32c" : "fp64") + ":s" + std::to_string(sb) +
         ":n" + std::to_string(nb) + (excl ? ":e0" : "");
}

// The kernel configuration of the batch for a precision: from the autotune
// cache when it holds this batch's key, else the default (occupancy-limited
// grid; Newton-3 row blocks).  The cache stores
// the work list as ni: 4 one-tile items, 8 two-tile items, 3 Newton-3 row
// blocks.
void batch_config(nbr_ctx* c, int prec, double eps2) {
  BatchState& b = c->bat;
  const int pi = prec == kFP32C ? 1 : 0;
  if (b.cfg_ok[pi]) return;
  ForceConfig t{0, 0, 0};
  if (tune_get(batch_key(prec, b.nsys, b.max_ns, eps2 == 0.0), &t) &&
      (t.ni == 4 || t.ni == 8 || t.ni == 3)) {
    b.wide[pi] = t.ni == 8 ? 1 : t.ni == 3 ? 2 : 0;
    b.per_sm[pi] = t.split;
  } else {
    // Defaults from the 4096-system workload on B200: FP32C 1888 GPairs/s
    // with one-tile items, 2045 with two-tile items, 2471 with Newton-3 row
    // blocks; FP64 837 with one-tile items, 787 with two-tile items, 1153
    // with Newton-3 row blocks.
    b.wide[pi] = 2;
    b.per_sm[pi] = 0;
  }
  b.cfg_ok[pi] = true;
}

// Sets the kernel's shared-memory attribute (once per kernel variant),
// allocates the Newton-3 scratch at its first use, and returns the
// persistent grid: resident CTAs per SM (the configured count, at most the
// occupancy limit) x SMs, or 0 if the scratch allocation failed.  Called
// before any stream capture.
int batch_grid(nbr_ctx* c, int prec, double eps2) {
  BatchState& b = c->bat;
  batch_config(c, prec, eps2);
  const int pi = prec == kFP32C ? 1 : 0, ei = eps2 == 0.0 ? 1 : 0, wi = b.wide[pi];
  BatchState::N3List& l3 = b.n3[pi];
  if (wi == 2 && l3.slots > 0 && !l3.d_rea) {
    cudaError_t e = cudaSuccess;
    if (!b.d_act) e = dalloc((void**)&b.d_act, 3 * b.s.n_pad * sizeof(double));
    if (e == cudaSuccess) e = dalloc((void**)&l3.d_rea, (size_t)l3.slots * 3 * kTile * sizeof(double));
    if (e != cudaSuccess) {
      dfree(l3.d_rea);
      l3.d_rea = nullptr;
      return 0;
    }
  }
  int& occ = b.occ[pi][ei][wi];
  if (occ == 0) {
    const void* fn = batch_kernel(prec, eps2 == 0.0, wi);
    const size_t smem = batch_smem(prec);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kBWarps * 32, smem) != cudaSuccess ||
        per < 1)
      per = 1;
    occ = per;
  }
  const int per = b.per_sm[pi] > 0 ? std::min(b.per_sm[pi], occ) : occ;
  return per * c->sms;
}

// One batched force evaluation (mode 0: a only; 1: leapfrog step into the
// other buffer).
int batch_eval(nbr_ctx* c, int prec, double G, double eps2, int mode, double kick, double drift,
               int* kernels) {
  BatchState& b = c->bat;
  SysState& s = b.s;
  const int a = s.cur, o = 1 - s.cur;
  cudaError_t e = cudaSuccess;
  if (prec == kFP32C && !s.rec_ok[a]) {
    e = launch_kick_drift((long long)s.n, (long long)s.n_pad, s.pos[a][0], s.pos[a][1], s.pos[a][2],
                          s.mass, nullptr, nullptr, nullptr, 0.0, 0.0, nullptr, nullptr, nullptr,
                          nullptr, nullptr, nullptr, s.rec[a], s.org[a], c->stream);
    if (kernels) ++*kernels;
    if (e != cudaSuccess) return cuda_fail(c, e, "batch pack");
    s.rec_ok[a] = true;
  }
  e = cudaMemsetAsync(b.d_head, 0, sizeof(unsigned), c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "batch queue reset");
  BatchParams p{};
  p.x = s.pos[a][0]; p.y = s.pos[a][1]; p.z = s.pos[a][2]; p.m = s.mass;
  p.rec = s.rec[a]; p.org = s.org[a];
  const int grid = batch_grid(c, prec, eps2);  // also settles the configuration
  if (grid == 0) return fail(c, NBR_ERR_CUDA, "batch Newton-3 scratch allocation");
  const int pi = prec == kFP32C ? 1 : 0, wi = b.wide[pi];
  const BatchState::N3List& l3 = b.n3[pi];
  p.poff = b.d_poff; p.nreal = b.d_nreal;
  p.items = wi == 2 ? l3.d_items : b.d_items[wi];
  p.n_items = wi == 2 ? l3.n_items : b.n_items[wi];
  p.act = b.d_act; p.rea = l3.d_rea; p.rea_off = l3.d_rea_off; p.n_pad = (long long)s.n_pad;
  p.n3_rows = prec == kFP32C ? 2 : 1;
  p.head = b.d_head;
  p.mode = mode; p.G = G; p.kick = kick; p.drift = drift;
  p.ax = s.acc[0]; p.ay = s.acc[1]; p.az = s.acc[2];
  p.vx = s.vel[0]; p.vy = s.vel[1]; p.vz = s.vel[2];
  p.xn = s.pos[o][0]; p.yn = s.pos[o][1]; p.zn = s.pos[o][2];
  p.rec_next = (mode == 1 && prec == kFP32C) ? s.rec[o] : nullptr;
  p.org_next = s.org[o];
  p.err = c->d_err;
  JStream js{};
  pipeline_params(js);
  p.wait_ns = js.wait_ns;
  p.skip_tile = js.skip_tile;
  NBR_CHECKED_ONLY(p.len = (long long)s.cap; p.nsys = (int)b.nsys;
                   p.rea_len = l3.d_rea ? l3.slots * 3 * kTile : 0;)
  e = launch_batch(prec, wi, p, eps2, grid, c->stream);
  if (kernels) ++*kernels;
  if (e != cudaSuccess) return cuda_fail(c, e, "batch force launch");
  if (wi == 2 && l3.n_tiles > 0) {
    const unsigned blocks = (unsigned)((l3.n_tiles + 3) / 4);
    k_batch_n3_reduce<<<blocks, 128, 0, c->stream>>>(p, l3.d_tiles, l3.n_tiles);
    e = cudaGetLastError();
    if (kernels) ++*kernels;
    if (e != cudaSuccess) return cuda_fail(c, e, "batch Newton-3 epilogue launch");
  }
  if (mode == 1) {
    s.cur = o;
    s.rec_ok[o] = (prec == kFP32C);
    s.rec_ok[a] = false;
  }
  return NBR_OK;
}

}  // namespace

void nbr::BatchState::release() {
  s.release();
  dfree(d_poff);
  dfree(d_nreal);
  dfree(d_sys_of_tile);
  dfree(d_items[0]);
  dfree(d_items[1]);
  for (N3List& l : n3) {
    dfree(l.d_items);
    dfree(l.d_tiles);
    dfree(l.d_rea_off);
    dfree(l.d_rea);
  }
  dfree(d_act);
  dfree(d_head);
  dfree(d_red);
  *this = BatchState();
}

extern "C" {

int nbr_batch_upload(nbr_ctx* c, size_t nsys, const size_t* offsets, const double* x,
                     const double* y, const double* z, const double* vx, const double* vy,
                     const double* vz, const double* m) {
  TraceRange trace_range("nbr_batch_upload");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  if (nsys == 0 || !offsets || !x || !y || !z || !m)
    return fail(c, NBR_ERR_INVALID_ARG, "empty batch or NULL array");
  if ((vx || vy || vz) && !(vx && vy && vz))
    return fail(c, NBR_ERR_INVALID_ARG, "velocities must be all given or all NULL");
  if (offsets[0] != 0) return fail(c, NBR_ERR_INVALID_ARG, "offsets[0] must be 0");
  if (nsys >= (size_t)kN3Item) return fail(c, NBR_ERR_INVALID_ARG, "too many systems");
  for (size_t s = 0; s < nsys; ++s) {
    if (offsets[s + 1] <= offsets[s]) return fail(c, NBR_ERR_INVALID_ARG, "every system needs >= 1 particle");
    if (offsets[s + 1] - offsets[s] > (size_t)1 << 30) return fail(c, NBR_ERR_INVALID_ARG, "system too large");
  }
  const size_t n = offsets[nsys];
  if (!finite_array(x, n) || !finite_array(y, n) || !finite_array(z, n) || !finite_array(m, n) ||
      (vx && (!finite_array(vx, n) || !finite_array(vy, n) || !finite_array(vz, n))))
    return fail(c, NBR_ERR_NONFINITE, "input contains NaN or Inf");
  for (size_t i = 0; i < n; ++i)
    if (m[i] < 0.0) return fail(c, NBR_ERR_INVALID_ARG, "negative mass");
  cudaSetDevice(c->device);
  BatchState& b = c->bat;
  b.release();
  b.nsys = nsys;
  b.n_real = n;
  b.off.assign(offsets, offsets + nsys + 1);
  b.poff.assign(nsys + 1, 0);
  double pairs = 0.0;
  for (size_t s = 0; s < nsys; ++s) {
    const long long ns = (long long)(offsets[s + 1] - offsets[s]);
    b.poff[s + 1] = b.poff[s] + ((ns + kTile - 1) / kTile) * kTile;
    pairs += double(ns) * double(ns - 1);
  }
  b.pairs_per_eval = pairs;
  const size_t np = (size_t)b.poff[nsys];
  cudaError_t e = b.s.reserve(np);
  if (e != cudaSuccess) {
    b.release();  // no half-built batch is left behind
    return cuda_fail(c, e, "batch allocation");
  }
  // Host staging in the padded layout.
  std::vector<double> h(b.s.n_pad, 0.0);
  auto put = [&](double* d, const double* src) {
    if (e != cudaSuccess) return;
    std::fill(h.begin(), h.end(), 0.0);
    if (src)
      for (size_t s = 0; s < nsys; ++s)
        std::memcpy(&h[b.poff[s]], src + offsets[s], (offsets[s + 1] - offsets[s]) * sizeof(double));
    e = cudaMemcpyAsync(d, h.data(), b.s.n_pad * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // h is reused
  };
  put(b.s.pos[0][0], x); put(b.s.pos[0][1], y); put(b.s.pos[0][2], z);
  put(b.s.vel[0], vx); put(b.s.vel[1], vy); put(b.s.vel[2], vz);
  put(b.s.mass, m);
  for (int d = 0; d < 3 && e == cudaSuccess; ++d) {
    e = cudaMemsetAsync(b.s.pos[1][d], 0, b.s.n_pad * sizeof(double), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.s.acc[d], 0, b.s.n_pad * sizeof(double), c->stream);
  }
  if (e != cudaSuccess) {
    b.release();
    return cuda_fail(c, e, "batch upload");
  }
  // Work items ordered by cost (receiver slots x system size), largest first:
  // list 0 with one-tile items only, list 1 pairing a system's tiles into
  // two-tile items (a system's odd last tile stays a one-tile item); lists 2
  // (FP64) and 3 (FP32C) with Newton-3 row blocks of R = 1 or 2 tiles for the
  // systems of R + 1 tiles or more (cost: the own tiles' ordered pairs, and
  // each later tile's pairs at the rotation's ~1.5x the work per pair), and
  // list 0's (FP64) or list 1's (FP32C) items for the rest.
  std::vector<int2> lists[4];
  std::vector<int2> n3_tiles[2];
  std::vector<long long> rea_off[2] = {std::vector<long long>(nsys, -1),
                                       std::vector<long long>(nsys, -1)};
  long long slots[2] = {0, 0};
  for (int wl = 0; wl < 4; ++wl) {
    std::vector<int2> items;
    std::vector<double> cost;
    const int q = wl - 2;                 // Newton-3 list of precision index q
    const int rows = wl == 3 ? 2 : 1;     // tiles per row block
    const bool pairs = wl == 1 || wl == 3;  // two-tile items for the other systems
    for (size_t s = 0; s < nsys; ++s) {
      const long long ns = (long long)(offsets[s + 1] - offsets[s]);
      const long long nt = (ns + kTile - 1) / kTile;
      if (q >= 0 && nt >= rows + 1) {
        rea_off[q][s] = slots[q];
        for (long long blk = 0; rows * blk < nt; ++blk) {
          const long long own = std::min<long long>(rows, nt - rows * blk);
          const long long later = std::max<long long>(0, nt - rows * blk - rows);
          slots[q] += later;
          items.push_back(make_int2((int)s | kN3Item, (int)blk));
          cost.push_back(double(rows) * kTile * (double(own) + 1.5 * double(later)) * kTile);
        }
        for (long long t = 0; t < nt; ++t) n3_tiles[q].push_back(make_int2((int)s, (int)t));
        continue;
      }
      for (long long t = 0; t < nt;) {
        const int tile = (int)(b.poff[s] / kTile + t);
        if (pairs && t + 1 < nt) {
          items.push_back(make_int2((int)s | kWideItem, tile));
          cost.push_back(2.0 * kTile * double(ns));
          t += 2;
        } else {
          const long long r = std::min<long long>(kTile, ns - t * kTile);
          items.push_back(make_int2((int)s, tile));
          cost.push_back(double(r > 64 ? kTile : r > 32 ? 64 : r > 16 ? 32 : 16) * double(ns));
          t += 1;
        }
      }
    }
    std::vector<int> order(items.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int bb) { return cost[a] > cost[bb]; });
    lists[wl].resize(items.size());
    for (size_t k = 0; k < order.size(); ++k) lists[wl][k] = items[order[k]];
  }
  std::vector<int> nreal(nsys);
  b.max_ns = 0;
  for (size_t s = 0; s < nsys; ++s) {
    nreal[s] = (int)(offsets[s + 1] - offsets[s]);
    b.max_ns = std::max(b.max_ns, nreal[s]);
  }
  int2** dl[4] = {&b.d_items[0], &b.d_items[1], &b.n3[0].d_items, &b.n3[1].d_items};
  b.n_items[0] = (int)lists[0].size();
  b.n_items[1] = (int)lists[1].size();
  for (int q = 0; q < 2; ++q) {
    b.n3[q].n_items = (int)lists[2 + q].size();
    b.n3[q].n_tiles = (int)n3_tiles[q].size();
    b.n3[q].slots = slots[q];
  }
  e = dalloc((void**)&b.d_poff, (nsys + 1) * sizeof(long long));
  if (e == cudaSuccess) e = dalloc((void**)&b.d_nreal, nsys * sizeof(int));
  for (int wl = 0; wl < 4 && e == cudaSuccess; ++wl)
    e = dalloc((void**)dl[wl], lists[wl].size() * sizeof(int2));
  for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
    if (!n3_tiles[q].empty()) e = dalloc((void**)&b.n3[q].d_tiles, n3_tiles[q].size() * sizeof(int2));
    if (e == cudaSuccess) e = dalloc((void**)&b.n3[q].d_rea_off, nsys * sizeof(long long));
  }
  if (e == cudaSuccess) e = dalloc((void**)&b.d_head, 256);
  if (e == cudaSuccess) e = dalloc((void**)&b.d_red, nsys * 9 * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.d_poff, b.poff.data(), (nsys + 1) * sizeof(long long),
                        cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.d_nreal, nreal.data(), nsys * sizeof(int), cudaMemcpyHostToDevice, c->stream);
  for (int wl = 0; wl < 4 && e == cudaSuccess; ++wl)
    e = cudaMemcpyAsync(*dl[wl], lists[wl].data(), lists[wl].size() * sizeof(int2),
                        cudaMemcpyHostToDevice, c->stream);
  for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
    if (!n3_tiles[q].empty())
      e = cudaMemcpyAsync(b.n3[q].d_tiles, n3_tiles[q].data(), n3_tiles[q].size() * sizeof(int2),
                          cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b.n3[q].d_rea_off, rea_off[q].data(), nsys * sizeof(long long),
                          cudaMemcpyHostToDevice, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    b.release();
    return cuda_fail(c, e, "batch tables");
  }
  b.s.cur = 0;
  b.s.rec_ok[0] = b.s.rec_ok[1] = false;
  b.acc_ok = false;
  return NBR_OK;
}

int nbr_batch_download(nbr_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                       double* vz) {
  TraceRange trace_range("nbr_batch_download");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  BatchState& b = c->bat;
  if (b.nsys == 0) return fail(c, NBR_ERR_NO_SYSTEM, "no batch uploaded");
  cudaSetDevice(c->device);
  std::vector<double> h(b.s.n_pad);
  cudaError_t e = cudaSuccess;
  auto get = [&](double* dst, const double* d) {
    if (!dst || e != cudaSuccess) return;
    e = cudaMemcpyAsync(h.data(), d, b.s.n_pad * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return;
    for (size_t s = 0; s < b.nsys; ++s)
      std::memcpy(dst + b.off[s], &h[b.poff[s]], (b.off[s + 1] - b.off[s]) * sizeof(double));
  };
  const int a = b.s.cur;
  get(x, b.s.pos[a][0]); get(y, b.s.pos[a][1]); get(z, b.s.pos[a][2]);
  get(vx, b.s.vel[0]); get(vy, b.s.vel[1]); get(vz, b.s.vel[2]);
  return e == cudaSuccess ? NBR_OK : cuda_fail(c, e, "batch download");
}

int nbr_batch_forces(nbr_ctx* c, int precision, double G, double eps2, int want_force, double* ax,
                     double* ay, double* az) {
  TraceRange trace_range("nbr_batch_forces");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  if (precision != NBR_FP64 && precision != NBR_FP32C)
    return fail(c, NBR_ERR_INVALID_ARG, "unknown precision");
  if (!(eps2 >= 0.0) || !std::isfinite(eps2) || !std::isfinite(G))
    return fail(c, NBR_ERR_INVALID_ARG, "eps2 must be finite and >= 0, G finite");
  BatchState& b = c->bat;
  if (b.nsys == 0) return fail(c, NBR_ERR_NO_SYSTEM, "no batch uploaded");
  cudaSetDevice(c->device);
  int rc = batch_eval(c, precision, G, eps2, 0, 0.0, 0.0, nullptr);
  if (rc) return rc;
  rc = check_device_error(c);
  if (rc) return rc;
  b.acc_ok = true;
  b.acc_prec = precision;
  b.acc_G = G;
  b.acc_eps2 = eps2;
  std::vector<double> h(b.s.n_pad), mh;
  cudaError_t e = cudaSuccess;
  if (want_force) {
    mh.resize(b.s.n_pad);
    e = cudaMemcpyAsync(mh.data(), b.s.mass, b.s.n_pad * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  }
  auto get = [&](double* dst, const double* d) {
    if (!dst || e != cudaSuccess) return;
    e = cudaMemcpyAsync(h.data(), d, b.s.n_pad * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return;
    for (size_t s = 0; s < b.nsys; ++s)
      for (size_t k = 0; k < b.off[s + 1] - b.off[s]; ++k) {
        const size_t i = (size_t)b.poff[s] + k;
        dst[b.off[s] + k] = want_force ? h[i] * mh[i] : h[i];
      }
  };
  get(ax, b.s.acc[0]); get(ay, b.s.acc[1]); get(az, b.s.acc[2]);
  return e == cudaSuccess ? NBR_OK : cuda_fail(c, e, "batch forces download");
}

int nbr_batch_run(nbr_ctx* c, int precision, double dt, size_t steps, double G, double eps2,
                  nbr_run_stats* stats) {
  TraceRange trace_range("nbr_batch_run");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  if (precision != NBR_FP64 && precision != NBR_FP32C)
    return fail(c, NBR_ERR_INVALID_ARG, "unknown precision");
  if (!std::isfinite(dt) || !(eps2 >= 0.0) || !std::isfinite(eps2) || !std::isfinite(G))
    return fail(c, NBR_ERR_INVALID_ARG, "dt, G must be finite, eps2 finite and >= 0");
  BatchState& b = c->bat;
  if (b.nsys == 0) return fail(c, NBR_ERR_NO_SYSTEM, "no batch uploaded");
  cudaSetDevice(c->device);
  nbr_run_stats st{};
  if (steps > 0) {
    // Configure the kernel (shared-memory attribute, grid) before capture.
    batch_grid(c, precision, eps2);
    const bool fsal = b.acc_ok && b.acc_prec == precision && b.acc_G == G && b.acc_eps2 == eps2;
    SysState& s = b.s;
    const int cur0 = s.cur;
    const bool r0 = s.rec_ok[0], r1 = s.rec_ok[1];
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(c, e, "begin capture");
    int kernels = 0, rc = NBR_OK;
    double evals = 0;
    const bool fp32 = precision == kFP32C;
    if (fsal) {
      const int a = s.cur, o = 1 - s.cur;
      e = launch_kick_drift((long long)s.n, (long long)s.n_pad, s.pos[a][0], s.pos[a][1],
                            s.pos[a][2], s.mass, s.acc[0], s.acc[1], s.acc[2], 0.5 * dt, dt,
                            s.vel[0], s.vel[1], s.vel[2], s.pos[o][0], s.pos[o][1], s.pos[o][2],
                            fp32 ? s.rec[o] : nullptr, fp32 ? s.org[o] : nullptr, c->stream);
      ++kernels;
      if (e != cudaSuccess) rc = cuda_fail(c, e, "batch kick-drift");
      s.cur = o;
      s.rec_ok[o] = fp32;
      s.rec_ok[a] = false;
    } else {
      rc = batch_eval(c, precision, G, eps2, 1, 0.5 * dt, dt, &kernels);
      evals += 1;
    }
    for (size_t k = 1; k < steps && rc == NBR_OK; ++k) {
      rc = batch_eval(c, precision, G, eps2, 1, dt, dt, &kernels);
      evals += 1;
    }
    if (rc == NBR_OK) {
      rc = batch_eval(c, precision, G, eps2, 1, 0.5 * dt, 0.0, &kernels);
      evals += 1;
    }
    cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
    if (rc != NBR_OK || ee != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      s.cur = cur0;
      s.rec_ok[0] = r0;
      s.rec_ok[1] = r1;
      return rc != NBR_OK ? rc : cuda_fail(c, ee, "end capture");
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      s.cur = cur0;
      s.rec_ok[0] = r0;
      s.rec_ok[1] = r1;
      return cuda_fail(c, e, "graph instantiate");
    }
    e = cudaEventRecord(c->ev0, c->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(exec);
    if (e != cudaSuccess) {
      b.acc_ok = false;
      return cuda_fail(c, e, "graph launch");
    }
    rc = check_device_error(c);
    if (rc) {
      b.acc_ok = false;
      return rc;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    st.gpu_ms = ms;
    st.kernels = kernels;
    st.force_evals = evals;
    st.pairs = evals * b.pairs_per_eval;
    b.acc_ok = true;
    b.acc_prec = precision;
    b.acc_G = G;
    b.acc_eps2 = eps2;
  }
  if (stats) *stats = st;
  return NBR_OK;
}

int nbr_batch_set_config(nbr_ctx* c, int precision, int wide, int ctas_per_sm) {
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  if (precision != NBR_FP64 && precision != NBR_FP32C)
    return fail(c, NBR_ERR_INVALID_ARG, "unknown precision");
  if (wide < -1 || wide > 2 || ctas_per_sm < 0)
    return fail(c, NBR_ERR_INVALID_ARG, "wide must be -1, 0, 1 or 2 and ctas_per_sm >= 0");
  BatchState& b = c->bat;
  const int pi = precision == kFP32C ? 1 : 0;
  if (wide < 0) {
    b.cfg_ok[pi] = false;  // back to the autotune cache or the default
    return NBR_OK;
  }
  b.wide[pi] = wide;
  b.per_sm[pi] = ctas_per_sm;
  b.cfg_ok[pi] = true;
  return NBR_OK;
}

int nbr_batch_autotune(nbr_ctx* c, int precision, double eps2) {
  TraceRange trace_range("nbr_batch_autotune");
  if (!c) return fail(nullptr, NBR_ERR_INVALID_ARG, "ctx is NULL");
  if (precision != NBR_FP64 && precision != NBR_FP32C)
    return fail(c, NBR_ERR_INVALID_ARG, "unknown precision");
  if (!(eps2 >= 0.0) || !std::isfinite(eps2)) return fail(c, NBR_ERR_INVALID_ARG, "bad eps2");
  BatchState& b = c->bat;
  if (b.nsys == 0) return fail(c, NBR_ERR_NO_SYSTEM, "no batch uploaded");
  cudaSetDevice(c->device);
  const int pi = precision == kFP32C ? 1 : 0;
  int best_w = -1, best_p = 0;
  float best_ms = 1e30f;
  for (int w = 0; w < 3; ++w) {
    b.wide[pi] = w;
    b.per_sm[pi] = 0;
    b.cfg_ok[pi] = true;
    if (batch_grid(c, precision, eps2) == 0) continue;
    const int occ = b.occ[pi][eps2 == 0.0 ? 1 : 0][w];
    for (int per = 1; per <= occ; ++per) {
      b.per_sm[pi] = per;
      float tot = 0.f;
      bool ok = true;
      for (int rep = 0; rep < 3 && ok; ++rep) {
        cudaEventRecord(c->ev0, c->stream);
        ok = batch_eval(c, precision, 1.0, eps2, 0, 0.0, 0.0, nullptr) == NBR_OK;
        cudaEventRecord(c->ev1, c->stream);
        ok = ok && check_device_error(c) == NBR_OK;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        if (rep > 0) tot += ms;  // the first repetition warms up
      }
      if (ok && tot < best_ms) {
        best_ms = tot;
        best_w = w;
        best_p = per;
      }
    }
  }
  b.acc_ok = false;
  if (best_w < 0) {
    b.cfg_ok[pi] = false;
    return fail(c, NBR_ERR_CUDA, "no batch configuration ran");
  }
  b.wide[pi] = best_w;
  b.per_sm[pi] = best_p;
  b.cfg_ok[pi] = true;
  tune_put(batch_key(precision, b.nsys, b.max_ns, eps2 == 0.0),
           ForceConfig{best_w == 2 ? 3 : best_w ? 8 : 4, kBWarps, best_p});
  return NBR_OK;
}

int nbr_batch_diagnostics(nbr_ctx* c, double G, double eps2, nbr_diag* out) {
  TraceRange trace_range("nbr_batch_diagnostics");
  if (!c || !out) return fail(c, NBR_ERR_INVALID_ARG, "NULL argument");
  if (!(eps2 >= 0.0) || !std::isfinite(eps2)) return fail(c, NBR_ERR_INVALID_ARG, "bad eps2");
  BatchState& b = c->bat;
  if (b.nsys == 0) return fail(c, NBR_ERR_NO_SYSTEM, "no batch uploaded");
  cudaSetDevice(c->device);
  const int a = b.s.cur;
  k_batch_diag<<<(unsigned)b.nsys, 256, 0, c->stream>>>(
      b.s.pos[a][0], b.s.pos[a][1], b.s.pos[a][2], b.s.vel[0], b.s.vel[1], b.s.vel[2], b.s.mass,
      b.d_poff, b.d_nreal, G, eps2, b.d_red);
  cudaError_t e = cudaGetLastError();
  std::vector<double> h(b.nsys * 9);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.data(), b.d_red, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "batch diagnostics");
  for (size_t s = 0; s < b.nsys; ++s) {
    const double* r = &h[s * 9];
    out[s].T = r[0];
    out[s].P[0] = r[1]; out[s].P[1] = r[2]; out[s].P[2] = r[3];
    out[s].L[0] = r[4]; out[s].L[1] = r[5]; out[s].L[2] = r[6];
    out[s].M = r[7];
    out[s].U = r[8];
    out[s].E = r[0] + r[8];
  }
  return NBR_OK;
}

}  // extern "C"
