// nbr_kernels.cuh -- launch parameters shared by the kernels and the host.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

namespace nbr {

enum Precision : int { kFP64 = 0, kFP32C = 1 };

// Fields that only checked builds carry: the allocated lengths the kernels
// test their indices against (see NBR_IN in nbr_device.cuh).
#ifdef NBR_CHECKED
#define NBR_CHECKED_FIELD(decl) decl;
#define NBR_CHECKED_ONLY(stmt) stmt
#else
#define NBR_CHECKED_FIELD(decl)
#define NBR_CHECKED_ONLY(stmt)
#endif

// Receivers ("i" particles): FP64 positions, read-only during the launch.
// Arrays are allocated to a multiple of 1024 entries.
struct IParticles {
  const double* x;
  const double* y;
  const double* z;
  const double* m;  // receiver masses (used for force output and the pack)
  long long n;      // real receivers; entries >= n are padding
  NBR_CHECKED_FIELD(long long len)  // entries allocated from x, y, z, m on
};

// Sources ("j" particles), streamed tile by tile.  FP64 form: SoA arrays padded
// with zero-mass particles to ntiles * kTile.  FP32C form: the pair-duplicated
// records (3 x 16 B per particle) plus one FP64 origin per tile.
struct JStream {
  const double* x;
  const double* y;
  const double* z;
  const double* m;
  const float4* rec;
  const double4* origin;
  int ntiles;
  unsigned long long wait_ns;  // limit of one bounded tile wait
  int skip_tile;               // test hook: this CTA-local tile is never copied (-1: off)
  NBR_CHECKED_FIELD(long long len)  // source entries allocated (x..m; rec 3 len, origin len / kTile)
};

// What happens to each receiver's summed acceleration.
struct Epilogue {
  int mode;            // 0: write a (or m a);  1: leapfrog kick then drift;
                       // 2: Euler (drift with the old velocity, then kick)
  double G;
  double* ax; double* ay; double* az;   // acceleration (or force) out
  int want_force;      // mode 0: multiply by the receiver mass
  // mode 1: v += kick * a;  x' = x + drift * v  (x' into the other buffer)
  double kick, drift;
  double* vx; double* vy; double* vz;
  double* xn; double* yn; double* zn;
  float4* rec_next;    // FP32C records for x' (nullptr: not needed)
  double4* origin_next;
  // split-j reduction
  double* part;        // [split][3][n_pad]
  unsigned* counters;  // one per CTA chunk, zero between launches
  long long n_pad;
  int* err;            // device error word
  NBR_CHECKED_FIELD(long long part_len)  // doubles allocated in part
  NBR_CHECKED_FIELD(long long cnt_len)   // counters allocated
  NBR_CHECKED_FIELD(long long rec_len)   // particles allocated in rec_next
};

struct ForceConfig {
  int ni;      // receivers per thread (4 or 8); 1 selects the small-N kernel
  int warps;   // warps per CTA (2, 4 or 8); for the small-N kernel: lane groups F (2, 4, 8)
  int split;   // j-range splits (>= 1)
  // Large kernels only (ni 4 / 8): sources per stage of the tile ring (the
  // j-tile: 64, 128 or 256) and the unroll depth of the source loop (2, 4 or
  // 8); 0 takes the default (128; unroll 4 for FP32C, 2 for FP64).  Other
  // values than the defaults exist for the default large configurations,
  // FP32C (8, 2) and FP64 (4, 4).
  int tile = 0;
  int unroll = 0;
};
// Default j-tile and unroll depth of the large kernels.
constexpr int kDefaultTileJ = 128;
inline int default_unroll(int precision) { return precision == kFP32C ? 4 : 2; }

// The small-N kernel: kSmallWarps warps per CTA, kSmallNI receivers per lane,
// F lane groups per warp sharing each tile's sources: 128 * kSmallNI / F
// receivers per CTA.
constexpr int kSmallWarps = 4;
constexpr int kSmallNI = 4;
// The Newton-3 kernels (ForceConfig ni = 3, FP32C and FP64): blocks of kN3Block
// particles, kN3Warps row blocks per CTA (one per warp), up to `cols` column
// blocks per CTA (n3_cols, n3_slice_cols: at most kN3MaxCols).
constexpr int kN3Warps = 8;
constexpr int kN3F64Warps = 2 * kN3Warps;  // FP64: two warps per row block
constexpr int kN3Block = 256;
constexpr int kN3MaxCols = 32;
struct N3Params {
  long long nb;  // blocks holding real particles: ceil(n / kN3Block)
  int cols;      // column blocks per CTA
  int g0, g1;    // row groups [g0, g1) of this launch (all: 0, ceil(nb / kN3Warps))
  double* act;   // action partials [cta][row block][3][kN3Block]
  double* rea;   // reaction partials [cta][column block][3][kN3Block]
  // Launch order of a whole-system launch: CTA blockIdx.x does (row group,
  // chunk) number order[blockIdx.x] of the group-major numbering and writes
  // its partial sums at index blockIdx.x; slot[] is the inverse (group-major
  // number -> partial-sum index) for the reduction.  nullptr: identity.
  const int* order;
  const int* slot;
  NBR_CHECKED_FIELD(long long act_len)  // doubles from act (through rea's end)
  NBR_CHECKED_FIELD(long long dst_len)  // doubles of a slice reduction's destination
};
// The Newton-3 partial sums grow as N^2 (8.4 GB at 2^20 particles).  Up to
// kN3SingleMaxDoubles one launch covers the system; above it the evaluation
// runs in row-group slices of at most kN3SliceMaxDoubles each, whose partial
// accelerations accumulate in slice order in an FP64 buffer (3 x 8 B per
// particle), so the scratch stays bounded at any N.
constexpr long long kN3SingleMaxDoubles = 9LL << 27;  // 9 GiB
constexpr long long kN3SliceMaxDoubles = 1LL << 28;   // 2 GiB
// Largest system the Newton-3 kernel is the default for.
constexpr long long kN3MaxN = 1LL << 23;
// Smallest system the default configuration gives the Newton-3 kernel.
constexpr long long kN3MinN = 16384;
// Column chunks (CTAs) of row group g.
__host__ __device__ inline int n3_chunks(long long nb, int cols, int g) {
  const long long left = nb - (long long)g * kN3Warps;
  return left <= 0 ? 0 : (int)((left + cols - 1) / cols);
}
// Column blocks per CTA (1 .. kN3MaxCols) for nb blocks on the current
// device: the width whose grid a model of the launch finishes first (see
// nbr_kernels.cu).  Memoized per (nb, SM count); a host function.
int n3_cols(long long nb);
// The model's cost of every CTA of the Newton-3 grid for nb blocks in chunks
// of `cols` (group-major order), in units of one column block's pair work.
void n3_cta_costs(long long nb, int cols, std::vector<double>& cost);
// The model's finishing time of that grid launched longest CTA first (ties in
// group-major order) on `sms` SMs, one CTA each at a time.
double n3_makespan(long long nb, int cols, int sms);
// That launch order: order[launch index] = group-major CTA index.
void n3_launch_order(long long nb, int cols, std::vector<int>& order);
// The model's efficiency of the whole-system Newton-3 grid for nb blocks on
// the current device: the pair work spread evenly over the SMs divided by the
// grid's finishing time (1 at best).  A host function.
double n3_grid_efficiency(long long nb);
// n3_cols, n3_slice_cols and n3_grid_efficiency for a device of `sms` SMs
// (host functions; no device needed).
int n3_cols_for(long long nb, int sms);
int n3_slice_cols_for(long long nb, int V, int sms);
double n3_grid_efficiency_for(long long nb, int sms);
// Column blocks per CTA of the row-group slices of V (the multi-GPU partition
// and the banded evaluation): the width whose slices the model finishes with
// the best worst-case efficiency when W = 2, 4, 8 or V ranks (those <= V)
// each launch their consecutive share of the slices (group-major order).
// The same for every world size of one V, so the sums stay bit-identical
// across world sizes.  Memoized per (nb, V, SM count); a host function.
int n3_slice_cols(long long nb, int V);
// CTAs of a Newton-3 launch and the doubles its partial sums need.
inline long long n3_ctas(long long nb, int cols) {
  long long t = 0;
  for (int g = 0; (long long)g * kN3Warps < nb; ++g) t += n3_chunks(nb, cols, g);
  return t;
}
inline long long n3_scratch_doubles(long long nb) {
  const int cols = n3_cols(nb);
  return n3_ctas(nb, cols) * (long long)(kN3Warps + cols) * 3 * kN3Block;
}
// CTAs of the row groups [g0, g1).
inline long long n3_ctas_range(long long nb, int cols, int g0, int g1) {
  long long t = 0;
  for (int g = g0; g < g1; ++g) t += n3_chunks(nb, cols, g);
  return t;
}
// Row groups [g0, g1) of slice v of V: consecutive groups with about the same
// number of CTAs (the same pair work) in each slice; slices may be empty.
inline void n3_slice_groups(long long nb, int cols, int v, int V, int* g0, int* g1) {
  const int groups = (int)((nb + kN3Warps - 1) / kN3Warps);
  const long long total = n3_ctas(nb, cols);
  auto start = [&](int s) {
    if (s <= 0) return 0;
    if (s >= V) return groups;
    const long long target = (total * s + V - 1) / V;  // first CTA of slice s
    long long acc = 0;
    int g = 0;
    while (g < groups && acc < target) acc += n3_chunks(nb, cols, g++);
    return g;
  };
  *g0 = start(v);
  *g1 = start(v + 1);
}
// Doubles of partial-sum scratch of slices [v0, v1) of V (one launch).
inline long long n3_slices_scratch_doubles(long long nb, int v0, int v1, int V) {
  const int cols = n3_slice_cols(nb, V);
  int g0 = 0, g1 = 0, g = 0;
  n3_slice_groups(nb, cols, v0, V, &g0, &g);
  n3_slice_groups(nb, cols, v1 - 1, V, &g, &g1);
  return n3_ctas_range(nb, cols, g0, g1) * (long long)(kN3Warps + cols) * 3 * kN3Block;
}
inline long long n3_slice_scratch_doubles(long long nb, int v, int V) {
  return n3_slices_scratch_doubles(nb, v, v + 1, V);
}
// One Newton-3 force evaluation over all n_pad receivers of ip against the
// same particles in js (FP32C: their records; FP64: their x, y, z, m arrays),
// with the epilogue ep: the pair kernel, then the per-particle reduction.
// scratch holds n3_scratch_doubles(ceil(n / kN3Block)) doubles; order is the
// grid's launch order (n3_launch_order, on the device).
// FP32C: warps = kN3Warps (one warp per row block) or kN3F64Warps (two).
cudaError_t launch_force_n3(int precision, int warps, double eps2, const IParticles& ip,
                            const JStream& js, const Epilogue& ep, double* scratch,
                            long long scratch_len, const int* order, cudaStream_t stream);
// Newton-3 partial accelerations (not G-scaled) of every particle from the
// pairs of slice `slice` of `nslices` (n3_slice_groups): stored into dst[d *
// ld + i] (i < n rounded up to 256), or added to it (accumulate); scratch
// holds n3_slice_scratch_doubles doubles.
cudaError_t launch_n3_slice(int precision, int warps, double eps2, const IParticles& ip,
                            const JStream& js, int* err, int slice, int nslices, double* scratch,
                            long long scratch_len, double* dst, long long ld, long long dst_len,
                            bool accumulate, cudaStream_t stream);
// Slices [v0, v1) in one pair launch (the same partial sums as one launch per
// slice): slice v's partials into dst + (v - v0) 3 ld; scratch holds
// n3_slices_scratch_doubles doubles.
cudaError_t launch_n3_slices(int precision, int warps, double eps2, const IParticles& ip,
                             const JStream& js, int* err, int v0, int v1, int nslices,
                             double* scratch, long long scratch_len, double* dst, long long ld,
                             long long dst_len, bool accumulate, cudaStream_t stream);
// The epilogue of the large kernels on the receivers ip, from V partial
// accelerations per particle summed in slice order: src[v * vstride + d * ld + i].
cudaError_t launch_sum_finish(const IParticles& ip, const Epilogue& ep, const double* src, int V,
                              long long vstride, long long ld, long long src_len,
                              cudaStream_t stream);
// Kernel attributes that must be set once per device, outside stream capture.
cudaError_t configure_kernels();

// The persistent small-system run (nbr_persist.cu): the whole nbr_run step
// loop of a system of at most kPersistMaxN particles (FP64 or FP32C) in one
// cooperative launch.  ForceConfig ni = kPersistNI with warps = lane groups (4, 8, 16)
// forces it; it is the default for such systems.
// ForceConfig split = warps per CTA of that launch (8 or 16; 0: default).
constexpr int kPersistNI = 2;
constexpr long long kPersistMaxN = 4096;
constexpr int kPersistDefaultWarps = 16;

// Receivers one CTA of a configuration covers.
inline long long force_chunk(const ForceConfig& c) {
  return c.ni == 1 ? 32LL * kSmallWarps * kSmallNI / (c.warps > 0 ? c.warps : 1)
                   : 32LL * c.ni * c.warps;
}

// Host-side launchers (nbr_kernels.cu).
cudaError_t launch_force(int precision, double eps2, const ForceConfig& cfg, const IParticles& ip,
                         const JStream& js, const Epilogue& ep, cudaStream_t stream);
// v += kick a; x' = x + drift v (x' may alias nothing; pass xn = x to pack in place
// with drift = 0); writes FP32C records of x' when rec_next != nullptr.
cudaError_t launch_kick_drift(long long n, long long n_pad, const double* x, const double* y,
                              const double* z, const double* m, const double* ax,
                              const double* ay, const double* az, double kick, double drift,
                              double* vx, double* vy, double* vz, double* xn, double* yn,
                              double* zn, float4* rec_next, double4* origin_next,
                              cudaStream_t stream);
// Outputs of a potential launch.
struct PotentialOut {
  double G;
  double* phi;         // phi_i (nullptr: not written)
  double* blocksum;    // per receiver chunk: sum of 1/2 m_i phi_i
  double* part;        // [split][n_pad] split partials
  unsigned* counters;  // one per receiver chunk, zero between launches
  long long n_pad;
  int* err;            // device error word
  NBR_CHECKED_FIELD(long long part_len)
  NBR_CHECKED_FIELD(long long cnt_len)
  NBR_CHECKED_FIELD(long long blocksum_len)
};
// Receivers per thread and warps per CTA of the potential kernel; a receiver
// chunk (one blocksum entry) is 32 * kPotNI * kPotWarps particles.
constexpr int kPotNI = 4, kPotWarps = 4;
// phi_i = -G sum_{j != i} m_j / sqrt(r^2 + eps2) in FP64 over receivers ip
// against the FP64 source stream js (x, y, z, m; the receivers themselves).
cudaError_t launch_potential(int split, const IParticles& ip, const JStream& js,
                             const PotentialOut& po, double eps2, cudaStream_t stream);
// Per-block partial sums of T, P, L, M (FP64): 8 values per block into part.
cudaError_t launch_moments(long long n, long long n_pad, const double* x, const double* y,
                           const double* z, const double* vx, const double* vy, const double* vz,
                           const double* m, double* part, cudaStream_t stream);
// Sums nblocks rows of `width` doubles in block order (deterministic).
cudaError_t launch_rowsum(const double* part, int nblocks, int width, double* out,
                          cudaStream_t stream);
// Sets bit 0 of *flags if any x, y, z, (vx, vy, vz,) m entry is NaN or Inf,
// bit 1 if a mass is negative (vx may be null: no velocities).
cudaError_t launch_validate(long long n, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz,
                            const double* m, int* flags, int sms, cudaStream_t stream);
size_t force_smem_bytes(int precision, const ForceConfig& cfg);
// Resident CTAs per SM of the force kernel for this configuration (0 on error).
int force_blocks_per_sm(int precision, double eps2, const ForceConfig& cfg);
bool force_config_supported(int precision, const ForceConfig& cfg);

}  // namespace nbr
