// nbr_ctx.h -- internal definition of nbr_ctx and its device state.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "nbr.h"
#include "nbr_kernels.cuh"

namespace nbr {

// Device state of one particle system (or of a batch of systems stored back to
// back).  Positions are double-buffered: a force evaluation reads buffer
// `cur` and its fused kick/drift epilogue writes buffer 1 - cur.  Every array
// holds n_pad entries (per-particle arrays kRangeSlack more); entries >= n are
// zero-mass padding at the origin.
// Zeroed entries allocated past n_pad in every per-particle array (see
// SysState::reserve).
constexpr size_t kRangeSlack = 1024;

struct SysState {
  size_t n = 0, n_pad = 0, cap = 0;
  int ntiles = 0;
  double* pos[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  double* vel[3] = {nullptr, nullptr, nullptr};
  double* acc[3] = {nullptr, nullptr, nullptr};
  double* mass = nullptr;
  float4* rec[2] = {nullptr, nullptr};     // FP32C source records of each buffer
  double4* org[2] = {nullptr, nullptr};    // FP64 tile origins of each buffer
  int cur = 0;
  bool rec_ok[2] = {false, false};

  cudaError_t reserve(size_t n);
  cudaError_t clear_padding(cudaStream_t st);
  void release();
};

// Scratch reused across calls: split partial sums, split arrival counters,
// diagnostic partial sums.
struct Scratch {
  double* part = nullptr;
  size_t part_cap = 0;
  unsigned* cnt = nullptr;
  size_t cnt_cap = 0;
  double* red = nullptr;
  size_t red_cap = 0;

  cudaError_t need_part(size_t doubles);
  cudaError_t need_counters(size_t count);
  cudaError_t need_red(size_t doubles);
  void release();
};

// Batched independent systems (nbr_batch_*).  Each system is padded to whole
// tiles, so a tile never mixes systems.
struct BatchState {
  SysState s;                        // all systems' particles (padded layout)
  size_t nsys = 0;
  size_t n_real = 0;                 // sum of the real sizes
  std::vector<size_t> off;           // real offsets (host), nsys + 1
  std::vector<long long> poff;       // padded offsets (host), nsys + 1
  long long* d_poff = nullptr;       // padded offsets (device), nsys + 1
  int* d_nreal = nullptr;            // real size of each system (device)
  int* d_sys_of_tile = nullptr;      // system index of every padded tile
  // Work queues of (system | kWideItem flag, first receiver tile), cost
  // ordered: [0] one-tile items only, [1] two-tile items where a system has
  // two tiles left.
  int2* d_items[2] = {nullptr, nullptr};
  int n_items[2] = {0, 0};
  // Newton-3 work per precision ([0] FP64: one-tile row blocks of the systems
  // of two tiles or more, the others' items as in list 0; [1] FP32C: two-tile
  // row blocks of the systems of three tiles or more, the others' items as in
  // list 1): the queue of (system | kN3Item, row block) and other items, the
  // Newton-3 systems' tiles (system, local tile) for the epilogue kernel, each
  // system's first reaction slot (-1: none), the slot count, and the slots
  // [slots][3][128] (allocated at first use).
  struct N3List {
    int2* d_items = nullptr;
    int n_items = 0;
    int2* d_tiles = nullptr;
    int n_tiles = 0;
    long long* d_rea_off = nullptr;
    long long slots = 0;
    double* d_rea = nullptr;
  };
  N3List n3[2];
  double* d_act = nullptr;           // Newton-3 action sums [3][n_pad] (at first use)
  int max_ns = 0;                    // largest system
  unsigned* d_head = nullptr;        // work-queue heads
  double* d_red = nullptr;           // per-system diagnostic sums
  bool acc_ok = false;
  int acc_prec = 0;
  double acc_G = 0.0, acc_eps2 = 0.0;
  double pairs_per_eval = 0.0;
  // Kernel configuration per precision: wide items, resident CTAs per SM
  // (0: the occupancy limit); chosen from the autotune cache or the default
  // at first use.
  bool cfg_ok[2] = {false, false};
  int wide[2] = {1, 1};
  int per_sm[2] = {0, 0};
  int occ[2][2][3] = {};              // occupancy limit per (precision, eps == 0, wide)

  void release();
};

// An NVTX range around a public call (visible to Nsight tools; a no-op when
// none is attached).
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

// Autotune cache (a JSON file shared by the processes on a host).
bool tune_get(const std::string& key, ForceConfig* out);
void tune_put(const std::string& key, const ForceConfig& cfg);

int fail(nbr_ctx* c, int code, const std::string& msg);
int cuda_fail(nbr_ctx* c, cudaError_t e, const char* where);
cudaError_t dalloc(void** p, size_t bytes);
void dfree(void* p);
bool finite_array(const double* a, size_t n);
int check_device_error(nbr_ctx* c);
// Bounded-wait limit and tile-skip test hook from the environment.
void pipeline_params(JStream& js);
// The persistent small-system run (nbr_persist.cu): whether it serves an
// nbr_run of this system, and the run itself (the schedule of nbr_run's
// launch sequence; cc/dd/lf the Yoshida tables for DKD).
bool persistent_run_applies(nbr_ctx* c, int precision, size_t n);
int run_persistent(nbr_ctx* c, int precision, int scheme, double dt, size_t steps, double G,
                   double eps2, bool fsal, const double* cc, const double* dd, int lf,
                   nbr_run_stats* st);

}  // namespace nbr

namespace nbr {
// Identity of a captured nbr_run launch sequence: the call's arguments, the
// host-side state it starts from and every device address it bakes in.
struct RunKey {
  int precision = -1, scheme = -1, order = 0;
  double dt = 0.0, G = 0.0, eps2 = 0.0;
  size_t steps = 0, n = 0, cap = 0;
  bool fsal = false;
  int cur = 0;
  bool rec_ok[2] = {false, false};
  ForceConfig cfg{0, 0, 0};
  unsigned long long wait_ns = 0;
  int skip_tile = -1;
  const void* ptr[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool operator==(const RunKey& o) const;
};
// The last nbr_run graph, replayed while the key matches.
struct RunGraph {
  cudaGraphExec_t exec = nullptr;
  RunKey key;
  int cur_after = 0;
  bool rec_after[2] = {false, false};
  int kernels = 0;
  double evals = 0.0;
  void release();
};
}  // namespace nbr

struct nbr_ctx {
  int device = 0;
  int sms = 148;
  bool coop = false;       // the device supports cooperative launches
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  nbr::SysState sys;       // the uploaded system
  nbr::SysState ij;        // scratch for nbr_accel_ij
  nbr::Scratch scr;
  nbr::BatchState bat;
  int* d_err = nullptr;    // device error word (nbr::kErr*)
  // First-same-as-last: sys.acc holds G-scaled accelerations of the current
  // positions for (acc_prec, acc_G, acc_eps2).
  bool acc_ok = false;
  int acc_prec = 0;
  double acc_G = 0.0, acc_eps2 = 0.0;
  nbr::ForceConfig override_cfg[2] = {{0, 0, 0}, {0, 0, 0}};
  nbr::RunGraph run_graph;
  // Launch order of the whole-system Newton-3 grid (longest CTA first) for
  // n3_order_nb blocks, then its inverse; written before any graph capture
  // (n3_order_prepare, the only writer), read by the pair and reduce kernels.
  int* n3_order = nullptr;
  long long n3_order_cap = 0;    // ints allocated
  long long n3_order_nb = -1;    // blocks the table holds the order of
};
