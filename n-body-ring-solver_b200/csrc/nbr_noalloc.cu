// nbr_noalloc.cu -- a force evaluation that allocates nothing.
//
// nbr_forces_noalloc runs the split-j force kernel of nbr_forces with all of
// its scratch memory (padded copies of the inputs, the FP32C source records
// and tile origins, the per-split partial sums, the split arrival counters
// and the error word) in one file-scope device array, so a call makes no
// cudaMalloc, cudaFree or other allocating call.  It is for callers that
// cannot let a library allocate device memory: a host application whose
// memory pool owns every device allocation and forbids foreign cudaMalloc
// calls, a process running under a fixed device-memory budget, or a
// latency-critical loop that cannot afford the device-wide synchronisation
// cudaMalloc and cudaFree can imply.  The caller still provides the inputs and
// the outputs.
//
// The array (kScratchBytes, about 8.5 MB) is part of the library image: every
// GPU that loads the library holds it until the process exits.  Every call on
// a device shares it and it keeps the last call's contents; what must start
// at zero (padding, counters, error word) is cleared by each call.  Calls that
// overlap on the same GPU (several streams or host threads) race on it and
// must be serialised by the caller.
#include "nbr.h"
#include "nbr_ctx.h"
#include "nbr_device.cuh"
#include "nbr_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

using namespace nbr;

namespace {

constexpr long long kMaxN = NBR_NOALLOC_MAX_N;
constexpr int kMaxSplit = 8;
constexpr int kMaxDevices = 64;
constexpr size_t kArr = size_t(kMaxN) * sizeof(double);
constexpr size_t kOffX = 0;
constexpr size_t kOffY = kOffX + kArr;
constexpr size_t kOffZ = kOffY + kArr;
constexpr size_t kOffM = kOffZ + kArr;
constexpr size_t kOffPart = kOffM + kArr;                        // [kMaxSplit][3][n_pad] doubles
constexpr size_t kOffRec = kOffPart + size_t(kMaxSplit) * 3 * kArr;  // 3 float4 per particle
constexpr size_t kOffOrg = kOffRec + size_t(kMaxN) * 3 * sizeof(float4);
constexpr size_t kOffCnt = kOffOrg + size_t(kMaxN / kTile) * sizeof(double4);
constexpr size_t kCounters = 1024;
constexpr size_t kOffErr = kOffCnt + kCounters * sizeof(unsigned);
constexpr size_t kScratchBytes = kOffErr + 256;
static_assert(kMaxN % 1024 == 0, "the limit must be a whole number of padding blocks");
static_assert(kOffRec % 256 == 0 && kOffOrg % 256 == 0 && kOffCnt % 256 == 0 && kOffErr % 256 == 0,
              "scratch regions stay 256-byte aligned");

// The scratch.  In host code this name is a host-side stand-in, not a device
// address: host code only uses the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (with that device current) on its first call and kept for the life
// of the process.  A cudaDeviceReset on that device unloads the module and
// invalidates the kept address, so a caller must not use this entry point on
// a device after resetting it.
int scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_scratch_addr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[device];
  return NBR_OK;
}

}  // namespace

extern "C" int nbr_forces_noalloc(int precision, size_t n, const double* x, const double* y,
                                  const double* z, const double* m, double G, double eps2,
                                  double* ax, double* ay, double* az, void* stream) {
  TraceRange trace_range("nbr_forces_noalloc");
  if (precision != NBR_FP64 && precision != NBR_FP32C)
    return fail(nullptr, NBR_ERR_INVALID_ARG, "unknown precision");
  if (n > size_t(kMaxN))
    return fail(nullptr, NBR_ERR_INVALID_ARG,
                "n = " + std::to_string(n) + " is above the no-allocation limit of " +
                    std::to_string(kMaxN) + " particles (NBR_NOALLOC_MAX_N)");
  if (n == 0) return NBR_OK;
  if (!x || !y || !z || !m || !ax || !ay || !az)
    return fail(nullptr, NBR_ERR_INVALID_ARG, "NULL array");
  if (!(eps2 >= 0.0) || !std::isfinite(eps2) || !std::isfinite(G))
    return fail(nullptr, NBR_ERR_INVALID_ARG, "eps2 must be finite and >= 0, G finite");
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDevice");
  if (device < 0 || device >= kMaxDevices)
    return fail(nullptr, NBR_ERR_UNSUPPORTED, "device index above 63");
  unsigned char* base = nullptr;
  int rc = scratch_address(device, &base);
  if (rc) return rc;
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaDeviceGetAttribute(SM count)");

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long nn = (long long)n;
  const long long n_pad = ((nn + 1023) / 1024) * 1024;
  const int ntiles = (int)((nn + kTile - 1) / kTile);
  double* X = reinterpret_cast<double*>(base + kOffX);
  double* Y = reinterpret_cast<double*>(base + kOffY);
  double* Z = reinterpret_cast<double*>(base + kOffZ);
  double* M = reinterpret_cast<double*>(base + kOffM);
  double* part = reinterpret_cast<double*>(base + kOffPart);
  float4* rec = reinterpret_cast<float4*>(base + kOffRec);
  double4* org = reinterpret_cast<double4*>(base + kOffOrg);
  unsigned* cnt = reinterpret_cast<unsigned*>(base + kOffCnt);
  int* err = reinterpret_cast<int*>(base + kOffErr);

  // Padded copies of the inputs (the tile ring reads whole 128-particle tiles),
  // padding zeroed, counters and error word cleared.
  const size_t B = n * sizeof(double), P = size_t(n_pad - nn) * sizeof(double);
  const double* src[4] = {x, y, z, m};
  double* dst[4] = {X, Y, Z, M};
  for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
    e = cudaMemcpyAsync(dst[k], src[k], B, cudaMemcpyDefault, st);
    if (e == cudaSuccess && P) e = cudaMemsetAsync(dst[k] + n, 0, P, st);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, kCounters * sizeof(unsigned), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "no-allocation staging");

  if (precision == NBR_FP32C) {
    e = launch_kick_drift(nn, n_pad, X, Y, Z, M, nullptr, nullptr, nullptr, 0.0, 0.0, nullptr,
                          nullptr, nullptr, nullptr, nullptr, nullptr, rec, org, st);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "no-allocation pack");
  }
  ForceConfig cfg = precision == NBR_FP32C ? ForceConfig{8, 2, 1} : ForceConfig{4, 4, 1};
  const long long chunk = 32LL * cfg.ni * cfg.warps;
  const long long chunks = (nn + chunk - 1) / chunk;
  const long long want = (16LL * sms + chunks - 1) / chunks;  // ~8 waves of 2 CTAs per SM
  cfg.split = (int)std::max<long long>(1, std::min<long long>({want, (long long)kMaxSplit,
                                                               (long long)ntiles}));
  IParticles ip{X, Y, Z, M, nn};
  JStream js{X, Y, Z, M, rec, org, ntiles, kWaitLimitNs, -1};
  pipeline_params(js);  // NBR_WAIT_LIMIT_MS, and the NBR_TEST_SKIP_TILE test hook
  Epilogue ep{};
  ep.mode = 0;
  ep.G = G;
  ep.ax = ax; ep.ay = ay; ep.az = az;
  ep.want_force = 0;
  ep.part = part;
  ep.counters = cnt;
  ep.n_pad = n_pad;
  ep.err = err;
  NBR_CHECKED_ONLY(ip.len = kMaxN; js.len = kMaxN; ep.part_len = (long long)kMaxSplit * 3 * kMaxN;
                   ep.cnt_len = (long long)kCounters;)
  e = launch_force(precision, eps2, cfg, ip, js, ep, st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "no-allocation force launch");

  int h = 0;
  e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "no-allocation force");
  if (h == kErrBounds)
    return fail(nullptr, NBR_ERR_BOUNDS, "a kernel index was outside its array (checked build)");
  if (h != kErrNone)
    return fail(nullptr, NBR_ERR_TIMEOUT, "a j-tile copy did not complete within the wait limit");
  return NBR_OK;
}
