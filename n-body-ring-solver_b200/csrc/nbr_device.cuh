// nbr_device.cuh -- sm_100a device helpers shared by the N-body kernels.
//
//  * packed FP32 pair arithmetic (add/sub/mul/fma .f32x2, PTX ISA 8.6,
//    sm_100+): one instruction operates on two particles held in a 64-bit
//    register pair, which halves the issue slots the FP32 pipe needs;
//  * the MUFU reciprocal square root (rsqrt.approx.ftz.f32);
//  * mbarrier + cp.async.bulk (1-D TMA) primitives for the shared-memory
//    j-tile ring.  No multicast form is used anywhere;
//  * bounded waits: every spin has a wall-clock limit after which the kernel
//    records an error code for the host and stops consuming tiles.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nbr {

// Particles per j-tile; also the group size the FP32 tile origins are taken over.
constexpr int kTile = 128;
// Default wall-clock limit of one bounded wait, in nanoseconds (%globaltimer).
constexpr unsigned long long kWaitLimitNs = 4000000000ull;

// Device error codes (written with atomicCAS(err, 0, code): first one wins).
enum : int {
  kErrNone = 0,
  kErrTileWait = 1,    // a j-tile's bulk copy did not complete in time
  kErrDrainWait = 2,   // draining in-flight copies after an abort timed out
  kErrBounds = 3,      // checked builds: an index outside its array (access skipped)
  kErrGridWait = 4,    // a grid-wide barrier of a persistent launch did not complete in time
};

typedef unsigned long long u64;

// ----------------------------------------------------------------- f32x2 ----
__device__ __forceinline__ u64 pack2(float lo, float hi) {
  u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(u64 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ u64 add2(u64 a, u64 b) {
  u64 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 sub2(u64 a, u64 b) {
  u64 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
  u64 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
  u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
// MUFU reciprocal square root of each half.
__device__ __forceinline__ float rsqrt_mufu(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ u64 rsqrt2(u64 v) {
  float lo, hi;
  unpack2(v, lo, hi);
  return pack2(rsqrt_mufu(lo), rsqrt_mufu(hi));
}

// Knuth TwoSum of the packed pair (hi + p): hi <- rounded sum, lo += the
// rounding error.  Six packed adds; exact error term for round-to-nearest.
__device__ __forceinline__ void two_sum2(u64& hi, u64& lo, u64 p) {
  u64 s = add2(hi, p);
  u64 bp = sub2(s, hi);
  u64 ap = sub2(s, bp);
  u64 e = add2(sub2(hi, ap), sub2(p, bp));
  lo = add2(lo, e);
  hi = s;
}

// --------------------------------------------------------------- timing -----
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ------------------------------------------------------- mbarrier + bulk ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the barrier phase with the given parity; gives up after limit_ns
// and returns false (the caller records the error).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity,
                                                  unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}
// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void record_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// Checked builds (-DNBR_CHECKED, libnbr_checked.so) test every array index
// against the array's allocated length, passed with the launch, before the
// access; a failing index is recorded (kErrBounds) and the access skipped.
// In normal builds NBR_IN is the constant true and the length expression is
// never compiled.
__device__ __forceinline__ bool in_bounds(long long idx, long long len, int* err) {
  if (idx >= 0 && idx < len) return true;
  record_error(err, kErrBounds);
  return false;
}
#ifdef NBR_CHECKED
#define NBR_IN(idx, len, err) (::nbr::in_bounds((long long)(idx), (long long)(len), (err)))
#else
#define NBR_IN(idx, len, err) true
#endif

}  // namespace nbr
