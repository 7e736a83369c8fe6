// Small device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include "rfxb_inst.h"

namespace rfxb {

// Physical constants of the reference (rfx/core/yee.py:117-118).
constexpr double kEps0 = 8.8541878128e-12;
constexpr double kMu0 = 1.25663706212e-6;

__device__ __forceinline__ void cp_async4(float* sdst, const float* gsrc) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// 16-byte copy; both addresses must be 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- TMA (cp.async.bulk.tensor) and mbarrier helpers ----------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(addr), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(addr), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}
// Default poll limit of a pipeline wait (each poll may suspend the thread for
// a hardware-defined time): a wait that never completes gives up instead of
// hanging the launch.
constexpr int kWaitLimit = 1 << 22;
// Bounded wait: false if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t parity, int limit = kWaitLimit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(addr, parity)) return true;
  return false;
}
// Mbarrier phases carried from one work item to the next by a CTA that
// processes several (the persistent kernels): bit s of `stage` is the parity
// of the next completion of plane stage s, bit s of `ring` that of psi ring
// slot s.  A CTA that runs one item starts from zero.
struct StepPhases {
  uint32_t stage = 0u;
  uint32_t ring = 0u;
};

// Fault injection of the bounded-wait test (the defaults in every other
// launch): the CTA whose block index is `cta` does not issue the TMA boxes
// of plane xa of its first item, so its wait on that plane runs out after
// `wait_limit` polls and the CTA takes the time-out path.
struct StepFault {
  int cta = -1;
  int wait_limit = kWaitLimit;
};

// Yee updates with their rounding spelled out (products and fused
// multiply-adds written as intrinsics, nothing left to contraction), so every
// kernel that updates a cell, the one-step and the two-step kernels alike,
// produces the same bits.
// a * pa - b * pb: one component of a curl
__device__ __forceinline__ float yee_diff2(float a, float pa, float b, float pb) {
  return __fmaf_rn(a, pa, -__fmul_rn(b, pb));
}
// H^{n+1/2} = H^{n-1/2} - ch * curl E
__device__ __forceinline__ float yee_h(float h, float ch, float curl) { return __fmaf_rn(-ch, curl, h); }
// E^{n+1} = ca * E^n + cb * curl H
__device__ __forceinline__ float yee_e(float ca, float e, float cb, float curl) {
  return __fmaf_rn(cb, curl, __fmul_rn(ca, e));
}

// Buffer selector of a forward step launch: the field state is read from
// F[in] and written to F[out] (0 and 1: the ping-pong pair; 2: the
// intermediate state of a two-step pass), the CPML psi are read from parity
// `psi` and written to psi ^ 1.
__host__ __device__ constexpr int step_sel(int in, int out, int psi) { return in | (out << 2) | (psi << 4); }
__host__ __device__ constexpr int sel_in(int s) { return s & 3; }
__host__ __device__ constexpr int sel_out(int s) { return (s >> 2) & 3; }
__host__ __device__ constexpr int sel_psi(int s) { return (s >> 4) & 1; }

// 4-D tiled TMA load of one box into shared memory, completing on an mbarrier.
// The innermost coordinate c0 must be a multiple of 4 (16 bytes of float).
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* tmap, int c0, int c1, int c2, int c3,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
      : "memory");
}

// Which slab of a CPML axis a coordinate falls in: returns side (0 lo, 1 hi)
// and the layer index in that face's (hi pre-flipped) profile, or -1.
__device__ __forceinline__ int cpml_side(int x, int nax, int n, int& s) {
  if (x < n) { s = x; return 0; }
  if (x >= nax - n) { s = x - (nax - n); return 1; }
  return -1;
}

__device__ __forceinline__ long long psi_index_x(const RfxbInst& P, int side, int q, int s, int j, int k) {
  return ((long long)((side * 2 + q) * P.ncp + s) * P.ny + j) * P.zs + k;
}
__device__ __forceinline__ long long psi_index_y(const RfxbInst& P, int side, int q, int s, int i, int k) {
  return ((long long)((side * 2 + q) * P.nx + i) * P.ncp + s) * P.zs + k;
}
__device__ __forceinline__ long long psi_index_z(const RfxbInst& P, int side, int q, int s, int i, int j) {
  return ((long long)((side * 2 + q) * P.nx + i) * P.ny + j) * P.ncp4 + s;
}

// Copy a descriptor into shared memory (word-wise, all threads help).
__device__ __forceinline__ void load_inst(RfxbInst& dst, const RfxbInst* src, int tid, int nthr) {
  static_assert(sizeof(RfxbInst) % 4 == 0, "descriptor must be word sized");
  const int nw = sizeof(RfxbInst) / 4;
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(&dst);
  for (int t = tid; t < nw; t += nthr) d[t] = __ldg(s + t);
}

}  // namespace rfxb
