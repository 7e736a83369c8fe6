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
  return ((long long)((side * 2 + q) * P.nx + i) * P.ny + j) * P.ncp + s;
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
