// Field-energy reduction over a box of one instance's current state: the
// interior-energy stop of rfx's run_until_decay (rfx/simulation.py:2493-2505,
// U = sum of E^2 + H^2 over the non-CPML slice), on the device.
//
// Grid-stride over the box cells in the padded layout, float64 accumulation
// per thread, warp-shuffle and shared-memory block reduction, one float64
// atomic add per block into the caller's accumulator.
#include "rfxb_common.cuh"

namespace rfxb {

__global__ void __launch_bounds__(256) box_energy_kernel(RfxbInst P, int par, int i0, int i1, int j0, int j1, int k0,
                                                         int k1, double* __restrict__ out) {
  const int nk = k1 - k0, nj = j1 - j0;
  const long long total = (long long)(i1 - i0) * nj * nk;
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = k0 + (int)(t % nk);
    const long long r = t / nk;
    const int j = j0 + (int)(r % nj);
    const int i = i0 + (int)(r / nj);
    const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const float v = P.F[par][c][e];
      s = fmaf(v, v, s);
    }
    acc += (double)s;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ double part[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    acc = lane < (int)(blockDim.x >> 5) ? part[lane] : 0.0;
    for (int o = 4; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) atomicAdd(out, acc);
  }
}

}  // namespace rfxb
