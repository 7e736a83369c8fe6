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
                                                         int k1, const double* __restrict__ wx,
                                                         const double* __restrict__ wy,
                                                         const double* __restrict__ wz, double* __restrict__ out) {
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
    // graded lane: weighted by the cell volume dx[i] dy[j] dz[k]
    acc += wx ? (double)s * (wx[i] * wy[j] * wz[k]) : (double)s;
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

// Net outgoing co-located Poynting flux through the six faces of a box
// (rfx/simulation.py:2521-2540 _radiated_power): grid-stride over the face
// cells of faces x_lo, x_hi, y_lo, y_hi, z_lo, z_hi (tangential ranges
// half-open), float32 products as in the reference, float64 accumulation,
// one atomic add per block.
__global__ void __launch_bounds__(256) box_flux_kernel(RfxbInst P, int par, int i0, int i1, int j0, int j1, int k0,
                                                       int k1, double* __restrict__ out) {
  const int ni = i1 - i0, nj = j1 - j0, nk = k1 - k0;
  const long long fx = (long long)nj * nk, fy = (long long)ni * nk, fz = (long long)ni * nj;
  const long long total = 2 * (fx + fy + fz);
  const float* const* F = P.F[par];
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    long long u = t;
    int axis, hi;
    if (u < 2 * fx) { axis = 0; hi = u >= fx; u -= hi ? fx : 0; }
    else if ((u -= 2 * fx) < 2 * fy) { axis = 1; hi = u >= fy; u -= hi ? fy : 0; }
    else { u -= 2 * fy; axis = 2; hi = u >= fz; u -= hi ? fz : 0; }
    int i, j, k;
    if (axis == 0) { i = hi ? i1 : i0; j = j0 + (int)(u / nk); k = k0 + (int)(u % nk); }
    else if (axis == 1) { i = i0 + (int)(u / nk); j = hi ? j1 : j0; k = k0 + (int)(u % nk); }
    else { i = i0 + (int)(u / nj); j = j0 + (int)(u % nj); k = hi ? k1 : k0; }
    const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
    float s;
    if (axis == 0) s = __fmul_rn(F[1][e], F[5][e]) - __fmul_rn(F[2][e], F[4][e]);        // Ey Hz - Ez Hy
    else if (axis == 1) s = __fmul_rn(F[2][e], F[3][e]) - __fmul_rn(F[0][e], F[5][e]);   // Ez Hx - Ex Hz
    else s = __fmul_rn(F[0][e], F[4][e]) - __fmul_rn(F[1][e], F[3][e]);                 // Ex Hy - Ey Hx
    acc += hi ? (double)s : -(double)s;
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

// Poynting-flux monitor accumulation for one step (rfx/simulation.py:1590-
// 1642): E1, E2 at the plane, H1, H2 averaged over the plane and the one
// before it in float32, each multiplied by its complex128 step factor and
// added to the complex128 accumulators.  One thread per region cell.
__global__ void flux_kernel(const RfxbInst* __restrict__ insts, const RfxbFluxPlane* __restrict__ planes,
                            int nplanes, int n, int par) {
  int q = 0;
  while (q + 1 < nplanes && planes[q + 1].block0 <= (int)blockIdx.x) ++q;
  const RfxbFluxPlane& M = planes[q];
  const RfxbInst& P = insts[M.inst];
  const int c = (blockIdx.x - M.block0) * blockDim.x + threadIdx.x;
  const int cells = M.n1 * M.n2;
  if (c >= cells) return;
  const int a = M.lo1 + c / M.n2, b = M.lo2 + c % M.n2;
  long long e, em1;
  auto at = [&](int plane) {
    int i, j, k;
    if (M.axis == 0) { i = plane; j = a; k = b; }
    else if (M.axis == 1) { i = a; j = plane; k = b; }
    else { i = a; j = b; k = plane; }
    return P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
  };
  e = at(M.index);
  em1 = at(M.im1);
  float v[4];
  v[0] = P.F[par][M.comp[0]][e];
  v[1] = P.F[par][M.comp[1]][e];
  v[2] = (P.F[par][M.comp[2]][em1] + P.F[par][M.comp[2]][e]) * 0.5f;
  v[3] = (P.F[par][M.comp[3]][em1] + P.F[par][M.comp[3]][e]) * 0.5f;
  const double2* kn = M.kern + (long long)n * 2 * M.nf;
  for (int f = 0; f < M.nf; ++f) {
    const double2 ke = kn[f], kh = kn[M.nf + f];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const double2 k2 = t < 2 ? ke : kh;
      double2* acc = M.acc + ((long long)t * M.nf + f) * cells + c;
      double2 s = *acc;
      s.x += (double)v[t] * k2.x;
      s.y += (double)v[t] * k2.y;
      *acc = s;
    }
  }
}

// NTFF Huygens-box accumulation for one step (rfx/farfield.py:208-313): on
// each face the four tangential components times the step's complex64 factor
// (E factor for the two E components, H factor, half a step later, for the
// two H components), Kahan-added to the complex64 running sums per real and
// imaginary part.  One thread per face cell; a thread's 4 components are
// adjacent (32 B), so a warp reads and writes 1 KB runs per frequency.
__global__ void __launch_bounds__(256) ntff_kernel(const RfxbInst* __restrict__ insts,
                                                   const RfxbNtffFace* __restrict__ faces, int nfaces, int n,
                                                   int par) {
  int q = 0;
  while (q + 1 < nfaces && faces[q + 1].block0 <= (int)blockIdx.x) ++q;
  const RfxbNtffFace& A = faces[q];
  const RfxbInst& P = insts[A.inst];
  const int c = (blockIdx.x - A.block0) * blockDim.x + threadIdx.x;
  const int cells = A.n1 * A.n2;
  if (c >= cells) return;
  const int a = A.lo1 + c / A.n2, b = A.lo2 + c % A.n2;
  int i, j, k;
  if (A.axis == 0) { i = A.index; j = a; k = b; }
  else if (A.axis == 1) { i = a; j = A.index; k = b; }
  else { i = a; j = b; k = A.index; }
  const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
  float v[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) v[t] = P.F[par][A.comp[t]][e];
  const float2* ph = A.phase + (long long)n * 2 * A.nf;
  for (int f = 0; f < A.nf; ++f) {
    const float2 we = __ldg(ph + f), wh = __ldg(ph + A.nf + f);
    float4* sp = reinterpret_cast<float4*>(A.acc + ((long long)f * cells + c) * 4);
    float4* rp = reinterpret_cast<float4*>(A.cmp + ((long long)f * cells + c) * 4);
#pragma unroll
    for (int h = 0; h < 2; ++h) {    // h = 0: the E pair, h = 1: the H pair
      const float2 w = h == 0 ? we : wh;
      float4 s = sp[h], r = rp[h];
      float* sv = reinterpret_cast<float*>(&s);
      float* rv = reinterpret_cast<float*>(&r);
#pragma unroll
      for (int u = 0; u < 4; ++u) {  // (re, im) of the two components
        const float val = __fmul_rn(v[2 * h + (u >> 1)], (u & 1) ? w.y : w.x);
        const float y = val - rv[u];
        const float t = sv[u] + y;
        rv[u] = (t - sv[u]) - y;
        sv[u] = t;
      }
      sp[h] = s;
      rp[h] = r;
    }
  }
}

}  // namespace rfxb
