// Two-step forward pass of the CPML-free interior (temporal blocking, depth 2).
//
// One CTA owns a (TY x 32) tile of the (y, z) plane over an x range [xa, xb)
// and advances it from step n to step n+2 in one pass over HBM: E^n,
// H^{n-1/2} and ca/cb are read once with a two-cell halo, the intermediate
// state (E^{n+1}, H^{n+1/2}) lives in shared memory on the tile plus the halo
// its second step needs, and only (E^{n+2}, H^{n+3/2}) of the tile are
// written.  The halo cells of the first step are recomputed by every CTA
// that needs them (overlapped tiling), from step-n values that no CTA of the
// pass overwrites (the pass reads F[par] and writes F[par ^ 1]).
//
// The march along x skews the second step one plane behind the first.  At
// plane p the CTA computes, each phase over its region of (y, z) cells:
//   H^{n+1/2}(p)   rows y0-2 .. y0+TY,   columns z0-2 .. z0+32
//   E^{n+1}(p)     rows y0-1 .. y0+TY,   columns z0-1 .. z0+32
//   H^{n+3/2}(p-1) rows y0-1 .. y0+TY-1, columns z0-1 .. z0+31
//   E^{n+2}(p-1)   the tile
// with the arithmetic of the one-step kernel (rfx/core/yee.py:226-291 and
// :347-404 through the shared rounding helpers), so every value equals the
// one the one-step kernel computes, bit for bit.
//
// The host gives this kernel only tiles whose cells, halo included, lie in no
// CPML slab and hold no source, probe or gradient-history cell, in plans with
// uniform H coefficients; cells at a grid face take the guarded path (zero
// outside the grid, PEC faces) and a PEC edge mask applies to every E cell as
// in the one-step kernel.  Everything else runs two one-step launches per
// pass through the intermediate buffer F[2].
// Where a one-step neighbour or a per-step observer (DFT plane, flux monitor,
// NTFF face) reads this tile's intermediate state, the CTA also stores it to
// F[2] (RfxbWork2::mid).
#include "rfxb_common.cuh"

namespace rfxb {

#define RFXB_D2W 40   // staged row: z in [z0 - 4, z0 + 36)
#define RFXB_D2I 36   // row pitch of the intermediate arrays (35 columns used at most)
#define RFXB_D2NS 3   // pipeline stages: planes p, p+1 and p+2 in flight

template <int TY>
struct Fwd2Dims {
  static constexpr int NE = 3 * (TY + 4) * RFXB_D2W;
  static constexpr int NH = 3 * (TY + 3) * RFXB_D2W;
  static constexpr int NC = 2 * (TY + 2) * RFXB_D2W;
  static constexpr int PH = (NE + NH) % 32 ? 32 - (NE + NH) % 32 : 32;   // cab on a 128-byte boundary
  static constexpr unsigned BYTES = 4u * (NE + NH + NC);
};

template <int TY>
struct __align__(128) Fwd2Stage {
  float e[3][TY + 4][RFXB_D2W];   // E^n, rows y0-2 .. y0+TY+1
  float h[3][TY + 3][RFXB_D2W];   // H^{n-1/2}, rows y0-2 .. y0+TY
  float pad[Fwd2Dims<TY>::PH];
  float cab[2][TY + 2][RFXB_D2W]; // ca, cb, rows y0-1 .. y0+TY
};

template <int TY>
struct Fwd2Smem {
  Fwd2Stage<TY> st[RFXB_D2NS];          // plane p in stage p % 3
  float h1[2][3][TY + 3][RFXB_D2I];     // H^{n+1/2}: [y - (y0-2)][z - (z0-2)], slot p & 1
  float e1[2][3][TY + 2][RFXB_D2I];     // E^{n+1}:   [y - (y0-1)][z - (z0-1)]
  float h2[2][3][TY + 1][RFXB_D2I];     // H^{n+3/2}: [y - (y0-1)][z - (z0-1)]
  float cabt[2][2][TY][RFXB_TZ];        // ca, cb of the tile, kept for the second step one plane on
  float ytab[2][TY + 3];                // yh, ye at y0-2 .. y0+TY
  float ztab[2][RFXB_D2I];              // zh, ze at z0-2 .. z0+32
  RfxbInst P;
  unsigned long long mbar[RFXB_D2NS];
};

size_t fwd2_step_smem_bytes() { return sizeof(Fwd2Smem<8>); }

// Issue the TMA boxes of plane ip (one thread): E and H of the field block of
// parity par with the two-step boxes, ca/cb with the two-step coefficient box.
template <int TY>
__device__ __forceinline__ void tma_stage2(Fwd2Smem<TY>& S, const CUtensorMap* tm, int par, int y0, int z0, int ip) {
  const int s = (ip + RFXB_D2NS) % RFXB_D2NS;   // ip >= -2
  const uint32_t mb = smem_u32(&S.mbar[s]);
  mbar_expect_tx(mb, Fwd2Dims<TY>::BYTES);
  // map coordinates: (z, j + 1, i + 1, component)
  tma_load_4d(smem_u32(&S.st[s].e[0][0][0]), tm + RFXB_MAP_E2 + par, z0 - 4, y0 - 1, ip + 1, 0, mb);
  tma_load_4d(smem_u32(&S.st[s].h[0][0][0]), tm + RFXB_MAP_H2 + par, z0 - 4, y0 - 1, ip + 1, 3, mb);
  tma_load_4d(smem_u32(&S.st[s].cab[0][0][0]), tm + RFXB_MAP_C2, z0 - 4, y0, ip + 1, 0, mb);
}

// The cells of a phase region: its 32 middle columns row by row, one warp
// per row and one lane per column (so every shared-memory row access is 32
// consecutive words), and its NEDGE edge columns one cell per thread on the
// last threads.  f(r, c) is called with the region's row and column;
// edge(k) is the column of edge k.
template <int TY, int ROWS, int C0, int NEDGE>
__device__ __forceinline__ void for_region(int ty, int lane, int tid, auto&& edge, auto&& f) {
#pragma unroll
  for (int r = ty; r < ROWS; r += TY) f(r, C0 + lane);
  constexpr int e0 = 32 * TY - NEDGE * ROWS;
  static_assert(e0 >= 0, "more edge cells than threads");
  if (tid >= e0) {
    const int e = tid - e0;
    f(e / NEDGE, edge(e % NEDGE));
  }
}

// PEC faces of the E update (rfx/boundaries/pec.py:13-47), as the one-step
// kernel applies them.
__device__ __forceinline__ void pec_faces(unsigned pec, int i, int j, int k, int nx, int ny, int nz, float& ex,
                                          float& ey, float& ez) {
  if ((pec & 1u) && (i == 0 || i == nx - 1)) { ey = 0.f; ez = 0.f; }
  if ((pec & 2u) && (j == 0 || j == ny - 1)) { ex = 0.f; ez = 0.f; }
  if ((pec & 4u) && (k == 0 || k == nz - 1)) { ex = 0.f; ey = 0.f; }
  if ((pec & 4u) && k == nz - 1) ez = 0.f;
}

// PEC edge mask of one E cell (rfx/boundaries/pec.py:179-208), as the
// one-step kernel applies it after the PEC faces.
__device__ __forceinline__ void edge_mask(unsigned m, float& ex, float& ey, float& ez) {
  if (m) {
    ex = ex * (1.f - (float)(m & 1u));
    ey = ey * (1.f - (float)((m >> 1) & 1u));
    ez = ez * (1.f - (float)((m >> 2) & 1u));
  }
}

// One work item.  EDGE: the item's cells reach a grid face (no CPML on that
// axis): cells outside the grid stay zero (the guards the one-step kernel
// reads) and E takes the PEC faces; otherwise every computed cell is an
// interior cell and those checks are compiled out.
template <int TY, bool EDGE>
__device__ __forceinline__ void fwd2_item(Fwd2Smem<TY>& S, const RfxbWork2& w, const CUtensorMap* __restrict__ maps,
                                          int par) {
  constexpr int NT = 32 * TY;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + lane;
  const RfxbInst& P = S.P;
  const int y0 = w.y0, z0 = w.z0, xa = w.xa, xb = w.xb;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const unsigned pec = P.pec_axes;
  const unsigned char* emask = P.emask;   // PEC edge mask bits (1 ex, 2 ey, 4 ez) or null
  const CUtensorMap* tm = maps + (size_t)w.inst * RFXB_NMAPS;
  const int producer = NT - 32;   // lane 0 of the last warp issues the boxes
  const int wlim = kWaitLimit;
  // planes are staged in order xa-2, xa-1, ..., xb+1 (from -2 on at the low
  // x face): plane p is the ((p - xa + 2) / 3)-th fill of stage (p + 3) % 3
  auto stg = [](int p) { return (p + RFXB_D2NS) % RFXB_D2NS; };
  auto sparity = [&](int p) -> uint32_t { return (uint32_t)(((p - xa + 2) / RFXB_D2NS) & 1); };
  if (tid == producer)
    for (int p = xa - 2; p <= min(xa, xb + 1); ++p) tma_stage2<TY>(S, tm, par, y0, z0, p);
  // spacing tables (entries -1 .. n exist; the cells beyond are zero anyway)
  for (int t = tid; t < TY + 3; t += NT) {
    const int j = min(max(y0 - 2 + t, -1), ny);
    S.ytab[0][t] = __ldg(P.yh + j);
    S.ytab[1][t] = __ldg(P.ye + j);
  }
  for (int t = tid; t < 35; t += NT) {
    const int k = min(max(z0 - 2 + t, -1), nz);
    S.ztab[0][t] = __ldg(P.zh + k);
    S.ztab[1][t] = __ldg(P.ze + k);
  }
  auto xclamp = [&](int i) { return min(max(i, -1), nx); };
  const float ch = P.ch0;
  float* Fo = P.F[par ^ 1][0];
  float* Fm = P.F[2][0];
  const long long cs = P.cs;
  // the tile cell of this thread in phase 4 and in the stores
  const int jt = y0 + ty, kt = z0 + lane;
  const bool own = !EDGE || (jt < ny && kt < nz);
  const long long e_row = P.off0 + (long long)jt * P.zs + kt;
  auto inside = [&](int i, int j, int k) {
    return !EDGE || ((unsigned)i < (unsigned)nx && (unsigned)j < (unsigned)ny && (unsigned)k < (unsigned)nz);
  };
  // x spacing entries: plane p (loaded one plane ahead) and plane p-1
  float xh_n = __ldg(P.xh + xclamp(xa - 2)), xe_n = __ldg(P.xe + xclamp(xa - 2));
  float xh_q = 0.f, xe_q = 0.f;
  // edge columns of the phase regions (region column indices)
  auto edge1 = [](int k) { return k < 2 ? k : 34; };   // z0-2, z0-1, z0+32
  auto edge2 = [](int k) { return k ? 33 : 0; };       // z0-1, z0+32
  auto edge3 = [](int) { return 0; };                  // z0-1

  for (int p = xa - 2; p <= xb; ++p) {
    // planes p and p+1 are needed (p+1 is the furthest); p was waited for in
    // the previous iteration, except in the first
    bool ok = mbar_wait_bounded(smem_u32(&S.mbar[stg(p + 1)]), sparity(p + 1), wlim);
    if (p == xa - 2) ok = ok && mbar_wait_bounded(smem_u32(&S.mbar[stg(p)]), sparity(p), wlim);
    if (__syncthreads_or(!ok)) {
      // a wait ran out: flag the launch and drain the boxes in flight
      if (tid == 0) {
        atomicOr(P.status, 1);
        const int last = min(xb + 1, max(xa, p + 1));
        for (int r = (p == xa - 2 ? p : p + 1); r <= last; ++r)
          mbar_wait_bounded(smem_u32(&S.mbar[stg(r)]), sparity(r), wlim);
      }
      return;
    }
    // every thread is done with iteration p-1, so plane p-1's stage is free
    if (tid == producer && p >= xa - 1 && p + 2 <= xb + 1) tma_stage2<TY>(S, tm, par, y0, z0, p + 2);
    const float xh = xh_n, xe = xe_n;
    if (p + 1 <= xb) { xh_n = __ldg(P.xh + xclamp(p + 1)); xe_n = __ldg(P.xe + xclamp(p + 1)); }

    // ---- phase 1: H^{n+1/2}(p), rows y0-2 .. y0+TY, columns z0-2 .. z0+32 ----
    {
      const Fwd2Stage<TY>& A = S.st[stg(p)];
      const Fwd2Stage<TY>& B = S.st[stg(p + 1)];
      auto& H1 = S.h1[p & 1];
      for_region<TY, TY + 3, 2, 3>(ty, lane, tid, edge1, [&](int r, int q) {
        if (!inside(p, y0 - 2 + r, z0 - 2 + q)) {
          H1[0][r][q] = 0.f; H1[1][r][q] = 0.f; H1[2][r][q] = 0.f;
          return;
        }
        const int lz = q + 2;                   // staged column: z - (z0-4)
        const float Ex = A.e[0][r][lz], Ey = A.e[1][r][lz], Ez = A.e[2][r][lz];
        const float dEz_y = A.e[2][r + 1][lz] - Ez;
        const float dEy_z = A.e[1][r][lz + 1] - Ey;
        const float dEx_z = A.e[0][r][lz + 1] - Ex;
        const float dEz_x = B.e[2][r][lz] - Ez;
        const float dEy_x = B.e[1][r][lz] - Ey;
        const float dEx_y = A.e[0][r + 1][lz] - Ex;
        const float yh = S.ytab[0][r], zh = S.ztab[0][q];
        H1[0][r][q] = yee_h(A.h[0][r][lz], ch, yee_diff2(dEz_y, yh, dEy_z, zh));
        H1[1][r][q] = yee_h(A.h[1][r][lz], ch, yee_diff2(dEx_z, zh, dEz_x, xh));
        H1[2][r][q] = yee_h(A.h[2][r][lz], ch, yee_diff2(dEy_x, xh, dEx_y, yh));
      });
    }
    __syncthreads();

    // ---- phase 2: E^{n+1}(p), rows y0-1 .. y0+TY, columns z0-1 .. z0+32 ----
    if (p >= xa - 1) {
      const Fwd2Stage<TY>& A = S.st[stg(p)];
      const auto& H1 = S.h1[p & 1];
      const auto& H1m = S.h1[(p - 1) & 1];
      auto& E1 = S.e1[p & 1];
      for_region<TY, TY + 2, 1, 2>(ty, lane, tid, edge2, [&](int r, int q) {
        const int j = y0 - 1 + r, k = z0 - 1 + q;
        if (!inside(p, j, k)) {
          E1[0][r][q] = 0.f; E1[1][r][q] = 0.f; E1[2][r][q] = 0.f;
          return;
        }
        const int hr = r + 1, hq = q + 1;       // the same cell in H1 / the tables
        const float hx = H1[0][hr][hq], hy = H1[1][hr][hq], hz = H1[2][hr][hq];
        const float dHz_y = hz - H1[2][hr - 1][hq];
        const float dHy_z = hy - H1[1][hr][hq - 1];
        const float dHx_z = hx - H1[0][hr][hq - 1];
        const float dHz_x = hz - H1m[2][hr][hq];
        const float dHy_x = hy - H1m[1][hr][hq];
        const float dHx_y = hx - H1[0][hr - 1][hq];
        const float ye = S.ytab[1][hr], ze = S.ztab[1][hq];
        const float cx_ = yee_diff2(dHz_y, ye, dHy_z, ze);
        const float cy_ = yee_diff2(dHx_z, ze, dHz_x, xe);
        const float cz_ = yee_diff2(dHy_x, xe, dHx_y, ye);
        const float cav = A.cab[0][r][q + 3], cbv = A.cab[1][r][q + 3];
        float ex = yee_e(cav, A.e[0][hr][q + 3], cbv, cx_);
        float ey = yee_e(cav, A.e[1][hr][q + 3], cbv, cy_);
        float ez = yee_e(cav, A.e[2][hr][q + 3], cbv, cz_);
        if (EDGE) pec_faces(pec, p, j, k, nx, ny, nz, ex, ey, ez);
        if (emask) edge_mask(emask[P.off0 + (long long)p * P.ps + (long long)j * P.zs + k], ex, ey, ez);
        E1[0][r][q] = ex;
        E1[1][r][q] = ey;
        E1[2][r][q] = ez;
      });
      // the tile's ca / cb for its second step one plane on (plane p's stage
      // takes plane p+3 before that)
      S.cabt[p & 1][0][ty][lane] = A.cab[0][ty + 1][lane + 4];
      S.cabt[p & 1][1][ty][lane] = A.cab[1][ty + 1][lane + 4];
    }
    __syncthreads();

    // ---- phase 3: H^{n+3/2}(p-1), rows y0-1 .. y0+TY-1, columns z0-1 .. z0+31 ----
    const int q = p - 1;
    if (q >= xa - 1) {
      const auto& E1 = S.e1[q & 1];
      const auto& E1n = S.e1[p & 1];
      const auto& H1 = S.h1[q & 1];
      auto& H2 = S.h2[q & 1];
      for_region<TY, TY + 1, 1, 1>(ty, lane, tid, edge3, [&](int r, int s) {
        if (!inside(q, y0 - 1 + r, z0 - 1 + s)) {
          H2[0][r][s] = 0.f; H2[1][r][s] = 0.f; H2[2][r][s] = 0.f;
          return;
        }
        const float Ex = E1[0][r][s], Ey = E1[1][r][s], Ez = E1[2][r][s];
        const float dEz_y = E1[2][r + 1][s] - Ez;
        const float dEy_z = E1[1][r][s + 1] - Ey;
        const float dEx_z = E1[0][r][s + 1] - Ex;
        const float dEz_x = E1n[2][r][s] - Ez;
        const float dEy_x = E1n[1][r][s] - Ey;
        const float dEx_y = E1[0][r + 1][s] - Ex;
        const float yh = S.ytab[0][r + 1], zh = S.ztab[0][s + 1];
        H2[0][r][s] = yee_h(H1[0][r + 1][s + 1], ch, yee_diff2(dEz_y, yh, dEy_z, zh));
        H2[1][r][s] = yee_h(H1[1][r + 1][s + 1], ch, yee_diff2(dEx_z, zh, dEz_x, xh_q));
        H2[2][r][s] = yee_h(H1[2][r + 1][s + 1], ch, yee_diff2(dEy_x, xh_q, dEx_y, yh));
      });
    }
    __syncthreads();

    // ---- phase 4: E^{n+2}(p-1) on the tile, and the stores ----
    if (q >= xa && own) {
      const auto& H2 = S.h2[q & 1];
      const auto& H2m = S.h2[(q - 1) & 1];
      const auto& E1 = S.e1[q & 1];
      const int r = ty + 1, s = lane + 1;      // in H2 / E1: y - (y0-1), z - (z0-1)
      const float hx = H2[0][r][s], hy = H2[1][r][s], hz = H2[2][r][s];
      const float dHz_y = hz - H2[2][r - 1][s];
      const float dHy_z = hy - H2[1][r][s - 1];
      const float dHx_z = hx - H2[0][r][s - 1];
      const float dHz_x = hz - H2m[2][r][s];
      const float dHy_x = hy - H2m[1][r][s];
      const float dHx_y = hx - H2[0][r - 1][s];
      const float ye = S.ytab[1][ty + 2], ze = S.ztab[1][lane + 2];
      const float cx_ = yee_diff2(dHz_y, ye, dHy_z, ze);
      const float cy_ = yee_diff2(dHx_z, ze, dHz_x, xe_q);
      const float cz_ = yee_diff2(dHy_x, xe_q, dHx_y, ye);
      const float cav = S.cabt[q & 1][0][ty][lane], cbv = S.cabt[q & 1][1][ty][lane];
      float ex = yee_e(cav, E1[0][r][s], cbv, cx_);
      float ey = yee_e(cav, E1[1][r][s], cbv, cy_);
      float ez = yee_e(cav, E1[2][r][s], cbv, cz_);
      if (EDGE) pec_faces(pec, q, jt, kt, nx, ny, nz, ex, ey, ez);
      if (emask) edge_mask(emask[e_row + (long long)q * P.ps], ex, ey, ez);
      const long long e = e_row + (long long)q * P.ps;
      Fo[e] = ex;
      Fo[cs + e] = ey;
      Fo[2 * cs + e] = ez;
      Fo[3 * cs + e] = hx;
      Fo[4 * cs + e] = hy;
      Fo[5 * cs + e] = hz;
      // the intermediate state of plane q where a one-step neighbour or an
      // observer reads it
      if ((w.mid & RFXB_MID_ALL) || (q == xa && (w.mid & RFXB_MID_LO)) || (q == xb - 1 && (w.mid & RFXB_MID_HI))) {
        const auto& H1 = S.h1[q & 1];
        Fm[e] = E1[0][r][s];
        Fm[cs + e] = E1[1][r][s];
        Fm[2 * cs + e] = E1[2][r][s];
        Fm[3 * cs + e] = H1[0][r + 1][s + 1];
        Fm[4 * cs + e] = H1[1][r + 1][s + 1];
        Fm[5 * cs + e] = H1[2][r + 1][s + 1];
      }
    }
    xh_q = xh;
    xe_q = xe;
  }
}

template <int TY>
__global__ void __launch_bounds__(32 * TY, 3)
fwd2_step_kernel(const RfxbInst* __restrict__ insts, const RfxbWork2* __restrict__ work,
                 const CUtensorMap* __restrict__ maps, int n, int par) {
  extern __shared__ __align__(128) unsigned char fwd2_smem_raw[];
  Fwd2Smem<TY>& S = *reinterpret_cast<Fwd2Smem<TY>*>(fwd2_smem_raw);
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const RfxbWork2 w = work[blockIdx.x];
  if (tid == 0) {
    for (int q = 0; q < RFXB_D2NS; ++q) mbar_init(smem_u32(&S.mbar[q]), 1);
    mbar_fence_init();
  }
  load_inst(S.P, insts + w.inst, tid, 32 * TY);
  __syncthreads();
  if (w.mid & RFXB_MID_EDGE) fwd2_item<TY, true>(S, w, maps, par);
  else fwd2_item<TY, false>(S, w, maps, par);
}

template __global__ void fwd2_step_kernel<8>(const RfxbInst*, const RfxbWork2*, const CUtensorMap*, int, int);

}  // namespace rfxb
