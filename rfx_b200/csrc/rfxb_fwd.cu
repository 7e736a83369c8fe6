// Forward time step of the Yee/CPML leapfrog: one fused kernel per step.
//
// One CTA owns a (TY x 32) tile of the (y, z) plane and marches along x over
// an x range [xa, xb).  For each x plane i it
//   1. keeps a 4-stage cp.async pipeline of the input planes i-1 .. i+2 in
//      shared memory, 16-byte copies of: E with a one-cell halo on every side,
//      H with the low y/z halo, and the ca/cb coefficients of the tile;
//   2. computes H^{n+1/2} on the tile plus the low y row / low z column halo
//      (rfx/core/yee.py:226-291 / :411-453, then rfx/boundaries/cpml.py:804-1065);
//   3. computes E^{n+1} on the tile from those H values and the H of plane
//      i-1 kept in registers (rfx/core/yee.py:347-404 / :456-492, then
//      rfx/boundaries/cpml.py:522-801), applies the PEC faces
//      (rfx/boundaries/pec.py:13-47), the PEC edge mask (pec.py:179-208),
//      soft sources (rfx/simulation.py:1518-1523) and probes (:1565-1567).
// Fields and psi are ping-ponged between two buffers, so halo cells
// recomputed by a neighbour CTA always read step-n values.  CPML work is
// confined to CTAs whose tile touches a y/z slab and to x-slab planes.
#include "rfxb_common.cuh"

namespace rfxb {

#define RFXB_NSTAGE 4
#define RFXB_EW 40   // staged E row: z in [z0 - 4, z0 + 36)
#define RFXB_HW 36   // staged H row: z in [z0 - 4, z0 + 32)

// float counts padded so every array of a stage starts on a 128-byte boundary
// (the alignment TMA writes into shared memory need)
__host__ __device__ constexpr int pad128(int nfloats) { return (nfloats % 32) ? 32 - (nfloats % 32) : 0; }

template <int TY>
struct FwdStageDims {
  static constexpr int NE = 3 * (TY + 2) * RFXB_EW;
  static constexpr int NH = 3 * (TY + 1) * RFXB_HW;
  static constexpr int NC = 2 * TY * RFXB_TZ;
  static constexpr int PE = pad128(NE) ? pad128(NE) : 32;
  static constexpr int PH = pad128(NE + PE + NH) ? pad128(NE + PE + NH) : 32;
  static constexpr unsigned BYTES = 4u * (NE + NH + NC);   // bytes the TMA boxes deliver
};

template <int TY>
struct __align__(128) FwdStage {
  float e[3][TY + 2][RFXB_EW];   // ex ey ez, rows y0-1 .. y0+TY
  float pe[FwdStageDims<TY>::PE];
  float h[3][TY + 1][RFXB_HW];   // hx hy hz (H^{n-1/2}), rows y0-1 .. y0+TY-1
  float ph[FwdStageDims<TY>::PH];
  float cab[2][TY][RFXB_TZ];     // ca cb, rows y0 .. y0+TY-1, z from z0
};

template <int TY>
struct FwdSmem {
  FwdStage<TY> st[RFXB_NSTAGE];      // plane p lives in stage (p + 1) & 3
  float h[3][TY + 1][RFXB_TZ + 1];   // H^{n+1/2} of plane i: [y - y0 + 1][z - z0 + 1]
  RfxbInst P;
  unsigned long long mbar[RFXB_NSTAGE];
};

__device__ __forceinline__ int stage_of(int p) { return (p + 1) & (RFXB_NSTAGE - 1); }

// Per-CTA constants kept in registers.
struct FwdCtx {
  int nx, ny, nz, zs, ncp, par;
  long long ps, off0, cs;
  const float* Fi;
  float* Fo;
  const float* ch;
  float ch0;
  bool cpx, cpy, cpz;      // CPML axis active (y/z: and this tile touches a slab)
};

// H^{n+1/2} components selected by MASK (1 hx, 2 hy, 4 hz) at (i, jj, kk).
// (ly, lz): the cell's row and z index in the staged planes (lz = k - z0 + 4).
template <int TY, int MASK>
__device__ __forceinline__ void h_cell(const RfxbInst& P, const FwdSmem<TY>& S, const FwdCtx& C,
                                       int b0, int b1, int i, int jj, int kk, int ly, int lz,
                                       float xh, float yh, float zh, bool write_psi,
                                       float& hx, float& hy, float& hz) {
  const FwdStage<TY>& A = S.st[b0];
  const FwdStage<TY>& B = S.st[b1];
  const float Ex = A.e[0][ly][lz], Ey = A.e[1][ly][lz], Ez = A.e[2][ly][lz];
  const float dEz_y = A.e[2][ly + 1][lz] - Ez;
  const float dEy_z = A.e[1][ly][lz + 1] - Ey;
  const float dEx_z = A.e[0][ly][lz + 1] - Ex;
  const float dEz_x = B.e[2][ly][lz] - Ez;
  const float dEy_x = B.e[1][ly][lz] - Ey;
  const float dEx_y = A.e[0][ly + 1][lz] - Ex;
  float chc = C.ch0;
  if (C.ch) chc = C.ch[C.off0 + (long long)i * C.ps + (long long)jj * C.zs + kk];
  if (MASK & 1) hx = A.h[0][ly][lz] - chc * (dEz_y * yh - dEy_z * zh);
  if (MASK & 2) hy = A.h[1][ly][lz] - chc * (dEx_z * zh - dEz_x * xh);
  if (MASK & 4) hz = A.h[2][ly][lz] - chc * (dEy_x * xh - dEx_y * yh);
  const int n = C.ncp;
  const int par = C.par;
  int s, sd;
  if (C.cpx) {
    sd = cpml_side(i, C.nx, n, s);
    if (sd >= 0) {
      const float* tb = P.cpb + (size_t)sd * 3 * n;
      const float b = __ldg(tb + s), c = __ldg(tb + n + s), km = __ldg(tb + 2 * n + s);
      const float ib = P.ib[sd];
      if (MASK & 2) {  // Hy += ch psi(dEz/dx)
        const long long q = psi_index_x(P, sd, 0, s, jj, kk);
        const float g = dEz_x * ib;
        const float p = b * P.psH[par][0][q] + c * g;
        if (write_psi) P.psH[par ^ 1][0][q] = p;
        hy = hy + chc * p;
        hy = hy + chc * km * g;
      }
      if (MASK & 4) {  // Hz -= ch psi(dEy/dx)
        const long long q = psi_index_x(P, sd, 1, s, jj, kk);
        const float g = dEy_x * ib;
        const float p = b * P.psH[par][0][q] + c * g;
        if (write_psi) P.psH[par ^ 1][0][q] = p;
        hz = hz - chc * p;
        hz = hz - chc * km * g;
      }
    }
  }
  if (C.cpy) {
    sd = cpml_side(jj, C.ny, n, s);
    if (sd >= 0) {
      const float* tb = P.cpb + (size_t)(2 + sd) * 3 * n;
      const float b = __ldg(tb + s), c = __ldg(tb + n + s), km = __ldg(tb + 2 * n + s);
      const float ib = P.ib[2 + sd];
      if (MASK & 1) {  // Hx -= ch psi(dEz/dy)
        const long long q = psi_index_y(P, sd, 0, s, i, kk);
        const float g = dEz_y * ib;
        const float p = b * P.psH[par][1][q] + c * g;
        if (write_psi) P.psH[par ^ 1][1][q] = p;
        hx = hx - chc * p;
        hx = hx - chc * (km * g);
      }
      if (MASK & 4) {  // Hz += ch psi(dEx/dy)
        const long long q = psi_index_y(P, sd, 1, s, i, kk);
        const float g = dEx_y * ib;
        const float p = b * P.psH[par][1][q] + c * g;
        if (write_psi) P.psH[par ^ 1][1][q] = p;
        hz = hz + chc * p;
        hz = hz + chc * (km * g);
      }
    }
  }
  if (C.cpz) {
    sd = cpml_side(kk, C.nz, n, s);
    if (sd >= 0) {
      const float* tb = P.cpb + (size_t)(4 + sd) * 3 * n;
      const float b = __ldg(tb + s), c = __ldg(tb + n + s), km = __ldg(tb + 2 * n + s);
      const float ib = P.ib[4 + sd];
      if (MASK & 1) {  // Hx += ch psi(dEy/dz)
        const long long q = psi_index_z(P, sd, 0, s, i, jj);
        const float g = dEy_z * ib;
        const float p = b * P.psH[par][2][q] + c * g;
        if (write_psi) P.psH[par ^ 1][2][q] = p;
        hx = hx + chc * p;
        hx = hx + chc * (km * g);
      }
      if (MASK & 2) {  // Hy -= ch psi(dEx/dz)
        const long long q = psi_index_z(P, sd, 1, s, i, jj);
        const float g = dEx_z * ib;
        const float p = b * P.psH[par][2][q] + c * g;
        if (write_psi) P.psH[par ^ 1][2][q] = p;
        hy = hy - chc * p;
        hy = hy - chc * (km * g);
      }
    }
  }
}

// Stage plane ip of the input state with 16-byte copies.  Every copy starts on
// a 16-byte boundary: off0, ps, zs, cs and z0 are multiples of 32 elements.
// Rows past the grid read the zero guard row j = ny.
template <int TY>
__device__ __forceinline__ void load_stage(FwdSmem<TY>& S, const FwdCtx& C, const float* ca, const float* cb,
                                           int y0, int z0, int ip, int tid) {
  FwdStage<TY>& D = S.st[stage_of(ip)];
  const long long pb = C.off0 + (long long)ip * C.ps;
  constexpr int RE = (TY + 2) * 10, RH = (TY + 1) * 9, RC = TY * 8;
  constexpr int NE = 3 * RE, NH = 3 * RH, NC = 2 * RC;
  for (int t = tid; t < NE + NH + NC; t += 32 * TY) {
    if (t < NE) {
      const int c = t / RE, u = t - c * RE, r = u / 10, q = u - r * 10;
      const int jj = min(y0 - 1 + r, C.ny);
      cp_async16(&D.e[c][r][4 * q], C.Fi + c * C.cs + pb + (long long)jj * C.zs + (z0 - 4 + 4 * q));
    } else if (t < NE + NH) {
      const int v = t - NE, c = v / RH, u = v - c * RH, r = u / 9, q = u - r * 9;
      const int jj = min(y0 - 1 + r, C.ny);
      cp_async16(&D.h[c][r][4 * q], C.Fi + (3 + c) * C.cs + pb + (long long)jj * C.zs + (z0 - 4 + 4 * q));
    } else {
      const int v = t - NE - NH, c = v / RC, u = v - c * RC, r = u / 8, q = u - r * 8;
      const int jj = min(y0 + r, C.ny);
      cp_async16(&D.cab[c][r][4 * q], (c ? cb : ca) + pb + (long long)jj * C.zs + (z0 + 4 * q));
    }
  }
}

// Issue the TMA boxes of plane ip into its stage (one thread).  Tensor maps of
// an instance: [0|1] field block of parity 0|1 with the E box, [2|3] the same
// with the H box, [4] the coefficient block with the ca/cb box.
template <int TY>
__device__ __forceinline__ void tma_stage(FwdSmem<TY>& S, const CUtensorMap* tm, int par, int y0, int z0, int ip) {
  const int s = stage_of(ip);
  const uint32_t mb = smem_u32(&S.mbar[s]);
  mbar_expect_tx(mb, FwdStageDims<TY>::BYTES);
  tma_load_4d(smem_u32(&S.st[s].e[0][0][0]), tm + par, z0 - 4, y0, ip + 1, 0, mb);
  tma_load_4d(smem_u32(&S.st[s].h[0][0][0]), tm + 2 + par, z0 - 4, y0, ip + 1, 3, mb);
  tma_load_4d(smem_u32(&S.st[s].cab[0][0][0]), tm + 4, z0, y0 + 1, ip + 1, 0, mb);
}

// Planes are loaded in order xa-1, xa, ...; stage (p+1)&3 completes its
// k-th fill on mbarrier phase k, so plane p waits on parity ((p-xa+1)/4) & 1.
__device__ __forceinline__ uint32_t stage_parity(int p, int xa) { return (uint32_t)(((p - xa + 1) >> 2) & 1); }

template <int TY, bool TMA>
__global__ void __launch_bounds__(32 * TY, 4)
fwd_step_kernel(const RfxbInst* __restrict__ insts, const RfxbWork* __restrict__ work,
                const CUtensorMap* __restrict__ maps, int n, int par) {
  __shared__ FwdSmem<TY> S;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + lane;
  const RfxbWork w = work[blockIdx.x];
  load_inst(S.P, insts + w.inst, tid, 32 * TY);
  if (TMA && tid == 0) {
    for (int q = 0; q < RFXB_NSTAGE; ++q) mbar_init(smem_u32(&S.mbar[q]), 1);
    mbar_fence_init();
  }
  __syncthreads();
  const CUtensorMap* tm = maps + (size_t)w.inst * RFXB_NMAPS;
  const RfxbInst& P = S.P;
  FwdCtx C;
  C.nx = P.nx; C.ny = P.ny; C.nz = P.nz; C.zs = P.zs; C.ncp = P.ncp; C.par = par;
  C.ps = P.ps; C.off0 = P.off0; C.cs = P.cs;
  C.Fi = P.F[par][0];
  C.Fo = P.F[par ^ 1][0];
  C.ch = P.ch;
  C.ch0 = P.ch0;
  const int y0 = w.y0, z0 = w.z0;
  C.cpx = C.ncp > 0 && (P.cpml_axes & 1u);
  C.cpy = C.ncp > 0 && (P.cpml_axes & 2u) && (y0 - 1 < C.ncp || y0 + TY - 1 >= C.ny - C.ncp);
  C.cpz = C.ncp > 0 && (P.cpml_axes & 4u) && (z0 - 1 < C.ncp || z0 + 31 >= C.nz - C.ncp);
  const float* ca = P.ca;
  const float* cb = P.cb;
  const int j = y0 + ty, k = z0 + lane;
  const bool own = (j < C.ny) && (k < C.nz);
  const int ly = ty + 1, lz = lane + 4, lh = lane + 1;
  // spacing table entries of this thread's column and of the halo cells
  const float yh = own ? __ldg(P.yh + j) : 0.f, ye = own ? __ldg(P.ye + j) : 0.f;
  const float zh = own ? __ldg(P.zh + k) : 0.f, ze = own ? __ldg(P.ze + k) : 0.f;
  const bool row_halo = (ty == 0) && (y0 >= 1) && (k < C.nz);
  const float yh_row = row_halo ? __ldg(P.yh + y0 - 1) : 0.f;
  const int hcw = TY > 1 ? 1 : 0;                       // warp computing the z halo column
  const bool col_halo = (ty == hcw) && (lane < TY) && (z0 >= 1) && (y0 + lane < C.ny);
  const float yh_col = col_halo ? __ldg(P.yh + y0 + lane) : 0.f;
  const float zh_col = col_halo ? __ldg(P.zh + z0 - 1) : 0.f;

  // Sources and probes whose (j, k) is this thread's column.
  unsigned smask = 0u, pmask = 0u;
  if (own) {
    const int ns = min(P.nsrc, 32);
    for (int s = 0; s < ns; ++s) {
      const int4 c = __ldg(P.src + s);
      if (c.y == j && c.z == k) smask |= 1u << s;
    }
    const int np = min(P.nprb, 32);
    for (int p = 0; p < np; ++p) {
      const int4 c = __ldg(P.prb + p);
      if (c.y == j && c.z == k) pmask |= 1u << p;
    }
  }
  const bool src_tail = P.nsrc > 32, prb_tail = P.nprb > 32;
  const unsigned pec = P.pec_axes;
  const bool pec_j = ((pec & 2u) != 0) && (j == 0 || j == C.ny - 1);
  const bool pec_k0 = ((pec & 4u) != 0) && (k == 0 || k == C.nz - 1);
  const bool pec_kz = ((pec & 4u) != 0) && (k == C.nz - 1);

  const int xa = w.xa, xb = w.xb;
  // A wait that runs out marks the launch failed and leaves the CTA after
  // draining the boxes it issued (a stalled copy cannot be waited out forever).
  auto bail = [&](int last_issued, int from) {
    if (tid == 0) {
      atomicOr(P.status, 1);
      for (int p = from; p <= last_issued; ++p) mbar_wait_bounded(smem_u32(&S.mbar[stage_of(p)]), stage_parity(p, xa));
    }
  };
  if (TMA) {
    if (tid == 0) {
      for (int p = xa - 1; p <= min(xa + 2, C.nx); ++p) tma_stage<TY>(S, tm, par, y0, z0, p);
    }
    const bool ok = mbar_wait_bounded(smem_u32(&S.mbar[stage_of(xa - 1)]), stage_parity(xa - 1, xa)) &&
                    mbar_wait_bounded(smem_u32(&S.mbar[stage_of(xa)]), stage_parity(xa, xa));
    if (__syncthreads_or(!ok)) { bail(min(xa + 2, C.nx), xa - 1); return; }
  } else {
    // pipeline: planes xa-1 and xa (group 0), xa+1 (group 1), xa+2 (group 2)
    load_stage<TY>(S, C, ca, cb, y0, z0, xa - 1, tid);
    load_stage<TY>(S, C, ca, cb, y0, z0, xa, tid);
    cp_async_commit();
    load_stage<TY>(S, C, ca, cb, y0, z0, xa + 1, tid);
    cp_async_commit();
    if (xa + 2 <= C.nx) load_stage<TY>(S, C, ca, cb, y0, z0, xa + 2, tid);
    cp_async_commit();
    cp_async_wait<2>();
    __syncthreads();
  }

  // H of plane xa-1 at this column (computed, not stored: its owner stores it).
  float hy_prev = 0.f, hz_prev = 0.f;
  if (xa > 0 && own) {
    float hx_, hy_, hz_;
    const float xhp = __ldg(P.xh + xa - 1);
    h_cell<TY, 6>(P, S, C, stage_of(xa - 1), stage_of(xa), xa - 1, j, k, ly, lz, xhp, yh, zh, false,
                  hx_, hy_, hz_);
    hy_prev = hy_;
    hz_prev = hz_;
  }

  const bool has_hist = P.hist != nullptr && (n - P.hist_step0) >= 0 && (n - P.hist_step0) < P.hist_nsteps;
  const bool has_emask = P.emask != nullptr;

  for (int i = xa; i < xb; ++i) {
    if (TMA) {
      // plane i+1 has landed; after the barrier every thread is done with
      // plane i-1, whose stage takes plane i+3
      const bool ok = mbar_wait_bounded(smem_u32(&S.mbar[stage_of(i + 1)]), stage_parity(i + 1, xa));
      if (__syncthreads_or(!ok)) { bail(min(i + 2, C.nx), i + 1); return; }
      if (tid == 0 && i + 3 <= C.nx) tma_stage<TY>(S, tm, par, y0, z0, i + 3);
    } else {
      cp_async_wait<1>();   // planes up to i+1 have landed (i+2 may be in flight)
      __syncthreads();      // ... for every thread; plane i-1's stage is free
      if (i + 3 <= C.nx) load_stage<TY>(S, C, ca, cb, y0, z0, i + 3, tid);
      cp_async_commit();
    }
    const int b0 = stage_of(i), b1 = stage_of(i + 1);
    const float xh = __ldg(P.xh + i), xe = __ldg(P.xe + i);

    // ---- H phase ----
    float hx = 0.f, hy = 0.f, hz = 0.f;
    const long long e = C.off0 + (long long)i * C.ps + (long long)j * C.zs + k;
    if (own) {
      h_cell<TY, 7>(P, S, C, b0, b1, i, j, k, ly, lz, xh, yh, zh, true, hx, hy, hz);
      C.Fo[3 * C.cs + e] = hx;
      C.Fo[4 * C.cs + e] = hy;
      C.Fo[5 * C.cs + e] = hz;
    }
    S.h[0][ly][lh] = hx;
    S.h[1][ly][lh] = hy;
    S.h[2][ly][lh] = hz;
    if (ty == 0) {  // halo row j = y0 - 1: hx, hz
      float a = 0.f, bq = 0.f, cq = 0.f;
      if (row_halo) h_cell<TY, 5>(P, S, C, b0, b1, i, y0 - 1, k, 0, lz, xh, yh_row, zh, false, a, bq, cq);
      S.h[0][0][lh] = a;
      S.h[2][0][lh] = cq;
    }
    if (ty == hcw && lane < TY) {  // halo column k = z0 - 1: hx, hy
      float a = 0.f, bq = 0.f, cq = 0.f;
      if (col_halo) h_cell<TY, 3>(P, S, C, b0, b1, i, y0 + lane, z0 - 1, lane + 1, 3, xh, yh_col, zh_col, false,
                                  a, bq, cq);
      S.h[0][lane + 1][0] = a;
      S.h[1][lane + 1][0] = bq;
    }
    __syncthreads();

    // ---- E phase ----
    if (own) {
      const FwdStage<TY>& A = S.st[b0];
      const float Ex = A.e[0][ly][lz], Ey = A.e[1][ly][lz], Ez = A.e[2][ly][lz];
      const float dHz_y = hz - S.h[2][ly - 1][lh];
      const float dHy_z = hy - S.h[1][ly][lh - 1];
      const float dHx_z = hx - S.h[0][ly][lh - 1];
      const float dHz_x = hz - hz_prev;
      const float dHy_x = hy - hy_prev;
      const float dHx_y = hx - S.h[0][ly - 1][lh];
      const float cx = dHz_y * ye - dHy_z * ze;
      const float cy = dHx_z * ze - dHz_x * xe;
      const float cz = dHy_x * xe - dHx_y * ye;
      const float cav = A.cab[0][ty][lane], cbv = A.cab[1][ty][lane];
      float ex = cav * Ex + cbv * cx;
      float ey = cav * Ey + cbv * cy;
      float ez = cav * Ez + cbv * cz;
      const int ncp = C.ncp;
      if (C.cpx || C.cpy || C.cpz) {
        int s, sd;
        float ce = 0.f;
        bool ce_loaded = false;
        if (C.cpx) {
          sd = cpml_side(i, C.nx, ncp, s);
          if (sd >= 0) {
            ce = P.ce[e];
            ce_loaded = true;
            const float* tb = P.cpb + (size_t)sd * 3 * ncp;
            const float b = __ldg(tb + s), c = __ldg(tb + ncp + s), km = __ldg(tb + 2 * ncp + s);
            const float ib = P.ib[sd];
            {  // Ey -= ce psi(dHz/dx)
              const long long q = psi_index_x(P, sd, 0, s, j, k);
              const float g = dHz_x * ib;
              const float p = b * P.psE[par][0][q] + c * g;
              P.psE[par ^ 1][0][q] = p;
              ey = ey - ce * p;
              ey = ey - ce * km * g;
            }
            {  // Ez += ce psi(dHy/dx)
              const long long q = psi_index_x(P, sd, 1, s, j, k);
              const float g = dHy_x * ib;
              const float p = b * P.psE[par][0][q] + c * g;
              P.psE[par ^ 1][0][q] = p;
              ez = ez + ce * p;
              ez = ez + ce * km * g;
            }
          }
        }
        if (C.cpy) {
          sd = cpml_side(j, C.ny, ncp, s);
          if (sd >= 0) {
            if (!ce_loaded) { ce = P.ce[e]; ce_loaded = true; }
            const float* tb = P.cpb + (size_t)(2 + sd) * 3 * ncp;
            const float b = __ldg(tb + s), c = __ldg(tb + ncp + s), km = __ldg(tb + 2 * ncp + s);
            const float ib = P.ib[2 + sd];
            {  // Ex += ce psi(dHz/dy)
              const long long q = psi_index_y(P, sd, 0, s, i, k);
              const float g = dHz_y * ib;
              const float p = b * P.psE[par][1][q] + c * g;
              P.psE[par ^ 1][1][q] = p;
              ex = ex + ce * p;
              ex = ex + ce * (km * g);
            }
            {  // Ez -= ce psi(dHx/dy)
              const long long q = psi_index_y(P, sd, 1, s, i, k);
              const float g = dHx_y * ib;
              const float p = b * P.psE[par][1][q] + c * g;
              P.psE[par ^ 1][1][q] = p;
              ez = ez - ce * p;
              ez = ez - ce * (km * g);
            }
          }
        }
        if (C.cpz) {
          sd = cpml_side(k, C.nz, ncp, s);
          if (sd >= 0) {
            if (!ce_loaded) { ce = P.ce[e]; ce_loaded = true; }
            const float* tb = P.cpb + (size_t)(4 + sd) * 3 * ncp;
            const float b = __ldg(tb + s), c = __ldg(tb + ncp + s), km = __ldg(tb + 2 * ncp + s);
            const float ib = P.ib[4 + sd];
            {  // Ex -= ce psi(dHy/dz)
              const long long q = psi_index_z(P, sd, 0, s, i, j);
              const float g = dHy_z * ib;
              const float p = b * P.psE[par][2][q] + c * g;
              P.psE[par ^ 1][2][q] = p;
              ex = ex - ce * p;
              ex = ex - ce * (km * g);
            }
            {  // Ey += ce psi(dHx/dz)
              const long long q = psi_index_z(P, sd, 1, s, i, j);
              const float g = dHx_z * ib;
              const float p = b * P.psE[par][2][q] + c * g;
              P.psE[par ^ 1][2][q] = p;
              ey = ey + ce * p;
              ey = ey + ce * (km * g);
            }
          }
        }
      }
      // PEC faces
      if ((pec & 1u) && (i == 0 || i == C.nx - 1)) { ey = 0.f; ez = 0.f; }
      if (pec_j) { ex = 0.f; ez = 0.f; }
      if (pec_k0) { ex = 0.f; ey = 0.f; }
      if (pec_kz) ez = 0.f;
      if (has_emask) {
        const unsigned m = P.emask[e];
        if (m) {
          ex = ex * (1.f - (float)(m & 1u));
          ey = ey * (1.f - (float)((m >> 1) & 1u));
          ez = ez * (1.f - (float)((m >> 2) & 1u));
        }
      }
      if (has_hist) {
        if (i >= P.hb[0] && i < P.hb[1] && j >= P.hb[2] && j < P.hb[3] && k >= P.hb[4] && k < P.hb[5]) {
          const int sy = P.hb[3] - P.hb[2], sz = P.hb[5] - P.hb[4];
          const int hc = (P.hb[1] - P.hb[0]) * sy * sz;
          const int ci = ((i - P.hb[0]) * sy + (j - P.hb[2])) * sz + (k - P.hb[4]);
          float* hp = P.hist + (long long)(n - P.hist_step0) * P.hist_ld + ci;
          hp[0] = Ex; hp[hc] = Ey; hp[2 * hc] = Ez;
          hp[3 * hc] = cx; hp[4 * hc] = cy; hp[5 * hc] = cz;
        }
      }
      if (pmask | smask | (unsigned)src_tail | (unsigned)prb_tail) {
        auto sample = [&](int p, int pre) {
          const int4 c = __ldg(P.prb + p);
          if (c.x != i || ((c.w >> 4) & 1) != pre) return;
          const int comp = c.w & 7;
          const float v = comp == 0 ? ex : comp == 1 ? ey : comp == 2 ? ez : comp == 3 ? hx : comp == 4 ? hy : hz;
          P.prb_out[(long long)n * P.prb_ld + p] = v;
        };
        auto inject = [&](int s) {
          const int4 c = __ldg(P.src + s);
          if (c.x != i) return;
          const float v = __ldg(P.srcw + (long long)n * P.src_ld + s);
          if (c.w == 0) ex = ex + v; else if (c.w == 1) ey = ey + v; else ez = ez + v;
        };
        if (P.prb_out) {
          for (unsigned m = pmask; m; m &= m - 1) sample(__ffs(m) - 1, 1);
          if (prb_tail)
            for (int p = 32; p < P.nprb; ++p) { const int4 c = __ldg(P.prb + p); if (c.y == j && c.z == k) sample(p, 1); }
        }
        for (unsigned m = smask; m; m &= m - 1) inject(__ffs(m) - 1);
        if (src_tail)
          for (int s = 32; s < P.nsrc; ++s) { const int4 c = __ldg(P.src + s); if (c.y == j && c.z == k) inject(s); }
        if (P.prb_out) {
          for (unsigned m = pmask; m; m &= m - 1) sample(__ffs(m) - 1, 0);
          if (prb_tail)
            for (int p = 32; p < P.nprb; ++p) { const int4 c = __ldg(P.prb + p); if (c.y == j && c.z == k) sample(p, 0); }
        }
      }
      C.Fo[e] = ex;
      C.Fo[C.cs + e] = ey;
      C.Fo[2 * C.cs + e] = ez;
    }
    hy_prev = hy;
    hz_prev = hz;
  }
  if (!TMA) cp_async_wait<0>();
}

// Running DFT of one plane per launch entry, Kahan-compensated
// (the plain sum of rfx/simulation.py:1574-1588 / rfx/nonuniform.py:1458-1472).
__global__ void dft_kernel(const RfxbInst* __restrict__ insts, const RfxbDftPlane* __restrict__ planes,
                           int nplanes, int n, int par) {
  int q = 0;
  while (q + 1 < nplanes && planes[q + 1].block0 <= (int)blockIdx.x) ++q;
  const RfxbDftPlane& D = planes[q];
  const RfxbInst& P = insts[D.inst];
  const int c = (blockIdx.x - D.block0) * blockDim.x + threadIdx.x;
  const int cells = D.n1 * D.n2;
  if (c >= cells) return;
  const int a = c / D.n2, b = c - a * D.n2;
  int i, j, k;
  if (D.axis == 0) { i = D.index; j = a; k = b; }
  else if (D.axis == 1) { i = a; j = D.index; k = b; }
  else { i = a; j = b; k = D.index; }
  const float v = P.F[par][D.comp][P.off0 + (long long)i * P.ps + (long long)j * P.zs + k];
  const float2* ph = D.phase + (long long)n * D.nf;
  for (int f = 0; f < D.nf; ++f) {
    const float2 w = __ldg(ph + f);
    const long long o = (long long)f * cells + c;
    float2 s = D.acc[o], r = D.cmp[o];
    float y = v * w.x - r.x;
    float t = s.x + y;
    r.x = (t - s.x) - y;
    s.x = t;
    y = v * w.y - r.y;
    t = s.y + y;
    r.y = (t - s.y) - y;
    s.y = t;
    D.acc[o] = s;
    D.cmp[o] = r;
  }
}

// Reference layout (nx, ny, nz) <-> internal padded layout.
__global__ void pack_kernel(float* __restrict__ dst, const float* __restrict__ src, RfxbInst P) {
  const long long total = (long long)P.nx * P.ny * P.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % P.nz);
    const long long r = t / P.nz;
    const int j = (int)(r % P.ny);
    const int i = (int)(r / P.ny);
    dst[P.off0 + (long long)i * P.ps + (long long)j * P.zs + k] = src[t];
  }
}

__global__ void unpack_kernel(float* __restrict__ dst, const float* __restrict__ src, RfxbInst P) {
  const long long total = (long long)P.nx * P.ny * P.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % P.nz);
    const long long r = t / P.nz;
    const int j = (int)(r % P.ny);
    const int i = (int)(r / P.ny);
    dst[t] = src[P.off0 + (long long)i * P.ps + (long long)j * P.zs + k];
  }
}

// Per-cell update coefficients in float32 with the reference's operation order:
// ca, cb from rfx/core/yee.py:387-393, ce from rfx/boundaries/cpml.py:536,
// ch from rfx/boundaries/cpml.py:818.
__global__ void coef_kernel(RfxbInst P, float* ca, float* cb, float* ce, float* ch,
                            const float* __restrict__ eps_r, const float* __restrict__ sigma,
                            const float* __restrict__ mu_r, const unsigned char* __restrict__ emask_ref,
                            unsigned char* emask, float dtf) {
  const long long total = (long long)P.nx * P.ny * P.nz;
  const float eps0 = (float)kEps0, mu0 = (float)kMu0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % P.nz);
    const long long r = t / P.nz;
    const int j = (int)(r % P.ny);
    const int i = (int)(r / P.ny);
    const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
    const float eps = eps_r[t] * eps0;
    const float s2 = (sigma[t] * dtf) / (2.0f * eps);
    ca[e] = (1.0f - s2) / (1.0f + s2);
    cb[e] = (dtf / eps) / (1.0f + s2);
    ce[e] = dtf / eps;
    if (ch) ch[e] = dtf / (mu_r[t] * mu0);
    if (emask) emask[e] = emask_ref ? emask_ref[t] : (unsigned char)0;
  }
}

// Explicit template instantiations used by the host side.
template __global__ void fwd_step_kernel<8, true>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);
template __global__ void fwd_step_kernel<8, false>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);

}  // namespace rfxb
