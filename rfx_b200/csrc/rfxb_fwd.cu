// Forward time step of the Yee/CPML leapfrog: one fused kernel per step.
//
// One CTA owns a (TY x 32) tile of the (y, z) plane and marches along x over
// an x range [xa, xb).  For each x plane it
//   1. stages E^n of planes i and i+1 (with a one-cell y/z halo) in shared
//      memory through cp.async, prefetching plane i+2 one iteration ahead;
//   2. computes H^{n+1/2} on the tile plus the low y row / low z column halo
//      (rfx/core/yee.py:226-291 / :411-453, then rfx/boundaries/cpml.py:804-1065);
//   3. computes E^{n+1} on the tile from those H values and the H of plane
//      i-1 kept in registers (rfx/core/yee.py:347-404 / :456-492, then
//      rfx/boundaries/cpml.py:522-801), applies the PEC faces
//      (rfx/boundaries/pec.py:13-47), the PEC edge mask (pec.py:179-208),
//      soft sources (rfx/simulation.py:1518-1523) and probes (:1565-1567).
// Fields and H-side CPML psi are ping-ponged between two buffers, so halo
// cells recomputed by a neighbour CTA always read step-n values.
#include "rfxb_common.cuh"

namespace rfxb {

#define RFXB_NSTAGE 4

// One pipeline stage holds everything the step reads from plane i of the
// input state: E with a one-cell halo on every side, H with the low y/z halo,
// and the ca/cb coefficients of the tile.
template <int TY>
struct FwdStage {
  float e[3][TY + 2][RFXB_TZ + 2];     // [ex,ey,ez][y - y0 + 1][z - z0 + 1]
  float h[3][TY + 1][RFXB_TZ + 1];     // [hx,hy,hz][y - y0 + 1][z - z0 + 1] (H^{n-1/2})
  float cab[2][TY][RFXB_TZ];           // [ca,cb][y - y0][z - z0]
};

template <int TY>
struct FwdSmem {
  FwdStage<TY> st[RFXB_NSTAGE];        // planes i-1 .. i+2 (buffer (p + 1) & 3)
  float h[3][TY + 1][RFXB_TZ + 1];     // H^{n+1/2} of plane i with the low y/z halo
  RfxbInst P;
};

__device__ __forceinline__ int stage_of(int p) { return (p + 1) & (RFXB_NSTAGE - 1); }

// H^{n+1/2} components selected by MASK (1 hx, 2 hy, 4 hz) at (i, jj, kk).
// E of plane i is in buffer b0 and of plane i+1 in b1; (ly, lz) are the
// cell's shared-memory coordinates.  psi is written only for owned cells.
template <int TY, int MASK>
__device__ __forceinline__ void h_cell(const RfxbInst& P, const FwdSmem<TY>& S, int par,
                                       int b0, int b1, int i, int jj, int kk, int ly, int lz,
                                       bool write_psi, float& hx, float& hy, float& hz) {
  const FwdStage<TY>& A = S.st[b0];
  const FwdStage<TY>& B = S.st[b1];
  const float Ex = A.e[0][ly][lz], Ey = A.e[1][ly][lz], Ez = A.e[2][ly][lz];
  const float dEz_y = A.e[2][ly + 1][lz] - Ez;
  const float dEy_z = A.e[1][ly][lz + 1] - Ey;
  const float dEx_z = A.e[0][ly][lz + 1] - Ex;
  const float dEz_x = B.e[2][ly][lz] - Ez;
  const float dEy_x = B.e[1][ly][lz] - Ey;
  const float dEx_y = A.e[0][ly + 1][lz] - Ex;
  float chc = P.ch0;
  if (P.ch) chc = P.ch[P.off0 + (long long)i * P.ps + (long long)jj * P.zs + kk];
  const float xh = __ldg(P.xh + i), yh = __ldg(P.yh + jj), zh = __ldg(P.zh + kk);
  if (MASK & 1) hx = A.h[0][ly][lz] - chc * (dEz_y * yh - dEy_z * zh);
  if (MASK & 2) hy = A.h[1][ly][lz] - chc * (dEx_z * zh - dEz_x * xh);
  if (MASK & 4) hz = A.h[2][ly][lz] - chc * (dEy_x * xh - dEx_y * yh);
  const int n = P.ncp;
  if (n == 0) return;
  int s, sd;
  if (P.cpml_axes & 1u) {
    sd = cpml_side(i, P.nx, n, s);
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
  if (P.cpml_axes & 2u) {
    sd = cpml_side(jj, P.ny, n, s);
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
  if (P.cpml_axes & 4u) {
    sd = cpml_side(kk, P.nz, n, s);
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

// Stage plane ip of the input state: E (rows y0-1..y0+TY, cols z0-1..z0+32),
// H (rows y0-1..y0+TY-1, cols z0-1..z0+31) and ca/cb of the tile.  Rows past
// the grid read the zero guard row j = ny.
template <int TY>
__device__ __forceinline__ void load_stage(const RfxbInst& P, FwdSmem<TY>& S, const float* const* F,
                                           int y0, int z0, int ip, int ty, int lane) {
  FwdStage<TY>& D = S.st[stage_of(ip)];
  const long long pbase = P.off0 + (long long)ip * P.ps + (z0 - 1);
  for (int r = ty; r < TY + 2; r += TY) {
    const int jj = min(y0 - 1 + r, P.ny);
    const long long rb = pbase + (long long)jj * P.zs;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cp_async4(&D.e[c][r][lane], F[c] + rb + lane);
      if (lane < 2) cp_async4(&D.e[c][r][32 + lane], F[c] + rb + 32 + lane);
    }
    if (r < TY + 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cp_async4(&D.h[c][r][lane], F[3 + c] + rb + lane);
        if (lane == 0) cp_async4(&D.h[c][r][32], F[3 + c] + rb + 32);
      }
    }
  }
  {
    const int jj = min(y0 + ty, P.ny);
    const long long o = P.off0 + (long long)ip * P.ps + (long long)jj * P.zs + z0 + lane;
    cp_async4(&D.cab[0][ty][lane], P.ca + o);
    cp_async4(&D.cab[1][ty][lane], P.cb + o);
  }
}

template <int TY>
__global__ void __launch_bounds__(32 * TY)
fwd_step_kernel(const RfxbInst* __restrict__ insts, const RfxbWork* __restrict__ work, int n, int par) {
  __shared__ FwdSmem<TY> S;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + lane;
  const RfxbWork w = work[blockIdx.x];
  load_inst(S.P, insts + w.inst, tid, 32 * TY);
  __syncthreads();
  const RfxbInst& P = S.P;
  const int j = w.y0 + ty, k = w.z0 + lane;
  const bool own = (j < P.ny) && (k < P.nz);
  const int ly = ty + 1, lz = lane + 1;

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
  const float* const* Fin = P.F[par];
  float* const* Fout = P.F[par ^ 1];

  const int xa = w.xa, xb = w.xb;
  // pipeline: planes xa-1 and xa (group 0), xa+1 (group 1), xa+2 (group 2)
  load_stage<TY>(P, S, Fin, w.y0, w.z0, xa - 1, ty, lane);
  load_stage<TY>(P, S, Fin, w.y0, w.z0, xa, ty, lane);
  cp_async_commit();
  load_stage<TY>(P, S, Fin, w.y0, w.z0, xa + 1, ty, lane);
  cp_async_commit();
  if (xa + 2 <= P.nx) load_stage<TY>(P, S, Fin, w.y0, w.z0, xa + 2, ty, lane);
  cp_async_commit();
  cp_async_wait<2>();
  __syncthreads();

  // H of plane xa-1 at this column (computed, not stored: its owner stores it).
  float hy_prev = 0.f, hz_prev = 0.f;
  if (xa > 0 && own) {
    float hx_, hy_, hz_;
    h_cell<TY, 6>(P, S, par, stage_of(xa - 1), stage_of(xa), xa - 1, j, k, ly, lz, false, hx_, hy_, hz_);
    hy_prev = hy_;
    hz_prev = hz_;
  }

  const bool has_hist = P.hist != nullptr && (n - P.hist_step0) >= 0 && (n - P.hist_step0) < P.hist_nsteps;

  for (int i = xa; i < xb; ++i) {
    cp_async_wait<1>();   // planes up to i+1 have landed (i+2 may be in flight)
    __syncthreads();      // ... for every thread; plane i-1's stage is free
    if (i + 3 <= P.nx) load_stage<TY>(P, S, Fin, w.y0, w.z0, i + 3, ty, lane);
    cp_async_commit();
    const int b0 = stage_of(i), b1 = stage_of(i + 1);

    // ---- H phase ----
    float hx = 0.f, hy = 0.f, hz = 0.f;
    const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
    if (own) {
      h_cell<TY, 7>(P, S, par, b0, b1, i, j, k, ly, lz, true, hx, hy, hz);
      Fout[3][e] = hx;
      Fout[4][e] = hy;
      Fout[5][e] = hz;
    }
    S.h[0][ly][lz] = hx;
    S.h[1][ly][lz] = hy;
    S.h[2][ly][lz] = hz;
    if (ty == 0) {  // halo row j = y0 - 1: hx, hz
      float a = 0.f, bq = 0.f, cq = 0.f;
      const int jh = w.y0 - 1;
      if (jh >= 0 && k < P.nz) h_cell<TY, 5>(P, S, par, b0, b1, i, jh, k, 0, lz, false, a, bq, cq);
      S.h[0][0][lz] = a;
      S.h[1][0][lz] = 0.f;
      S.h[2][0][lz] = cq;
    }
    if (ty == (TY > 1 ? 1 : 0) && lane < TY) {  // halo column k = z0 - 1: hx, hy
      float a = 0.f, bq = 0.f, cq = 0.f;
      const int jc = w.y0 + lane, kh = w.z0 - 1;
      if (kh >= 0 && jc < P.ny) h_cell<TY, 3>(P, S, par, b0, b1, i, jc, kh, lane + 1, 0, false, a, bq, cq);
      S.h[0][lane + 1][0] = a;
      S.h[1][lane + 1][0] = bq;
      S.h[2][lane + 1][0] = 0.f;
    }
    __syncthreads();

    // ---- E phase ----
    if (own) {
      const FwdStage<TY>& A = S.st[b0];
      const float Ex = A.e[0][ly][lz], Ey = A.e[1][ly][lz], Ez = A.e[2][ly][lz];
      const float dHz_y = hz - S.h[2][ly - 1][lz];
      const float dHy_z = hy - S.h[1][ly][lz - 1];
      const float dHx_z = hx - S.h[0][ly][lz - 1];
      const float dHz_x = hz - hz_prev;
      const float dHy_x = hy - hy_prev;
      const float dHx_y = hx - S.h[0][ly - 1][lz];
      const float xe = __ldg(P.xe + i), ye = __ldg(P.ye + j), ze = __ldg(P.ze + k);
      const float cx = dHz_y * ye - dHy_z * ze;
      const float cy = dHx_z * ze - dHz_x * xe;
      const float cz = dHy_x * xe - dHx_y * ye;
      const float ca = A.cab[0][ty][lane], cb = A.cab[1][ty][lane];
      float ex = ca * Ex + cb * cx;
      float ey = ca * Ey + cb * cy;
      float ez = ca * Ez + cb * cz;
      const int ncp = P.ncp;
      if (ncp) {
        int s, sd;
        float ce = 0.f;
        bool ce_loaded = false;
        if (P.cpml_axes & 1u) {
          sd = cpml_side(i, P.nx, ncp, s);
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
        if (P.cpml_axes & 2u) {
          sd = cpml_side(j, P.ny, ncp, s);
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
        if (P.cpml_axes & 4u) {
          sd = cpml_side(k, P.nz, ncp, s);
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
      if (P.pec_axes & 1u) if (i == 0 || i == P.nx - 1) { ey = 0.f; ez = 0.f; }
      if (P.pec_axes & 2u) if (j == 0 || j == P.ny - 1) { ex = 0.f; ez = 0.f; }
      if (P.pec_axes & 4u) {
        if (k == 0 || k == P.nz - 1) { ex = 0.f; ey = 0.f; }
        if (k == P.nz - 1) ez = 0.f;
      }
      if (P.emask) {
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
        if (prb_tail) for (int p = 32; p < P.nprb; ++p) { const int4 c = __ldg(P.prb + p); if (c.y == j && c.z == k) sample(p, 1); }
      }
      for (unsigned m = smask; m; m &= m - 1) inject(__ffs(m) - 1);
      if (src_tail) for (int s = 32; s < P.nsrc; ++s) { const int4 c = __ldg(P.src + s); if (c.y == j && c.z == k) inject(s); }
      if (P.prb_out) {
        for (unsigned m = pmask; m; m &= m - 1) sample(__ffs(m) - 1, 0);
        if (prb_tail) for (int p = 32; p < P.nprb; ++p) { const int4 c = __ldg(P.prb + p); if (c.y == j && c.z == k) sample(p, 0); }
      }
      Fout[0][e] = ex;
      Fout[1][e] = ey;
      Fout[2][e] = ez;
    }
    hy_prev = hy;
    hz_prev = hz;
  }
  cp_async_wait<0>();
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
template __global__ void fwd_step_kernel<8>(const RfxbInst*, const RfxbWork*, int, int);
template __global__ void fwd_step_kernel<4>(const RfxbInst*, const RfxbWork*, int, int);

}  // namespace rfxb
