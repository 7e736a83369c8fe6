// Forward time step of the Yee/CPML leapfrog: one fused kernel per step.
//
// One CTA owns a (TY x 32) tile of the (y, z) plane and marches along x over
// an x range [xa, xb).  For each x plane i it
//   1. keeps a 4-stage pipeline of the input planes i-1 .. i+2 in shared
//      memory: E with a one-cell halo on every side, H with the low y/z halo,
//      and the ca/cb coefficients of the tile (TMA boxes, or 16-byte cp.async
//      copies in the generic mode);
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
//
// Modes (template MODE):
//   0  generic: cp.async staging, psi read and written in global memory;
//   1  TMA staging, no CPML in the launch;
//   2  TMA staging, and the psi of every CPML plane/tile (plus ce) arrive by
//      TMA into a two-slot ring one plane ahead, so the slab cells see no
//      global-load latency.  The host selects it when no tile touches both
//      slabs of an axis and the z layers fit the ring.
#include "rfxb_common.cuh"

namespace rfxb {

#define RFXB_NSTAGE 4
#define RFXB_EW 40   // staged E row: z in [z0 - 4, z0 + 36)
#define RFXB_HW 36   // staged H row: z in [z0 - 4, z0 + 32)
#define RFXB_ZPMAX 16  // largest z-psi row (layers rounded up to 4) mode 2 stages

// float counts padded so every array of a stage starts on a 128-byte boundary
// (the alignment TMA writes into shared memory need)
__host__ __device__ constexpr int pad128(int nfloats) { return (nfloats % 32) ? 32 - (nfloats % 32) : 0; }
__host__ __device__ constexpr int up32(int nfloats) { return (nfloats + 31) / 32 * 32; }

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
  unsigned char em[TY][RFXB_TZ]; // PEC edge-mask bits of the tile (staged only when the plan has a mask)
};

template <int TY>
struct FwdSmem {
  FwdStage<TY> st[RFXB_NSTAGE];      // plane p lives in stage (p + 1) & 3
  float h[3][TY + 1][RFXB_TZ + 1];   // H^{n+1/2} of plane i: [y - y0 + 1][z - z0 + 1]
  // mode 2: the y / z CPML profiles (b, c/cell, (1/kappa-1)/cell, on) of the
  // halo cells, fixed along the x march: row y0-1 per lane, column z0-1 per
  // row (each entry written and read by the same thread)
  float4 hcp_row[2][RFXB_TZ];
  float4 hcp_col[2][TY];
  RfxbInst P;
  unsigned long long mbar[RFXB_NSTAGE];
  unsigned long long pbar[2];        // psi ring (mode 2)
};

// One slot of the mode-2 psi ring (floats, 128-byte aligned sub-arrays):
//   HX/HY [q][TY+1][36]  H-side psi of the x / y slab, rows y0-1.., z from z0-4
//   HZ    [q][TY+1][n4]  H-side psi of the z slab, rows y0-1.., layer s
//   EX/EY [q][TY][32]    E-side psi of the x / y slab on the tile
//   EZ    [q][TY][n4]    E-side psi of the z slab
//   CE    [TY][32]       ce of the tile
template <int TY>
struct PsiSlot {
  static constexpr int HX = 0;
  static constexpr int HY = HX + up32(2 * (TY + 1) * RFXB_HW);
  static constexpr int HZ = HY + up32(2 * (TY + 1) * RFXB_HW);
  static constexpr int EX = HZ + up32(2 * (TY + 1) * RFXB_ZPMAX);
  static constexpr int EY = EX + up32(2 * TY * RFXB_TZ);
  static constexpr int EZ = EY + up32(2 * TY * RFXB_TZ);
  static constexpr int CE = EZ + up32(2 * TY * RFXB_ZPMAX);
  static constexpr int FLOATS = CE + up32(TY * RFXB_TZ);
  static constexpr unsigned BH = 4u * 2 * (TY + 1) * RFXB_HW;   // bytes of an HX / HY box
  static constexpr unsigned BE = 4u * 2 * TY * RFXB_TZ;         // bytes of an EX / EY box
  static constexpr unsigned BC = 4u * TY * RFXB_TZ;             // bytes of the CE box
};

template <int TY>
__host__ __device__ constexpr size_t fwd_smem_bytes(int mode) {
  return sizeof(FwdSmem<TY>) + (mode == 2 ? 2 * sizeof(float) * PsiSlot<TY>::FLOATS : 0);
}

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

// H^{n+1/2} components selected by MASK (1 hx, 2 hy, 4 hz) at (i, jj, kk),
// CPML read from global memory (mode 0).
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
  if (MASK & 1) hx = yee_h(A.h[0][ly][lz], chc, yee_diff2(dEz_y, yh, dEy_z, zh));
  if (MASK & 2) hy = yee_h(A.h[1][ly][lz], chc, yee_diff2(dEx_z, zh, dEz_x, xh));
  if (MASK & 4) hz = yee_h(A.h[2][ly][lz], chc, yee_diff2(dEy_x, xh, dEx_y, yh));
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

// Mode-2 CPML state of one axis at one cell: whether the cell is in the slab,
// its profile (b, c/cell, (1/kappa-1)/cell) and the element offset of its
// psi entry q = 0 (q = 1 is one q-stride further).
struct CpAx {
  bool on;
  float4 c;
  int off;
};

// Yee part of H^{n+1/2} at one cell plus its mode-2 CPML corrections.  The
// staged psi are read at slot row r (0 = row y0-1), z column lz of the H
// boxes and layer sz of the z box; new psi (WRITE) go to the other parity.
template <int TY, int MASK, bool WRITE>
__device__ __forceinline__ void h_cell2(const RfxbInst& P, const FwdSmem<TY>& S, const float* PS, const FwdCtx& C,
                                        int b0, int b1, int ly, int lz, int r, int sz, float chc,
                                        float xh, float yh, float zh, const CpAx& X, const CpAx& Y, const CpAx& Z,
                                        float& hx, float& hy, float& hz) {
  using L = PsiSlot<TY>;
  const FwdStage<TY>& A = S.st[b0];
  const FwdStage<TY>& B = S.st[b1];
  const float Ex = A.e[0][ly][lz], Ey = A.e[1][ly][lz], Ez = A.e[2][ly][lz];
  const float dEz_y = A.e[2][ly + 1][lz] - Ez;
  const float dEy_z = A.e[1][ly][lz + 1] - Ey;
  const float dEx_z = A.e[0][ly][lz + 1] - Ex;
  const float dEz_x = B.e[2][ly][lz] - Ez;
  const float dEy_x = B.e[1][ly][lz] - Ey;
  const float dEx_y = A.e[0][ly + 1][lz] - Ex;
  if (MASK & 1) hx = yee_h(A.h[0][ly][lz], chc, yee_diff2(dEz_y, yh, dEy_z, zh));
  if (MASK & 2) hy = yee_h(A.h[1][ly][lz], chc, yee_diff2(dEx_z, zh, dEz_x, xh));
  if (MASK & 4) hz = yee_h(A.h[2][ly][lz], chc, yee_diff2(dEy_x, xh, dEx_y, yh));
  constexpr int RH = (TY + 1) * RFXB_HW;   // q stride of an H box
  const int par = C.par;
  if (X.on) {   // Hy += ch psi(dEz/dx) [q0], Hz -= ch psi(dEy/dx) [q1]
    const int o = r * RFXB_HW + lz;
    const int qs = P.ncp * P.ny * P.zs;
    if (MASK & 2) {
      const float p = X.c.x * PS[L::HX + o] + X.c.y * dEz_x;
      if (WRITE) P.psH[par ^ 1][0][X.off] = p;
      hy = hy + chc * p;
      hy = hy + chc * (X.c.z * dEz_x);
    }
    if (MASK & 4) {
      const float p = X.c.x * PS[L::HX + RH + o] + X.c.y * dEy_x;
      if (WRITE) P.psH[par ^ 1][0][X.off + qs] = p;
      hz = hz - chc * p;
      hz = hz - chc * (X.c.z * dEy_x);
    }
  }
  if (Y.on) {   // Hx -= ch psi(dEz/dy) [q0], Hz += ch psi(dEx/dy) [q1]
    const int o = r * RFXB_HW + lz;
    const int qs = P.nx * P.ncp * P.zs;
    if (MASK & 1) {
      const float p = Y.c.x * PS[L::HY + o] + Y.c.y * dEz_y;
      if (WRITE) P.psH[par ^ 1][1][Y.off] = p;
      hx = hx - chc * p;
      hx = hx - chc * (Y.c.z * dEz_y);
    }
    if (MASK & 4) {
      const float p = Y.c.x * PS[L::HY + RH + o] + Y.c.y * dEx_y;
      if (WRITE) P.psH[par ^ 1][1][Y.off + qs] = p;
      hz = hz + chc * p;
      hz = hz + chc * (Y.c.z * dEx_y);
    }
  }
  if (Z.on) {   // Hx += ch psi(dEy/dz) [q0], Hy -= ch psi(dEx/dz) [q1]
    const int n4 = P.ncp4;
    const int o = r * n4 + sz;
    const int qs = P.nx * P.ny * n4;
    if (MASK & 1) {
      const float p = Z.c.x * PS[L::HZ + o] + Z.c.y * dEy_z;
      if (WRITE) P.psH[par ^ 1][2][Z.off] = p;
      hx = hx + chc * p;
      hx = hx + chc * (Z.c.z * dEy_z);
    }
    if (MASK & 2) {
      const float p = Z.c.x * PS[L::HZ + (TY + 1) * n4 + o] + Z.c.y * dEx_z;
      if (WRITE) P.psH[par ^ 1][2][Z.off + qs] = p;
      hy = hy - chc * p;
      hy = hy - chc * (Z.c.z * dEx_z);
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
// with the H box, [4] the coefficient block with the ca/cb box; the
// intermediate block (fin = 2) has its own E and H box maps.
template <int TY, bool EM>
__device__ __forceinline__ void tma_stage(FwdSmem<TY>& S, const CUtensorMap* tm, int fin, int y0, int z0, int ip) {
  const int s = stage_of(ip);
  const uint32_t mb = smem_u32(&S.mbar[s]);
  const int me = fin < 2 ? fin : RFXB_MAP_MIDE, mh = fin < 2 ? 2 + fin : RFXB_MAP_MIDH;
  mbar_expect_tx(mb, FwdStageDims<TY>::BYTES + (EM ? (unsigned)(TY * RFXB_TZ) : 0u));
  if (EM) tma_load_4d(smem_u32(&S.st[s].em[0][0]), tm + RFXB_MAP_EMASK, z0, y0 + 1, ip + 1, 0, mb);
  tma_load_4d(smem_u32(&S.st[s].e[0][0][0]), tm + me, z0 - 4, y0, ip + 1, 0, mb);
  tma_load_4d(smem_u32(&S.st[s].h[0][0][0]), tm + mh, z0 - 4, y0, ip + 1, 3, mb);
  tma_load_4d(smem_u32(&S.st[s].cab[0][0][0]), tm + 4, z0, y0 + 1, ip + 1, 0, mb);
}

// Planes are loaded in order xa-1, xa, ...; stage (p+1)&3 completes its
// k-th fill on mbarrier phase k, so plane p waits on parity ((p-xa+1)/4) & 1.
__device__ __forceinline__ uint32_t stage_parity(int p, int xa) { return (uint32_t)(((p - xa + 1) >> 2) & 1); }

// Which CPML slab of an axis a CTA's cells (rows y0-1 .. y0+TY-1, or z
// columns z0-1 .. z0+31) reach: the side, or -1.  The host guarantees at most
// one side per axis for mode 2.
__device__ __forceinline__ int tile_side(int lo, int hi, int n, int ncp) {
  if (lo < ncp) return 0;
  if (hi >= n - ncp) return 1;
  return -1;
}

// Issue the mode-2 psi boxes of plane p into ring slot `slot` (one thread):
// H and E psi of the x slab when p is in it, of the y / z slab the tile
// reaches, and the ce tile.  Returns whether anything was issued.
template <int TY>
__device__ __forceinline__ void psi_issue(float* slot, uint32_t mb, const CUtensorMap* tm, const RfxbInst& P,
                                          int par, int y0, int z0, int p, bool cpx, int ysd, int zsd) {
  using L = PsiSlot<TY>;
  const int ncp = P.ncp, n4 = P.ncp4;
  int s = 0;
  const int xsd = cpx ? cpml_side(p, P.nx, ncp, s) : -1;
  unsigned bytes = L::BC;
  if (xsd >= 0) bytes += L::BH + L::BE;
  if (ysd >= 0) bytes += L::BH + L::BE;
  if (zsd >= 0) bytes += 4u * 2 * (TY + 1) * n4 + 4u * 2 * TY * n4;
  mbar_expect_tx(mb, bytes);
  if (xsd >= 0) {
    tma_load_4d(smem_u32(slot + L::HX), tm + RFXB_MAP_PSH + 0 + par, z0 - 4, y0 - 1, s, 2 * xsd, mb);
    tma_load_4d(smem_u32(slot + L::EX), tm + RFXB_MAP_PSE + 0 + par, z0, y0, s, 2 * xsd, mb);
  }
  if (ysd >= 0) {
    const int jb = ysd ? P.ny - ncp : 0;
    tma_load_4d(smem_u32(slot + L::HY), tm + RFXB_MAP_PSH + 2 + par, z0 - 4, y0 - 1 - jb, p, 2 * ysd, mb);
    tma_load_4d(smem_u32(slot + L::EY), tm + RFXB_MAP_PSE + 2 + par, z0, y0 - jb, p, 2 * ysd, mb);
  }
  if (zsd >= 0) {
    tma_load_4d(smem_u32(slot + L::HZ), tm + RFXB_MAP_PSH + 4 + par, 0, y0 - 1, p, 2 * zsd, mb);
    tma_load_4d(smem_u32(slot + L::EZ), tm + RFXB_MAP_PSE + 4 + par, 0, y0, p, 2 * zsd, mb);
  }
  tma_load_4d(smem_u32(slot + L::CE), tm + 10, z0, y0 + 1, p + 1, 2, mb);
}

template <int MODE>
struct FwdBounds { static constexpr int MIN_CTAS = 4; };
template <>
struct FwdBounds<2> { static constexpr int MIN_CTAS = 3; };

// One work item (a (TY x 32) tile over an x range) of the forward step.
// Returns false when a bounded wait ran out: the status word is then set and
// every box the CTA issued has been waited for, so the caller must leave.
// EM: the launch's plans have PEC edge masks, staged by TMA with the planes
// (TMA modes); without EM the mask (if any) is read from global memory.
template <int TY, int MODE, bool EM>
__device__ __forceinline__ bool fwd_item(FwdSmem<TY>& S, float* ring, const RfxbInst* __restrict__ insts,
                                         const RfxbWork w, const CUtensorMap* __restrict__ maps, int n, int sel,
                                         StepPhases& ph, const StepFault& fault, bool first_item) {
  constexpr bool TMA = MODE != 0;
  using L = PsiSlot<TY>;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + lane;
  load_inst(S.P, insts + w.inst, tid, 32 * TY);
  __syncthreads();
  const int wlim = fault.wait_limit;
  // the thread that issues the TMA boxes: lane 0 of the last warp (warps 0
  // and 1 compute the halo row and column of H)
  const int producer = 32 * (TY - 1);
  const bool skip_first = first_item && (int)blockIdx.x == fault.cta;
  const CUtensorMap* tm = maps + (size_t)w.inst * RFXB_NMAPS;
  const RfxbInst& P = S.P;
  FwdCtx C;
  // fields in F[fin] -> F[fout], psi parity par -> par ^ 1
  const int fin = sel_in(sel), fout = sel_out(sel), par = sel_psi(sel);
  C.nx = P.nx; C.ny = P.ny; C.nz = P.nz; C.zs = P.zs; C.ncp = P.ncp; C.par = par;
  C.ps = P.ps; C.off0 = P.off0; C.cs = P.cs;
  C.Fi = P.F[fin][0];
  C.Fo = P.F[fout][0];
  C.ch = P.ch;
  C.ch0 = P.ch0;
  const int y0 = w.y0, z0 = w.z0;
  C.cpx = MODE != 1 && C.ncp > 0 && (P.cpml_axes & 1u);
  C.cpy = MODE != 1 && C.ncp > 0 && (P.cpml_axes & 2u) && (y0 - 1 < C.ncp || y0 + TY - 1 >= C.ny - C.ncp);
  C.cpz = MODE != 1 && C.ncp > 0 && (P.cpml_axes & 4u) && (z0 - 1 < C.ncp || z0 + 31 >= C.nz - C.ncp);
  const float* ca = P.ca;
  const float* cb = P.cb;
  const int j = y0 + ty, k = z0 + lane;
  const bool own = (j < C.ny) && (k < C.nz);
  const int ly = ty + 1, lz = lane + 4, lh = lane + 1;
  // spacing table entries of this thread's column and of the halo cells
  const float yh = own ? __ldg(P.yh + j) : 0.f, ye = own ? __ldg(P.ye + j) : 0.f;
  const float zh = own ? __ldg(P.zh + k) : 0.f, ze = own ? __ldg(P.ze + k) : 0.f;
  // The halo H is split over four warps so that none carries more than one
  // extra component: row j = y0-1 hx by warp 0 and hz by warp 2, column
  // k = z0-1 hx by warp 1 and hy by warp 3 (lanes < TY); the TMA producer is
  // the last warp.
  static_assert(TY >= 4, "the halo split needs four warps");
  const int hcw = 1;                                    // warp writing the column halo profiles
  const bool row_w = ty == 0;
  const bool row_halo = row_w && (y0 >= 1) && (k < C.nz);
  const float yh_row = row_halo ? __ldg(P.yh + y0 - 1) : 0.f;
  const bool col_w = (ty == 1) && (lane < TY);
  const bool col_halo = col_w && (z0 >= 1) && (y0 + lane < C.ny);
  const float yh_col = col_halo ? __ldg(P.yh + y0 + lane) : 0.f;
  const float zh_col = col_halo ? __ldg(P.zh + z0 - 1) : 0.f;

  // Mode-2 CPML state: the slab side this tile reaches per axis, and this
  // thread's own-cell profile and psi offsets (y and z are fixed along the
  // x march; x is per plane).
  const int ysd = (MODE == 2 && C.cpy) ? tile_side(y0 - 1, y0 + TY - 1, C.ny, C.ncp) : -1;
  const int zsd = (MODE == 2 && C.cpz) ? tile_side(z0 - 1, z0 + 31, C.nz, C.ncp) : -1;
  const int jb = ysd == 1 ? C.ny - C.ncp : 0;
  const int kb = zsd == 1 ? C.nz - C.ncp : 0;
  CpAx cyo{false, make_float4(0.f, 0.f, 0.f, 0.f), 0}, czo{false, make_float4(0.f, 0.f, 0.f, 0.f), 0};
  if (MODE == 2) {
    const int sy = j - jb, sz = k - kb;
    if (own && ysd >= 0 && sy >= 0 && sy < C.ncp) {
      cyo.on = true;
      cyo.c = __ldg(P.cpt + (2 + ysd) * C.ncp + sy);
      cyo.off = (2 * ysd * C.nx * C.ncp + sy) * C.zs + k;   // + i * ncp * zs per plane
    }
    if (own && zsd >= 0 && sz >= 0 && sz < C.ncp) {
      czo.on = true;
      czo.c = __ldg(P.cpt + (4 + zsd) * C.ncp + sz);
      czo.off = (2 * zsd * C.nx * C.ny + j) * P.ncp4 + sz;    // + i * ny * ncp4 per plane
    }
  }
  const bool psi_tile = ysd >= 0 || zsd >= 0;   // every plane needs the psi ring
  // y / z profiles of the halo cells, fixed along the x march, into shared
  // memory once per item: row y0-1 at this lane's column (warp 0) and column
  // z0-1 at row y0+lane (warp hcw); .w = 1 where the cell is in the slab
  if (MODE == 2) {
    const float4 off = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ty == 0) {
      float4 a = off, b = off;
      if ((y0 >= 1) && (k < C.nz)) {
        const int sy = y0 - 1 - jb;
        if (ysd >= 0 && sy >= 0 && sy < C.ncp) { a = __ldg(P.cpt + (2 + ysd) * C.ncp + sy); a.w = 1.f; }
        if (czo.on) { b = czo.c; b.w = 1.f; }
        else if (zsd >= 0 && k - kb >= 0 && k - kb < C.ncp) {   // own lane past the grid edge only
          b = __ldg(P.cpt + (4 + zsd) * C.ncp + (k - kb));
          b.w = 1.f;
        }
      }
      S.hcp_row[0][lane] = a;
      S.hcp_row[1][lane] = b;
    }
    if ((ty == (TY > 1 ? 1 : 0)) && (lane < TY)) {
      float4 a = off, b = off;
      if ((z0 >= 1) && (y0 + lane < C.ny)) {
        const int sy = y0 + lane - jb, sz = z0 - 1 - kb;
        if (ysd >= 0 && sy >= 0 && sy < C.ncp) { a = __ldg(P.cpt + (2 + ysd) * C.ncp + sy); a.w = 1.f; }
        if (zsd >= 0 && sz >= 0 && sz < C.ncp) { b = __ldg(P.cpt + (4 + zsd) * C.ncp + sz); b.w = 1.f; }
      }
      S.hcp_col[0][lane] = a;
      S.hcp_col[1][lane] = b;
    }
  }

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
  // completion parity of the stage holding plane p (planes load in order
  // xa-1, xa, ...: the k-th fill of a stage in this item is k phases past
  // the phase the previous items left it in)
  auto sparity = [&](int p) -> uint32_t {
    return ((ph.stage >> stage_of(p)) ^ (uint32_t)((p - xa + 1) >> 2)) & 1u;
  };
  // psi ring bookkeeping (mode 2; identical in every thread): which planes
  // need psi, the next phase parity of each slot, and fills in flight
  auto psi_need = [&](int p) {
    if (MODE != 2 || p < 0 || p >= C.nx) return false;
    return psi_tile || (C.cpx && (p < C.ncp || p >= C.nx - C.ncp));
  };
  unsigned& pph = ph.ring;
  unsigned pout = 0u;
  auto psi_fill = [&](int p) {
    if (!psi_need(p)) return;
    if (tid == producer)
      psi_issue<TY>(ring + (p & 1) * L::FLOATS, smem_u32(&S.pbar[p & 1]), tm, P, par, y0, z0, p, C.cpx, ysd, zsd);
    pout |= 1u << (p & 1);
  };
  auto psi_wait = [&](int p) -> bool {
    if (!psi_need(p)) return true;
    const int s = p & 1;
    const bool ok = mbar_wait_bounded(smem_u32(&S.pbar[s]), (pph >> s) & 1u, wlim);
    if (ok) {
      pph ^= 1u << s;
      pout &= ~(1u << s);
    }
    return ok;
  };
  // A wait that runs out marks the launch failed and leaves the CTA after
  // draining the boxes it issued (a stalled copy cannot be waited out forever).
  auto bail = [&](int last_issued, int from) {
    if (tid == 0) {
      atomicOr(P.status, 1);
      for (int p = from; p <= last_issued; ++p) mbar_wait_bounded(smem_u32(&S.mbar[stage_of(p)]), sparity(p), wlim);
      for (int s = 0; s < 2; ++s)
        if (pout & (1u << s)) mbar_wait_bounded(smem_u32(&S.pbar[s]), (pph >> s) & 1u, wlim);
    }
  };
  if (TMA) {
    if (tid == producer) {
      for (int p = xa - 1; p <= min(xa + 2, xb); ++p)
        if (!(skip_first && p == xa)) tma_stage<TY, EM>(S, tm, fin, y0, z0, p);
    }
    psi_fill(xa - 1);
    psi_fill(xa);
    const bool ok = mbar_wait_bounded(smem_u32(&S.mbar[stage_of(xa - 1)]), sparity(xa - 1), wlim) &&
                    mbar_wait_bounded(smem_u32(&S.mbar[stage_of(xa)]), sparity(xa), wlim) && psi_wait(xa - 1);
    if (__syncthreads_or(!ok)) { bail(min(xa + 2, xb), xa - 1); return false; }
  } else {
    // pipeline: planes xa-1 and xa (group 0), xa+1 (group 1), xa+2 (group 2)
    load_stage<TY>(S, C, ca, cb, y0, z0, xa - 1, tid);
    load_stage<TY>(S, C, ca, cb, y0, z0, xa, tid);
    cp_async_commit();
    load_stage<TY>(S, C, ca, cb, y0, z0, xa + 1, tid);
    cp_async_commit();
    if (xa + 2 <= xb) load_stage<TY>(S, C, ca, cb, y0, z0, xa + 2, tid);
    cp_async_commit();
    cp_async_wait<2>();
    __syncthreads();
  }

  // x-slab profile of plane p (mode 2; uniform over the CTA)
  auto x_ax = [&](int p) {
    CpAx a{false, make_float4(0.f, 0.f, 0.f, 0.f), 0};
    int s = 0;
    const int sd = C.cpx ? cpml_side(p, C.nx, C.ncp, s) : -1;
    if (sd >= 0) {
      a.on = true;
      a.c = __ldg(P.cpt + sd * C.ncp + s);
      a.off = (2 * sd * C.ncp + s) * C.ny * C.zs + j * C.zs + k;
    }
    return a;
  };

  // H of plane xa-1 at this column (computed, not stored: its owner stores it).
  float hy_prev = 0.f, hz_prev = 0.f;
  if (xa > 0 && own) {
    float hx_, hy_, hz_;
    const float xhp = __ldg(P.xh + xa - 1);
    if (MODE == 2) {
      const float chc = C.ch ? C.ch[C.off0 + (long long)(xa - 1) * C.ps + (long long)j * C.zs + k] : C.ch0;
      const CpAx cx = x_ax(xa - 1);
      h_cell2<TY, 6, false>(P, S, ring + ((xa - 1) & 1) * L::FLOATS, C, stage_of(xa - 1), stage_of(xa), ly, lz, ly,
                            k - kb, chc, xhp, yh, zh, cx, cyo, czo, hx_, hy_, hz_);
    } else {
      h_cell<TY, 6>(P, S, C, stage_of(xa - 1), stage_of(xa), xa - 1, j, k, ly, lz, xhp, yh, zh, false,
                    hx_, hy_, hz_);
    }
    hy_prev = hy_;
    hz_prev = hz_;
  }

  const bool has_hist = P.hist != nullptr && (n - P.hist_step0) >= 0 && (n - P.hist_step0) < P.hist_nsteps;
  const bool has_emask = P.emask != nullptr;

  // the x spacing entries and x-slab profile of the next plane are loaded one
  // plane ahead, so no plane starts by waiting on a global load
  const float* xh_tab = P.xh;
  const float* xe_tab = P.xe;
  float xh_n = __ldg(xh_tab + xa), xe_n = __ldg(xe_tab + xa);
  CpAx cx_n{false, make_float4(0.f, 0.f, 0.f, 0.f), 0};
  if (MODE == 2) cx_n = x_ax(xa);

  for (int i = xa; i < xb; ++i) {
    if (TMA) {
      // plane i+1 has landed (and plane i's psi); after the barrier every
      // thread is done with plane i-1, whose stage takes plane i+3 and whose
      // psi slot takes plane i+1
      const bool ok = mbar_wait_bounded(smem_u32(&S.mbar[stage_of(i + 1)]), sparity(i + 1), wlim) && psi_wait(i);
      if (__syncthreads_or(!ok)) { bail(min(i + 2, xb), i + 1); return false; }
      if (tid == producer && i + 3 <= xb) tma_stage<TY, EM>(S, tm, fin, y0, z0, i + 3);
      if (i + 1 < xb) psi_fill(i + 1);
    } else {
      cp_async_wait<1>();   // planes up to i+1 have landed (i+2 may be in flight)
      __syncthreads();      // ... for every thread; plane i-1's stage is free
      if (i + 3 <= xb) load_stage<TY>(S, C, ca, cb, y0, z0, i + 3, tid);
      cp_async_commit();
    }
    const int b0 = stage_of(i), b1 = stage_of(i + 1);
    const float xh = xh_n, xe = xe_n;
    if (i + 1 < xb) { xh_n = __ldg(xh_tab + i + 1); xe_n = __ldg(xe_tab + i + 1); }
    const float* PS = ring + (i & 1) * L::FLOATS;
    CpAx cx{false, make_float4(0.f, 0.f, 0.f, 0.f), 0}, cy = cyo, cz = czo;
    if (MODE == 2) {
      cx = cx_n;
      if (i + 1 < xb) cx_n = x_ax(i + 1);
      cy.off += i * C.ncp * C.zs;
      cz.off += i * C.ny * P.ncp4;
    }

    // ---- H phase ----
    float hx = 0.f, hy = 0.f, hz = 0.f;
    const long long e = C.off0 + (long long)i * C.ps + (long long)j * C.zs + k;
    if (own) {
      if (MODE == 2) {
        const float chc = C.ch ? C.ch[e] : C.ch0;
        h_cell2<TY, 7, true>(P, S, PS, C, b0, b1, ly, lz, ly, k - kb, chc, xh, yh, zh, cx, cy, cz, hx, hy, hz);
      } else {
        h_cell<TY, 7>(P, S, C, b0, b1, i, j, k, ly, lz, xh, yh, zh, true, hx, hy, hz);
      }
      C.Fo[3 * C.cs + e] = hx;
      C.Fo[4 * C.cs + e] = hy;
      C.Fo[5 * C.cs + e] = hz;
    }
    S.h[0][ly][lh] = hx;
    S.h[1][ly][lh] = hy;
    S.h[2][ly][lh] = hz;
    if (ty == 0) {  // halo row j = y0 - 1: hx, hz
      float a = 0.f, bq = 0.f, cq = 0.f;
      if (row_halo) {
        if (MODE == 2) {
          const int jr = y0 - 1;
          const float chc = C.ch ? C.ch[C.off0 + (long long)i * C.ps + (long long)jr * C.zs + k] : C.ch0;
          const float4 qy = S.hcp_row[0][lane], qz = S.hcp_row[1][lane];
          const CpAx ry{qy.w != 0.f, qy, 0}, rz{qz.w != 0.f, qz, 0};
          h_cell2<TY, 5, false>(P, S, PS, C, b0, b1, 0, lz, 0, k - kb, chc, xh, yh_row, zh, cx, ry, rz, a, bq, cq);
        } else {
          h_cell<TY, 5>(P, S, C, b0, b1, i, y0 - 1, k, 0, lz, xh, yh_row, zh, false, a, bq, cq);
        }
      }
      S.h[0][0][lh] = a;
      S.h[2][0][lh] = cq;
    }
    if (ty == hcw && lane < TY) {  // halo column k = z0 - 1: hx, hy
      float a = 0.f, bq = 0.f, cq = 0.f;
      if (col_halo) {
        if (MODE == 2) {
          const int jc = y0 + lane, kc = z0 - 1;
          const float chc = C.ch ? C.ch[C.off0 + (long long)i * C.ps + (long long)jc * C.zs + kc] : C.ch0;
          const float4 qy = S.hcp_col[0][lane], qz = S.hcp_col[1][lane];
          const CpAx ry{qy.w != 0.f, qy, 0}, rz{qz.w != 0.f, qz, 0};
          h_cell2<TY, 3, false>(P, S, PS, C, b0, b1, lane + 1, 3, lane + 1, kc - kb, chc, xh, yh_col, zh_col, cx, ry,
                                rz, a, bq, cq);
        } else {
          h_cell<TY, 3>(P, S, C, b0, b1, i, y0 + lane, z0 - 1, lane + 1, 3, xh, yh_col, zh_col, false, a, bq, cq);
        }
      }
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
      const float cx_ = yee_diff2(dHz_y, ye, dHy_z, ze);
      const float cy_ = yee_diff2(dHx_z, ze, dHz_x, xe);
      const float cz_ = yee_diff2(dHy_x, xe, dHx_y, ye);
      const float cav = A.cab[0][ty][lane], cbv = A.cab[1][ty][lane];
      float ex = yee_e(cav, Ex, cbv, cx_);
      float ey = yee_e(cav, Ey, cbv, cy_);
      float ez = yee_e(cav, Ez, cbv, cz_);
      const int ncp = C.ncp;
      // CPML-E correction of each component before its ce scaling (the
      // factor d ce / d eps_r multiplies in the gradient) and this cell's ce
      float kx = 0.f, ky = 0.f, kz = 0.f, ceh = 0.f;
      if (MODE == 2) {
        if (cx.on || cy.on || cz.on) {
          const float ce = PS[L::CE + ty * RFXB_TZ + lane];
          ceh = ce;
          constexpr int RE = TY * RFXB_TZ;   // q stride of an E box
          const int o = ty * RFXB_TZ + lane;
          if (cx.on) {   // Ey -= ce psi(dHz/dx) [q0], Ez += ce psi(dHy/dx) [q1]
            const int qs = ncp * C.ny * C.zs;
            const float p0 = cx.c.x * PS[L::EX + o] + cx.c.y * dHz_x;
            const float p1 = cx.c.x * PS[L::EX + RE + o] + cx.c.y * dHy_x;
            P.psE[par ^ 1][0][cx.off] = p0;
            P.psE[par ^ 1][0][cx.off + qs] = p1;
            ey = ey - ce * p0;
            ey = ey - ce * (cx.c.z * dHz_x);
            ez = ez + ce * p1;
            ez = ez + ce * (cx.c.z * dHy_x);
            ky -= p0 + cx.c.z * dHz_x;
            kz += p1 + cx.c.z * dHy_x;
          }
          if (cy.on) {   // Ex += ce psi(dHz/dy) [q0], Ez -= ce psi(dHx/dy) [q1]
            const int qs = C.nx * ncp * C.zs;
            const float p0 = cy.c.x * PS[L::EY + o] + cy.c.y * dHz_y;
            const float p1 = cy.c.x * PS[L::EY + RE + o] + cy.c.y * dHx_y;
            P.psE[par ^ 1][1][cy.off] = p0;
            P.psE[par ^ 1][1][cy.off + qs] = p1;
            ex = ex + ce * p0;
            ex = ex + ce * (cy.c.z * dHz_y);
            ez = ez - ce * p1;
            ez = ez - ce * (cy.c.z * dHx_y);
            kx += p0 + cy.c.z * dHz_y;
            kz -= p1 + cy.c.z * dHx_y;
          }
          if (cz.on) {   // Ex -= ce psi(dHy/dz) [q0], Ey += ce psi(dHx/dz) [q1]
            const int n4 = P.ncp4;
            const int qs = C.nx * C.ny * n4;
            const int oz = ty * n4 + (k - kb);
            const float p0 = cz.c.x * PS[L::EZ + oz] + cz.c.y * dHy_z;
            const float p1 = cz.c.x * PS[L::EZ + TY * n4 + oz] + cz.c.y * dHx_z;
            P.psE[par ^ 1][2][cz.off] = p0;
            P.psE[par ^ 1][2][cz.off + qs] = p1;
            ex = ex - ce * p0;
            ex = ex - ce * (cz.c.z * dHy_z);
            ey = ey + ce * p1;
            ey = ey + ce * (cz.c.z * dHx_z);
            kx -= p0 + cz.c.z * dHy_z;
            ky += p1 + cz.c.z * dHx_z;
          }
        }
      } else if (C.cpx || C.cpy || C.cpz) {
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
              ky -= p + km * g;
            }
            {  // Ez += ce psi(dHy/dx)
              const long long q = psi_index_x(P, sd, 1, s, j, k);
              const float g = dHy_x * ib;
              const float p = b * P.psE[par][0][q] + c * g;
              P.psE[par ^ 1][0][q] = p;
              ez = ez + ce * p;
              ez = ez + ce * km * g;
              kz += p + km * g;
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
              kx += p + km * g;
            }
            {  // Ez -= ce psi(dHx/dy)
              const long long q = psi_index_y(P, sd, 1, s, i, k);
              const float g = dHx_y * ib;
              const float p = b * P.psE[par][1][q] + c * g;
              P.psE[par ^ 1][1][q] = p;
              ez = ez - ce * p;
              ez = ez - ce * (km * g);
              kz -= p + km * g;
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
              kx -= p + km * g;
            }
            {  // Ey += ce psi(dHx/dz)
              const long long q = psi_index_z(P, sd, 1, s, i, j);
              const float g = dHx_z * ib;
              const float p = b * P.psE[par][2][q] + c * g;
              P.psE[par ^ 1][2][q] = p;
              ey = ey + ce * p;
              ey = ey + ce * (km * g);
              ky += p + km * g;
            }
          }
        }
        ceh = ce;
      }
      // PEC faces
      if ((pec & 1u) && (i == 0 || i == C.nx - 1)) { ey = 0.f; ez = 0.f; }
      if (pec_j) { ex = 0.f; ez = 0.f; }
      if (pec_k0) { ex = 0.f; ey = 0.f; }
      if (pec_kz) ez = 0.f;
      if (has_emask) {
        const unsigned m = (TMA && EM) ? (unsigned)A.em[ty][lane] : (unsigned)P.emask[e];
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
          // d E^{n+1} / d eps_r = dca E^n + dcb curl + dce corr, and
          // dce / dcb = (1 + sigma dt / (2 eps))^2 = (ce / cb)^2: the
          // recorded curl carries the CPML term so that the reverse step's
          // dca E + dcb curl is the whole derivative (ceh = 0 off the slabs)
          const float rr = ceh != 0.f ? (ceh / cbv) * (ceh / cbv) : 0.f;
          hp[3 * hc] = cx_ + rr * kx; hp[4 * hc] = cy_ + rr * ky; hp[5 * hc] = cz_ + rr * kz;
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
  if (TMA) {   // the phases this item advanced: stage s filled by planes xa-1 .. xb
    const int T = xb - xa + 2;
    for (int st = 0; st < RFXB_NSTAGE; ++st) {
      const int fills = T / RFXB_NSTAGE + ((((st - xa) % RFXB_NSTAGE + RFXB_NSTAGE) % RFXB_NSTAGE) < T % RFXB_NSTAGE ? 1 : 0);
      ph.stage ^= (uint32_t)(fills & 1) << st;
    }
  }
  __syncthreads();   // every thread is done with the stages and P before the next item reuses them
  return true;
}

template <int TY, int MODE>
__device__ __forceinline__ void fwd_init_barriers(FwdSmem<TY>& S, int tid) {
  if (MODE != 0 && tid == 0) {
    for (int q = 0; q < RFXB_NSTAGE; ++q) mbar_init(smem_u32(&S.mbar[q]), 1);
    if (MODE == 2) { mbar_init(smem_u32(&S.pbar[0]), 1); mbar_init(smem_u32(&S.pbar[1]), 1); }
    mbar_fence_init();
  }
  __syncthreads();
}

// One launch per step and variant: CTA b runs work item b.  `sel` selects
// the field buffers and the psi parity (step_sel).
template <int TY, int MODE, bool EM>
__global__ void __launch_bounds__(32 * TY, FwdBounds<MODE>::MIN_CTAS)
fwd_step_kernel(const RfxbInst* __restrict__ insts, const RfxbWork* __restrict__ work,
                const CUtensorMap* __restrict__ maps, int n, int sel) {
  extern __shared__ __align__(128) unsigned char fwd_smem_raw[];
  FwdSmem<TY>& S = *reinterpret_cast<FwdSmem<TY>*>(fwd_smem_raw);
  float* ring = reinterpret_cast<float*>(fwd_smem_raw + sizeof(FwdSmem<TY>));   // mode 2: 2 slots
  fwd_init_barriers<TY, MODE>(S, threadIdx.y * 32 + threadIdx.x);
  StepPhases ph;
  fwd_item<TY, MODE, EM>(S, ring, insts, work[blockIdx.x], maps, n, sel, ph, StepFault{}, true);
}

// Whether a work item can be run: its instance exists and its tile and x
// range lie inside that instance's grid on the tiling of the lists.
template <int TY>
__device__ __forceinline__ bool work_item_valid(const RfxbWork& w, const RfxbInst* insts, int n_inst) {
  if (w.inst < 0 || w.inst >= n_inst) return false;
  const RfxbInst& I = insts[w.inst];
  return w.y0 >= 0 && w.y0 < I.ny && w.y0 % TY == 0 && w.z0 >= 0 && w.z0 < I.nz && w.z0 % RFXB_TZ == 0 &&
         w.xa >= 0 && w.xa < w.xb && w.xb <= I.nx;
}

// Persistent forward step: one launch per step of exactly as many CTAs as
// fit on the GPU at once.  Each CTA takes items from the two lists of the
// step -- queue 0 the tiles that reach a CPML slab (the staged-psi path of
// mode 2), queue 1 the CPML-free tiles (mode 1) -- through fetch counters in
// device memory until both are empty.  The first `plain_ctas` CTAs (one per
// SM when the block scheduler spreads the first wave) try queue 1 first,
// the others queue 0, so latency-bound CPML tiles and bandwidth-bound plain
// tiles share every SM; a CTA whose queue is empty helps with the other.
// An item outside its instance's grid is skipped and flagged (status bit 2).
// The last CTA to finish clears the counters for the next launch.
template <int TY, bool EM>
__global__ void __launch_bounds__(32 * TY, 3)
fwd_persist_kernel(const RfxbInst* __restrict__ insts, int n_inst, RfxbFwdQueues Q,
                   const CUtensorMap* __restrict__ maps, int n, int sel) {
  extern __shared__ __align__(128) unsigned char fwd_smem_raw[];
  FwdSmem<TY>& S = *reinterpret_cast<FwdSmem<TY>*>(fwd_smem_raw);
  float* ring = reinterpret_cast<float*>(fwd_smem_raw + sizeof(FwdSmem<TY>));
  __shared__ int pick[2];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  fwd_init_barriers<TY, 2>(S, tid);
  StepPhases ph;
  StepFault fault;
  fault.cta = Q.fault_cta;
  fault.wait_limit = Q.wait_limit;
  const int first = (int)blockIdx.x < Q.plain_ctas ? 1 : 0;
  bool first_item = true;
  bool ok = true;
  while (ok) {
    if (tid == 0) {
      pick[0] = -1;
      for (int t = 0; t < 2; ++t) {
        const int q = t == 0 ? first : 1 - first;
        if (*(volatile int*)&Q.ctr[q] >= Q.count[q]) continue;   // drained (counters only grow): no ticket
        const int k = atomicAdd(&Q.ctr[q], 1);
        if (k < Q.count[q]) { pick[0] = q; pick[1] = k; break; }
      }
    }
    __syncthreads();
    const int q = pick[0], k = pick[1];
    __syncthreads();
    if (q < 0) break;
    const RfxbWork w = Q.list[q][k];
    if (!work_item_valid<TY>(w, insts, n_inst)) {
      if (tid == 0) atomicOr(Q.status, 2);
      continue;
    }
    ok = q == 0 ? fwd_item<TY, 2, EM>(S, ring, insts, w, maps, n, sel, ph, fault, first_item)
                : fwd_item<TY, 1, EM>(S, ring, insts, w, maps, n, sel, ph, fault, first_item);
    first_item = false;
  }
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&Q.ctr[2], 1) == (int)gridDim.x - 1) {
      Q.ctr[0] = 0;
      Q.ctr[1] = 0;
      Q.ctr[2] = 0;
      __threadfence();
    }
  }
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
template __global__ void fwd_step_kernel<8, 0, false>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int,
                                                      int);
template __global__ void fwd_step_kernel<8, 1, false>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int,
                                                      int);
template __global__ void fwd_step_kernel<8, 1, true>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);
template __global__ void fwd_step_kernel<8, 2, false>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int,
                                                      int);
template __global__ void fwd_step_kernel<8, 2, true>(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);

template __global__ void fwd_persist_kernel<8, false>(const RfxbInst*, int, RfxbFwdQueues, const CUtensorMap*, int,
                                                       int);
template __global__ void fwd_persist_kernel<8, true>(const RfxbInst*, int, RfxbFwdQueues, const CUtensorMap*, int,
                                                      int);

size_t fwd_step_smem_bytes(int mode) { return fwd_smem_bytes<8>(mode); }

}  // namespace rfxb
