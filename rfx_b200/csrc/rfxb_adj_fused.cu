// Fused reverse step of the adjoint: the same tiling, x-march, staged plane
// pipeline and halo recomputation as the forward step kernel.
//
// The transpose of one forward step (see rfxb_adj.cu for the derivation)
// has the forward's dependency shape with the roles swapped:
//   phase A (H-like, needs aE at x and x+1 along each axis):
//     aH1 = aH + C_H^T(cb aEm) + sum_slabs [r_E(x) - r_E(x+1)]
//     r_E = ib (c nu + s ce km aE_t),  nu = aPsiE + s ce aE_t,  aPsiE' = b nu
//   phase B (E-like, needs p = ch aH1 at x and x-1 along each axis):
//     aE  = ca aEm + C_E^T(p) + sum_slabs [r_H(x-1) - r_H(x)]
//     r_H = ib (c nu + s km p_t),       nu = aPsiH + s p_t,       aPsiH' = b nu
// followed by the probe cotangent of y_{n-1}, the source adjoint and the
// PEC/edge mask.  Adjoint fields and psi are ping-ponged like the forward
// state, so halo cells recomputed by a neighbour CTA read step-consistent
// values.  The eps_r gradient over the recorded region is accumulated in
// phase A from the forward history.
//
// The CPML terms of each relation are evaluated once per cell: the y / z
// relations are exchanged between neighbouring cells through shared memory,
// the x relations are carried along the march.  Modes (template MODE):
//   0  cp.async staging (4 planes), psi and ce read from global memory;
//   1  TMA staging (4 planes), psi and ce read from global memory;
//   2  TMA staging (3 planes) plus a two-slot ring that brings, one plane
//      ahead, every adjoint psi and ce value the plane's CPML terms read, so
//      no slab cell waits on a global load.  The host selects it when no
//      tile reaches both slabs of an axis;
//   3  TMA staging (4 planes) with the CPML code compiled out, for the
//      tiles and x ranges whose reverse step touches no slab (the host runs
//      them beside variant 2 or 1 on a second stream);
//   4  variant 2 for tiles that reach no y slab: the y relations and the
//      edge-mask staging compiled out and the ring without its y-slab
//      arrays (57 KB of shared memory; three CTAs per SM at 80 registers,
//      measured faster than four at 64 with spills; a third stream).
#include <algorithm>

#include "rfxb_common.cuh"

namespace rfxb {

#define RFXB_ANSTAGE 4
#define RFXB_AEW 40
#define RFXB_AHW 36

__host__ __device__ constexpr int apad128(int nfloats) { return (nfloats % 32) ? 32 - (nfloats % 32) : 32; }
__host__ __device__ constexpr int up32(int nfloats) { return (nfloats + 31) / 32 * 32; }

template <int TY>
struct AdjDims {
  static constexpr int NE = 3 * (TY + 2) * RFXB_AEW;
  static constexpr int NB = (TY + 2) * RFXB_AEW;
  static constexpr int NH = 3 * (TY + 1) * RFXB_AHW;
  static constexpr int NC = TY * RFXB_TZ;
  static constexpr int P0 = apad128(NE);
  static constexpr int P1 = apad128(NE + P0 + NB);
  static constexpr int P2 = apad128(NE + P0 + NB + P1 + NH);
  static constexpr unsigned BYTES = 4u * (NE + NB + NH + NC);
};

// One plane stage; EMS: with the tile's PEC edge-mask bits (staged only when
// the plan has a mask; variant 4 has no room for them).
template <int TY, bool EMS>
struct __align__(128) AdjStage {
  float ae[3][TY + 2][RFXB_AEW];   // masked adjoint E, rows y0-1 .. y0+TY, z from z0-4
  float p0[AdjDims<TY>::P0];
  float cbp[TY + 2][RFXB_AEW];     // cb on the same footprint
  float p1[AdjDims<TY>::P1];
  float ah[3][TY + 1][RFXB_AHW];   // adjoint H, rows y0-1 .. y0+TY-1, z from z0-4
  float p2[AdjDims<TY>::P2];
  float ca[TY][RFXB_TZ];           // ca of the tile
  unsigned char em[TY][RFXB_TZ];   // PEC edge-mask bits of the tile
};
template <int TY>
struct __align__(128) AdjStage<TY, false> {
  float ae[3][TY + 2][RFXB_AEW];
  float p0[AdjDims<TY>::P0];
  float cbp[TY + 2][RFXB_AEW];
  float p1[AdjDims<TY>::P1];
  float ah[3][TY + 1][RFXB_AHW];
  float p2[AdjDims<TY>::P2];
  float ca[TY][RFXB_TZ];
};

// The plane stages come last so that a kernel using fewer of them (modes 2
// and 4) allocates only those, followed by its psi ring (modes 2, 4) or the
// exchange array of the CPML terms (modes 0, 1): r_E / r_H of the y and z
// relations (y q0, y q1, z q0, z q1) at rows y0-1 .. y0+TY, columns
// z0-1 .. z0+32.
template <int TY>
using AdjExchange = float[4][TY + 2][RFXB_TZ + 2];

template <int TY, bool EMS>
struct AdjSmem {
  float p[3][TY + 1][RFXB_TZ + 1];   // ch * aH1 of plane i, [y - y0 + 1][z - z0 + 1]
  RfxbInst P;
  AdjInst A;
  unsigned long long mbar[RFXB_ANSTAGE];
  unsigned long long pbar[2];        // psi ring (modes 2, 4)
  AdjStage<TY, EMS> st[RFXB_ANSTAGE];
};

// Plane p lives in stage (p + 1) mod NST.
template <int NST>
__device__ __forceinline__ int astage_of(int p) { return (p + 1) % NST; }
// Planes are loaded in order xa-1, xa, ...; a stage completes its k-th fill on
// mbarrier phase k.
template <int NST>
__device__ __forceinline__ uint32_t astage_parity(int p, int xa) { return (uint32_t)(((p - xa + 1) / NST) & 1); }

// One slot of the mode-2 psi ring: everything the CPML terms of plane p read
// (floats, 128-byte aligned sub-arrays; zp = the launch's largest z-psi row):
//   EY  [q][TY+2][40]  adjoint E-side psi of the y slab, rows y0-1.., z from z0-4
//   HY  [q][TY+1][36]  adjoint H-side psi of the y slab, rows y0-1.., z from z0-4
//   EXN [q][TY+1][36]  adjoint E-side psi of the x slab at plane p+1
//   HX  [q][TY][32]    adjoint H-side psi of the x slab on the tile
//   CE  [TY+2][40]     ce of plane p on the E footprint
//   CEN [TY+1][36]     ce of plane p+1 on the H footprint
//   EZ  [q][TY+2][n4]  adjoint E-side psi of the z slab, layer s
//   HZ  [q][TY+1][n4]  adjoint H-side psi of the z slab
// (YS false, variant 4: no EY / HY arrays.)
template <int TY, bool YS>
struct APsiSlot {
  static constexpr int EY = 0;
  static constexpr int HY = EY + (YS ? up32(2 * (TY + 2) * RFXB_AEW) : 0);
  static constexpr int EXN = HY + (YS ? up32(2 * (TY + 1) * RFXB_AHW) : 0);
  static constexpr int HX = EXN + up32(2 * (TY + 1) * RFXB_AHW);
  static constexpr int CE = HX + up32(2 * TY * RFXB_TZ);
  static constexpr int CEN = CE + up32((TY + 2) * RFXB_AEW);
  static constexpr int EZ = CEN + up32((TY + 1) * RFXB_AHW);
  __host__ __device__ static constexpr int HZ(int zp) { return EZ + up32(2 * (TY + 2) * zp); }
  __host__ __device__ static constexpr int FLOATS(int zp) { return HZ(zp) + up32(2 * (TY + 1) * zp); }
};

struct AdjCtx {
  int nx, ny, nz, zs, ncp, par, apar;
  long long ps, off0, cs;
  const float* ch;
  float ch0;
  bool cpx, cpy, cpz;
};

__device__ __forceinline__ long long cell_index(const AdjCtx& C, int i, int j, int k) {
  return C.off0 + (long long)i * C.ps + (long long)j * C.zs + k;
}

__device__ __forceinline__ long long psi_q(const RfxbInst& P, int axis, int sd, int q, int s, int i, int j, int k) {
  if (axis == 0) return psi_index_x(P, sd, q, s, j, k);
  if (axis == 1) return psi_index_y(P, sd, q, s, i, k);
  return psi_index_z(P, sd, q, s, i, j);
}

// r_E of one CPML-E relation at cell (i, j, k) whose masked adjoint E
// component t is at: the transposed psi recursion and kappa term.
__device__ __forceinline__ float r_e(const RfxbInst& P, const AdjInst& A, const AdjCtx& C, int axis, int q, float sgn,
                                     int i, int j, int k, float at, bool write) {
  const int coord = axis == 0 ? i : axis == 1 ? j : k;
  const int nax = axis == 0 ? C.nx : axis == 1 ? C.ny : C.nz;
  if (coord < 0 || coord >= nax) return 0.f;
  int s;
  const int sd = cpml_side(coord, nax, C.ncp, s);
  if (sd < 0) return 0.f;
  const float4 cf = __ldg(P.cpt + (2 * axis + sd) * C.ncp + s);
  const float ce = P.ce[cell_index(C, i, j, k)];
  const long long qi = psi_q(P, axis, sd, q, s, i, j, k);
  const float nu = A.aPsiE[C.par][axis][qi] + sgn * ce * at;
  if (write) A.aPsiE[C.par ^ 1][axis][qi] = cf.x * nu;
  return cf.y * nu + sgn * ce * (cf.z * at);
}

// r_H of one CPML-H relation at cell (i, j, k) with p_t = ch aH1_t there.
__device__ __forceinline__ float r_h(const RfxbInst& P, const AdjInst& A, const AdjCtx& C, int axis, int q, float sgn,
                                     int i, int j, int k, float pt, bool write) {
  const int coord = axis == 0 ? i : axis == 1 ? j : k;
  const int nax = axis == 0 ? C.nx : axis == 1 ? C.ny : C.nz;
  if (coord < 0 || coord >= nax) return 0.f;
  int s;
  const int sd = cpml_side(coord, nax, C.ncp, s);
  if (sd < 0) return 0.f;
  const float4 cf = __ldg(P.cpt + (2 * axis + sd) * C.ncp + s);
  const long long qi = psi_q(P, axis, sd, q, s, i, j, k);
  const float nu = A.aPsiH[C.par][axis][qi] + sgn * pt;
  if (write) A.aPsiH[C.par ^ 1][axis][qi] = cf.x * nu;
  return cf.y * nu + sgn * (cf.z * pt);
}

// r_E / r_H with the folded profile (b, c/cell, (1/kappa-1)/cell) of the
// staged-psi forward: c' nu + s ce k' a_t and c' nu + s k' p_t.  Zero outside
// the grid and outside the slab.
__device__ __forceinline__ float re_eval(const RfxbInst& P, const AdjInst& A, const AdjCtx& C, int axis, int q,
                                         float sgn, int i, int j, int k, float at, float ce, bool write) {
  const int coord = axis == 0 ? i : axis == 1 ? j : k;
  const int nax = axis == 0 ? C.nx : axis == 1 ? C.ny : C.nz;
  if (coord < 0 || coord >= nax) return 0.f;
  int s;
  const int sd = cpml_side(coord, nax, C.ncp, s);
  if (sd < 0) return 0.f;
  const float4 cf = __ldg(P.cpt + (2 * axis + sd) * C.ncp + s);
  const long long qi = psi_q(P, axis, sd, q, s, i, j, k);
  const float nu = __ldg(A.aPsiE[C.par][axis] + qi) + sgn * ce * at;
  if (write) A.aPsiE[C.par ^ 1][axis][qi] = cf.x * nu;
  return cf.y * nu + sgn * ce * (cf.z * at);
}

__device__ __forceinline__ float rh_eval(const RfxbInst& P, const AdjInst& A, const AdjCtx& C, int axis, int q,
                                         float sgn, int i, int j, int k, float pt, bool write) {
  const int coord = axis == 0 ? i : axis == 1 ? j : k;
  const int nax = axis == 0 ? C.nx : axis == 1 ? C.ny : C.nz;
  if (coord < 0 || coord >= nax) return 0.f;
  int s;
  const int sd = cpml_side(coord, nax, C.ncp, s);
  if (sd < 0) return 0.f;
  const float4 cf = __ldg(P.cpt + (2 * axis + sd) * C.ncp + s);
  const long long qi = psi_q(P, axis, sd, q, s, i, j, k);
  const float nu = __ldg(A.aPsiH[C.par][axis] + qi) + sgn * pt;
  if (write) A.aPsiH[C.par ^ 1][axis][qi] = cf.x * nu;
  return cf.y * nu + sgn * (cf.z * pt);
}

// Whether a cell lies in a CPML slab of an active axis other than x.
__device__ __forceinline__ bool in_yz_slab(const AdjCtx& C, int j, int k) {
  return (C.cpy && (j < C.ncp || j >= C.ny - C.ncp)) || (C.cpz && (k < C.ncp || k >= C.nz - C.ncp));
}

// Phase A at (i, jj, kk): aH1 components selected by MASK (1 hx, 2 hy, 4 hz).
// With CP, the CPML-E^T terms are evaluated here at the cell and its +1
// neighbours (the prologue plane); without, the caller adds them.
template <int TY, int MASK, bool CP = true, class SM>
__device__ __forceinline__ void adj_a_cell(const RfxbInst& P, const AdjInst& A, const SM& S,
                                           const AdjCtx& C, int b0, int b1, int i, int jj, int kk, int ly, int lz,
                                           float xe0, float xe1, float ye0, float ye1, float ze0, float ze1,
                                           bool own, float& ahx, float& ahy, float& ahz) {
  const auto& X = S.st[b0];
  const auto& Y = S.st[b1];
  const float cb0 = X.cbp[ly][lz];
  const float ax0 = X.ae[0][ly][lz], ay0 = X.ae[1][ly][lz], az0 = X.ae[2][ly][lz];
  const float qx = cb0 * ax0, qy = cb0 * ay0, qz = cb0 * az0;
  const float cbx = Y.cbp[ly][lz];
  const float ay_x1 = Y.ae[1][ly][lz], az_x1 = Y.ae[2][ly][lz];
  const float cby = X.cbp[ly + 1][lz];
  const float ax_y1 = X.ae[0][ly + 1][lz], az_y1 = X.ae[2][ly + 1][lz];
  const float cbz = X.cbp[ly][lz + 1];
  const float ax_z1 = X.ae[0][ly][lz + 1], ay_z1 = X.ae[1][ly][lz + 1];
  if (MASK & 1) ahx = X.ah[0][ly][lz] + ((ze0 * qy - ze1 * (cbz * ay_z1)) - (ye0 * qz - ye1 * (cby * az_y1)));
  if (MASK & 2) ahy = X.ah[1][ly][lz] + ((xe0 * qz - xe1 * (cbx * az_x1)) - (ze0 * qx - ze1 * (cbz * ax_z1)));
  if (MASK & 4) ahz = X.ah[2][ly][lz] + ((ye0 * qx - ye1 * (cby * ax_y1)) - (xe0 * qy - xe1 * (cbx * ay_x1)));
  // CPML-E^T: aH_h(x) += r_E(x) - r_E(x + 1 along the axis); own cells write aPsiE'
  if (!CP) return;
  if (C.cpx) {
    if (own || (MASK & 4)) ahz += r_e(P, A, C, 0, 0, -1.f, i, jj, kk, ay0, own) -
                                  r_e(P, A, C, 0, 0, -1.f, i + 1, jj, kk, ay_x1, false);   // (ey <- hz)
    if (own || (MASK & 2)) ahy += r_e(P, A, C, 0, 1, +1.f, i, jj, kk, az0, own) -
                                  r_e(P, A, C, 0, 1, +1.f, i + 1, jj, kk, az_x1, false);   // (ez <- hy)
  }
  if (C.cpy) {
    if (own || (MASK & 4)) ahz += r_e(P, A, C, 1, 0, +1.f, i, jj, kk, ax0, own) -
                                  r_e(P, A, C, 1, 0, +1.f, i, jj + 1, kk, ax_y1, false);   // (ex <- hz)
    if (own || (MASK & 1)) ahx += r_e(P, A, C, 1, 1, -1.f, i, jj, kk, az0, own) -
                                  r_e(P, A, C, 1, 1, -1.f, i, jj + 1, kk, az_y1, false);   // (ez <- hx)
  }
  if (C.cpz) {
    if (own || (MASK & 2)) ahy += r_e(P, A, C, 2, 0, -1.f, i, jj, kk, ax0, own) -
                                  r_e(P, A, C, 2, 0, -1.f, i, jj, kk + 1, ax_z1, false);   // (ex <- hy)
    if (own || (MASK & 1)) ahx += r_e(P, A, C, 2, 1, +1.f, i, jj, kk, ay0, own) -
                                  r_e(P, A, C, 2, 1, +1.f, i, jj, kk + 1, ay_z1, false);   // (ey <- hx)
  }
}

template <int TY, class SM>
__device__ __forceinline__ void adj_load_stage(SM& S, const AdjCtx& C, const float* aF0, const float* ca,
                                               const float* cb, int y0, int z0, int ip, int tid) {
  auto& D = S.st[astage_of<RFXB_ANSTAGE>(ip)];
  const long long pb = C.off0 + (long long)ip * C.ps;
  constexpr int RE = (TY + 2) * 10, RH = (TY + 1) * 9, RC = TY * 8;
  constexpr int NE = 4 * RE, NH = 3 * RH, NC = RC;
  for (int t = tid; t < NE + NH + NC; t += 32 * TY) {
    if (t < NE) {
      const int c = t / RE, u = t - c * RE, r = u / 10, q = u - r * 10;
      const int jj = min(y0 - 1 + r, C.ny);
      const long long off = pb + (long long)jj * C.zs + (z0 - 4 + 4 * q);
      if (c < 3) cp_async16(&D.ae[c][r][4 * q], aF0 + c * C.cs + off);
      else cp_async16(&D.cbp[r][4 * q], cb + off);
    } else if (t < NE + NH) {
      const int v = t - NE, c = v / RH, u = v - c * RH, r = u / 9, q = u - r * 9;
      const int jj = min(y0 - 1 + r, C.ny);
      cp_async16(&D.ah[c][r][4 * q], aF0 + (3 + c) * C.cs + pb + (long long)jj * C.zs + (z0 - 4 + 4 * q));
    } else {
      const int v = t - NE - NH, r = v / 8, q = v - r * 8;
      const int jj = min(y0 + r, C.ny);
      cp_async16(&D.ca[r][4 * q], ca + pb + (long long)jj * C.zs + (z0 + 4 * q));
    }
  }
}

// TMA boxes of plane ip (one thread): adjoint E and H of parity apar, cb with
// the E footprint, ca of the tile.
template <int TY, int NST, bool EMS>
__device__ __forceinline__ void adj_tma_stage(AdjSmem<TY, EMS>& S, const CUtensorMap* tm, int apar, int y0, int z0,
                                              int ip) {
  const int s = astage_of<NST>(ip);
  const uint32_t mb = smem_u32(&S.mbar[s]);
  const bool em = EMS && S.P.emask != nullptr;
  mbar_expect_tx(mb, AdjDims<TY>::BYTES + (em ? (unsigned)(TY * RFXB_TZ) : 0u));
  if constexpr (EMS) {
    if (em) tma_load_4d(smem_u32(&S.st[s].em[0][0]), tm + RFXB_MAP_EMASK, z0, y0 + 1, ip + 1, 0, mb);
  }
  tma_load_4d(smem_u32(&S.st[s].ae[0][0][0]), tm + 5 + apar, z0 - 4, y0, ip + 1, 0, mb);
  tma_load_4d(smem_u32(&S.st[s].cbp[0][0]), tm + 9, z0 - 4, y0, ip + 1, 1, mb);
  tma_load_4d(smem_u32(&S.st[s].ah[0][0][0]), tm + 7 + apar, z0 - 4, y0, ip + 1, 3, mb);
  tma_load_4d(smem_u32(&S.st[s].ca[0][0]), tm + 10, z0, y0 + 1, ip + 1, 0, mb);
}

// r_E / r_H of one relation from a given old psi (modes 2, 4: staged); the new
// psi goes to the other parity at index qi.
__device__ __forceinline__ float re_core(const AdjInst& A, const AdjCtx& C, int axis, const float4& cf, long long qi,
                                         float psi, float sgn, float ce, float at, bool write) {
  const float nu = psi + sgn * ce * at;
  if (write) A.aPsiE[C.par ^ 1][axis][qi] = cf.x * nu;
  return cf.y * nu + sgn * ce * (cf.z * at);
}
__device__ __forceinline__ float rh_core(const AdjInst& A, const AdjCtx& C, int axis, const float4& cf, long long qi,
                                         float psi, float sgn, float pt, bool write) {
  const float nu = psi + sgn * pt;
  if (write) A.aPsiH[C.par ^ 1][axis][qi] = cf.x * nu;
  return cf.y * nu + sgn * (cf.z * pt);
}

// Which CPML slab of an axis the cells lo..hi of a CTA reach: side or -1
// (modes 2 and 4 guarantee at most one side per axis).
__device__ __forceinline__ int atile_side(int lo, int hi, int n, int ncp) {
  if (lo < ncp) return 0;
  if (hi >= n - ncp) return 1;
  return -1;
}

// Issue the mode-2 ring boxes of plane p (one thread).
template <int TY, bool YS>
__device__ __forceinline__ void apsi_issue(float* slot, uint32_t mb, const CUtensorMap* tm, const AdjCtx& C, int zp4,
                                           int y0, int z0, int p, bool yz_tile, int ysd, int zsd, int n4) {
  using L = APsiSlot<TY, YS>;
  const int par = C.par;
  int sx = 0, sn = 0;
  const int xsd = C.cpx ? cpml_side(p, C.nx, C.ncp, sx) : -1;
  const int xnd = (C.cpx && p + 1 < C.nx) ? cpml_side(p + 1, C.nx, C.ncp, sn) : -1;
  unsigned bytes = 0;
  if (yz_tile) bytes += 4u * (TY + 2) * RFXB_AEW;
  if (ysd >= 0) bytes += 4u * 2 * (TY + 2) * RFXB_AEW + 4u * 2 * (TY + 1) * RFXB_AHW;
  if (zsd >= 0) bytes += 4u * 2 * (TY + 2) * n4 + 4u * 2 * (TY + 1) * n4;
  if (xnd >= 0) bytes += 4u * 2 * (TY + 1) * RFXB_AHW + 4u * (TY + 1) * RFXB_AHW;
  if (xsd >= 0) bytes += 4u * 2 * TY * RFXB_TZ;
  mbar_expect_tx(mb, bytes);
  if (yz_tile) tma_load_4d(smem_u32(slot + L::CE), tm + 9, z0 - 4, y0, p + 1, 2, mb);
  if (ysd >= 0) {
    const int jb = ysd ? C.ny - C.ncp : 0;
    tma_load_4d(smem_u32(slot + L::EY), tm + RFXB_MAP_APE + 2 + par, z0 - 4, y0 - 1 - jb, p, 2 * ysd, mb);
    tma_load_4d(smem_u32(slot + L::HY), tm + RFXB_MAP_APH + 2 + par, z0 - 4, y0 - 1 - jb, p, 2 * ysd, mb);
  }
  if (zsd >= 0) {
    tma_load_4d(smem_u32(slot + L::EZ), tm + RFXB_MAP_APE + 4 + par, 0, y0 - 1, p, 2 * zsd, mb);
    tma_load_4d(smem_u32(slot + L::HZ(zp4)), tm + RFXB_MAP_APH + 4 + par, 0, y0 - 1, p, 2 * zsd, mb);
  }
  if (xnd >= 0) {
    tma_load_4d(smem_u32(slot + L::EXN), tm + RFXB_MAP_APE + 0 + par, z0 - 4, y0 - 1, sn, 2 * xnd, mb);
    tma_load_4d(smem_u32(slot + L::CEN), tm + 23, z0 - 4, y0, p + 2, 2, mb);
  }
  if (xsd >= 0) tma_load_4d(smem_u32(slot + L::HX), tm + RFXB_MAP_APH + 0 + par, z0, y0, sx, 2 * xsd, mb);
}

template <int MODE>
struct AdjBounds { static constexpr int MIN_CTAS = 4; };
template <>
struct AdjBounds<2> { static constexpr int MIN_CTAS = 3; };
template <>
struct AdjBounds<4> { static constexpr int MIN_CTAS = 3; };   // 80 registers, no spills (measured 0.6 % faster than 4)

// One work item of the reverse step (see the forward's fwd_item): returns
// false when a bounded wait ran out (status set, every issued box waited
// for); the caller must then leave.  The shared memory at `raw` holds the
// layout of this mode; the mbarriers sit at the same offsets in every mode.
template <int TY, int MODE>
__device__ __forceinline__ bool adj_item(unsigned char* raw, const RfxbInst* __restrict__ insts,
                                         const AdjInst* __restrict__ adjs, const RfxbWork w,
                                         const CUtensorMap* __restrict__ maps, int n, int par, int apar, int zp,
                                         StepPhases& ph, const StepFault& fault, bool first_item) {
  constexpr bool TMA = MODE != 0;
  constexpr bool RING = MODE == 2 || MODE == 4;       // psi ring
  constexpr bool YS = MODE != 4;                      // y-slab relations compiled in
  constexpr int NST = RING ? 3 : RFXB_ANSTAGE;        // plane stages
  using L = APsiSlot<TY, YS>;
  using SM = AdjSmem<TY, MODE != 4>;
  SM& S = *reinterpret_cast<SM*>(raw);
  float* ring = reinterpret_cast<float*>(&S.st[NST]);   // modes 2, 4: two psi slots after the stages
  auto& rx = *reinterpret_cast<AdjExchange<TY>*>(&S.st[NST]);   // modes 0, 1: the exchange array
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + lane;
  load_inst(S.P, insts + w.inst, tid, 32 * TY);
  {
    const int nw = sizeof(AdjInst) / 4;
    const int* s = reinterpret_cast<const int*>(adjs + w.inst);
    int* d = reinterpret_cast<int*>(&S.A);
    for (int t = tid; t < nw; t += 32 * TY) d[t] = __ldg(s + t);
  }
  __syncthreads();
  const int wlim = fault.wait_limit;
  // the thread that issues the TMA boxes: lane 0 of the last warp (warps 0
  // and 1 compute the halo row and column of phase A)
  const int producer = 32 * (TY - 1);
  const bool skip_first = first_item && (int)blockIdx.x == fault.cta;
  const CUtensorMap* tm = maps + (size_t)w.inst * RFXB_NMAPS;
  const RfxbInst& P = S.P;
  const AdjInst& A = S.A;
  AdjCtx C;
  C.nx = P.nx; C.ny = P.ny; C.nz = P.nz; C.zs = P.zs; C.ncp = P.ncp; C.par = par; C.apar = apar;
  C.ps = P.ps; C.off0 = P.off0; C.cs = P.cs;
  C.ch = P.ch;
  C.ch0 = P.ch0;
  const int y0 = w.y0, z0 = w.z0;
  // the +1 neighbours of the tile (row y0+TY, column z0+32) also read CPML terms
  C.cpx = MODE != 3 && C.ncp > 0 && (P.cpml_axes & 1u);
  C.cpy = MODE != 3 && YS && C.ncp > 0 && (P.cpml_axes & 2u) && (y0 - 1 < C.ncp || y0 + TY >= C.ny - C.ncp);
  C.cpz = MODE != 3 && C.ncp > 0 && (P.cpml_axes & 4u) && (z0 - 1 < C.ncp || z0 + 32 >= C.nz - C.ncp);
  const float* aF0 = A.aF[apar][0];
  float* aFo = A.aF[apar ^ 1][0];
  const int j = y0 + ty, k = z0 + lane;
  const bool own = (j < C.ny) && (k < C.nz);
  const int ly = ty + 1, lz = lane + 4, lh = lane + 1;
  auto chat = [&](int i_, int j_, int k_) { return C.ch ? C.ch[cell_index(C, i_, j_, k_)] : C.ch0; };
  const float ye0 = own ? __ldg(P.ye + j) : 0.f, ye1 = own ? __ldg(P.ye + j + 1) : 0.f;
  const float ze0 = own ? __ldg(P.ze + k) : 0.f, ze1 = own ? __ldg(P.ze + k + 1) : 0.f;
  const float yh0 = own ? __ldg(P.yh + j) : 0.f, yhm = own ? __ldg(P.yh + j - 1) : 0.f;
  const float zh0 = own ? __ldg(P.zh + k) : 0.f, zhm = own ? __ldg(P.zh + k - 1) : 0.f;
  const bool row_halo = (ty == 0) && (y0 >= 1) && (k < C.nz);
  const float ye0_r = row_halo ? __ldg(P.ye + y0 - 1) : 0.f, ye1_r = row_halo ? __ldg(P.ye + y0) : 0.f;
  const float ze0_r = row_halo ? __ldg(P.ze + k) : 0.f, ze1_r = row_halo ? __ldg(P.ze + k + 1) : 0.f;
  const int hcw = TY > 1 ? 1 : 0;
  const bool col_halo = (ty == hcw) && (lane < TY) && (z0 >= 1) && (y0 + lane < C.ny);
  const float ye0_c = col_halo ? __ldg(P.ye + y0 + lane) : 0.f, ye1_c = col_halo ? __ldg(P.ye + y0 + lane + 1) : 0.f;
  const float ze0_c = col_halo ? __ldg(P.ze + z0 - 1) : 0.f, ze1_c = col_halo ? __ldg(P.ze + z0) : 0.f;
  const unsigned pec = P.pec_axes;
  const bool pec_j = ((pec & 2u) != 0) && (j == 0 || j == C.ny - 1);
  const bool pec_k0 = ((pec & 4u) != 0) && (k == 0 || k == C.nz - 1);
  const bool pec_kz = ((pec & 4u) != 0) && (k == C.nz - 1);
  // probes (cotangent injection) and sources (adjoint read-out) on this column
  unsigned pmask = 0u, smask = 0u;
  if (own) {
    const int np = min(P.nprb, 32);
    for (int q = 0; q < np; ++q) { const int4 c = __ldg(P.prb + q); if (c.y == j && c.z == k) pmask |= 1u << q; }
    const int ns = min(P.nsrc, 32);
    for (int q = 0; q < ns; ++q) { const int4 c = __ldg(P.src + q); if (c.y == j && c.z == k) smask |= 1u << q; }
  }
  const bool prb_tail = P.nprb > 32, src_tail = P.nsrc > 32;
  const bool in_gyz = P.grad && j >= P.hb[2] && j < P.hb[3] && k >= P.hb[4] && k < P.hb[5];
  const bool hist_ok = P.hist && (n - P.hist_step0) >= 0 && (n - P.hist_step0) < P.hist_nsteps;

  const int xa = w.xa, xb = w.xb;
  const float* ca = P.ca;
  const float* cb = P.cb;
  // mode-2 psi ring: the slab side this tile reaches per axis, and the
  // bookkeeping of the two slots (identical in every thread)
  const bool yz_tile = C.cpy || C.cpz;
  const int ysd = (RING && C.cpy) ? atile_side(y0 - 1, y0 + TY, C.ny, C.ncp) : -1;
  const int zsd = (RING && C.cpz) ? atile_side(z0 - 1, z0 + 32, C.nz, C.ncp) : -1;
  const int n4 = P.ncp4;
  auto xslab = [&](int p) { return C.cpx && p >= 0 && p < C.nx && (p < C.ncp || p >= C.nx - C.ncp); };
  auto psi_need = [&](int p) {
    if (!RING || p < 0 || p >= C.nx) return false;
    return yz_tile || xslab(p) || xslab(p + 1);
  };
  unsigned& pph = ph.ring;
  unsigned pout = 0u;
  // completion parity of the stage holding plane p (the k-th fill of a stage
  // in this item is k phases past where the previous items left it)
  auto sparity = [&](int p) -> uint32_t {
    return ((ph.stage >> astage_of<NST>(p)) ^ (uint32_t)((p - xa + 1) / NST)) & 1u;
  };
  auto psi_fill = [&](int p) {
    if (!psi_need(p)) return;
    if (tid == producer)
      apsi_issue<TY, YS>(ring + (p & 1) * L::FLOATS(zp), smem_u32(&S.pbar[p & 1]), tm, C, zp, y0, z0, p, yz_tile, ysd,
                     zsd, n4);
    pout |= 1u << (p & 1);
  };
  auto psi_wait = [&](int p) -> bool {
    if (!psi_need(p)) return true;
    const int sl = p & 1;
    const bool ok = mbar_wait_bounded(smem_u32(&S.pbar[sl]), (pph >> sl) & 1u, wlim);
    if (ok) {
      pph ^= 1u << sl;
      pout &= ~(1u << sl);
    }
    return ok;
  };
  auto bail = [&](int last_issued, int from) {
    if (tid == 0) {
      atomicOr(P.status, 1);
      for (int p = from; p <= last_issued; ++p)
        mbar_wait_bounded(smem_u32(&S.mbar[astage_of<NST>(p)]), sparity(p), wlim);
      for (int sl = 0; sl < 2; ++sl)
        if (pout & (1u << sl)) mbar_wait_bounded(smem_u32(&S.pbar[sl]), (pph >> sl) & 1u, wlim);
    }
  };
  if (TMA) {
    if (tid == producer)
      for (int p = xa - 1; p <= min(xa + NST - 2, xb); ++p)
        if (!(skip_first && p == xa)) adj_tma_stage<TY, NST>(S, tm, apar, y0, z0, p);
    psi_fill(xa);
    const bool ok = mbar_wait_bounded(smem_u32(&S.mbar[astage_of<NST>(xa - 1)]), sparity(xa - 1), wlim) &&
                    mbar_wait_bounded(smem_u32(&S.mbar[astage_of<NST>(xa)]), sparity(xa), wlim);
    if (__syncthreads_or(!ok)) { bail(min(xa + NST - 2, xb), xa - 1); return false; }
  } else {
    adj_load_stage<TY>(S, C, aF0, ca, cb, y0, z0, xa - 1, tid);
    adj_load_stage<TY>(S, C, aF0, ca, cb, y0, z0, xa, tid);
    cp_async_commit();
    adj_load_stage<TY>(S, C, aF0, ca, cb, y0, z0, xa + 1, tid);
    cp_async_commit();
    if (xa + 2 <= xb) adj_load_stage<TY>(S, C, aF0, ca, cb, y0, z0, xa + 2, tid);
    cp_async_commit();
    cp_async_wait<2>();
    __syncthreads();
  }

  // phase A of plane xa-1 at this column: p and r_H there (not stored)
  float py_prev = 0.f, pz_prev = 0.f, rhy_prev = 0.f, rhz_prev = 0.f;
  if (xa > 0 && own) {
    float a1, a2, a3;
    const int im = xa - 1;
    adj_a_cell<TY, 6>(P, A, S, C, astage_of<NST>(im), astage_of<NST>(xa), im, j, k, ly, lz, __ldg(P.xe + im),
                      __ldg(P.xe + xa), ye0, ye1, ze0, ze1, false, a1, a2, a3);
    if (P.g) {   // H-probe cotangent of y_n at plane xa-1
      for (unsigned m = pmask; m; m &= m - 1) {
        const int q = __ffs(m) - 1;
        const int4 c = __ldg(P.prb + q);
        if (c.x == im && (c.w & 7) >= 4) {
          const float gv = __ldg(P.g + (long long)n * P.g_ld + q);
          if ((c.w & 7) == 4) a2 += gv; else a3 += gv;
        }
      }
      if (prb_tail)
        for (int q = 32; q < P.nprb; ++q) {
          const int4 c = __ldg(P.prb + q);
          if (c.x == im && c.y == j && c.z == k && (c.w & 7) >= 4) {
            const float gv = __ldg(P.g + (long long)n * P.g_ld + q);
            if ((c.w & 7) == 4) a2 += gv; else a3 += gv;
          }
        }
    }
    const float chc = chat(im, j, k);
    py_prev = chc * a2;
    pz_prev = chc * a3;
    if (C.cpx) {
      rhy_prev = r_h(P, A, C, 0, 0, +1.f, im, j, k, py_prev, false);
      rhz_prev = r_h(P, A, C, 0, 1, -1.f, im, j, k, pz_prev, false);
    }
  }

  // The x relations of CPML-E^T are carried along the march: r_E of plane i
  // at this column (q0: ey <- hz, q1: ez <- hy) and at this thread's halo
  // cell (row y0-1: q0; column z0-1: q1) is evaluated one plane ahead; the
  // CTA owning a plane writes its psi when it evaluates it.
  float rx0 = 0.f, rx1 = 0.f, rxh = 0.f;
  if (C.cpx) {
    const auto& X0 = S.st[astage_of<NST>(xa)];
    if (own) {
      const float ce = P.ce[cell_index(C, xa, j, k)];
      rx0 = re_eval(P, A, C, 0, 0, -1.f, xa, j, k, X0.ae[1][ly][lz], ce, true);
      rx1 = re_eval(P, A, C, 0, 1, +1.f, xa, j, k, X0.ae[2][ly][lz], ce, true);
    }
    if (row_halo)
      rxh = re_eval(P, A, C, 0, 0, -1.f, xa, y0 - 1, k, X0.ae[1][0][lz], P.ce[cell_index(C, xa, y0 - 1, k)], false);
    if (col_halo)
      rxh = re_eval(P, A, C, 0, 1, +1.f, xa, y0 + lane, z0 - 1, X0.ae[2][lane + 1][3],
                    P.ce[cell_index(C, xa, y0 + lane, z0 - 1)], false);
  }

  // x spacing entries of the next plane, loaded one plane ahead
  const float* xe_tab = P.xe;
  const float* xh_tab = P.xh;
  float xe1_n = __ldg(xe_tab + xa + 1), xhm_n = __ldg(xh_tab + xa - 1);
  float xe0_n = __ldg(xe_tab + xa), xh0_n = __ldg(xh_tab + xa);

  for (int i = xa; i < xb; ++i) {
    const float xe0 = xe0_n, xe1 = xe1_n, xh0 = xh0_n, xhm = xhm_n;
    if (i + 1 < xb) {
      xe0_n = xe1;
      xhm_n = xh0;
      xe1_n = __ldg(xe_tab + i + 2);
      xh0_n = __ldg(xh_tab + i + 1);
    }
    if (TMA) {
      // plane i+1 (and plane i's psi) have landed; after the barrier plane
      // i-1's stage takes plane i+NST-1 and its psi slot plane i+1
      const bool ok = mbar_wait_bounded(smem_u32(&S.mbar[astage_of<NST>(i + 1)]), sparity(i + 1), wlim) && psi_wait(i);
      if (__syncthreads_or(!ok)) { bail(min(i + NST - 2, xb), i + 1); return false; }
      if (tid == producer && i + NST - 1 <= xb) adj_tma_stage<TY, NST>(S, tm, apar, y0, z0, i + NST - 1);
      if (i + 1 < xb) psi_fill(i + 1);
    } else {
      cp_async_wait<1>();
      __syncthreads();
      if (i + 3 <= xb) adj_load_stage<TY>(S, C, aF0, ca, cb, y0, z0, i + 3, tid);
      cp_async_commit();
    }
    const int b0 = astage_of<NST>(i), b1 = astage_of<NST>(i + 1);
    const float* PS = ring + (i & 1) * L::FLOATS(zp);
    // Mode 2: r_E / r_H of the y (axes bit 1) and z (bit 2) relations at
    // footprint position (r, c) = (jj - y0 + 1, kk - z0 + 1), evaluated from
    // the staged plane and the psi ring; .x .y: y relations q0 q1, .z .w: z
    // relations q0 q1; zero outside the grid and the slabs.  Each cell reads
    // its neighbours' relations this way, so no exchange barrier is needed.
    auto re_at = [&](int r, int c, int axes, bool write) -> float4 {
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      const int jj = y0 - 1 + r, kk = z0 - 1 + c;
      if (jj < 0 || jj >= C.ny || kk < 0 || kk >= C.nz) return v;
      int sy = 0, sz = 0;
      const int dy = ((axes & 1) && C.cpy) ? cpml_side(jj, C.ny, C.ncp, sy) : -1;
      const int dz = ((axes & 2) && C.cpz) ? cpml_side(kk, C.nz, C.ncp, sz) : -1;
      if (dy < 0 && dz < 0) return v;
      const auto& X = S.st[b0];
      const float ce = PS[L::CE + r * RFXB_AEW + c + 3];
      const float ax = X.ae[0][r][c + 3];
      if (dy >= 0) {
        const float4 cf = __ldg(P.cpt + (2 + dy) * C.ncp + sy);
        const int o = r * RFXB_AEW + c + 3;
        v.x = re_core(A, C, 1, cf, write ? psi_q(P, 1, dy, 0, sy, i, jj, kk) : 0, PS[L::EY + o], +1.f, ce, ax,
                      write);                                                           // ex <- hz
        v.y = re_core(A, C, 1, cf, write ? psi_q(P, 1, dy, 1, sy, i, jj, kk) : 0,
                      PS[L::EY + (TY + 2) * RFXB_AEW + o], -1.f, ce, X.ae[2][r][c + 3], write);   // ez <- hx
      }
      if (dz >= 0) {
        const float4 cf = __ldg(P.cpt + (4 + dz) * C.ncp + sz);
        const int o = r * n4 + sz;
        v.z = re_core(A, C, 2, cf, write ? psi_q(P, 2, dz, 0, sz, i, jj, kk) : 0, PS[L::EZ + o], -1.f, ce, ax,
                      write);                                                           // ex <- hy
        v.w = re_core(A, C, 2, cf, write ? psi_q(P, 2, dz, 1, sz, i, jj, kk) : 0, PS[L::EZ + (TY + 2) * n4 + o],
                      +1.f, ce, X.ae[1][r][c + 3], write);                              // ey <- hx
      }
      return v;
    };
    auto rh_at = [&](int r, int c, int axes, bool write) -> float4 {
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      const int jj = y0 - 1 + r, kk = z0 - 1 + c;
      if (jj < 0 || jj >= C.ny || kk < 0 || kk >= C.nz) return v;
      int sy = 0, sz = 0;
      const int dy = ((axes & 1) && C.cpy) ? cpml_side(jj, C.ny, C.ncp, sy) : -1;
      const int dz = ((axes & 2) && C.cpz) ? cpml_side(kk, C.nz, C.ncp, sz) : -1;
      if (dy < 0 && dz < 0) return v;
      const float p0 = S.p[0][r][c];
      if (dy >= 0) {
        const float4 cf = __ldg(P.cpt + (2 + dy) * C.ncp + sy);
        const int o = r * RFXB_AHW + c + 3;
        v.x = rh_core(A, C, 1, cf, write ? psi_q(P, 1, dy, 0, sy, i, jj, kk) : 0, PS[L::HY + o], -1.f, p0,
                      write);                                                           // hx <- ez
        v.y = rh_core(A, C, 1, cf, write ? psi_q(P, 1, dy, 1, sy, i, jj, kk) : 0,
                      PS[L::HY + (TY + 1) * RFXB_AHW + o], +1.f, S.p[2][r][c], write);  // hz <- ex
      }
      if (dz >= 0) {
        const float4 cf = __ldg(P.cpt + (4 + dz) * C.ncp + sz);
        const int hz = L::HZ(zp), o = r * n4 + sz;
        v.z = rh_core(A, C, 2, cf, write ? psi_q(P, 2, dz, 0, sz, i, jj, kk) : 0, PS[hz + o], +1.f, p0,
                      write);                                                           // hx <- ey
        v.w = rh_core(A, C, 2, cf, write ? psi_q(P, 2, dz, 1, sz, i, jj, kk) : 0, PS[hz + (TY + 1) * n4 + o],
                      -1.f, S.p[1][r][c], write);                                       // hy <- ex
      }
      return v;
    };
    const long long e = cell_index(C, i, j, k);

    // x relations of plane i+1 (written by this CTA when it owns that plane)
    float nx0 = 0.f, nx1 = 0.f, nxh = 0.f;
    if (RING && xslab(i + 1)) {   // psi and ce of plane i+1 from the ring
      const auto& Y1 = S.st[b1];
      const bool wr = i + 1 < xb;
      int sx;
      const int sd = cpml_side(i + 1, C.nx, C.ncp, sx);
      const float4 cf = __ldg(P.cpt + sd * C.ncp + sx);
      constexpr int RQ = (TY + 1) * RFXB_AHW;
      auto xnext = [&](int r, int zc, int jj, int kk, float at0, float at1, bool write, float& v0, float& v1) {
        const float ce = PS[L::CEN + r * RFXB_AHW + zc];
        v0 = re_core(A, C, 0, cf, psi_q(P, 0, sd, 0, sx, i + 1, jj, kk), PS[L::EXN + r * RFXB_AHW + zc], -1.f, ce,
                     at0, write);
        v1 = re_core(A, C, 0, cf, psi_q(P, 0, sd, 1, sx, i + 1, jj, kk), PS[L::EXN + RQ + r * RFXB_AHW + zc], +1.f,
                     ce, at1, write);
      };
      if (own) xnext(ly, lz, j, k, Y1.ae[1][ly][lz], Y1.ae[2][ly][lz], wr, nx0, nx1);
      float d0 = 0.f, d1 = 0.f;
      if (row_halo) { xnext(0, lz, y0 - 1, k, Y1.ae[1][0][lz], 0.f, false, d0, d1); nxh = d0; }
      if (col_halo) {
        xnext(lane + 1, 3, y0 + lane, z0 - 1, 0.f, Y1.ae[2][lane + 1][3], false, d0, d1);
        nxh = d1;
      }
    } else if (!RING && C.cpx && i + 1 < C.nx) {
      const auto& Y1 = S.st[b1];
      const bool wr = i + 1 < xb;
      if (own) {
        const float ce = P.ce[e + C.ps];
        nx0 = re_eval(P, A, C, 0, 0, -1.f, i + 1, j, k, Y1.ae[1][ly][lz], ce, wr);
        nx1 = re_eval(P, A, C, 0, 1, +1.f, i + 1, j, k, Y1.ae[2][ly][lz], ce, wr);
      }
      if (row_halo)
        nxh = re_eval(P, A, C, 0, 0, -1.f, i + 1, y0 - 1, k, Y1.ae[1][0][lz],
                      P.ce[cell_index(C, i + 1, y0 - 1, k)], false);
      if (col_halo)
        nxh = re_eval(P, A, C, 0, 1, +1.f, i + 1, y0 + lane, z0 - 1, Y1.ae[2][lane + 1][3],
                      P.ce[cell_index(C, i + 1, y0 + lane, z0 - 1)], false);
    }

    // Modes 0 / 1: r_E of the y / z relations at the tile, its +1 row /
    // column and the halo cells, once per cell into the exchange array (own
    // cells write their psi)
    if (!RING && yz_tile) {
      const auto& X = S.st[b0];
      auto re_fill = [&](int r, int c, bool write) {
        const int jj = y0 - 1 + r, kk = z0 - 1 + c;
        float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
        if (jj >= 0 && jj < C.ny && kk >= 0 && kk < C.nz && in_yz_slab(C, jj, kk)) {
          const float ce = P.ce[cell_index(C, i, jj, kk)];
          const float ax = X.ae[0][r][c + 3], ay = X.ae[1][r][c + 3], az = X.ae[2][r][c + 3];
          if (C.cpy) {
            v0 = re_eval(P, A, C, 1, 0, +1.f, i, jj, kk, ax, ce, write);   // ex <- hz
            v1 = re_eval(P, A, C, 1, 1, -1.f, i, jj, kk, az, ce, write);   // ez <- hx
          }
          if (C.cpz) {
            v2 = re_eval(P, A, C, 2, 0, -1.f, i, jj, kk, ax, ce, write);   // ex <- hy
            v3 = re_eval(P, A, C, 2, 1, +1.f, i, jj, kk, ay, ce, write);   // ey <- hx
          }
        }
        rx[0][r][c] = v0;
        rx[1][r][c] = v1;
        rx[2][r][c] = v2;
        rx[3][r][c] = v3;
      };
      re_fill(ly, lh, own);
      constexpr int W = RFXB_TZ + 2;
      // the extra cells go to the last warps (warps 0 and 1 carry the phase-A
      // halo row and column, the middle warps the phase-B extras)
      const int t = tid - (32 * TY - (2 * W + 2 * TY));
      if (t >= 0) {
        if (t < W) re_fill(0, t, false);
        else if (t < 2 * W) re_fill(TY + 1, t - W, false);
        else if (t < 2 * W + TY) re_fill(t - 2 * W + 1, 0, false);
        else re_fill(t - 2 * W - TY + 1, W - 1, false);
      }
      __syncthreads();
    }

    // ---- phase A ----
    float ahx = 0.f, ahy = 0.f, ahz = 0.f;
    float4 rown = make_float4(0.f, 0.f, 0.f, 0.f);   // mode 2: this cell's y / z r_E
    if (own) {
      adj_a_cell<TY, 7, false>(P, A, S, C, b0, b1, i, j, k, ly, lz, xe0, xe1, ye0, ye1, ze0, ze1, true, ahx, ahy,
                               ahz);
      if (C.cpx) { ahz += rx0 - nx0; ahy += rx1 - nx1; }
      if (RING) {
        if (yz_tile) {
          rown = re_at(ly, lh, 3, true);
          if (C.cpy) {
            const float4 ry = re_at(ly + 1, lh, 1, false);
            ahz += rown.x - ry.x;
            ahx += rown.y - ry.y;
          }
          if (C.cpz) {
            const float4 rz = re_at(ly, lh + 1, 2, false);
            ahy += rown.z - rz.z;
            ahx += rown.w - rz.w;
          }
        }
      } else {
        if (C.cpy) {
          ahz += rx[0][ly][lh] - rx[0][ly + 1][lh];
          ahx += rx[1][ly][lh] - rx[1][ly + 1][lh];
        }
        if (C.cpz) {
          ahy += rx[2][ly][lh] - rx[2][ly][lh + 1];
          ahx += rx[3][ly][lh] - rx[3][ly][lh + 1];
        }
      }
      if (P.g && (pmask || prb_tail)) {   // H-probe cotangent of y_n
        for (unsigned m = pmask; m; m &= m - 1) {
          const int q = __ffs(m) - 1;
          const int4 c = __ldg(P.prb + q);
          if (c.x == i && (c.w & 7) >= 3) {
            const float gv = __ldg(P.g + (long long)n * P.g_ld + q);
            if ((c.w & 7) == 3) ahx += gv; else if ((c.w & 7) == 4) ahy += gv; else ahz += gv;
          }
        }
        if (prb_tail)
          for (int q = 32; q < P.nprb; ++q) {
            const int4 c = __ldg(P.prb + q);
            if (c.x == i && c.y == j && c.z == k && (c.w & 7) >= 3) {
              const float gv = __ldg(P.g + (long long)n * P.g_ld + q);
              if ((c.w & 7) == 3) ahx += gv; else if ((c.w & 7) == 4) ahy += gv; else ahz += gv;
            }
          }
      }
      aFo[3 * C.cs + e] = ahx;
      aFo[4 * C.cs + e] = ahy;
      aFo[5 * C.cs + e] = ahz;
      if (in_gyz && hist_ok && i >= P.hb[0] && i < P.hb[1]) {
        const int sy = P.hb[3] - P.hb[2], sz = P.hb[5] - P.hb[4];
        const int hc = (P.hb[1] - P.hb[0]) * sy * sz;
        const int ci = ((i - P.hb[0]) * sy + (j - P.hb[2])) * sz + (k - P.hb[4]);
        const float* hp = P.hist + (long long)(n - P.hist_step0) * P.hist_ld + ci;
        const float dca = P.dca[ci], dcb = P.dcb[ci];
        const auto& X = S.st[b0];
        const double acc = (double)X.ae[0][ly][lz] * ((double)dca * hp[0] + (double)dcb * hp[3 * hc]) +
                           (double)X.ae[1][ly][lz] * ((double)dca * hp[hc] + (double)dcb * hp[4 * hc]) +
                           (double)X.ae[2][ly][lz] * ((double)dca * hp[2 * hc] + (double)dcb * hp[5 * hc]);
        P.grad[ci] += acc;
      }
    }
    const float chc = own ? chat(i, j, k) : 0.f;
    S.p[0][ly][lh] = chc * ahx;
    S.p[1][ly][lh] = chc * ahy;
    S.p[2][ly][lh] = chc * ahz;
    if (ty == 0) {   // halo row j = y0 - 1: hx, hz
      float a1 = 0.f, a2 = 0.f, a3 = 0.f;
      float chr = 0.f;
      if (row_halo) {
        adj_a_cell<TY, 5, false>(P, A, S, C, b0, b1, i, y0 - 1, k, 0, lz, xe0, xe1, ye0_r, ye1_r, ze0_r, ze1_r,
                                 false, a1, a2, a3);
        if (C.cpx) a3 += rxh - nxh;
        if (RING) {   // row y0 is this thread's own row: its r_E is rown
          if (C.cpy) {
            const float4 r0 = re_at(0, lh, 1, false);
            a3 += r0.x - rown.x;
            a1 += r0.y - rown.y;
          }
          if (C.cpz) a1 += re_at(0, lh, 2, false).w - re_at(0, lh + 1, 2, false).w;
        } else {
          if (C.cpy) {
            a3 += rx[0][0][lh] - rx[0][1][lh];
            a1 += rx[1][0][lh] - rx[1][1][lh];
          }
          if (C.cpz) a1 += rx[3][0][lh] - rx[3][0][lh + 1];
        }
        chr = chat(i, y0 - 1, k);
        if (P.g) {
          for (int q = 0; q < P.nprb; ++q) {
            const int4 c = __ldg(P.prb + q);
            if (c.x == i && c.y == y0 - 1 && c.z == k && ((c.w & 7) == 3 || (c.w & 7) == 5)) {
              const float gv = __ldg(P.g + (long long)n * P.g_ld + q);
              if ((c.w & 7) == 3) a1 += gv; else a3 += gv;
            }
          }
        }
      }
      S.p[0][0][lh] = chr * a1;
      S.p[2][0][lh] = chr * a3;
    }
    if (ty == hcw && lane < TY) {   // halo column k = z0 - 1: hx, hy
      float a1 = 0.f, a2 = 0.f, a3 = 0.f;
      float chz = 0.f;
      if (col_halo) {
        adj_a_cell<TY, 3, false>(P, A, S, C, b0, b1, i, y0 + lane, z0 - 1, lane + 1, 3, xe0, xe1, ye0_c, ye1_c,
                                 ze0_c, ze1_c, false, a1, a2, a3);
        const int r = lane + 1;
        if (C.cpx) a2 += rxh - nxh;
        if (RING) {
          if (C.cpy) a1 += re_at(r, 0, 1, false).y - re_at(r + 1, 0, 1, false).y;
          if (C.cpz) {
            const float4 z0v = re_at(r, 0, 2, false), z1v = re_at(r, 1, 2, false);
            a2 += z0v.z - z1v.z;
            a1 += z0v.w - z1v.w;
          }
        } else {
          if (C.cpy) a1 += rx[1][r][0] - rx[1][r + 1][0];
          if (C.cpz) {
            a2 += rx[2][r][0] - rx[2][r][1];
            a1 += rx[3][r][0] - rx[3][r][1];
          }
        }
        chz = chat(i, y0 + lane, z0 - 1);
        if (P.g) {
          for (int q = 0; q < P.nprb; ++q) {
            const int4 c = __ldg(P.prb + q);
            if (c.x == i && c.y == y0 + lane && c.z == z0 - 1 && ((c.w & 7) == 3 || (c.w & 7) == 4)) {
              const float gv = __ldg(P.g + (long long)n * P.g_ld + q);
              if ((c.w & 7) == 3) a1 += gv; else a2 += gv;
            }
          }
        }
      }
      S.p[0][lane + 1][0] = chz * a1;
      S.p[1][lane + 1][0] = chz * a2;
    }
    __syncthreads();

    // Modes 0 / 1: r_H of the y / z relations at the tile and the low halo
    // row / column (rows y0-1 .. y0+TY-1, columns z0-1 .. z0+31), once per
    // cell into the exchange array
    if (!RING && yz_tile) {
      auto rh_fill = [&](int r, int c, bool write, bool ny_, bool nz_) {
        const int jj = y0 - 1 + r, kk = z0 - 1 + c;
        float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
        if (jj >= 0 && jj < C.ny && kk >= 0 && kk < C.nz && in_yz_slab(C, jj, kk)) {
          if (C.cpy && ny_) {
            v0 = rh_eval(P, A, C, 1, 0, -1.f, i, jj, kk, S.p[0][r][c], write);   // hx <- ez
            v1 = rh_eval(P, A, C, 1, 1, +1.f, i, jj, kk, S.p[2][r][c], write);   // hz <- ex
          }
          if (C.cpz && nz_) {
            v2 = rh_eval(P, A, C, 2, 0, +1.f, i, jj, kk, S.p[0][r][c], write);   // hx <- ey
            v3 = rh_eval(P, A, C, 2, 1, -1.f, i, jj, kk, S.p[1][r][c], write);   // hy <- ex
          }
        }
        rx[0][r][c] = v0;
        rx[1][r][c] = v1;
        rx[2][r][c] = v2;
        rx[3][r][c] = v3;
      };
      rh_fill(ly, lh, own, true, true);
      const int t = tid - 64;   // warps 2 and 3
      if (t >= 0 && t < RFXB_TZ) rh_fill(0, t + 1, false, true, false);                     // row y0-1: y relations
      else if (t >= RFXB_TZ && t < RFXB_TZ + TY) rh_fill(t - RFXB_TZ + 1, 0, false, false, true);   // column z0-1
      __syncthreads();
    }

    // ---- phase B ----
    float py = 0.f, pz = 0.f;
    float rhy = 0.f, rhz = 0.f;
    if (own) {
      const auto& X = S.st[b0];
      const float px = S.p[0][ly][lh];
      py = S.p[1][ly][lh];
      pz = S.p[2][ly][lh];
      const float px_ym = S.p[0][ly - 1][lh], pz_ym = S.p[2][ly - 1][lh];
      const float px_zm = S.p[0][ly][lh - 1], py_zm = S.p[1][ly][lh - 1];
      const float cav = X.ca[ty][lane];
      float ax = cav * X.ae[0][ly][lz] + ((zh0 * py - zhm * py_zm) - (yh0 * pz - yhm * pz_ym));
      float ay = cav * X.ae[1][ly][lz] + ((xh0 * pz - xhm * pz_prev) - (zh0 * px - zhm * px_zm));
      float az = cav * X.ae[2][ly][lz] + ((yh0 * px - yhm * px_ym) - (xh0 * py - xhm * py_prev));
      if (C.cpx) {   // (hy <- ez, +1, q0), (hz <- ey, -1, q1): aE(x) += r(x-1) - r(x)
        if (RING) {
          if (xslab(i)) {
            int sx;
            const int sd = cpml_side(i, C.nx, C.ncp, sx);
            const float4 cf = __ldg(P.cpt + sd * C.ncp + sx);
            const int o = ty * RFXB_TZ + lane;
            rhy = rh_core(A, C, 0, cf, psi_q(P, 0, sd, 0, sx, i, j, k), PS[L::HX + o], +1.f, py, true);
            rhz = rh_core(A, C, 0, cf, psi_q(P, 0, sd, 1, sx, i, j, k), PS[L::HX + TY * RFXB_TZ + o], -1.f, pz, true);
          }
        } else {
          rhy = rh_eval(P, A, C, 0, 0, +1.f, i, j, k, py, true);
          rhz = rh_eval(P, A, C, 0, 1, -1.f, i, j, k, pz, true);
        }
        az += rhy_prev - rhy;
        ay += rhz_prev - rhz;
      }
      if (RING) {
        if (yz_tile) {
          const float4 rh = rh_at(ly, lh, 3, true);
          if (C.cpy) {   // (hx <- ez, -1, q0), (hz <- ex, +1, q1)
            const float4 ry = rh_at(ly - 1, lh, 1, false);
            az += ry.x - rh.x;
            ax += ry.y - rh.y;
          }
          if (C.cpz) {   // (hx <- ey, +1, q0), (hy <- ex, -1, q1)
            const float4 rz = rh_at(ly, lh - 1, 2, false);
            ay += rz.z - rh.z;
            ax += rz.w - rh.w;
          }
        }
      } else {
        if (C.cpy) {   // (hx <- ez, -1, q0), (hz <- ex, +1, q1)
          az += rx[0][ly - 1][lh] - rx[0][ly][lh];
          ax += rx[1][ly - 1][lh] - rx[1][ly][lh];
        }
        if (C.cpz) {   // (hx <- ey, +1, q0), (hy <- ex, -1, q1)
          ay += rx[2][ly][lh - 1] - rx[2][ly][lh];
          ax += rx[3][ly][lh - 1] - rx[3][ly][lh];
        }
      }
      if (n >= 1 && (pmask | smask | (unsigned)prb_tail | (unsigned)src_tail)) {
        if (P.g) {   // E-probe cotangent of y_{n-1}
          for (unsigned m = pmask; m; m &= m - 1) {
            const int q = __ffs(m) - 1;
            const int4 c = __ldg(P.prb + q);
            if (c.x == i && (c.w & 7) < 3) {
              const float gv = __ldg(P.g + (long long)(n - 1) * P.g_ld + q);
              if ((c.w & 7) == 0) ax += gv; else if ((c.w & 7) == 1) ay += gv; else az += gv;
            }
          }
          if (prb_tail)
            for (int q = 32; q < P.nprb; ++q) {
              const int4 c = __ldg(P.prb + q);
              if (c.x == i && c.y == j && c.z == k && (c.w & 7) < 3) {
                const float gv = __ldg(P.g + (long long)(n - 1) * P.g_ld + q);
                if ((c.w & 7) == 0) ax += gv; else if ((c.w & 7) == 1) ay += gv; else az += gv;
              }
            }
        }
        if (P.src_adj) {
          for (unsigned m = smask; m; m &= m - 1) {
            const int q = __ffs(m) - 1;
            const int4 c = __ldg(P.src + q);
            if (c.x == i) P.src_adj[(long long)(n - 1) * P.src_ld + q] = c.w == 0 ? ax : c.w == 1 ? ay : az;
          }
          if (src_tail)
            for (int q = 32; q < P.nsrc; ++q) {
              const int4 c = __ldg(P.src + q);
              if (c.x == i && c.y == j && c.z == k)
                P.src_adj[(long long)(n - 1) * P.src_ld + q] = c.w == 0 ? ax : c.w == 1 ? ay : az;
            }
        }
      }
      if ((pec & 1u) && (i == 0 || i == C.nx - 1)) { ay = 0.f; az = 0.f; }
      if (pec_j) { ax = 0.f; az = 0.f; }
      if (pec_k0) { ax = 0.f; ay = 0.f; }
      if (pec_kz) az = 0.f;
      if (P.emask) {
        unsigned m;
        if constexpr (MODE == 4) m = (unsigned)P.emask[e];   // not staged on this variant
        else m = TMA ? (unsigned)X.em[ty][lane] : (unsigned)P.emask[e];
        if (m & 1u) ax = 0.f;
        if (m & 2u) ay = 0.f;
        if (m & 4u) az = 0.f;
      }
      aFo[e] = ax;
      aFo[C.cs + e] = ay;
      aFo[2 * C.cs + e] = az;
    }
    py_prev = py;
    pz_prev = pz;
    rhy_prev = rhy;
    rhz_prev = rhz;
    rx0 = nx0;
    rx1 = nx1;
    rxh = nxh;
  }
  if (!TMA) cp_async_wait<0>();
  if (TMA) {   // the phases this item advanced: stage s filled by planes xa-1 .. xb
    const int T = xb - xa + 2;
    for (int st = 0; st < NST; ++st) {
      const int fills = T / NST + ((((st - xa) % NST + NST) % NST) < T % NST ? 1 : 0);
      ph.stage ^= (uint32_t)(fills & 1) << st;
    }
  }
  __syncthreads();   // every thread is done with the stages, P and A before the next item reuses them
  return true;
}

template <int TY>
__device__ __forceinline__ void adj_init_barriers(unsigned char* raw, int nst, bool ring, int tid) {
  auto& S = *reinterpret_cast<AdjSmem<TY, true>*>(raw);
  if (tid == 0) {
    for (int q = 0; q < nst; ++q) mbar_init(smem_u32(&S.mbar[q]), 1);
    if (ring) { mbar_init(smem_u32(&S.pbar[0]), 1); mbar_init(smem_u32(&S.pbar[1]), 1); }
    mbar_fence_init();
  }
  __syncthreads();
}

// One launch per reverse step and variant: CTA b runs work item b.
template <int TY, int MODE>
__global__ void __launch_bounds__(32 * TY, AdjBounds<MODE>::MIN_CTAS)
adj_step_kernel(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
                const RfxbWork* __restrict__ work, const CUtensorMap* __restrict__ maps, int n, int par, int apar,
                int zp) {
  extern __shared__ __align__(128) unsigned char adj_smem_raw[];
  constexpr bool RING = MODE == 2 || MODE == 4;
  if (MODE != 0) adj_init_barriers<TY>(adj_smem_raw, RING ? 3 : RFXB_ANSTAGE, RING, threadIdx.y * 32 + threadIdx.x);
  StepPhases ph;
  adj_item<TY, MODE>(adj_smem_raw, insts, adjs, work[blockIdx.x], maps, n, par, apar, zp, ph, StepFault{}, true);
}

__device__ __forceinline__ bool adj_work_valid(const RfxbWork& w, const RfxbInst* insts, int n_inst, int ty) {
  if (w.inst < 0 || w.inst >= n_inst) return false;
  const RfxbInst& I = insts[w.inst];
  return w.y0 >= 0 && w.y0 < I.ny && w.y0 % ty == 0 && w.z0 >= 0 && w.z0 < I.nz && w.z0 % RFXB_TZ == 0 &&
         w.xa >= 0 && w.xa < w.xb && w.xb <= I.nx;
}

// Persistent reverse step: one launch per reverse step of as many CTAs as
// are resident.  Queue 0 holds the tiles that reach a y slab (variant 2),
// queue 1 the other CPML work (variant 4), queue 2 the CPML-free tiles
// (variant 3).  CTAs of role 0 (blocks [0, role_ctas), one per SM when the
// first wave spreads) take CPML-free items first, role 1 variant-4 items,
// role 2 variant-2 items; an emptied queue sends a CTA to the others, so the
// latency-bound CPML work and the bandwidth-bound plain work share every SM.
// Invalid items are skipped and flagged (status bit 2); the last CTA to
// finish clears the fetch counters for the next launch.
template <int TY>
__global__ void __launch_bounds__(32 * TY, 3)
adj_persist_kernel(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs, int n_inst,
                   RfxbAdjQueues Q, const CUtensorMap* __restrict__ maps, int n, int par, int apar) {
  extern __shared__ __align__(128) unsigned char adj_smem_raw[];
  __shared__ int pick[2];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  adj_init_barriers<TY>(adj_smem_raw, RFXB_ANSTAGE, true, tid);
  StepPhases ph;
  StepFault fault;
  fault.cta = Q.fault_cta;
  fault.wait_limit = Q.wait_limit;
  static constexpr int kOrder[3][3] = {{2, 1, 0}, {1, 0, 2}, {0, 1, 2}};
  const int role = min(2, (int)blockIdx.x / max(1, Q.role_ctas));
  bool first_item = true;
  bool ok = true;
  while (ok) {
    if (tid == 0) {
      pick[0] = -1;
      for (int t = 0; t < 3; ++t) {
        const int q = kOrder[role][t];
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
    if (!adj_work_valid(w, insts, n_inst, TY)) {
      if (tid == 0) atomicOr(Q.status, 2);
      continue;
    }
    if (q == 0) ok = adj_item<TY, 2>(adj_smem_raw, insts, adjs, w, maps, n, par, apar, Q.zp, ph, fault, first_item);
    else if (q == 1) ok = adj_item<TY, 4>(adj_smem_raw, insts, adjs, w, maps, n, par, apar, Q.zp, ph, fault, first_item);
    else ok = adj_item<TY, 3>(adj_smem_raw, insts, adjs, w, maps, n, par, apar, Q.zp, ph, fault, first_item);
    first_item = false;
  }
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&Q.ctr[3], 1) == (int)gridDim.x - 1) {
      Q.ctr[0] = 0;
      Q.ctr[1] = 0;
      Q.ctr[2] = 0;
      Q.ctr[3] = 0;
      __threadfence();
    }
  }
}

template __global__ void adj_step_kernel<8, 0>(const RfxbInst*, const AdjInst*, const RfxbWork*,
                                               const CUtensorMap*, int, int, int, int);
template __global__ void adj_step_kernel<8, 1>(const RfxbInst*, const AdjInst*, const RfxbWork*,
                                               const CUtensorMap*, int, int, int, int);
template __global__ void adj_step_kernel<8, 2>(const RfxbInst*, const AdjInst*, const RfxbWork*,
                                               const CUtensorMap*, int, int, int, int);
template __global__ void adj_step_kernel<8, 3>(const RfxbInst*, const AdjInst*, const RfxbWork*,
                                               const CUtensorMap*, int, int, int, int);
template __global__ void adj_step_kernel<8, 4>(const RfxbInst*, const AdjInst*, const RfxbWork*,
                                               const CUtensorMap*, int, int, int, int);
template __global__ void adj_persist_kernel<8>(const RfxbInst*, const AdjInst*, int, RfxbAdjQueues,
                                               const CUtensorMap*, int, int, int);

// Dynamic shared memory of a mode: the fixed part, the plane stages it uses
// and (modes 2, 4) the two ring slots sized for z-psi rows of zp floats, or
// (modes 0, 1) the exchange array.
size_t adj_step_smem_bytes(int mode, int zp) {
  if (mode == 5)   // the persistent kernel: the largest of variants 2, 3 and 4
    return std::max(std::max(adj_step_smem_bytes(2, zp), adj_step_smem_bytes(3, zp)), adj_step_smem_bytes(4, zp));
  using Lite = AdjSmem<8, false>;
  using Full = AdjSmem<8, true>;
  if (mode == 4)
    return offsetof(Lite, st) + 3 * sizeof(AdjStage<8, false>) +
           2 * sizeof(float) * (size_t)APsiSlot<8, false>::FLOATS(zp);
  const size_t fixed = offsetof(Full, st);
  if (mode == 2) return fixed + 3 * sizeof(AdjStage<8, true>) + 2 * sizeof(float) * (size_t)APsiSlot<8, true>::FLOATS(zp);
  if (mode == 3) return fixed + RFXB_ANSTAGE * sizeof(AdjStage<8, true>);
  return fixed + RFXB_ANSTAGE * sizeof(AdjStage<8, true>) + sizeof(AdjExchange<8>);
}

}  // namespace rfxb
