// Device-side descriptors shared by the forward, adjoint and DFT kernels.
//
// Internal state layout (one simulation, "instance"): every per-cell array
// (fields, coefficients) uses a padded copy of the reference's (nx, ny, nz)
// C-order layout with z fastest:
//
//   element(i, j, k) = off0 + i*ps + j*zs + k,   i in [-1, nx], j in [-1, ny]
//
// zs = round_up(nz + 1, 32) is the row stride (128-byte aligned rows), and
// ps = (ny + 2) * zs the plane stride.  Planes i = -1 and i = nx, rows j = -1
// and j = ny, and the row tail k in [nz, zs) are zero guards that are never
// written.  Because the element before a row start is the previous row's
// tail, k = -1 also reads zero.  The guards are exactly the reference's
// zero padding in _shift_fwd / _shift_bwd (rfx/core/yee.py:121-138), so the
// stencils carry no boundary branches.
#pragma once
#include <cstdint>
#include <cuda.h>   // CUtensorMap

#define RFXB_TZ 32          // tile extent along z (one warp)
#define RFXB_MAXC 6
// TMA descriptors per instance: [0|1] fields parity 0|1 with the E box,
// [2|3] with the H box, [4] coefficients with the ca/cb box, [5|6] adjoint
// fields with the E box, [7|8] with the H box, [9] cb with the E box,
// [10] one coefficient with the tile box, then the CPML psi of parity 0|1:
// [11|12] H-side x, [13|14] H-side y, [15|16] H-side z (H boxes), [17|18]
// E-side x, [19|20] E-side y, [21|22] E-side z (tile boxes); [23] one
// coefficient with the H box; then the adjoint psi of parity 0|1: [24|25]
// E-side x (H box), [26|27] E-side y (E box), [28|29] E-side z (E rows),
// [30|31] H-side x (tile box), [32|33] H-side y (H box), [34|35] H-side z
// (H rows); [36] the PEC edge-mask bytes with the tile box; [37] the
// intermediate field state of a two-step pass with the E box, [38] with the
// H box; the two-step kernel's boxes: [39|40] fields parity 0|1 with the
// two-step E box, [41|42] with the two-step H box, [43] coefficients with the
// two-step ca/cb box.
#define RFXB_NMAPS 44
#define RFXB_MAP_EMASK 36   // PEC edge mask bytes with the tile box
#define RFXB_MAP_MIDE 37
#define RFXB_MAP_MIDH 38
#define RFXB_MAP_E2 39
#define RFXB_MAP_H2 41
#define RFXB_MAP_C2 43
#define RFXB_MAP_PSH 11
#define RFXB_MAP_PSE 17
#define RFXB_MAP_APE 24
#define RFXB_MAP_APH 30

// CPML psi layout per axis (q = which of the two corrected components,
// n = layers, n4 = n rounded up to a multiple of 4):
//   x: ((side*2 + q)*n + s)*ny*zs + j*zs + k
//   y: ((side*2 + q)*nx + i)*n*zs + s*zs + k
//   z: ((side*2 + q)*nx + i)*ny*n4 + j*n4 + s
// Every row is a multiple of 16 bytes, so each axis is a TMA-tileable 4-D
// array (rows along k for x and y, along s for z).
struct RfxbInst {
  int nx, ny, nz, zs;
  long long ps;            // plane stride (elements)
  long long off0;          // element offset of cell (0,0,0)
  long long cs;            // component stride: F[p][c] = F[p][0] + c * cs (multiple of 32)
  float* F[3][6];          // ping-pong field buffers: ex ey ez hx hy hz; [2] the
                           // intermediate state of two-step passes (or null)
  const float* ca;         // per cell, E decay coefficient
  const float* cb;         // per cell, E curl coefficient
  const float* ce;         // per cell, dt/(eps_r eps0) for CPML-E
  const float* ch;         // per cell dt/(mu_r mu0), or null -> ch0
  float ch0;
  // inverse spacing tables; pointers address entry 0, entries -1 and n valid
  const float* xe; const float* xh;
  const float* ye; const float* yh;
  const float* ze; const float* zh;
  // CPML
  int ncp;                 // layers per face (0 = none)
  int ncp4;                // ncp rounded up to a multiple of 4 (z psi row length)
  unsigned cpml_axes;      // bit a set -> axis a absorbs
  const float* cpb;        // [face][3][ncp]: b, c, (1/kappa - 1); face = 2*axis + side
  const float4* cpt;       // [face][ncp]: (b, c / cell, (1/kappa - 1) / cell, 0)
  float ib[6];             // 1 / boundary cell size per face
  float* psH[2][3];        // H-side psi per axis, ping-pong
  float* psE[2][3];        // E-side psi per axis, ping-pong
  // PEC
  unsigned pec_axes;       // bit a set -> zero tangential E on both faces of axis a
  const unsigned char* emask;  // per cell bits (1 ex, 2 ey, 4 ez) zeroed, or null
  // sources: E_c[i,j,k] += w[n*src_ld + s]
  int nsrc;
  const int4* src;         // (i, j, k, comp)
  const float* srcw;
  int src_ld;
  // probes: out[n*prb_ld + p] = field; comp bits 0..2, bit 4 = sample before sources
  int nprb;
  const int4* prb;
  float* prb_out;
  int prb_ld;
  // gradient-region history: per step 6 * hcells floats (E_old xyz, curl xyz)
  int hb[6];               // i0 i1 j0 j1 k0 k1 (half-open), empty if i0 >= i1
  float* hist;
  long long hist_ld;
  int hist_step0;
  int hist_nsteps;
  // adjoint-only inputs
  const float* g;          // dJ/d(probe) table [n*g_ld + p]
  int g_ld;
  const float* dca;        // d ca / d eps_r over the gradient region
  const float* dcb;        // d cb / d eps_r over the gradient region
  double* grad;            // accumulated dJ/d eps_r over the gradient region
  float* src_adj;          // dJ/d w[n, s] output [n*src_ld + s]
  int* status;             // device status word: bit 0 = a pipeline wait ran out
};

struct AdjInst {           // adjoint state of one instance (same layouts as the forward state)
  float* aF[2][6];         // ping-pong: aex aey aez ahx ahy ahz (component stride cs)
  float* aPsiH[2][3];      // ping-pong
  float* aPsiE[2][3];
};

struct RfxbWork {          // one CTA: a (y, z) tile over an x range
  int inst;
  int y0, z0;
  int xa, xb;
};

// One CTA of the two-step kernel: a tile over an x range, advanced two time
// steps, and where the intermediate state must also be stored (the cells that
// one-step neighbours or per-step observers read): bit 0 every plane, bit 1
// plane xa, bit 2 plane xb-1; bit 3: the item's cells reach a grid face (the
// kernel then keeps cells outside the grid at zero and applies PEC faces).
#define RFXB_MID_ALL 1
#define RFXB_MID_LO 2
#define RFXB_MID_HI 4
#define RFXB_MID_EDGE 8
struct RfxbWork2 {
  int inst;
  int y0, z0;
  int xa, xb;
  int mid;
};

// Work queues of the persistent forward step (one launch per step).
struct RfxbFwdQueues {
  const RfxbWork* list[2];   // 0: tiles that reach a CPML slab (staged psi), 1: CPML-free tiles
  int count[2];
  int* ctr;                  // [3]: fetch counters of the two lists, CTAs finished (zero between launches)
  int* status;               // the group's status word (bit 1: a wait ran out, bit 2: an invalid item)
  int plain_ctas;            // CTAs from block 0 on that try the CPML-free list first
  int fault_cta;             // test only: block whose first item does not load its plane xa (-1: none)
  int wait_limit;            // polls of a bounded mbarrier wait
};

// Work queues of the persistent reverse step: 0 tiles that reach a y slab
// (variant 2), 1 the other CPML work (variant 4), 2 CPML-free tiles (variant 3).
struct RfxbAdjQueues {
  const RfxbWork* list[3];
  int count[3];
  int* ctr;                  // [4]: fetch counters of the three lists, CTAs finished
  int* status;
  int role_ctas;             // CTAs per role: blocks [r * role_ctas, (r+1) * role_ctas) have role r
  int fault_cta;
  int wait_limit;
  int zp;                    // largest z-psi row of the group (ring slot size)
};

struct RfxbNtffFace {      // one face of one instance's NTFF box
  int inst;
  int axis, index;         // normal axis and face plane
  int lo1, n1, lo2, n2;    // tangential ranges (x face: j, k; y face: i, k; z face: i, j)
  int nf;
  int comp[4];             // tangential E E H H component codes
  float2* acc;             // running sums (nf, n1, n2, 4) complex64
  float2* cmp;             // Kahan residuals, same layout
  const float2* phase;     // [n][2][nf]: E and H factors times dt
  int block0;              // first CTA of this face in the launch
};

struct RfxbFluxPlane {     // one Poynting-flux monitor of one instance
  int inst;
  int axis, index, im1;    // normal axis, E plane, the other H plane (index-1, or 0)
  int lo1, n1, lo2, n2;    // region on the tangential axes (reference order)
  int nf;
  int comp[4];             // E1 E2 H1 H2 component codes
  double2* acc;            // caller accumulator [4][nf][n1][n2] complex128
  const double2* kern;     // [n][2][nf]: E and H factors (phase * dt * window)
  int block0;              // first CTA of this monitor in the launch
};

struct RfxbDftPlane {      // one running-DFT plane of one instance
  int inst;
  int axis, index, comp;
  int nf;
  int n1, n2;              // plane extents (reference order)
  float2* acc;             // caller accumulator (nf, n1, n2) complex64
  float2* cmp;             // Kahan compensation, same shape
  const float2* phase;     // [n][nf]: (cos, sin) * dt of the sample time
  int block0;              // first CTA of this plane in the launch
};
