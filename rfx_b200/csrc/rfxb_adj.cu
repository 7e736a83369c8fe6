// Reverse-time adjoint of the forward step (the exact discrete transpose of
// rfxb_fwd.cu's arithmetic), replacing jax.grad through the scan
// (rfx/simulation.py:1972-2058, rfx/nonuniform.py:1755-1796).
//
// Forward step n maps u_n = (E, H, psi_H, psi_E) to u_{n+1}:
//   H1 = H - ch C_E E            ; psi_H' = b psi_H + c g(E) ; H' = H1 + s ch (psi_H' + km g)
//   E1 = ca E + cb C_H H'        ; psi_E' = b psi_E + c g(H') ; E2 = E1 + s ce (psi_E' + km g)
//   E' = M E2 + w_n              (M: PEC faces and edge mask)
// The adjoint sweep carries mu_{n+1} = dJ/du_{n+1} back to mu_n = S^T mu_{n+1}
// + Q^T g_{n-1} in two passes per step:
//   pass A (H-like): aH1 = aH + C_H^T(cb aEm) + CPML-E^T terms, aPsiE = b nu_E
//   pass B (E-like): aE  = ca aEm + C_E^T(ch aH1) + CPML-H^T terms, aPsiH = b nu_H
// where aEm = M aE.  The stored adjoint E is kept already masked.  The
// gradient d J / d eps_r over the recorded region is accumulated in pass A
// from the forward history (E^n and curl H^{n+1/2}) and the derivatives of ca
// and cb.  dJ/dw_{n-1} at each source cell is the raw mu_n there.
#include "rfxb_common.cuh"

namespace rfxb {

// Pass A: one thread per (j, k) column marching along x.
__global__ void __launch_bounds__(256)
adj_pass_a(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
           const RfxbWork* __restrict__ work, int n, int par, int apar) {
  const RfxbWork w = work[blockIdx.x];
  const RfxbInst& P = insts[w.inst];
  const AdjInst& A = adjs[w.inst];
  const int j = w.y0 + threadIdx.y, k = w.z0 + threadIdx.x;
  if (j >= P.ny || k >= P.nz) return;
  const int ncp = P.ncp;
  const float ye0 = __ldg(P.ye + j), ye1 = __ldg(P.ye + j + 1);
  const float ze0 = __ldg(P.ze + k), ze1 = __ldg(P.ze + k + 1);
  const bool in_hy = P.grad && j >= P.hb[2] && j < P.hb[3] && k >= P.hb[4] && k < P.hb[5];
  const int sy = P.hb[3] - P.hb[2], sz = P.hb[5] - P.hb[4];
  const int hc = (P.hb[1] - P.hb[0]) * sy * sz;
  const bool hist_ok = P.hist && (n - P.hist_step0) >= 0 && (n - P.hist_step0) < P.hist_nsteps;

  // H-probe injections of y_n (rows of g at step n) for this column.
  for (int i = w.xa; i < w.xb; ++i) {
    const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
    const long long ex1 = e + P.ps, ey1 = e + P.zs, ez1 = e + 1;
    const float cb0 = P.cb[e];
    const float qx = cb0 * A.aF[apar][0][e], qy = cb0 * A.aF[apar][1][e], qz = cb0 * A.aF[apar][2][e];
    const float cbx = P.cb[ex1], cby = P.cb[ey1], cbz = P.cb[ez1];
    const float qy_x1 = cbx * A.aF[apar][1][ex1], qz_x1 = cbx * A.aF[apar][2][ex1];
    const float qx_y1 = cby * A.aF[apar][0][ey1], qz_y1 = cby * A.aF[apar][2][ey1];
    const float qx_z1 = cbz * A.aF[apar][0][ez1], qy_z1 = cbz * A.aF[apar][1][ez1];
    const float xe0 = __ldg(P.xe + i), xe1 = __ldg(P.xe + i + 1);
    float ahx = A.aF[apar][3][e] + ((ze0 * qy - ze1 * qy_z1) - (ye0 * qz - ye1 * qz_y1));
    float ahy = A.aF[apar][4][e] + ((xe0 * qz - xe1 * qz_x1) - (ze0 * qx - ze1 * qx_z1));
    float ahz = A.aF[apar][5][e] + ((ye0 * qx - ye1 * qx_y1) - (xe0 * qy - xe1 * qy_x1));
    if (ncp) {
      // r(y) = ib (c nu + s ce km aE_t), nu = aPsiE + s ce aE_t, at slab cells y
      // aH_h(x) += r(x) - r(x + 1 along the axis)
      auto rel = [&](int axis, int q, int t, float sgn, int ii, int jj, int kk, bool own, float& r) {
        int s, sd;
        const int coord = axis == 0 ? ii : axis == 1 ? jj : kk;
        const int nax = axis == 0 ? P.nx : axis == 1 ? P.ny : P.nz;
        r = 0.f;
        if (coord < 0 || coord >= nax) return;
        if (!(P.cpml_axes & (1u << axis))) return;
        sd = cpml_side(coord, nax, ncp, s);
        if (sd < 0) return;
        const int face = 2 * axis + sd;
        const float* tb = P.cpb + (size_t)face * 3 * ncp;
        const float b = __ldg(tb + s), c = __ldg(tb + ncp + s), km = __ldg(tb + 2 * ncp + s);
        const long long ee = P.off0 + (long long)ii * P.ps + (long long)jj * P.zs + kk;
        const float ce = P.ce[ee];
        const float at = A.aF[apar][t][ee];
        long long qi;
        if (axis == 0) qi = psi_index_x(P, sd, q, s, jj, kk);
        else if (axis == 1) qi = psi_index_y(P, sd, q, s, ii, kk);
        else qi = psi_index_z(P, sd, q, s, ii, jj);
        const float nu = A.aPsiE[par][axis][qi] + sgn * ce * at;
        if (own) A.aPsiE[par ^ 1][axis][qi] = b * nu;
        r = P.ib[face] * (c * nu + sgn * ce * km * at);
      };
      float r0, r1;
      // x axis: (ey <- hz, -1, q0), (ez <- hy, +1, q1)
      rel(0, 0, 1, -1.f, i, j, k, true, r0); rel(0, 0, 1, -1.f, i + 1, j, k, false, r1); ahz += r0 - r1;
      rel(0, 1, 2, +1.f, i, j, k, true, r0); rel(0, 1, 2, +1.f, i + 1, j, k, false, r1); ahy += r0 - r1;
      // y axis: (ex <- hz, +1, q0), (ez <- hx, -1, q1)
      rel(1, 0, 0, +1.f, i, j, k, true, r0); rel(1, 0, 0, +1.f, i, j + 1, k, false, r1); ahz += r0 - r1;
      rel(1, 1, 2, -1.f, i, j, k, true, r0); rel(1, 1, 2, -1.f, i, j + 1, k, false, r1); ahx += r0 - r1;
      // z axis: (ex <- hy, -1, q0), (ey <- hx, +1, q1)
      rel(2, 0, 0, -1.f, i, j, k, true, r0); rel(2, 0, 0, -1.f, i, j, k + 1, false, r1); ahy += r0 - r1;
      rel(2, 1, 1, +1.f, i, j, k, true, r0); rel(2, 1, 1, +1.f, i, j, k + 1, false, r1); ahx += r0 - r1;
    }
    // H-probe injection of y_n
    if (P.g) {
      for (int p = 0; p < P.nprb; ++p) {
        const int4 c = __ldg(P.prb + p);
        if (c.x == i && c.y == j && c.z == k && (c.w & 7) >= 3) {
          const float gv = __ldg(P.g + (long long)n * P.g_ld + p);
          if ((c.w & 7) == 3) ahx += gv; else if ((c.w & 7) == 4) ahy += gv; else ahz += gv;
        }
      }
    }
    A.aF[apar][3][e] = ahx;
    A.aF[apar][4][e] = ahy;
    A.aF[apar][5][e] = ahz;
    // gradient over the recorded region
    if (in_hy && hist_ok && i >= P.hb[0] && i < P.hb[1]) {
      const int ci = ((i - P.hb[0]) * sy + (j - P.hb[2])) * sz + (k - P.hb[4]);
      const float* hp = P.hist + (long long)(n - P.hist_step0) * P.hist_ld + ci;
      const float dca = P.dca[ci], dcb = P.dcb[ci];
      const float ax = A.aF[apar][0][e], ay = A.aF[apar][1][e], az = A.aF[apar][2][e];
      double acc = (double)ax * ((double)dca * hp[0] + (double)dcb * hp[3 * hc])
                 + (double)ay * ((double)dca * hp[hc] + (double)dcb * hp[4 * hc])
                 + (double)az * ((double)dca * hp[2 * hc] + (double)dcb * hp[5 * hc]);
      P.grad[ci] += acc;
    }
  }
}

// Pass B: aE = ca aEm + C_E^T(ch aH1) + CPML-H^T, then the E-probe injection
// of y_{n-1}, the source adjoint dJ/dw_{n-1}, and the mask for storage.
__global__ void __launch_bounds__(256)
adj_pass_b(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
           const RfxbWork* __restrict__ work, int n, int par, int apar) {
  const RfxbWork w = work[blockIdx.x];
  const RfxbInst& P = insts[w.inst];
  const AdjInst& A = adjs[w.inst];
  const int j = w.y0 + threadIdx.y, k = w.z0 + threadIdx.x;
  if (j >= P.ny || k >= P.nz) return;
  const int ncp = P.ncp;
  const float yh0 = __ldg(P.yh + j), yhm = __ldg(P.yh + j - 1);
  const float zh0 = __ldg(P.zh + k), zhm = __ldg(P.zh + k - 1);
  for (int i = w.xa; i < w.xb; ++i) {
    const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
    const long long exm = e - P.ps, eym = e - P.zs, ezm = e - 1;
    auto chat = [&](long long ee) { return P.ch ? P.ch[ee] : P.ch0; };
    const float c0 = chat(e);
    const float px = c0 * A.aF[apar][3][e], py = c0 * A.aF[apar][4][e], pz = c0 * A.aF[apar][5][e];
    const float cxm = chat(exm), cym = chat(eym), czm = chat(ezm);
    const float py_xm = cxm * A.aF[apar][4][exm], pz_xm = cxm * A.aF[apar][5][exm];
    const float px_ym = cym * A.aF[apar][3][eym], pz_ym = cym * A.aF[apar][5][eym];
    const float px_zm = czm * A.aF[apar][3][ezm], py_zm = czm * A.aF[apar][4][ezm];
    const float xh0 = __ldg(P.xh + i), xhm = __ldg(P.xh + i - 1);
    const float ca = P.ca[e];
    float ax = ca * A.aF[apar][0][e] + ((zh0 * py - zhm * py_zm) - (yh0 * pz - yhm * pz_ym));
    float ay = ca * A.aF[apar][1][e] + ((xh0 * pz - xhm * pz_xm) - (zh0 * px - zhm * px_zm));
    float az = ca * A.aF[apar][2][e] + ((yh0 * px - yhm * px_ym) - (xh0 * py - xhm * py_xm));
    if (ncp) {
      // r(y) = ib (c nu + s km p_t), nu = aPsiH + s p_t, p = ch aH1
      // aE_e(x) += r(x - 1 along the axis) - r(x)
      auto rel = [&](int axis, int q, int t, float sgn, int ii, int jj, int kk, bool own, float& r) {
        int s, sd;
        const int coord = axis == 0 ? ii : axis == 1 ? jj : kk;
        const int nax = axis == 0 ? P.nx : axis == 1 ? P.ny : P.nz;
        r = 0.f;
        if (coord < 0 || coord >= nax) return;
        if (!(P.cpml_axes & (1u << axis))) return;
        sd = cpml_side(coord, nax, ncp, s);
        if (sd < 0) return;
        const int face = 2 * axis + sd;
        const float* tb = P.cpb + (size_t)face * 3 * ncp;
        const float b = __ldg(tb + s), c = __ldg(tb + ncp + s), km = __ldg(tb + 2 * ncp + s);
        const long long ee = P.off0 + (long long)ii * P.ps + (long long)jj * P.zs + kk;
        const float pt = chat(ee) * A.aF[apar][t][ee];
        long long qi;
        if (axis == 0) qi = psi_index_x(P, sd, q, s, jj, kk);
        else if (axis == 1) qi = psi_index_y(P, sd, q, s, ii, kk);
        else qi = psi_index_z(P, sd, q, s, ii, jj);
        const float nu = A.aPsiH[par][axis][qi] + sgn * pt;
        if (own) A.aPsiH[par ^ 1][axis][qi] = b * nu;
        r = P.ib[face] * (c * nu + sgn * km * pt);
      };
      float r0, r1;
      // x axis: (hy <- ez, +1, q0), (hz <- ey, -1, q1)
      rel(0, 0, 4, +1.f, i - 1, j, k, false, r0); rel(0, 0, 4, +1.f, i, j, k, true, r1); az += r0 - r1;
      rel(0, 1, 5, -1.f, i - 1, j, k, false, r0); rel(0, 1, 5, -1.f, i, j, k, true, r1); ay += r0 - r1;
      // y axis: (hx <- ez, -1, q0), (hz <- ex, +1, q1)
      rel(1, 0, 3, -1.f, i, j - 1, k, false, r0); rel(1, 0, 3, -1.f, i, j, k, true, r1); az += r0 - r1;
      rel(1, 1, 5, +1.f, i, j - 1, k, false, r0); rel(1, 1, 5, +1.f, i, j, k, true, r1); ax += r0 - r1;
      // z axis: (hx <- ey, +1, q0), (hy <- ex, -1, q1)
      rel(2, 0, 3, +1.f, i, j, k - 1, false, r0); rel(2, 0, 3, +1.f, i, j, k, true, r1); ay += r0 - r1;
      rel(2, 1, 4, -1.f, i, j, k - 1, false, r0); rel(2, 1, 4, -1.f, i, j, k, true, r1); ax += r0 - r1;
    }
    // E-probe injection of y_{n-1}
    if (P.g && n >= 1) {
      for (int p = 0; p < P.nprb; ++p) {
        const int4 c = __ldg(P.prb + p);
        if (c.x == i && c.y == j && c.z == k && (c.w & 7) < 3) {
          const float gv = __ldg(P.g + (long long)(n - 1) * P.g_ld + p);
          if ((c.w & 7) == 0) ax += gv; else if ((c.w & 7) == 1) ay += gv; else az += gv;
        }
      }
    }
    if (P.src_adj && n >= 1) {
      for (int s = 0; s < P.nsrc; ++s) {
        const int4 c = __ldg(P.src + s);
        if (c.x == i && c.y == j && c.z == k)
          P.src_adj[(long long)(n - 1) * P.src_ld + s] = c.w == 0 ? ax : c.w == 1 ? ay : az;
      }
    }
    // store M aE
    if (P.pec_axes & 1u) if (i == 0 || i == P.nx - 1) { ay = 0.f; az = 0.f; }
    if (P.pec_axes & 2u) if (j == 0 || j == P.ny - 1) { ax = 0.f; az = 0.f; }
    if (P.pec_axes & 4u) {
      if (k == 0 || k == P.nz - 1) { ax = 0.f; ay = 0.f; }
      if (k == P.nz - 1) az = 0.f;
    }
    if (P.emask) {
      const unsigned m = P.emask[e];
      if (m & 1u) ax = 0.f;
      if (m & 2u) ay = 0.f;
      if (m & 4u) az = 0.f;
    }
    A.aF[apar][0][e] = ax;
    A.aF[apar][1][e] = ay;
    A.aF[apar][2][e] = az;
  }
}

// mu_N = Q^T g_{N-1} on the E probes (H probes are injected by pass A of the
// first reverse step), dJ/dw_{N-1} at the sources, stored masked.
__global__ void adj_init_kernel(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
                                int ninst, int nlast, int apar) {
  const int q = blockIdx.x;
  if (q >= ninst) return;
  const RfxbInst& P = insts[q];
  const AdjInst& A = adjs[q];
  if (threadIdx.x != 0) return;
  // accumulate probe injections first (several probes may share a cell)
  if (P.g) {
    for (int p = 0; p < P.nprb; ++p) {
      const int4 c = P.prb[p];
      const int comp = c.w & 7;
      if (comp >= 3) continue;
      const long long e = P.off0 + (long long)c.x * P.ps + (long long)c.y * P.zs + c.z;
      A.aF[apar][comp][e] += P.g[(long long)nlast * P.g_ld + p];
    }
  }
  if (P.src_adj) {
    for (int s = 0; s < P.nsrc; ++s) {
      const int4 c = P.src[s];
      const long long e = P.off0 + (long long)c.x * P.ps + (long long)c.y * P.zs + c.z;
      P.src_adj[(long long)nlast * P.src_ld + s] = A.aF[apar][c.w][e];
    }
  }
  if (P.g) {
    for (int p = 0; p < P.nprb; ++p) {
      const int4 c = P.prb[p];
      const int comp = c.w & 7;
      if (comp >= 3) continue;
      const int i = c.x, j = c.y, k = c.z;
      const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
      bool zero = false;
      if ((P.pec_axes & 1u) && (i == 0 || i == P.nx - 1) && comp != 0) zero = true;
      if ((P.pec_axes & 2u) && (j == 0 || j == P.ny - 1) && comp != 1) zero = true;
      if ((P.pec_axes & 4u) && (k == 0 || k == P.nz - 1) && comp != 2) zero = true;
      if ((P.pec_axes & 4u) && k == P.nz - 1 && comp == 2) zero = true;
      if (P.emask && (P.emask[e] >> comp) & 1u) zero = true;
      if (zero) A.aF[apar][comp][e] = 0.f;
    }
  }
}

// Transpose of the running-DFT planes for sample s (the fields after step s:
// E^{s+1} after the sources, H^{s+1/2}): each plane cell receives
// sum_f Re(G_f) cos_f(s) dt + Im(G_f) sin_f(s) dt, added to the adjoint field
// of the current parity.  It lands where an E / H probe cotangent of sample s
// lands: an E component also feeds the source adjoint of a source on that
// cell, and is dropped where the PEC faces or the edge mask zero the
// component (the transposes of those zeroings, which the forward applies
// before the sources).  Planes may share cells, so the adds are atomic.
__global__ void dft_adj_kernel(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
                               const RfxbDftPlane* __restrict__ planes, int nplanes, int s, int apar) {
  int q = 0;
  while (q + 1 < nplanes && planes[q + 1].block0 <= (int)blockIdx.x) ++q;
  const RfxbDftPlane& D = planes[q];
  if (D.acc == nullptr) return;
  const int c = (blockIdx.x - D.block0) * blockDim.x + threadIdx.x;
  const int cells = D.n1 * D.n2;
  if (c >= cells) return;
  const float2* ph = D.phase + (long long)s * D.nf;
  float g = 0.f;
  for (int f = 0; f < D.nf; ++f) {
    const float2 G = D.acc[(long long)f * cells + c], w = __ldg(ph + f);
    g = fmaf(G.x, w.x, g);
    g = fmaf(G.y, w.y, g);
  }
  if (g == 0.f) return;
  const RfxbInst& P = insts[D.inst];
  const AdjInst& A = adjs[D.inst];
  const int a = c / D.n2, b = c - a * D.n2;
  int i, j, k;
  if (D.axis == 0) { i = D.index; j = a; k = b; }
  else if (D.axis == 1) { i = a; j = D.index; k = b; }
  else { i = a; j = b; k = D.index; }
  const int comp = D.comp;
  const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
  bool zero = false;
  if (comp < 3) {
    if (P.src_adj)
      for (int t = 0; t < P.nsrc; ++t) {
        const int4 sc = P.src[t];
        if (sc.x == i && sc.y == j && sc.z == k && sc.w == comp) atomicAdd(P.src_adj + (long long)s * P.src_ld + t, g);
      }
    if ((P.pec_axes & 1u) && (i == 0 || i == P.nx - 1) && comp != 0) zero = true;
    if ((P.pec_axes & 2u) && (j == 0 || j == P.ny - 1) && comp != 1) zero = true;
    if ((P.pec_axes & 4u) && (k == 0 || k == P.nz - 1) && comp != 2) zero = true;
    if ((P.pec_axes & 4u) && k == P.nz - 1 && comp == 2) zero = true;
    if (P.emask && (P.emask[e] >> comp) & 1u) zero = true;
  }
  if (!zero) atomicAdd(A.aF[apar][comp] + e, g);
}

// Transpose of the NTFF box for sample s: on every face cell each of the four
// tangential components receives sum_f Re(G) Re(w) + Im(G) Im(w) with w the E
// factor (E components) or the H factor (H components) of step s, injected as
// a DFT-plane cotangent is (E components: source adjoint, PEC / edge-mask
// drop).  Faces share their edge cells, so the adds are atomic.
__global__ void ntff_adj_kernel(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
                                const RfxbNtffFace* __restrict__ faces, int nfaces, int s, int apar) {
  int q = 0;
  while (q + 1 < nfaces && faces[q + 1].block0 <= (int)blockIdx.x) ++q;
  const RfxbNtffFace& F = faces[q];
  if (F.acc == nullptr) return;
  const int c = (blockIdx.x - F.block0) * blockDim.x + threadIdx.x;
  const int cells = F.n1 * F.n2;
  if (c >= cells) return;
  const int a = F.lo1 + c / F.n2, b = F.lo2 + c % F.n2;
  int i, j, k;
  if (F.axis == 0) { i = F.index; j = a; k = b; }
  else if (F.axis == 1) { i = a; j = F.index; k = b; }
  else { i = a; j = b; k = F.index; }
  const RfxbInst& P = insts[F.inst];
  const AdjInst& A = adjs[F.inst];
  const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
  const float2* ph = F.phase + (long long)s * 2 * F.nf;
  float g[4] = {0.f, 0.f, 0.f, 0.f};
  for (int f = 0; f < F.nf; ++f) {
    const float2 we = __ldg(ph + f), wh = __ldg(ph + F.nf + f);
    const float4* gp = reinterpret_cast<const float4*>(F.acc + ((long long)f * cells + c) * 4);
    const float4 g01 = gp[0], g23 = gp[1];
    g[0] = fmaf(g01.x, we.x, fmaf(g01.y, we.y, g[0]));
    g[1] = fmaf(g01.z, we.x, fmaf(g01.w, we.y, g[1]));
    g[2] = fmaf(g23.x, wh.x, fmaf(g23.y, wh.y, g[2]));
    g[3] = fmaf(g23.z, wh.x, fmaf(g23.w, wh.y, g[3]));
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (g[t] == 0.f) continue;
    const int comp = F.comp[t];
    bool zero = false;
    if (comp < 3) {
      if (P.src_adj)
        for (int u = 0; u < P.nsrc; ++u) {
          const int4 sc = P.src[u];
          if (sc.x == i && sc.y == j && sc.z == k && sc.w == comp)
            atomicAdd(P.src_adj + (long long)s * P.src_ld + u, g[t]);
        }
      if ((P.pec_axes & 1u) && (i == 0 || i == P.nx - 1) && comp != 0) zero = true;
      if ((P.pec_axes & 2u) && (j == 0 || j == P.ny - 1) && comp != 1) zero = true;
      if ((P.pec_axes & 4u) && (k == 0 || k == P.nz - 1) && comp != 2) zero = true;
      if ((P.pec_axes & 4u) && k == P.nz - 1 && comp == 2) zero = true;
      if (P.emask && (P.emask[e] >> comp) & 1u) zero = true;
    }
    if (!zero) atomicAdd(A.aF[apar][comp] + e, g[t]);
  }
}

// Transpose of the flux monitors for sample s: per region cell the E pair
// receives sum_f Re(G) Re(k_E) + Im(G) Im(k_E) on the monitor plane (source
// adjoint and PEC / edge-mask drop as for a DFT plane), the H pair the same
// with the H factor, split in halves over the two planes the forward
// averaged (both halves on plane 0 when the monitor is on plane 0).
__global__ void flux_adj_kernel(const RfxbInst* __restrict__ insts, const AdjInst* __restrict__ adjs,
                                const RfxbFluxPlane* __restrict__ planes, int nplanes, int s, int apar) {
  int q = 0;
  while (q + 1 < nplanes && planes[q + 1].block0 <= (int)blockIdx.x) ++q;
  const RfxbFluxPlane& M = planes[q];
  if (M.acc == nullptr) return;
  const int c = (blockIdx.x - M.block0) * blockDim.x + threadIdx.x;
  const int cells = M.n1 * M.n2;
  if (c >= cells) return;
  const int a = M.lo1 + c / M.n2, b = M.lo2 + c % M.n2;
  auto at = [&](int plane, int& i, int& j, int& k) {
    if (M.axis == 0) { i = plane; j = a; k = b; }
    else if (M.axis == 1) { i = a; j = plane; k = b; }
    else { i = a; j = b; k = plane; }
  };
  const double2* kn = M.kern + (long long)s * 2 * M.nf;
  double g[4] = {0.0, 0.0, 0.0, 0.0};
  for (int f = 0; f < M.nf; ++f) {
    const double2 ke = kn[f], kh = kn[M.nf + f];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const double2 G = M.acc[((long long)t * M.nf + f) * cells + c];
      const double2 w = t < 2 ? ke : kh;
      g[t] += G.x * w.x + G.y * w.y;
    }
  }
  const RfxbInst& P = insts[M.inst];
  const AdjInst& A = adjs[M.inst];
  int i, j, k;
  at(M.index, i, j, k);
  const long long e = P.off0 + (long long)i * P.ps + (long long)j * P.zs + k;
  for (int t = 0; t < 2; ++t) {   // E pair on the monitor plane
    const float v = (float)g[t];
    if (v == 0.f) continue;
    const int comp = M.comp[t];
    if (P.src_adj)
      for (int u = 0; u < P.nsrc; ++u) {
        const int4 sc = P.src[u];
        if (sc.x == i && sc.y == j && sc.z == k && sc.w == comp) atomicAdd(P.src_adj + (long long)s * P.src_ld + u, v);
      }
    bool zero = false;
    if ((P.pec_axes & 1u) && (i == 0 || i == P.nx - 1) && comp != 0) zero = true;
    if ((P.pec_axes & 2u) && (j == 0 || j == P.ny - 1) && comp != 1) zero = true;
    if ((P.pec_axes & 4u) && (k == 0 || k == P.nz - 1) && comp != 2) zero = true;
    if ((P.pec_axes & 4u) && k == P.nz - 1 && comp == 2) zero = true;
    if (P.emask && (P.emask[e] >> comp) & 1u) zero = true;
    if (!zero) atomicAdd(A.aF[apar][comp] + e, v);
  }
  int i1, j1, k1;
  at(M.im1, i1, j1, k1);
  const long long e1 = P.off0 + (long long)i1 * P.ps + (long long)j1 * P.zs + k1;
  for (int t = 2; t < 4; ++t) {   // H pair: (H(im1) + H(index)) / 2
    const float v = (float)(0.5 * g[t]);
    if (v == 0.f) continue;
    atomicAdd(A.aF[apar][M.comp[t]] + e1, v);
    atomicAdd(A.aF[apar][M.comp[t]] + e, v);
  }
}

}  // namespace rfxb
