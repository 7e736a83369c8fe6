"""Reverse-mode gradient of the oracle scan -- TEST INFRASTRUCTURE ONLY.

The reference obtains gradients with ``jax.grad`` through its scan
(rfx/simulation.py:1972-2058); that is, the transpose of every linear
operation of the step body, applied in reverse order.  This module writes
that transpose out for the oracle's own step (rfx/core/yee.py:226-404,
rfx/boundaries/cpml.py:522-1065, rfx/boundaries/pec.py:13-47, 179-208):

  forward  u_{n+1} = M (CE o UE o CH o UH)(u_n) + w_n,   y_n = Q u_{n+1}
  backward mu_n = UH^T CH^T UE^T CE^T M mu_{n+1} + Q^T g_{n-1}

with the eps_r derivative taken where the reference's autodiff takes it:
ca and cb of rfx/core/yee.py:387-393 (d ca/d eps_r, d cb/d eps_r) times the
recorded E^n and curl H^{n+1/2}, and, in CPML slab cells, the E-side
coefficient ce = dt/(eps_r eps0) of rfx/boundaries/cpml.py:536-546
(d ce/d eps_r = -ce/eps_r) times the recorded correction
sign * (psi + (1/kappa - 1) curl) of each axis.  It is used to check the
CUDA adjoint and as the CPU baseline of the forward+adjoint workload.
"""

from __future__ import annotations

import numpy as np

from .fdtd import (COMPONENTS, EPS_0, MU_0, _CPML_E, _CPML_H, _col, _sb, _sf, _slab, _Stepper)


def _coef_derivs(eps_r, sigma, dt):
    e = np.asarray(eps_r, np.float64)
    s = np.asarray(sigma, np.float64)
    L = s * dt / (2.0 * EPS_0 * e)
    return 2.0 * L / (e * (1.0 + L) ** 2), -dt * EPS_0 / (EPS_0 * e + s * dt / 2.0) ** 2


def _ce_deriv(eps_r, dt):
    """d ce / d eps_r of ce = dt / (eps_r eps0) (rfx/boundaries/cpml.py:536)."""
    e = np.asarray(eps_r, np.float64)
    return -dt / (EPS_0 * e * e)


class _RecStepper(_Stepper):
    """Forward stepper that records E^n and curl H^{n+1/2} over a box."""

    def __init__(self, *a, box, **kw):
        super().__init__(*a, **kw)
        self.box = tuple(slice(box[2 * d], box[2 * d + 1]) for d in range(3))
        self.hist = []

    def update_e(self):
        F, dt = self.F, self.g.dt
        hx, hy, hz = F["hx"], F["hy"], F["hz"]
        eps = self.eps_r * EPS_0
        s2 = self.sigma * dt / (2.0 * eps)
        ca = (1.0 - s2) / (1.0 + s2)
        cb = (dt / eps) / (1.0 + s2)
        if self.nu:
            t = self.tab
            iy, iz, ix = _col(t["inv_dy"], 1), _col(t["inv_dz"], 2), _col(t["inv_dx"], 0)
            cx = (hz - _sb(hz, 1)) * iy - (hy - _sb(hy, 2)) * iz
            cy = (hx - _sb(hx, 2)) * iz - (hz - _sb(hz, 0)) * ix
            cz = (hy - _sb(hy, 0)) * ix - (hx - _sb(hx, 1)) * iy
        else:
            dx = self.g.dx
            cx = (hz - _sb(hz, 1)) / dx - (hy - _sb(hy, 2)) / dx
            cy = (hx - _sb(hx, 2)) / dx - (hz - _sb(hz, 0)) / dx
            cz = (hy - _sb(hy, 0)) / dx - (hx - _sb(hx, 1)) / dx
        b = self.box
        self.hist.append(np.stack([F["ex"][b], F["ey"][b], F["ez"][b], cx[b], cy[b], cz[b]]).astype(np.float64))
        F["ex"] = ca * F["ex"] + cb * cx
        F["ey"] = ca * F["ey"] + cb * cy
        F["ez"] = ca * F["ez"] + cb * cz
        self.step_count += 1

    def cpml_e(self):
        """CPML-E pass that also records, over the box, the correction of
        each E component before its ce scaling (zero off the slabs)."""
        corr = {c: np.zeros(self.g.shape, np.float64) for c in ("ex", "ey", "ez")}
        if self.psi:
            ce = self.g.dt / (self.eps_r * EPS_0)
            self._apply_cpml(_CPML_E, ce, fwd=False, corr=corr)
        b = self.box
        self.hist[-1] = np.concatenate([self.hist[-1], np.stack([corr[c][b] for c in ("ex", "ey", "ez")])])


def _mask_e(st, aF):
    """Transpose of apply_pec + apply_pec_mask (diagonal 0/1)."""
    ax = st.pec_axes
    if "x" in ax:
        for c in ("ey", "ez"):
            aF[c][0] = 0.0
            aF[c][-1] = 0.0
    if "y" in ax:
        for c in ("ex", "ez"):
            aF[c][:, 0] = 0.0
            aF[c][:, -1] = 0.0
    if "z" in ax:
        for c in ("ex", "ey"):
            aF[c][:, :, 0] = 0.0
            aF[c][:, :, -1] = 0.0
        aF["ez"][:, :, -1] = 0.0
    if st.emask is not None:
        for c, m in zip(("ex", "ey", "ez"), st.emask):
            aF[c] = aF[c] * (1.0 - m)


def _cpml_transpose(st, aF, apsi, table, coef_full, fwd):
    """Transpose of _Stepper._apply_cpml: the corrected component's adjoint
    feeds the psi adjoint and the differentiated component's adjoint."""
    n = st.n
    new = {}
    for ax in range(3):
        if "xyz"[ax] not in st.cpml_axes:
            continue
        name = "xyz"[ax]
        for (fc, dc, sgn) in table[ax]:
            for side in ("lo", "hi"):
                b, c, kap, d = st.prof[f"{name}_{side}"]
                b = _col(b.astype(st.f), ax)
                c = _col(c.astype(st.f), ax)
                km = 1.0 / _col(kap.astype(st.f), ax) - 1.0
                sl = _slab(ax, side == "lo", n)
                cf = coef_full[sl] * sgn
                key = (fc, ax, side)
                a_t = aF[fc][sl]
                nu = apsi[key] + cf * a_t
                new[key] = b * nu
                a_g = (c * nu + cf * km * a_t) / d
                full = np.zeros_like(aF[dc])
                full[sl] = a_g
                if fwd:   # g = (E[x+1] - E[x]) / d
                    aF[dc] = aF[dc] + _sb(full, ax) - full
                else:     # g = (H[x] - H[x-1]) / d
                    aF[dc] = aF[dc] + full - _sf(full, ax)
    apsi.update(new)


def forward_adjoint(grid, materials, n_steps, *, nonuniform=False, boundary="cpml", cpml_axes="xyz",
                    pec_axes=None, sources=(), probes=(), pec_mask=None, box, objective_grad,
                    dtype=np.float64):
    """Forward run, then the reverse sweep.

    ``objective_grad(ts) -> g`` maps the probe traces (n_steps, n_probes) to
    dJ/dts.  Returns (ts, dJ/d eps_r over ``box``, dJ/d source table)."""
    if nonuniform:
        axes = cpml_axes if grid.cpml_layers > 0 else ""
        pec_axes = "xyz"
    else:
        axes = cpml_axes if boundary == "cpml" else ""
        pec_axes = "xyz" if pec_axes is None else pec_axes
    st = _RecStepper(grid, materials, dtype=dtype, nonuniform=nonuniform, cpml_axes=axes,
                     pec_axes=pec_axes, pec_mask=pec_mask, box=box)
    f = st.f
    ts = np.zeros((n_steps, len(probes)), f)
    for n in range(n_steps):
        st.update_h()
        st.cpml_h()
        st.update_e()
        st.cpml_e()
        st.pec()
        st.pec_mask()
        for (i, j, k, comp, wave) in sources:
            st.F[comp][i, j, k] = st.F[comp][i, j, k] + f.type(wave[n])
        for p, (i, j, k, comp) in enumerate(probes):
            ts[n, p] = st.F[comp][i, j, k]
    g = np.asarray(objective_grad(ts), np.float64)

    dt = grid.dt
    eps = st.eps_r * EPS_0
    s2 = st.sigma * dt / (2.0 * eps)
    ca = (1.0 - s2) / (1.0 + s2)
    cb = (dt / eps) / (1.0 + s2)
    ce = dt / (st.eps_r * EPS_0)
    ch = dt / (st.mu_r * MU_0)
    bx = st.box
    dca, dcb = _coef_derivs(st.eps_r[bx], st.sigma[bx], dt)
    dce = _ce_deriv(st.eps_r[bx], dt)
    aF = {c: np.zeros(grid.shape, f) for c in COMPONENTS}
    apsi = {k: np.zeros_like(v) for k, v in st.psi.items()}
    grad = np.zeros(dca.shape, np.float64)
    src_adj = np.zeros((n_steps, len(sources)), np.float64)

    def inject(n, e_part):
        for p, (i, j, k, comp) in enumerate(probes):
            if (comp[0] == "e") == e_part:
                aF[comp][i, j, k] += g[n, p]

    def record_src(n):
        for s, (i, j, k, comp, _) in enumerate(sources):
            src_adj[n, s] = aF[comp][i, j, k]

    inject(n_steps - 1, True)
    record_src(n_steps - 1)
    if st.nu:
        t = st.tab
        ix, iy, iz = _col(t["inv_dx"], 0), _col(t["inv_dy"], 1), _col(t["inv_dz"], 2)
        ixh, iyh, izh = _col(t["inv_dx_h"], 0), _col(t["inv_dy_h"], 1), _col(t["inv_dz_h"], 2)
    else:
        ix = iy = iz = ixh = iyh = izh = 1.0 / grid.dx
    for n in reversed(range(n_steps)):
        inject(n, False)                     # H part of Q^T g_n
        _mask_e(st, aF)                      # M^T
        _cpml_transpose(st, aF, apsi, _CPML_E, ce, fwd=False)   # CE^T
        # UE^T and the eps_r gradient
        h = st.hist[n]
        grad += sum(aF[c][bx] * (dca * h[q] + dcb * h[3 + q] + dce * h[6 + q]) for q, c in enumerate(("ex", "ey", "ez")))
        qx, qy, qz = cb * aF["ex"], cb * aF["ey"], cb * aF["ez"]
        # curl_x = dHz/dy - dHy/dz, curl_y = dHx/dz - dHz/dx, curl_z = dHy/dx - dHx/dy (backward diffs)
        vyx, vzx = iy * qx, iz * qx
        vzy, vxy = iz * qy, ix * qy
        vxz, vyz = ix * qz, iy * qz
        aF["hz"] = aF["hz"] + (vyx - _sf(vyx, 1)) - (vxy - _sf(vxy, 0))
        aF["hy"] = aF["hy"] - (vzx - _sf(vzx, 2)) + (vxz - _sf(vxz, 0))
        aF["hx"] = aF["hx"] + (vzy - _sf(vzy, 2)) - (vyz - _sf(vyz, 1))
        for c in ("ex", "ey", "ez"):
            aF[c] = ca * aF[c]
        _cpml_transpose(st, aF, apsi, _CPML_H, ch, fwd=True)    # CH^T
        # UH^T: H' = H - ch curl_E(E), forward diffs
        px, py, pz = ch * aF["hx"], ch * aF["hy"], ch * aF["hz"]
        ux_y, ux_z = iyh * px, izh * px
        uy_z, uy_x = izh * py, ixh * py
        uz_x, uz_y = ixh * pz, iyh * pz
        # curl_x = (Ez[j+1]-Ez[j]) iyh - (Ey[k+1]-Ey[k]) izh ; H -= ch curl
        aF["ez"] = aF["ez"] - (_sb(ux_y, 1) - ux_y) + (_sb(uy_x, 0) - uy_x)
        aF["ey"] = aF["ey"] + (_sb(ux_z, 2) - ux_z) - (_sb(uz_x, 0) - uz_x)
        aF["ex"] = aF["ex"] - (_sb(uy_z, 2) - uy_z) + (_sb(uz_y, 1) - uz_y)
        if n >= 1:
            inject(n - 1, True)
            record_src(n - 1)
    return ts, grad, src_adj
