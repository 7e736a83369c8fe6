"""NumPy restatement of the rfx scan body (uniform and graded lanes).

TEST INFRASTRUCTURE ONLY -- see the package docstring.  The arithmetic follows
the reference operation by operation so that a float32 run reproduces the
reference's float32 rounding pattern closely; ``dtype=np.float64`` gives the
FP64 oracle in which, as in the reference's float64 mode, the material arrays
and CPML profile coefficients keep their float32 values
(rfx/api/__init__.py precision docstring, rfx/boundaries/cpml.py:165-171) and
only the state and the arithmetic are promoted.

Reference anchors (paths relative to the rfx project root):
  grid geometry           rfx/grid.py:105-279
  graded grid             rfx/nonuniform.py:101-224, 274-422
  Yee updates             rfx/core/yee.py:121-138, 226-404, 411-492
  CPML                    rfx/boundaries/cpml.py:101-171, 346-478, 522-1065
  PEC / PEC mask          rfx/boundaries/pec.py:13-47, 90-208
  sources                 rfx/simulation.py:181-293, rfx/nonuniform.py:588-691,
                          rfx/sources/sources.py:31-103, 238-247
  uniform scan order      rfx/simulation.py:1255-1685, 1958-1977
  graded scan order       rfx/nonuniform.py:1256-1568
  DFT plane accumulation  rfx/simulation.py:1574-1588, rfx/nonuniform.py:1458-1472
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import NamedTuple

import numpy as np

# rfx/core/yee.py:117-118 and rfx/grid.py:8
EPS_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6
C0 = 299_792_458.0
# rfx/nonuniform.py:34 uses the constant implied by EPS_0/MU_0
C0_NU = 1.0 / math.sqrt(EPS_0 * MU_0)

COMPONENTS = ("ex", "ey", "ez", "hx", "hy", "hz")


# ---------------------------------------------------------------------------
# Grids
# ---------------------------------------------------------------------------

@dataclass
class UniformGrid:
    """Geometry of ``rfx.grid.Grid`` (rfx/grid.py:105-246)."""
    nx: int
    ny: int
    nz: int
    dx: float
    dt: float
    cpml_layers: int
    pads: tuple  # (x_lo, x_hi, y_lo, y_hi, z_lo, z_hi)

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    def position_to_index(self, pos):
        """rfx/grid.py:258-279: round-to-nearest plus the lo pad."""
        i = int(round(pos[0] / self.dx)) + self.pads[0]
        j = int(round(pos[1] / self.dx)) + self.pads[2]
        k = int(round(pos[2] / self.dx)) + self.pads[4]
        if not (0 <= i < self.nx and 0 <= j < self.ny and 0 <= k < self.nz):
            raise ValueError(f"position {pos} maps outside the grid")
        return (i, j, k)


def make_uniform_grid(domain, dx, cpml_layers=8, cpml_axes="xyz"):
    """rfx/grid.py:88-239 (3-D mode, no per-face overrides)."""
    dt = dx / (C0 * np.sqrt(3.0)) * 0.99
    pad = [cpml_layers if ax in cpml_axes else 0 for ax in "xyz"]
    nx = int(np.ceil(domain[0] / dx)) + 1 + 2 * pad[0]
    ny = int(np.ceil(domain[1] / dx)) + 1 + 2 * pad[1]
    nz = int(np.ceil(domain[2] / dx)) + 1 + 2 * pad[2]
    return UniformGrid(nx, ny, nz, float(dx), float(dt), int(cpml_layers),
                       (pad[0], pad[0], pad[1], pad[1], pad[2], pad[2]))


@dataclass
class NonUniformGrid:
    """Geometry of ``rfx.nonuniform.NonUniformGrid`` (rfx/nonuniform.py:37-98)."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dx_arr: np.ndarray
    dy_arr: np.ndarray
    dz: np.ndarray
    dt: float
    cpml_layers: int
    inv_dx: np.ndarray
    inv_dy: np.ndarray
    inv_dz: np.ndarray
    inv_dx_h: np.ndarray
    inv_dy_h: np.ndarray
    inv_dz_h: np.ndarray
    pads: tuple

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)


def profile_to_inv_arrays(profile_full):
    """rfx/nonuniform.py:187-224 (float32 arithmetic)."""
    arr = np.asarray(profile_full, dtype=np.float32)
    inv_local = np.float32(1.0) / arr
    inv_mean = np.float32(2.0) / (arr[:-1] + arr[1:])
    inv_d_h = np.concatenate([inv_local[:-1], np.zeros(1, np.float32)])
    inv_d_e = np.concatenate([inv_local[:1], inv_mean])
    return inv_d_e, inv_d_h


def _pad_profile(profile, pad_lo, pad_hi):
    """rfx/nonuniform.py:101-127 (concrete numpy branch)."""
    lo = np.full(pad_lo, float(profile[0]))
    hi = np.full(pad_hi, float(profile[-1]))
    return np.concatenate([lo, np.asarray(profile, dtype=np.float64), hi])


def _append_bounding_node(profile_full):
    """rfx/nonuniform.py:130-152."""
    return np.concatenate([profile_full, profile_full[-1:]])


def make_nonuniform_grid(domain_xy, dz_profile, dx, cpml_layers=8):
    """rfx/nonuniform.py:274-422 with uniform x/y and CPML on every face."""
    pad = int(cpml_layers)
    nxi = int(round(domain_xy[0] / dx))
    nyi = int(round(domain_xy[1] / dx))
    dx_full = _append_bounding_node(_pad_profile(np.full(nxi, float(dx)), pad, pad))
    dy_full = _append_bounding_node(_pad_profile(np.full(nyi, float(dx)), pad, pad))
    dz_full = _append_bounding_node(_pad_profile(np.asarray(dz_profile, np.float64), pad, pad))
    dt = float(0.99 / (C0_NU * np.sqrt(1 / float(np.min(dx_full)) ** 2
                                       + 1 / float(np.min(dy_full)) ** 2
                                       + 1 / float(np.min(dz_full)) ** 2)))
    ix, ixh = profile_to_inv_arrays(dx_full)
    iy, iyh = profile_to_inv_arrays(dy_full)
    iz, izh = profile_to_inv_arrays(dz_full)
    return NonUniformGrid(
        nx=len(dx_full), ny=len(dy_full), nz=len(dz_full),
        dx=float(dx), dy=float(dx),
        dx_arr=dx_full.astype(np.float32), dy_arr=dy_full.astype(np.float32),
        dz=dz_full.astype(np.float32), dt=dt, cpml_layers=pad,
        inv_dx=ix, inv_dy=iy, inv_dz=iz, inv_dx_h=ixh, inv_dy_h=iyh, inv_dz_h=izh,
        pads=(pad,) * 6)


# ---------------------------------------------------------------------------
# CPML profiles
# ---------------------------------------------------------------------------

class CPMLProfile(NamedTuple):
    sigma: np.ndarray
    kappa: np.ndarray
    alpha: np.ndarray
    b: np.ndarray
    c: np.ndarray


def cpml_profile(n_layers, dt, dx, order=3, kappa_max=1.0, R_asymptotic=1e-15):
    """rfx/boundaries/cpml.py:101-171 (concrete float64 branch, float32 out)."""
    eta = float(np.sqrt(MU_0 / EPS_0))
    d = n_layers * dx
    sigma_max = -float(np.log(R_asymptotic)) * (order + 1) / (2.0 * eta * d)
    sigma_max = sigma_max * kappa_max
    rho = 1.0 - np.arange(n_layers, dtype=np.float64) / max(n_layers - 1, 1)
    sigma = sigma_max * rho ** order
    kappa = 1.0 + (kappa_max - 1.0) * rho ** order
    alpha = 0.05 * (1.0 - rho)
    denom = sigma * kappa + kappa ** 2 * alpha
    b = np.exp(-(sigma / kappa + alpha) * dt / EPS_0)
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.where(denom > 1e-30, sigma * (b - 1.0) / denom, 0.0)
    f = np.float32
    return CPMLProfile(sigma.astype(f), kappa.astype(f), alpha.astype(f),
                       b.astype(f), c.astype(f))


def build_cpml(grid, kappa_max=1.0):
    """Per-face profiles and boundary cell sizes (rfx/boundaries/cpml.py:346-478).

    Returns ``{face: (b, c, kappa, cell_size)}`` with the hi faces pre-flipped
    (rfx/boundaries/cpml.py:404-409).  Uniform grids use ``dx`` on every face;
    graded grids use ``dx``, ``dy``, ``dz[0]``, ``dz[-1]``
    (rfx/boundaries/cpml.py:174-197).
    """
    n = grid.cpml_layers
    if isinstance(grid, NonUniformGrid):
        sizes = {"x": (grid.dx, grid.dx), "y": (grid.dy, grid.dy),
                 "z": (float(grid.dz[0]), float(grid.dz[-1]))}
    else:
        sizes = {a: (grid.dx, grid.dx) for a in "xyz"}
    out = {}
    for a in "xyz":
        lo = cpml_profile(n, grid.dt, sizes[a][0], kappa_max=kappa_max)
        hi = cpml_profile(n, grid.dt, sizes[a][1], kappa_max=kappa_max)
        out[a + "_lo"] = (lo.b, lo.c, lo.kappa, sizes[a][0])
        out[a + "_hi"] = (hi.b[::-1].copy(), hi.c[::-1].copy(), hi.kappa[::-1].copy(), sizes[a][1])
    return out


# ---------------------------------------------------------------------------
# Sources
# ---------------------------------------------------------------------------

def gaussian_pulse(t, f0, bandwidth=0.5, amplitude=1.0, cutoff=3.0):
    """rfx/sources/sources.py:56-103, evaluated in the dtype of ``t``."""
    tau = 1.0 / (f0 * bandwidth * math.pi)
    t0 = cutoff * tau
    arg = (t - t0) / tau
    return amplitude * (-2.0 * arg) * np.exp(-(arg ** 2))


def _times(n_steps, dt):
    """``jnp.arange(n_steps, dtype=float32) * dt`` (rfx/simulation.py:277)."""
    return np.arange(n_steps, dtype=np.float32) * dt


def _cell_cb(eps_r_cell, sigma_cell, dt):
    """rfx/simulation.py:181-194 in float32."""
    eps = np.float32(eps_r_cell) * EPS_0
    loss = np.float32(sigma_cell) * dt / (2.0 * eps)
    return np.float32((dt / eps) / (1.0 + loss))


def j_source_waveform(grid, idx, materials, n_steps, f0, bandwidth=0.5, amplitude=1.0):
    """``make_j_source`` (rfx/simulation.py:239-293): ``cb * pulse(n dt)``."""
    i, j, k = idx
    cb = _cell_cb(materials[0][i, j, k], materials[1][i, j, k], grid.dt)
    w = gaussian_pulse(_times(n_steps, grid.dt), f0, bandwidth, amplitude)
    return (cb * w).astype(np.float32)


def port_sigma(d_par, d_perp1, d_perp2, impedance):
    """rfx/sources/sources.py:31-45."""
    return d_par / (impedance * d_perp1 * d_perp2)


def port_source_waveform(grid, idx, materials, n_steps, f0, bandwidth=0.5, d_par=None):
    """``make_port_source`` (rfx/simulation.py:296-314): ``cb/d_par * pulse``."""
    i, j, k = idx
    cb = _cell_cb(materials[0][i, j, k], materials[1][i, j, k], grid.dt)
    d_par = grid.dx if d_par is None else d_par
    w = gaussian_pulse(_times(n_steps, grid.dt), f0, bandwidth)
    return ((cb / d_par) * w).astype(np.float32)


def current_source_waveform(grid, idx, component, materials, n_steps, f0, bandwidth=0.5):
    """``make_current_source`` (rfx/nonuniform.py:588-691): ``cb/dV * pulse``
    with the primal width on the component axis and dual widths across."""
    i, j, k = idx
    eps = float(materials[0][i, j, k]) * EPS_0
    sigma = float(materials[1][i, j, k])
    loss = sigma * grid.dt / (2.0 * eps)
    cb = (grid.dt / eps) / (1.0 + loss)
    p_axis = {"ex": 0, "ey": 1, "ez": 2}[component]
    profiles = (grid.dx_arr, grid.dy_arr, grid.dz)
    widths = []
    for a, ii in enumerate((i, j, k)):
        prof = np.asarray(profiles[a], dtype=np.float64)
        if a == p_axis:
            widths.append(float(prof[ii]))
        elif ii <= 0:
            widths.append(float(prof[0]))
        else:
            widths.append(float(0.5 * (prof[ii - 1] + prof[ii])))
    dV = widths[0] * widths[1] * widths[2]
    w = gaussian_pulse(_times(n_steps, grid.dt), f0, bandwidth)
    return ((cb / dV) * w).astype(np.float32)


# ---------------------------------------------------------------------------
# Stencil helpers
# ---------------------------------------------------------------------------

def _sf(a, ax):
    """``_shift_fwd`` (rfx/core/yee.py:121-128): a[i+1], zero past the end."""
    out = np.zeros_like(a)
    d = [slice(None)] * 3
    s = [slice(None)] * 3
    d[ax] = slice(0, -1)
    s[ax] = slice(1, None)
    out[tuple(d)] = a[tuple(s)]
    return out


def _sb(a, ax):
    """``_shift_bwd`` (rfx/core/yee.py:131-138): a[i-1], zero before the start."""
    out = np.zeros_like(a)
    d = [slice(None)] * 3
    s = [slice(None)] * 3
    d[ax] = slice(1, None)
    s[ax] = slice(0, -1)
    out[tuple(d)] = a[tuple(s)]
    return out


def tangential_edge_masks(cell_mask):
    """rfx/boundaries/pec.py:90-176 on non-periodic 3-D axes."""
    m = np.asarray(cell_mask, dtype=bool)
    out = []
    for ax in range(3):
        nb = _sb(m, ax) | _sf(m, ax)
        out.append(m & nb)
    return tuple(out)


def _slab(ax, lo, n):
    s = [slice(None)] * 3
    s[ax] = slice(0, n) if lo else slice(-n, None)
    return tuple(s)


def _col(v, ax):
    shp = [1, 1, 1]
    shp[ax] = -1
    return v.reshape(shp)


# ---------------------------------------------------------------------------
# One step
# ---------------------------------------------------------------------------

# (field corrected, field differentiated, sign) per CPML axis, in the order
# the reference applies them (rfx/boundaries/cpml.py:874-1043 and 604-777).
_CPML_H = {0: (("hy", "ez", +1), ("hz", "ey", -1)),
           1: (("hx", "ez", -1), ("hz", "ex", +1)),
           2: (("hx", "ey", +1), ("hy", "ex", -1))}
_CPML_E = {0: (("ey", "hz", -1), ("ez", "hy", +1)),
           1: (("ex", "hz", +1), ("ez", "hx", -1)),
           2: (("ex", "hy", -1), ("ey", "hx", +1))}


class _Stepper:
    def __init__(self, grid, materials, *, dtype, nonuniform, cpml_axes,
                 pec_axes, pec_mask, kappa_max=1.0, exact_materials=False):
        self.g = grid
        self.f = np.dtype(dtype)
        self.nu = nonuniform
        shape = grid.shape
        eps_r, sigma, mu_r = materials
        f = self.f
        # exact_materials keeps float64 material values (finite-difference
        # checks); otherwise they are float32 as in the reference.
        mdt = f if exact_materials else np.float32
        self.eps_r = np.asarray(eps_r, mdt).astype(f)
        self.sigma = np.asarray(sigma, mdt).astype(f)
        self.mu_r = np.asarray(mu_r, mdt).astype(f)
        self.F = {c: np.zeros(shape, f) for c in COMPONENTS}
        self.step_count = 0
        self.cpml_axes = cpml_axes
        self.pec_axes = pec_axes
        self.n = grid.cpml_layers
        self.psi = {}
        if cpml_axes and self.n > 0:
            self.prof = build_cpml(grid, kappa_max)
            for ax in range(3):
                if "xyz"[ax] not in cpml_axes:
                    continue
                for side in ("lo", "hi"):
                    sl_shape = list(shape)
                    sl_shape[ax] = self.n
                    for (fc, _, _) in _CPML_H[ax] + _CPML_E[ax]:
                        self.psi[(fc, ax, side)] = np.zeros(sl_shape, f)
        self.emask = None
        if pec_mask is not None:
            self.emask = tuple(m.astype(f) for m in tangential_edge_masks(pec_mask))
        if nonuniform:
            g = grid
            self.tab = {k: np.asarray(getattr(g, k), np.float32).astype(f) for k in
                        ("inv_dx", "inv_dy", "inv_dz", "inv_dx_h", "inv_dy_h", "inv_dz_h")}

    # rfx/core/yee.py:226-291 (uniform) and :411-453 (graded)
    def update_h(self):
        F, dt, f = self.F, self.g.dt, self.f
        ex, ey, ez = F["ex"], F["ey"], F["ez"]
        mu = self.mu_r * MU_0
        if self.nu:
            t = self.tab
            iyh, izh, ixh = _col(t["inv_dy_h"], 1), _col(t["inv_dz_h"], 2), _col(t["inv_dx_h"], 0)
            cx = (_sf(ez, 1) - ez) * iyh - (_sf(ey, 2) - ey) * izh
            cy = (_sf(ex, 2) - ex) * izh - (_sf(ez, 0) - ez) * ixh
            cz = (_sf(ey, 0) - ey) * ixh - (_sf(ex, 1) - ex) * iyh
        else:
            dx = self.g.dx
            cx = (_sf(ez, 1) - ez) / dx - (_sf(ey, 2) - ey) / dx
            cy = (_sf(ex, 2) - ex) / dx - (_sf(ez, 0) - ez) / dx
            cz = (_sf(ey, 0) - ey) / dx - (_sf(ex, 1) - ex) / dx
        k = dt / mu
        F["hx"] = F["hx"] - k * cx
        F["hy"] = F["hy"] - k * cy
        F["hz"] = F["hz"] - k * cz

    # rfx/core/yee.py:347-404 (uniform) and :456-492 (graded)
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
        F["ex"] = ca * F["ex"] + cb * cx
        F["ey"] = ca * F["ey"] + cb * cy
        F["ez"] = ca * F["ez"] + cb * cz
        self.step_count += 1

    def _apply_cpml(self, table, coef_full, fwd, corr=None):
        """rfx/boundaries/cpml.py:522-801 (E) and :804-1065 (H).  The curl
        slices read the field values from before this correction pass.
        ``corr`` (optional, per component float64 arrays of the grid shape)
        accumulates each correction before its coefficient scaling,
        sign * (psi + (1/kappa - 1) curl): the factor that d coef / d eps_r
        multiplies in the reference's autodiff of the same two adds."""
        F, n = self.F, self.n
        src = {c: F[c] for c in COMPONENTS}
        work = {c: F[c].copy() for c in COMPONENTS}
        for ax in range(3):
            if "xyz"[ax] not in self.cpml_axes:
                continue
            name = "xyz"[ax]
            for (fc, dc, sgn) in table[ax]:
                for side in ("lo", "hi"):
                    b, c, kap, d = self.prof[f"{name}_{side}"]
                    b = _col(b.astype(self.f), ax)
                    c = _col(c.astype(self.f), ax)
                    kap = _col(kap.astype(self.f), ax)
                    sl = _slab(ax, side == "lo", n)
                    a = src[dc]
                    if fwd:
                        curl = (_sf(a, ax)[sl] - a[sl]) / d
                    else:
                        curl = (a[sl] - _sb(a, ax)[sl]) / d
                    key = (fc, ax, side)
                    psi = b * self.psi[key] + c * curl
                    self.psi[key] = psi
                    cf = coef_full[sl]
                    if sgn < 0:
                        cf = -cf
                    km = (1.0 / kap - 1.0)
                    if ax == 0:
                        work[fc][sl] = work[fc][sl] + cf * psi
                        work[fc][sl] = work[fc][sl] + cf * km * curl
                    else:
                        work[fc][sl] = work[fc][sl] + cf * psi
                        work[fc][sl] = work[fc][sl] + cf * (km * curl)
                    if corr is not None:
                        corr[fc][sl] = corr[fc][sl] + sgn * (np.asarray(psi, np.float64)
                                                             + np.asarray(km * curl, np.float64))
        for c in COMPONENTS:
            F[c] = work[c]

    def cpml_h(self):
        if self.psi:
            ch = self.g.dt / (self.mu_r * MU_0)
            self._apply_cpml(_CPML_H, ch, fwd=True)

    def cpml_e(self):
        if self.psi:
            ce = self.g.dt / (self.eps_r * EPS_0)
            self._apply_cpml(_CPML_E, ce, fwd=False)

    # rfx/boundaries/pec.py:13-47
    def pec(self):
        F, ax = self.F, self.pec_axes
        if "x" in ax:
            for c in ("ey", "ez"):
                F[c][0, :, :] = 0.0
                F[c][-1, :, :] = 0.0
        if "y" in ax:
            for c in ("ex", "ez"):
                F[c][:, 0, :] = 0.0
                F[c][:, -1, :] = 0.0
        if "z" in ax:
            for c in ("ex", "ey"):
                F[c][:, :, 0] = 0.0
                F[c][:, :, -1] = 0.0
            F["ez"][:, :, -1] = 0.0

    # rfx/boundaries/pec.py:179-208
    def pec_mask(self):
        if self.emask is not None:
            for c, m in zip(("ex", "ey", "ez"), self.emask):
                self.F[c] = self.F[c] * (1.0 - m)


class OracleResult(NamedTuple):
    time_series: np.ndarray           # (n_steps, n_probes)
    dft_planes: list                  # [(n_freqs, n1, n2) complex]
    state: dict                       # final fields
    vi: np.ndarray | None             # (n_steps, n_ports, 2) pre-source V, I
    psi: dict
    flux: list | None = None          # per flux monitor: complex128 (4, n_freqs, n1, n2)
    ntff: dict | None = None          # NTFF faces: {"x_lo": ..., "c_x_lo": ...} complex64 (n_f, n1, n2, 4)


def _plane(a, axis, index):
    if axis == 0:
        return a[index, :, :]
    if axis == 1:
        return a[:, index, :]
    return a[:, :, index]


_FLUX_COMPONENTS = {0: ("ey", "ez", "hy", "hz"), 1: ("ez", "ex", "hz", "hx"), 2: ("ex", "ey", "hx", "hy")}


def flux_window_weight(step, total_steps, window, alpha):
    """rfx/core/dft_utils.py:8-50 (float32)."""
    if total_steps <= 1 or window == "rect":
        return np.float32(1.0)
    x = np.float32(step) / np.float32(max(total_steps - 1, 1))
    if window == "hann" or (window == "tukey" and alpha >= 1.0):
        return np.float32(0.5) * (np.float32(1.0) - np.cos(np.float32(2.0 * np.pi) * x))
    a = float(alpha)
    if a <= 0.0:
        return np.float32(1.0)
    if x < a / 2.0:
        return np.float32(0.5) * (np.float32(1.0) + np.cos(np.float32(np.pi) * (np.float32(2.0) * x / np.float32(a)
                                                                                - np.float32(1.0))))
    if x <= 1.0 - a / 2.0:
        return np.float32(1.0)
    return np.float32(0.5) * (np.float32(1.0) + np.cos(np.float32(np.pi) * (
        np.float32(2.0) * x / np.float32(a) - np.float32(2.0 / a) + np.float32(1.0))))


def _flux_step(F, mon, acc, step, dt, graded=False):
    """rfx/simulation.py:1590-1642: E at plane index, H averaged over index-1
    and index (float32), times exp(-j 2 pi f t) dt w (E, t = step dt) and
    exp(-j 2 pi f (t - dt/2)) dt w (H), accumulated in complex128.  On the
    graded lane (rfx/nonuniform.py:1483-1520) t = f32(step) * dt is rounded to
    float32."""
    axis, index, lo1, hi1, lo2, hi2, freqs, total, window, alpha = mon
    c = _FLUX_COMPONENTS[axis]
    im1 = max(index - 1, 0)

    def cut(a, plane):
        s = [slice(None)] * 3
        s[axis] = plane
        t = a[tuple(s)]
        return t[lo1:hi1, lo2:hi2]

    e1, e2 = cut(F[c[0]], index), cut(F[c[1]], index)
    h1 = (cut(F[c[2]], im1) + cut(F[c[2]], index)) * np.float32(0.5)
    h2 = (cut(F[c[3]], im1) + cut(F[c[3]], index)) * np.float32(0.5)
    f = np.asarray(freqs, np.float64)
    t = float(np.float32(step) * np.float32(dt)) if graded else float(step) * dt
    w = float(flux_window_weight(step, total, window, alpha))
    ke = np.exp(-1j * 2.0 * np.pi * f * t) * dt * w
    kh = np.exp(-1j * 2.0 * np.pi * f * (t - dt * 0.5)) * dt * w
    for q, (v, k) in enumerate(((e1, ke), (e2, ke), (h1, kh), (h2, kh))):
        acc[q] += np.asarray(v, np.float64)[None, :, :] * k[:, None, None]


NTFF_FACES = ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")
_NTFF_COMPONENTS = {0: ("ey", "ez", "hy", "hz"), 1: ("ex", "ez", "hx", "hz"), 2: ("ex", "ey", "hx", "hy")}


def ntff_init(box, dtype=np.float32):
    """Zeroed NTFF running sums and Kahan residuals (rfx/farfield.py:164-205):
    ``box`` = (i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, freqs); x faces are
    (n_f, nj, nk, 4), y faces (n_f, ni, nk, 4), z faces (n_f, ni, nj, 4);
    complex64 for float32 fields, complex128 for float64 ones
    (rfx/farfield.py:144-161 ntff_accum_dtype)."""
    i0, i1, j0, j1, k0, k1, freqs = box
    nf = len(freqs)
    cdt = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
    dims = {0: (j1 - j0, k1 - k0), 1: (i1 - i0, k1 - k0), 2: (i1 - i0, j1 - j0)}
    out = {}
    for q, name in enumerate(NTFF_FACES):
        out[name] = np.zeros((nf,) + dims[q // 2] + (4,), cdt)
        out["c_" + name] = np.zeros_like(out[name])
    return out


def ntff_phases(freqs, step, dt, dtype=np.float32):
    """E and H step factors of rfx/farfield.py:230-244: t = step dt,
    omega = 2 pi f, E factor exp(-1j omega t) dt, H factor
    exp(-1j omega (t + dt/2)) dt, in float32 arithmetic (or float64 for a
    float64 run)."""
    f = np.dtype(dtype).type
    d = f(dt)
    t = f(step) * d
    om = f(2 * np.pi) * np.asarray(freqs, dtype)
    th = f(t + d * f(0.5))
    out = []
    for tt in (t, th):
        a = (om * tt).astype(dtype).astype(np.float64)
        c = np.cos(a).astype(dtype) * d
        sn = -np.sin(a).astype(dtype) * d
        out.append((c.astype(dtype), sn.astype(dtype)))
    return out


def ntff_step(F, box, acc, step, dt):
    """One step of rfx/farfield.py:208-313: on each face the four tangential
    components times the step's factor (E factor for the E pair, H factor for
    the H pair), Kahan-added per real and imaginary part in the accumulators'
    real type (float32 for complex64 sums)."""
    i0, i1, j0, j1, k0, k1, freqs = box
    rt = np.float32 if acc["x_lo"].dtype == np.complex64 else np.float64
    (ce, se), (chh, sh) = ntff_phases(freqs, step, dt, rt)
    lo = (i0, j0, k0)
    hi = (i1, j1, k1)
    for q, name in enumerate(NTFF_FACES):
        ax = q // 2
        idx = hi[ax] if q & 1 else lo[ax]
        sl = [slice(i0, i1), slice(j0, j1), slice(k0, k1)]
        sl[ax] = idx
        vals = np.stack([np.asarray(F[c][tuple(sl)], rt) for c in _NTFF_COMPONENTS[ax]], axis=-1)
        wr = np.stack([ce, ce, chh, chh], axis=-1)[:, None, None, :]
        wi = np.stack([se, se, sh, sh], axis=-1)[:, None, None, :]
        s, c = acc[name], acc["c_" + name]
        for part, w in (("real", wr), ("imag", wi)):
            sv = getattr(s, part).astype(rt)
            cv = getattr(c, part).astype(rt)
            val = (vals[None] * w).astype(rt)
            y = (val - cv).astype(rt)
            t = (sv + y).astype(rt)
            cv = ((t - sv).astype(rt) - y).astype(rt)
            if part == "real":
                s.real, c.real = t, cv
            else:
                s.imag, c.imag = t, cv


def _run(st, n_steps, sources, probes, dft_planes, vi_ports, dft_time_offset,
         probes_before_dft, dx_vi, stop=None, flux_monitors=(), ntff=None):
    f = st.f
    cdt = np.complex64 if f == np.float32 else np.complex128
    ts = np.zeros((n_steps, len(probes)), f)
    accs = []
    for (axis, index, comp, freqs) in dft_planes:
        shp = list(st.g.shape)
        del shp[axis]
        accs.append(np.zeros([len(freqs)] + shp, cdt))
    vi = np.zeros((n_steps, len(vi_ports), 2), f) if vi_ports else None
    dt = st.g.dt
    flux_accs = [np.zeros((4, len(m[6]), m[3] - m[2], m[5] - m[4]), np.complex128) for m in flux_monitors]
    ntff_acc = ntff_init(ntff, f) if ntff is not None else None
    for n in range(n_steps):
        st.update_h()
        st.cpml_h()
        st.update_e()
        st.cpml_e()
        st.pec()
        st.pec_mask()
        F = st.F
        # Lumped-port V/I sampling happens before source injection
        # (rfx/simulation.py:1480-1500).
        for p, (i, j, k, comp) in enumerate(vi_ports or ()):
            v = -F[comp][i, j, k] * dx_vi
            if comp == "ez":
                iv = (F["hy"][i, j, k] - F["hy"][i - 1, j, k] - F["hx"][i, j, k] + F["hx"][i, j - 1, k]) * dx_vi
            elif comp == "ex":
                iv = (F["hz"][i, j, k] - F["hz"][i, j - 1, k] - F["hy"][i, j, k] + F["hy"][i, j, k - 1]) * dx_vi
            else:
                iv = (F["hx"][i, j, k] - F["hx"][i, j, k - 1] - F["hz"][i, j, k] + F["hz"][i - 1, j, k]) * dx_vi
            vi[n, p, 0] = v
            vi[n, p, 1] = iv
        for (i, j, k, comp, wave) in sources:
            F[comp][i, j, k] = F[comp][i, j, k] + f.type(wave[n])

        def _probes():
            for p, (i, j, k, comp) in enumerate(probes):
                ts[n, p] = F[comp][i, j, k]

        def _dft():
            t = np.float32(n + dft_time_offset) * np.float32(dt) if f == np.float32 \
                else float(n + dft_time_offset) * dt
            for q, (axis, index, comp, freqs) in enumerate(dft_planes):
                fr = np.asarray(freqs, dtype=f)
                arg = (fr * (-2.0 * math.pi)).astype(f) * t
                phase = (np.cos(arg) + 1j * np.sin(arg)).astype(cdt)
                plane = _plane(F[comp], axis, index)
                accs[q] = accs[q] + (plane[None, :, :] * phase[:, None, None]) * dt

        if probes_before_dft:
            _probes()
            _dft()
        else:
            _dft()
            _probes()
        for m, acc in zip(flux_monitors, flux_accs):
            _flux_step(F, m, acc, n + dft_time_offset, dt, graded=dft_time_offset == 0)
        if ntff is not None:
            ntff_step(F, ntff, ntff_acc, n, dt)
        if stop is not None and stop(n, F):
            ts = ts[:n + 1]
            vi = vi[:n + 1] if vi is not None else None
            break
    return OracleResult(ts, accs, {c: st.F[c].copy() for c in COMPONENTS}, vi, st.psi,
                        flux_accs if flux_monitors else None, ntff_acc)


def _set_fields(st, init_fields):
    """Start from given fields (a dict of the six components) instead of zero:
    a test device, not part of the reference's run."""
    for c, v in (init_fields or {}).items():
        st.F[c][...] = np.asarray(v, st.f)


def run_uniform(grid, materials, n_steps, *, boundary="cpml", cpml_axes="xyz",
                pec_axes=None, sources=(), probes=(), dft_planes=(), pec_mask=None,
                vi_ports=(), kappa_max=1.0, dtype=np.float32, exact_materials=False, flux_monitors=(),
                ntff=None, init_fields=None):
    """``rfx.simulation.run`` (rfx/simulation.py:1686-2138), scan body order of
    rfx/simulation.py:1255-1685.  ``pec_axes=None`` means all axes
    (rfx/simulation.py:684-691).  ``sources`` are ``(i, j, k, comp, waveform)``,
    ``probes`` ``(i, j, k, comp)``, ``dft_planes`` ``(axis, index, comp, freqs)``.
    The uniform DFT time stamp is ``(n+1) dt`` (rfx/simulation.py:1574).
    ``ntff`` = (i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, freqs) accumulates the
    Huygens box after the step's probes (rfx/simulation.py:1570-1572)."""
    if pec_axes is None:
        pec_axes = "xyz"
    st = _Stepper(grid, materials, dtype=dtype, nonuniform=False,
                  cpml_axes=cpml_axes if boundary == "cpml" else "",
                  pec_axes=pec_axes, pec_mask=pec_mask, kappa_max=kappa_max,
                  exact_materials=exact_materials)
    _set_fields(st, init_fields)
    return _run(st, n_steps, sources, probes, dft_planes, vi_ports, 1,
                probes_before_dft=True, dx_vi=grid.dx, flux_monitors=flux_monitors, ntff=ntff)


def run_nonuniform(grid, materials, n_steps, *, sources=(), probes=(), dft_planes=(),
                   pec_mask=None, kappa_max=1.0, dtype=np.float32, exact_materials=False, ntff=None,
                   flux_monitors=(), init_fields=None):
    """``rfx.nonuniform.run_nonuniform`` (rfx/nonuniform.py:1589-1804), scan body
    of rfx/nonuniform.py:1256-1568: PEC on every axis, DFT time stamp ``n dt``
    (rfx/nonuniform.py:1461), DFT before probes."""
    axes = "".join(a for a, p in zip("xyz", (grid.pads[0] + grid.pads[1],
                                             grid.pads[2] + grid.pads[3],
                                             grid.pads[4] + grid.pads[5])) if p > 0)
    st = _Stepper(grid, materials, dtype=dtype, nonuniform=True,
                  cpml_axes=axes if grid.cpml_layers > 0 else "",
                  pec_axes="xyz", pec_mask=pec_mask, kappa_max=kappa_max,
                  exact_materials=exact_materials)
    _set_fields(st, init_fields)
    return _run(st, n_steps, sources, probes, dft_planes, (), 0,
                probes_before_dft=False, dx_vi=grid.dx, ntff=ntff, flux_monitors=flux_monitors)


def _box_flux(F, flux_box):
    """Net outgoing co-located Poynting flux through the faces of the index
    box (i0, i1, j0, j1, k0, k1): float32 products, float64 sum
    (rfx/simulation.py:2513-2540, rfx/nonuniform.py:2171-2184)."""
    i0, i1, j0, j1, k0, k1 = flux_box
    f32 = np.float32
    g = {c: F[c] for c in COMPONENTS}
    jj, kk, ii = slice(j0, j1), slice(k0, k1), slice(i0, i1)

    def term(a, b, c, d, sel):
        return np.sum(((g[a][sel] * g[b][sel]).astype(f32) - (g[c][sel] * g[d][sel]).astype(f32))
                      .astype(np.float64))

    p = term("ey", "hz", "ez", "hy", (i1, jj, kk)) - term("ey", "hz", "ez", "hy", (i0, jj, kk))
    p += term("ez", "hx", "ex", "hz", (ii, j1, kk)) - term("ez", "hx", "ex", "hz", (ii, j0, kk))
    p += term("ex", "hy", "ey", "hx", (ii, jj, k1)) - term("ex", "hy", "ey", "hx", (ii, jj, k0))
    return float(p)


def run_until_decay_uniform(grid, materials, *, decay_by=1e-3, check_interval=50, min_steps=100,
                            max_steps=50_000, decay_energy_consecutive=2, monitor=None, boundary="pec",
                            cpml_axes="xyz", pec_axes=None, sources=(), probes=(), pec_mask=None,
                            dtype=np.float32, flux_box=None, flux_env_checks=4):
    """``rfx.simulation.run_until_decay`` (rfx/simulation.py:2198-2700), energy
    and point-field stops only.  Absorbing boundary: at step n with n+1 >=
    min_steps and n % check_interval == 0 the interior energy
    U = sum(E^2 + H^2) over the non-CPML slice (:2493-2505, summed here in
    float64) updates its running peak, and ``decay_energy_consecutive``
    consecutive checks with U < decay_by * peak stop the run (:2603-2622).
    Closed boundary: the squared field at ``monitor`` = (i, j, k, comp)
    (after the step's source injection) keeps a running peak every step, and a
    check step with value^2 < decay_by * peak stops (:2623-2633).
    ``flux_box`` = (i0, i1, j0, j1, k0, k1) selects the radiated-flux stop on
    an absorbing boundary (:2513-2540, 2580-2600): at every check step from
    the first, |net outgoing co-located Poynting flux| through the box faces
    (float32 products, float64 sum), enveloped by the maximum over the last
    ``flux_env_checks`` checks, against decay_by times its running peak,
    once n+1 >= min_steps.
    Returns (OracleResult, steps run)."""
    if pec_axes is None:
        pec_axes = "xyz"
    absorbing = boundary == "cpml"
    st = _Stepper(grid, materials, dtype=dtype, nonuniform=False,
                  cpml_axes=cpml_axes if absorbing else "",
                  pec_axes=pec_axes, pec_mask=pec_mask, kappa_max=1.0)
    p = grid.pads
    sl = (slice(p[0], grid.nx - p[1]), slice(p[2], grid.ny - p[3]), slice(p[4], grid.nz - p[5]))
    state = {"peak_U": 0.0, "below": 0, "peak_sq": 0.0, "steps": 0, "peak_flux": 0.0, "hist": []}

    def radiated_power(F):
        return _box_flux(F, flux_box)

    def stop(n, F):
        state["steps"] = n + 1
        if absorbing and flux_box is not None:
            if n % check_interval == 0:
                state["hist"].append(abs(radiated_power(F)))
                env = max(state["hist"][-flux_env_checks:])
                state["peak_flux"] = max(state["peak_flux"], env)
                if n + 1 >= min_steps and state["peak_flux"] > 0.0 and env < decay_by * state["peak_flux"]:
                    state["below"] += 1
                    if state["below"] >= decay_energy_consecutive:
                        return True
                else:
                    state["below"] = 0
            return False
        if absorbing:
            if n + 1 >= min_steps and n % check_interval == 0:
                U = float(sum(np.sum(np.asarray(F[c][sl], np.float64) ** 2) for c in COMPONENTS))
                state["peak_U"] = max(state["peak_U"], U)
                if U < decay_by * state["peak_U"]:
                    state["below"] += 1
                    if state["below"] >= decay_energy_consecutive:
                        return True
                else:
                    state["below"] = 0
            return False
        i, j, k, comp = monitor
        v2 = float(F[comp][i, j, k]) ** 2
        state["peak_sq"] = max(state["peak_sq"], v2)
        return (n + 1 >= min_steps and n % check_interval == 0 and state["peak_sq"] > 0.0
                and v2 < decay_by * state["peak_sq"])

    res = _run(st, max_steps, sources, probes, (), (), 1, probes_before_dft=True, dx_vi=grid.dx, stop=stop)
    return res, state["steps"]


def run_until_decay_nonuniform(grid, materials, *, decay_by=1e-3, check_interval=50, min_steps=100,
                               max_steps=50_000, decay_energy_consecutive=2, sources=(), probes=(),
                               pec_mask=None, dtype=np.float32, flux_box=None, flux_env_checks=4,
                               dx_arr=None, dy_arr=None):
    """``rfx.nonuniform.run_nonuniform_until_decay`` (rfx/nonuniform.py:1988-2260),
    energy and radiated-flux stops.  Checks fall after every ``check_interval``
    steps (and after the last, shorter chunk): the energy U = sum((E^2 + H^2)
    dV) over the non-CPML cells, dV = dx[i] dy[j] dz[k] from the padded
    per-axis cell sizes (``dx_arr``, ``dy_arr``: the x and y profiles of the
    grid, ``grid.dz`` for z), once ``min_steps`` are done, peak updated before
    the compare, ``decay_energy_consecutive`` consecutive checks below
    decay_by * peak stop; with ``flux_box`` (index box) the |net flux| is
    tracked from the first check, enveloped over the last ``flux_env_checks``
    checks, and gated on ``min_steps``.  Returns (OracleResult, steps run,
    [(steps, U, peak U), ...])."""
    axes = "".join(a for a, p in zip("xyz", (grid.pads[0] + grid.pads[1], grid.pads[2] + grid.pads[3],
                                             grid.pads[4] + grid.pads[5])) if p > 0)
    st = _Stepper(grid, materials, dtype=dtype, nonuniform=True,
                  cpml_axes=axes if grid.cpml_layers > 0 else "",
                  pec_axes="xyz", pec_mask=pec_mask, kappa_max=1.0)
    p = grid.pads
    sl = (slice(p[0], grid.nx - p[1]), slice(p[2], grid.ny - p[3]), slice(p[4], grid.nz - p[5]))
    dx_arr = np.full(grid.nx, grid.dx) if dx_arr is None else np.asarray(dx_arr, np.float64)
    dy_arr = np.full(grid.ny, grid.dx) if dy_arr is None else np.asarray(dy_arr, np.float64)
    dV = (dx_arr[sl[0], None, None] * dy_arr[None, sl[1], None] *
          np.asarray(grid.dz, np.float64)[None, None, sl[2]])
    state = {"peak_U": 0.0, "below": 0, "steps": 0, "peak_flux": 0.0, "hist": [], "checks": []}

    def stop(n, F):
        done = n + 1
        state["steps"] = done
        if done % check_interval != 0 and done != max_steps:
            return False
        if flux_box is not None:
            state["hist"].append(abs(_box_flux(F, flux_box)))
            env = max(state["hist"][-flux_env_checks:])
            state["peak_flux"] = max(state["peak_flux"], env)
            if done >= min_steps and state["peak_flux"] > 0.0 and env < decay_by * state["peak_flux"]:
                state["below"] += 1
                return state["below"] >= decay_energy_consecutive
            state["below"] = 0
            return False
        if done < min_steps:
            return False
        U = float(sum(np.sum(np.asarray(F[c][sl], np.float64) ** 2 * dV) for c in COMPONENTS))
        state["peak_U"] = max(state["peak_U"], U)
        state["checks"].append((done, U, state["peak_U"]))
        if U < decay_by * state["peak_U"]:
            state["below"] += 1
            return state["below"] >= decay_energy_consecutive
        state["below"] = 0
        return False

    src = []
    for (i, j, k, comp, w) in sources:
        w = np.asarray(w, np.float32)[:max_steps]
        src.append((i, j, k, comp, np.concatenate([w, np.zeros(max_steps - len(w), np.float32)])))
    res = _run(st, max_steps, src, probes, (), (), 0, probes_before_dft=False, dx_vi=grid.dx, stop=stop)
    return res, state["steps"], state["checks"]
