"""Grid geometry: the uniform ``Grid`` and the graded ``NonUniformGrid``.

Mirrors the reference's host-side geometry so callers can build a grid here
or hand in the reference's own objects (duck-typed on ``shape``, ``dx``,
``dt``, ``cpml_layers`` and the per-face pads).

  Grid                   rfx/grid.py:37-246
  make_nonuniform_grid   rfx/nonuniform.py:274-422
  _profile_to_inv_arrays rfx/nonuniform.py:187-224
"""

from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np

C0 = 299_792_458.0                     # rfx/grid.py:8
EPS_0 = 8.8541878128e-12               # rfx/core/yee.py:117
MU_0 = 1.25663706212e-6                # rfx/core/yee.py:118
C0_NU = 1.0 / math.sqrt(EPS_0 * MU_0)  # rfx/nonuniform.py:34


class Grid:
    """Uniform Yee grid with CPML padding (rfx/grid.py:37-246, 3-D mode)."""

    def __init__(self, freq_max: float, domain, dx: float | None = None, cpml_layers: int = 8,
                 cpml_axes: str = "xyz", kappa_max: float = 1.0, pec_faces=None, face_layers=None):
        self.freq_max = float(freq_max)
        self.domain = tuple(float(v) for v in domain)
        self.cpml_layers = int(cpml_layers)
        self.kappa_max = float(kappa_max)
        self.pec_faces = set(pec_faces or ())
        self.cpml_axes = "".join(a for a in "xyz" if a in cpml_axes)
        self.face_layers = {f: self.cpml_layers for f in ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")}
        self.face_layers.update(face_layers or {})
        for f, n in self.face_layers.items():
            if n > self.cpml_layers:
                raise ValueError(f"face_layers[{f!r}]={n} exceeds cpml_layers={self.cpml_layers}")
        self.dx = float(dx) if dx is not None else (C0 / self.freq_max) / 20.0
        self.dt = float(self.dx / (C0 * np.sqrt(3.0)) * 0.99)

        def pad(axis, side):
            face = f"{axis}_{side}"
            if face in self.pec_faces or axis not in self.cpml_axes:
                return 0
            return int(self.face_layers.get(face, self.cpml_layers))

        self.pad_x_lo, self.pad_x_hi = pad("x", "lo"), pad("x", "hi")
        self.pad_y_lo, self.pad_y_hi = pad("y", "lo"), pad("y", "hi")
        self.pad_z_lo, self.pad_z_hi = pad("z", "lo"), pad("z", "hi")
        self.axis_pads = (self.pad_x_lo, self.pad_y_lo, self.pad_z_lo)
        self.face_pads = (self.pad_x_lo, self.pad_x_hi, self.pad_y_lo, self.pad_y_hi,
                          self.pad_z_lo, self.pad_z_hi)
        self.nx = int(np.ceil(self.domain[0] / self.dx)) + 1 + self.pad_x_lo + self.pad_x_hi
        self.ny = int(np.ceil(self.domain[1] / self.dx)) + 1 + self.pad_y_lo + self.pad_y_hi
        self.nz = int(np.ceil(self.domain[2] / self.dx)) + 1 + self.pad_z_lo + self.pad_z_hi
        self.shape = (self.nx, self.ny, self.nz)

    def position_to_index(self, pos):
        """rfx/grid.py:258-279."""
        i = int(round(pos[0] / self.dx)) + self.pad_x_lo
        j = int(round(pos[1] / self.dx)) + self.pad_y_lo
        k = int(round(pos[2] / self.dx)) + self.pad_z_lo
        if not (0 <= i < self.nx and 0 <= j < self.ny and 0 <= k < self.nz):
            raise ValueError(f"position {pos} maps to grid index ({i}, {j}, {k}), outside the grid shape "
                             f"{self.shape}. Check the position lies inside the simulation domain.")
        return (i, j, k)

    def __repr__(self):
        return f"Grid(shape={self.shape}, dx={self.dx:.4e} m, dt={self.dt:.4e} s)"


class NonUniformGrid(NamedTuple):
    """Graded grid (rfx/nonuniform.py:37-98)."""
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
    pad_x_lo: int = 0
    pad_x_hi: int = 0
    pad_y_lo: int = 0
    pad_y_hi: int = 0
    pad_z_lo: int = 0
    pad_z_hi: int = 0

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)


def _profile_to_inv_arrays(profile_full):
    """(inv_d_e, inv_d_h) in float32 (rfx/nonuniform.py:187-224)."""
    arr = np.asarray(profile_full, dtype=np.float32)
    inv_local = np.float32(1.0) / arr
    inv_mean = np.float32(2.0) / (arr[:-1] + arr[1:])
    inv_d_h = np.concatenate([inv_local[:-1], np.zeros(1, np.float32)])
    inv_d_e = np.concatenate([inv_local[:1], inv_mean])
    return inv_d_e, inv_d_h


def _pad_profile(profile, pad_lo, pad_hi):
    """rfx/nonuniform.py:101-127."""
    return np.concatenate([np.full(pad_lo, float(profile[0])), np.asarray(profile, np.float64),
                           np.full(pad_hi, float(profile[-1]))])


def _append_bounding_node(profile_full):
    """rfx/nonuniform.py:130-152: one duplicate boundary cell."""
    return np.concatenate([profile_full, profile_full[-1:]])


def make_nonuniform_grid(domain_xy, dz_profile, dx, cpml_layers=8, *, dx_profile=None, dy_profile=None,
                         pec_faces=None, cpml_axes="xyz") -> NonUniformGrid:
    """rfx/nonuniform.py:274-422 (concrete numpy branch)."""
    pec = set(pec_faces or ())

    def pad(axis, side):
        if f"{axis}_{side}" in pec or axis not in cpml_axes:
            return 0
        return int(cpml_layers)

    pads = [pad(a, s) for a in "xyz" for s in ("lo", "hi")]
    if dx_profile is None:
        dxp = np.full(int(round(domain_xy[0] / dx)), float(dx))
    else:
        dxp = np.asarray(dx_profile, np.float64)
        if abs(dxp[0] - dx) > 1e-12 or abs(dxp[-1] - dx) > 1e-12:
            raise ValueError("dx_profile boundary cells must equal dx (CPML cells use the boundary spacing)")
    if dy_profile is None:
        dyp = np.full(int(round(domain_xy[1] / dx)), float(dx))
        dy_b = float(dx)
    else:
        dyp = np.asarray(dy_profile, np.float64)
        dy_b = float(dyp[0])
        if abs(dyp[-1] - dy_b) > 1e-12:
            raise ValueError("dy_profile boundary cells must match each other")
    dx_full = _append_bounding_node(_pad_profile(dxp, pads[0], pads[1]))
    dy_full = _append_bounding_node(_pad_profile(dyp, pads[2], pads[3]))
    dz_full = _append_bounding_node(_pad_profile(np.asarray(dz_profile, np.float64), pads[4], pads[5]))
    dt = float(0.99 / (C0_NU * np.sqrt(1 / float(np.min(dx_full)) ** 2 + 1 / float(np.min(dy_full)) ** 2
                                       + 1 / float(np.min(dz_full)) ** 2)))
    ix, ixh = _profile_to_inv_arrays(dx_full)
    iy, iyh = _profile_to_inv_arrays(dy_full)
    iz, izh = _profile_to_inv_arrays(dz_full)
    return NonUniformGrid(
        nx=len(dx_full), ny=len(dy_full), nz=len(dz_full), dx=float(dx), dy=dy_b,
        dx_arr=dx_full.astype(np.float32), dy_arr=dy_full.astype(np.float32), dz=dz_full.astype(np.float32),
        dt=dt, cpml_layers=int(cpml_layers), inv_dx=ix, inv_dy=iy, inv_dz=iz,
        inv_dx_h=ixh, inv_dy_h=iyh, inv_dz_h=izh,
        pad_x_lo=pads[0], pad_x_hi=pads[1], pad_y_lo=pads[2], pad_y_hi=pads[3],
        pad_z_lo=pads[4], pad_z_hi=pads[5])


def face_pads(grid):
    """(x_lo, x_hi, y_lo, y_hi, z_lo, z_hi) pads of either grid type."""
    if hasattr(grid, "face_pads"):
        return tuple(int(v) for v in grid.face_pads)
    return tuple(int(getattr(grid, f"pad_{a}_{s}", 0) or 0) for a in "xyz" for s in ("lo", "hi"))


def spacing_tables(grid):
    """Inverse spacing tables (xe, xh, ye, yh, ze, zh) for the step kernel.

    Graded grids pass their own E/H tables (rfx/nonuniform.py:187-224); a
    uniform grid divides every difference by dx, including the last forward
    difference whose far neighbour is the zero pad (rfx/core/yee.py:121-128).
    """
    if isinstance(grid, NonUniformGrid) or hasattr(grid, "inv_dx_h"):
        return tuple(np.asarray(getattr(grid, n), np.float32) for n in
                     ("inv_dx", "inv_dx_h", "inv_dy", "inv_dy_h", "inv_dz", "inv_dz_h"))
    nx, ny, nz = grid.shape
    inv = np.float32(1.0) / np.float32(grid.dx)
    return (np.full(nx, inv, np.float32), np.full(nx, inv, np.float32),
            np.full(ny, inv, np.float32), np.full(ny, inv, np.float32),
            np.full(nz, inv, np.float32), np.full(nz, inv, np.float32))
