"""CPML profiles (host setup, float64 arithmetic, float32 tables).

  _cpml_profile     rfx/boundaries/cpml.py:101-171
  init_cpml         rfx/boundaries/cpml.py:346-478
  per-face padding  rfx/boundaries/cpml.py:200-233 (no-op entries b=1, c=0, kappa=1)
  cell sizes        rfx/boundaries/cpml.py:174-197
"""

from __future__ import annotations

import numpy as np

from .engine import CPMLSetup
from .grid import EPS_0, MU_0, NonUniformGrid

FACES = ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")


def cpml_profile(n_layers, dt, dx, order=3, kappa_max=1.0, R_asymptotic=1e-15):
    """(sigma, kappa, alpha, b, c) as float32, computed in float64.

    Polynomial order 3, sigma_max = -ln(R) (m+1) / (2 eta d) scaled by
    kappa_max, alpha = 0.05 (1 - rho) (not scaled by eps0),
    b = exp(-(sigma/kappa + alpha) dt / eps0), c = sigma (b-1) / (sigma kappa + kappa^2 alpha).
    """
    eta = float(np.sqrt(MU_0 / EPS_0))
    d = n_layers * dx
    sigma_max = -float(np.log(R_asymptotic)) * (order + 1) / (2.0 * eta * d) * kappa_max
    rho = 1.0 - np.arange(n_layers, dtype=np.float64) / max(n_layers - 1, 1)
    sigma = sigma_max * rho ** order
    kappa = 1.0 + (kappa_max - 1.0) * rho ** order
    alpha = 0.05 * (1.0 - rho)
    denom = sigma * kappa + kappa ** 2 * alpha
    b = np.exp(-(sigma / kappa + alpha) * dt / EPS_0)
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.where(denom > 1e-30, sigma * (b - 1.0) / denom, 0.0)
    f = np.float32
    return sigma.astype(f), kappa.astype(f), alpha.astype(f), b.astype(f), c.astype(f)


def boundary_cell_sizes(grid):
    """(dx, dy, dz_lo, dz_hi) of the CPML faces (rfx/boundaries/cpml.py:174-197)."""
    dx = float(grid.dx)
    dy = float(getattr(grid, "dy", dx))
    dz = getattr(grid, "dz", None)
    if dz is not None and np.ndim(dz) > 0 and len(dz) > 0:
        return dx, dy, float(dz[0]), float(dz[-1])
    return dx, dy, dx, dx


def build_cpml(grid, axes="xyz", kappa_max=None, noop_faces=()) -> CPMLSetup | None:
    """Per-face tables for the kernel; hi faces pre-flipped.

    ``axes`` are the absorbing axes of the run; faces in ``noop_faces`` (PEC
    or PMC faces) get the identity profile, as in init_cpml.
    """
    n = int(grid.cpml_layers)
    if n <= 0 or not axes:
        return None
    if kappa_max is None:
        kappa_max = getattr(grid, "kappa_max", None) or 1.0
    face_layers = getattr(grid, "face_layers", None) or {f: n for f in FACES}
    dx, dy, dz_lo, dz_hi = boundary_cell_sizes(grid)
    sizes = {"x_lo": dx, "x_hi": dx, "y_lo": dy, "y_hi": dy, "z_lo": dz_lo, "z_hi": dz_hi}
    b = np.ones((6, n), np.float32)
    c = np.zeros((6, n), np.float32)
    k = np.ones((6, n), np.float32)
    for f, face in enumerate(FACES):
        if face in noop_faces:
            continue
        na = int(face_layers.get(face, n))
        _, kap, _, bb, cc = cpml_profile(na, grid.dt, sizes[face], kappa_max=kappa_max)
        if face.endswith("lo"):
            b[f, :na], c[f, :na], k[f, :na] = bb, cc, kap
        else:
            b[f, n - na:], c[f, n - na:], k[f, n - na:] = bb[::-1], cc[::-1], kap[::-1]
    return CPMLSetup(layers=n, axes="".join(a for a in "xyz" if a in axes), b=b, c=c, kappa=k,
                     cell=tuple(sizes[f] for f in FACES))
