"""The reference's two gradient-ladder witnesses, rebuilt from their producer
scripts so that the oracle and the CUDA adjoint can be checked against the
reference's own ``jax.grad`` numbers (``tests/golden/ad_fd_ladder.json`` and
``tests/golden/per_cell_snr.json``, copied from the reference's
``tests/fixtures/gradient_dx_ladder/``).

Both scenes are ``Simulation(freq_max=10e9, domain=(L, 0.012, 0.012),
boundary="cpml", cpml_layers=8, dx=lambda/n)`` with one soft Ez source
``GaussianPulse(f0=8e9, bandwidth=0.9)`` and one Ez probe, run through
``Simulation.forward(eps_override=...)``; the objective is
``|sum_n ts[n] exp(-j 2 pi 8e9 n dt)|^2`` with float32 time stamps:

* ``slab`` (scripts/diagnostics/gradient_dx_ladder/run_ladder.py:133-163):
  L = 60 mm, source at x = 12 mm, probe at x = 48 mm, an eps_r slab over
  x in [30, 36) mm spanning the whole transverse extent, CPML pads included;
  one scalar degree of freedom (the slab's eps_r), whose derivative is the sum
  of dJ/d eps_r over the slab cells;
* ``block`` (scripts/diagnostics/gradient_dx_ladder/per_cell_snr.py:210-260):
  L = 30 mm, source at x = 6 mm, probe at x = 24 mm, an eps_r = 4 block over
  [13, 19) x [3, 9) x [3, 9) mm, per-cell degrees of freedom.

Simulation.forward with CPML on every axis runs no PEC pass
(rfx/api/_execute.py:1420-1421) and drives a zero-impedance source through
make_j_source (rfx/api/_execute.py:1041-1050, rfx/simulation.py:239-293).
"""

from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass

import numpy as np

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
C0_LADDER = 2.998e8          # the producers' own speed of light for lambda
FREQ_MAX = 10e9
F_OBJ = 8e9
LAMBDA = C0_LADDER / FREQ_MAX
CPML = 8
NUM_PERIODS = 20.0


@dataclass
class LadderScene:
    kind: str
    n: int                   # lambda / dx
    grid: object             # oracle grid
    n_steps: int
    src: tuple
    prb: tuple
    box: tuple               # (i0, i1, j0, j1, k0, k1) of the degrees of freedom
    dx: float
    domain: tuple

    def materials(self, eps_value):
        """(eps_r, sigma, mu_r) float32 with eps_value over the box."""
        eps = np.ones(self.grid.shape, np.float32)
        i0, i1, j0, j1, k0, k1 = self.box
        eps[i0:i1, j0:j1, k0:k1] = np.float32(eps_value)
        z = np.zeros(self.grid.shape, np.float32)
        return eps, z, np.ones(self.grid.shape, np.float32)

    def source_wave(self, mats):
        return oracle.j_source_waveform(self.grid, self.src, mats, self.n_steps, f0=F_OBJ, bandwidth=0.9)

    def phasor(self):
        """exp(-j 2 pi f t) with t = float32(n) * float32(dt), in complex64
        (the producers' jnp arithmetic with x64 off)."""
        t = np.arange(self.n_steps, dtype=np.float32) * np.float32(self.grid.dt)
        arg = np.float32(-2.0 * math.pi * F_OBJ) * t
        return (np.cos(arg) + 1j * np.sin(arg)).astype(np.complex64)

    def objective(self, ts):
        """J = |sum ts[n] p[n]|^2 and dJ/dts (float64)."""
        p = self.phasor().astype(np.complex128)
        a = np.sum(np.asarray(ts, np.float64) * p)
        return float(abs(a) ** 2), 2.0 * np.real(np.conj(a) * p)


def _index(grid, pos, dx):
    return tuple(int(round(pos[a] / dx)) + grid.pads[2 * a] for a in range(3))


def _range(grid, axis, lo, hi, dx):
    coord = (np.arange(grid.shape[axis]) - grid.pads[2 * axis]) * dx
    sel = np.flatnonzero((coord >= lo) & (coord < hi))
    return int(sel[0]), int(sel[-1]) + 1


def ladder_scene(kind, n):
    dx = LAMBDA / n
    dom_x = 60e-3 if kind == "slab" else 30e-3
    domain = (dom_x, 12e-3, 12e-3)
    g = oracle.make_uniform_grid(domain, dx, cpml_layers=CPML)
    n_steps = int(np.ceil(NUM_PERIODS * (1.0 / FREQ_MAX) / g.dt))
    yc = 6e-3
    if kind == "slab":
        src = _index(g, (12e-3, yc, yc), dx)
        prb = _index(g, (48e-3, yc, yc), dx)
        i0, i1 = _range(g, 0, 30e-3, 36e-3, dx)
        box = (i0, i1, 0, g.shape[1], 0, g.shape[2])
    else:
        src = _index(g, (6e-3, yc, yc), dx)
        prb = _index(g, (24e-3, yc, yc), dx)
        box = (*_range(g, 0, 13e-3, 19e-3, dx), *_range(g, 1, 3e-3, 9e-3, dx), *_range(g, 2, 3e-3, 9e-3, dx))
    return LadderScene(kind, n, g, n_steps, src, prb, box, dx, domain)


def slab_fixture():
    """Rungs of the reference's scalar-slab ladder (jax.grad and FD)."""
    return json.load(open(os.path.join(GOLDEN, "ad_fd_ladder.json")))["rungs"]


def block_fixture():
    """Rungs of the reference's per-cell block ladder (|jax.grad| per cell)."""
    return json.load(open(os.path.join(GOLDEN, "per_cell_snr.json")))["rungs"]


def oracle_forward_adjoint(sc, eps_value, dtype=np.float32):
    """Oracle J and dJ/d eps_r over the box at eps_value."""
    from oracle.adjoint import forward_adjoint
    mats = sc.materials(eps_value)
    w = sc.source_wave(mats)
    captured = {}

    def og(ts):
        J, g = sc.objective(ts[:, 0])
        captured["J"] = J
        return g[:, None]

    _, grad, _ = forward_adjoint(sc.grid, mats, sc.n_steps, boundary="cpml", pec_axes="",
                                 sources=[(*sc.src, "ez", w)], probes=[(*sc.prb, "ez")], box=sc.box,
                                 objective_grad=og, dtype=dtype)
    return captured["J"], grad


def oracle_J(sc, eps_value, dtype=np.float32):
    mats = sc.materials(eps_value)
    w = sc.source_wave(mats)
    r = oracle.run_uniform(sc.grid, mats, sc.n_steps, boundary="cpml", pec_axes="",
                           sources=[(*sc.src, "ez", w)], probes=[(*sc.prb, "ez")], dtype=dtype)
    return sc.objective(r.time_series[:, 0])[0]
