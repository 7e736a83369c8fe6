"""Source waveforms and source specs (host tables, float32).

  GaussianPulse          rfx/sources/sources.py:56-103
  make_source            rfx/simulation.py:197-236 (raw field add)
  make_j_source          rfx/simulation.py:239-293 (cb-normalised)
  make_port_source       rfx/simulation.py:296-314 (cb / d_parallel)
  make_current_source    rfx/nonuniform.py:588-691 (cb / dV, mixed primal/dual volume)
  port_sigma / setup_lumped_port  rfx/sources/sources.py:31-45, 238-247
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from .grid import EPS_0


@dataclass(frozen=True)
class GaussianPulse:
    """Differentiated Gaussian ``-2 A ((t-t0)/tau) exp(-((t-t0)/tau)^2)``."""
    f0: float
    bandwidth: float = 0.5
    amplitude: float = 1.0
    cutoff: float = 3.0

    @property
    def tau(self) -> float:
        return 1.0 / (self.f0 * self.bandwidth * math.pi)

    @property
    def t0(self) -> float:
        return self.cutoff * self.tau

    def __call__(self, t):
        """Evaluated in the dtype of ``t`` (float32 tables, as in the reference)."""
        t = np.asarray(t)
        arg = (t - self.t0) / self.tau
        return self.amplitude * (-2.0 * arg) * np.exp(-(arg ** 2))


class SourceSpec(NamedTuple):
    """Soft source: ``E_component[i, j, k] += waveform[n]`` (rfx/simulation.py:44-54)."""
    i: int
    j: int
    k: int
    component: str
    waveform: np.ndarray


class LumpedPort(NamedTuple):
    position: tuple
    component: str
    impedance: float
    excitation: object


def _times(n_steps, dt):
    """``jnp.arange(n_steps, dtype=float32) * dt``: a float32 product, as JAX
    computes it with x64 off (rfx/simulation.py:277)."""
    return np.arange(n_steps, dtype=np.float32) * float(dt)


def _cell_cb(materials, idx, dt):
    """cb at a cell in float32 (rfx/simulation.py:181-194)."""
    i, j, k = idx
    eps = np.float32(np.asarray(materials.eps_r)[i, j, k]) * EPS_0
    sig = np.float32(np.asarray(materials.sigma)[i, j, k])
    loss = sig * dt / (2.0 * eps)
    return np.float32((dt / eps) / (1.0 + loss))


def make_source(grid, position, component, waveform_fn, n_steps, materials=None):
    idx = grid.position_to_index(position)
    w = np.asarray(waveform_fn(_times(n_steps, grid.dt)), np.float32)
    return SourceSpec(idx[0], idx[1], idx[2], component, w)


def make_j_source(grid, position, component, waveform_fn, n_steps, materials):
    idx = grid.position_to_index(position)
    cb = _cell_cb(materials, idx, grid.dt)
    w = (cb * np.asarray(waveform_fn(_times(n_steps, grid.dt)))).astype(np.float32)
    return SourceSpec(idx[0], idx[1], idx[2], component, w)


def port_sigma(d_par, d_perp1, d_perp2, impedance):
    return d_par / (impedance * d_perp1 * d_perp2)


def setup_lumped_port(grid, port: LumpedPort, materials):
    """Fold the port impedance into sigma at the port cell (float32 add)."""
    idx = grid.position_to_index(port.position)
    d = float(grid.dx)
    sigma = np.array(np.asarray(materials.sigma), dtype=np.float32, copy=True)
    sigma[idx] = sigma[idx] + np.float32(port_sigma(d, d, d, port.impedance))
    return materials._replace(sigma=sigma)


def make_port_source(grid, port: LumpedPort, materials, n_steps):
    idx = grid.position_to_index(port.position)
    cb = _cell_cb(materials, idx, grid.dt)
    d_par = float(grid.dx)
    w = ((cb / d_par) * np.asarray(port.excitation(_times(n_steps, grid.dt)))).astype(np.float32)
    return SourceSpec(idx[0], idx[1], idx[2], port.component, w)


def make_current_source(grid, position_ijk, component, waveform_fn, n_steps, materials):
    """Graded-grid current source; returns the reference's tuple form
    ``(i, j, k, component, waveform)``."""
    i, j, k = position_ijk
    eps = float(np.asarray(materials.eps_r)[i, j, k]) * EPS_0
    sigma = float(np.asarray(materials.sigma)[i, j, k])
    loss = sigma * grid.dt / (2.0 * eps)
    cb = (grid.dt / eps) / (1.0 + loss)
    p_axis = {"ex": 0, "ey": 1, "ez": 2}[component]
    widths = []
    for a, (prof, ii) in enumerate(zip((grid.dx_arr, grid.dy_arr, grid.dz), (i, j, k))):
        prof = np.asarray(prof, np.float64)
        if a == p_axis:
            widths.append(float(prof[ii]))
        elif ii <= 0:
            widths.append(float(prof[0]))
        else:
            widths.append(float(0.5 * (prof[ii - 1] + prof[ii])))
    dV = widths[0] * widths[1] * widths[2]
    w = ((cb / dV) * np.asarray(waveform_fn(_times(n_steps, grid.dt)))).astype(np.float32)
    return (i, j, k, component, w)
