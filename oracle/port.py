"""Lumped-port scenario of the reference's golden S11 fixture -- TEST INFRASTRUCTURE.

Rebuilds ``Simulation(freq_max=10e9, domain=(0.02,)*3, dx=0.02/15,
boundary="cpml", cpml_layers=6)`` with one 50-ohm ``ez`` port at
(0.0093, 0.0093, 0.0093) driven by ``GaussianPulse(f0=5e9, bandwidth=0.9)``
and ``forward(port_s11_freqs=[3..7] GHz, n_steps=1200)``, as in
``tests/test_lumped_rlc_ad.py:138-152`` of the reference, whose output is the
fixture ``tests/fixtures/golden_forward_no_rlc_s11.npy``.

The forward lane runs CPML on all axes with no PEC pass
(rfx/api/_execute.py:1420-1421), folds the port impedance into sigma
(rfx/sources/sources.py:238-247), drives the port cell with
``cb/dx * pulse`` (rfx/simulation.py:296-314), samples V and I before source
injection with the time stamp ``n dt`` (rfx/simulation.py:1447, 1480-1500) and
forms ``S11 = (V + Z0 I)/(V - Z0 I)`` (rfx/probes/probes.py:1240-1274).
"""

from __future__ import annotations

import numpy as np

from .fdtd import make_uniform_grid, port_sigma, port_source_waveform

GOLDEN_FREQS = np.array([3.0, 4.0, 5.0, 6.0, 7.0]) * 1e9
GOLDEN_STEPS = 1200
Z0 = 50.0


def golden_port_scenario():
    """Grid, materials (with the sigma fold), port index and waveform."""
    grid = make_uniform_grid((0.02, 0.02, 0.02), 0.02 / 15, cpml_layers=6)
    shape = grid.shape
    eps_r = np.ones(shape, np.float32)
    sigma = np.zeros(shape, np.float32)
    mu_r = np.ones(shape, np.float32)
    idx = grid.position_to_index((0.0093, 0.0093, 0.0093))
    sp = port_sigma(grid.dx, grid.dx, grid.dx, Z0)
    sigma[idx] = sigma[idx] + np.float32(sp)
    wave = port_source_waveform(grid, idx, (eps_r, sigma, mu_r), GOLDEN_STEPS,
                                f0=5e9, bandwidth=0.9)
    return grid, (eps_r, sigma, mu_r), idx, wave


def vi_dft(vi, dt, freqs, dtype=np.complex64):
    """In-scan V/I DFT of rfx/simulation.py:1480-1500, summed in step order.

    ``vi`` is ``(n_steps, 2)`` pre-source samples.  With x64 off the reference's
    float64 casts are no-ops, so the phase is float32 ``exp(-j 2 pi f n dt) * dt``.
    """
    n_steps = vi.shape[0]
    f32 = dtype == np.complex64
    fr = np.asarray(freqs, np.float32 if f32 else np.float64)
    v_acc = np.zeros(len(fr), dtype)
    i_acc = np.zeros(len(fr), dtype)
    for n in range(n_steps):
        if f32:
            t = np.float32(n) * np.float32(dt)
            arg = (fr * np.float32(-2.0 * np.pi)) * t
            ph = (np.cos(arg) + 1j * np.sin(arg)).astype(np.complex64) * np.complex64(dt)
        else:
            t = n * dt
            arg = fr * (-2.0 * np.pi) * t
            ph = (np.cos(arg) + 1j * np.sin(arg)) * dt
        v_acc = v_acc + vi[n, 0] * ph
        i_acc = i_acc + vi[n, 1] * ph
    return v_acc, i_acc


def s11_from_vi(v_dft, i_dft, z0=Z0):
    """rfx/probes/probes.py:1240-1274."""
    denom = v_dft - z0 * i_dft
    safe = np.where(np.abs(denom) > 0.0, denom, np.ones_like(denom))
    return (v_dft + z0 * i_dft) / safe
