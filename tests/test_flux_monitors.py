"""Poynting-flux monitors (rfx/probes/probes.py:476-680, accumulated as in
rfx/simulation.py:1590-1642): the oracle's running accumulators against a
post-hoc DFT of probe series, and the CUDA path against the oracle
(complex128 accumulators of the float32 fields, relative L2 below 1e-4),
including Tukey- and Hann-windowed monitors."""

import numpy as np
import pytest

import oracle
from tests.scenarios import rel_l2

TOL = 1e-4


def _scene(n_steps=260):
    dx = 1e-3
    g = oracle.make_uniform_grid((0.030, 0.022, 0.020), dx, cpml_layers=6)
    eps = np.ones(g.shape, np.float32)
    sig = np.zeros(g.shape, np.float32)
    mats = (eps, sig, np.ones(g.shape, np.float32))
    src = (12, g.ny // 2, g.nz // 2)
    w = oracle.j_source_waveform(g, src, mats, n_steps, f0=12e9, bandwidth=0.8)
    freqs = np.array([8e9, 12e9, 16e9])
    # (axis, index, lo1, hi1, lo2, hi2, freqs, total_steps, window, alpha)
    mons = [(0, 20, 8, g.ny - 8, 8, g.nz - 8, freqs, 0, "rect", 0.25),
            (0, 28, 8, g.ny - 8, 8, g.nz - 8, freqs, 0, "rect", 0.25),
            (2, g.nz // 2 + 3, 7, g.nx - 7, 7, g.ny - 7, freqs, n_steps, "tukey", 0.25),
            (1, g.ny // 2, 0, g.nx, 0, g.nz, freqs[:2], n_steps, "hann", 0.25)]
    return g, mats, [(*src, "ez", w)], mons


def test_oracle_flux_matches_post_hoc_dft():
    """The oracle's running flux accumulators equal a post-hoc DFT of probe
    series at the same cells (E at the plane, H averaged over the plane and
    the one before), with E sampled at (n+1) dt and H half a step earlier."""
    g, mats, srcs, mons = _scene()
    m = mons[0]
    axis, index, lo1, lo2, freqs = m[0], m[1], m[2], m[4], m[6]
    cells = [(lo1 + 3, lo2 + 5), (lo1 + 9, lo2 + 2)]
    probes = []
    for (a, b) in cells:
        probes += [(index, a, b, "ey"), (index, a, b, "ez"), (index - 1, a, b, "hy"), (index, a, b, "hy"),
                   (index - 1, a, b, "hz"), (index, a, b, "hz")]
    r = oracle.run_uniform(g, mats, 260, boundary="cpml", pec_axes="", sources=srcs, probes=probes,
                           flux_monitors=[m])
    ts = r.time_series.astype(np.float64)
    t = np.arange(1, 261) * g.dt
    ke = np.exp(-1j * 2 * np.pi * freqs[:, None] * t[None, :]) * g.dt
    kh = np.exp(-1j * 2 * np.pi * freqs[:, None] * (t[None, :] - g.dt / 2)) * g.dt
    acc = r.flux[0]
    for c, (a, b) in enumerate(cells):
        q = ts[:, 6 * c:6 * c + 6]
        h1 = ((r.time_series[:, 6 * c + 2] + r.time_series[:, 6 * c + 3]) * np.float32(0.5)).astype(np.float64)
        h2 = ((r.time_series[:, 6 * c + 4] + r.time_series[:, 6 * c + 5]) * np.float32(0.5)).astype(np.float64)
        for name, series, k, slot in (("e1", q[:, 0], ke, 0), ("e2", q[:, 1], ke, 1), ("h1", h1, kh, 2),
                                      ("h2", h2, kh, 3)):
            post = k @ series
            got = acc[slot][:, a - lo1, b - lo2]
            assert np.allclose(got, post, rtol=1e-10, atol=1e-12 * np.abs(post).max()), name


@pytest.mark.gpu
def test_flux_monitors_match_oracle(cuda):
    import rfx_b200
    g, mats, srcs, mons = _scene()
    ref = oracle.run_uniform(g, mats, 260, boundary="cpml", pec_axes="", sources=srcs, flux_monitors=mons)
    pg = rfx_b200.Grid(freq_max=10e9, domain=(0.030, 0.022, 0.020), dx=1e-3, cpml_layers=6)
    fms = [rfx_b200.init_flux_monitor(m[0], m[1], m[6], pg.shape, pg.dx, pg.dx, dft_total_steps=m[7],
                                      dft_window=m[8], dft_window_alpha=m[9], lo1=m[2], hi1=m[3], lo2=m[4], hi2=m[5])
           for m in mons]
    r = rfx_b200.run(pg, rfx_b200.MaterialArrays(*mats), 260, boundary="cpml", pec_axes="",
                     sources=[rfx_b200.SourceSpec(*s) for s in srcs], flux_monitors=fms)
    assert len(r.flux_monitors) == len(mons)
    errs = []
    for q, (fm, acc) in enumerate(zip(r.flux_monitors, ref.flux)):
        # the tangential E pair and H pair are compared jointly: with an Ez
        # source one member of each pair is orders of magnitude smaller
        # (numerical noise) and carries no meaning on its own
        for name, a, b in (("E", np.stack([fm.e1_dft, fm.e2_dft]), acc[:2]),
                           ("H", np.stack([fm.h1_dft, fm.h2_dft]), acc[2:])):
            e = rel_l2(a, b)
            print("monitor", q, name, "relL2", e)
            errs.append(e)
        sp = rfx_b200.flux_spectrum(fm)
        sp_ref = rfx_b200.flux_spectrum(fm._replace(e1_dft=acc[0], e2_dft=acc[1], h1_dft=acc[2], h2_dft=acc[3]))
        print("monitor", q, "flux", sp, "oracle", sp_ref)
        errs.append(rel_l2(sp, sp_ref) / 10)
    assert max(errs) < TOL
