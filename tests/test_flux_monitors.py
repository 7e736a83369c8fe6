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


def _graded_scene(n_steps=220):
    dz = np.concatenate([np.full(6, 1e-3), np.linspace(1e-3, 0.5e-3, 6), np.full(8, 0.5e-3)])
    g = oracle.make_nonuniform_grid((0.014, 0.012), dz, 1e-3, cpml_layers=4)
    eps = np.ones(g.shape, np.float32)
    eps[:, :, 10:14] = 2.5
    mats = (eps, np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    src = (g.nx // 2, g.ny // 2, 8)
    w = oracle.current_source_waveform(g, src, "ez", mats, n_steps, f0=40e9, bandwidth=0.8)
    f = np.array([30e9, 45e9])
    mons = [(2, 14, 4, g.nx - 4, 4, g.ny - 4, f, 0, "rect", 0.25),
            (0, g.nx // 2 + 3, 3, g.ny - 3, 3, g.nz - 3, f[:1], n_steps, "tukey", 0.25)]
    return g, mats, [(*src, "ez", w)], mons, dz


def test_oracle_graded_flux_matches_post_hoc_dft():
    """The graded lane samples at t = f32(n) * dt rounded to float32 (E) and
    half a step earlier (H), with the window weight of step n
    (rfx/nonuniform.py:1483-1520)."""
    g, mats, srcs, mons, _ = _graded_scene()
    m = mons[0]
    axis, index, lo1, lo2, freqs = m[0], m[1], m[2], m[4], m[6]
    a, b = lo1 + 4, lo2 + 3
    probes = [(a, b, index, "ex"), (a, b, index, "ey"), (a, b, index - 1, "hx"), (a, b, index, "hx"),
              (a, b, index - 1, "hy"), (a, b, index, "hy")]
    n = 200
    r = oracle.run_nonuniform(g, mats, n, sources=srcs, probes=probes, flux_monitors=[m])
    ts = r.time_series
    t = (np.arange(n, dtype=np.float32) * np.float32(g.dt)).astype(np.float64)
    ke = np.exp(-1j * 2 * np.pi * freqs[:, None] * t[None, :]) * g.dt
    kh = np.exp(-1j * 2 * np.pi * freqs[:, None] * (t[None, :] - g.dt / 2)) * g.dt
    h1 = ((ts[:, 2] + ts[:, 3]) * np.float32(0.5)).astype(np.float64)
    h2 = ((ts[:, 4] + ts[:, 5]) * np.float32(0.5)).astype(np.float64)
    for slot, series, k in ((0, ts[:, 0].astype(np.float64), ke), (1, ts[:, 1].astype(np.float64), ke),
                            (2, h1, kh), (3, h2, kh)):
        post = k @ series
        got = r.flux[0][slot][:, a - lo1, b - lo2]
        assert np.allclose(got, post, rtol=1e-10, atol=1e-12 * np.abs(post).max()), slot


@pytest.mark.gpu
def test_graded_flux_monitors_match_oracle(cuda):
    import rfx_b200
    g, mats, srcs, mons, dz = _graded_scene()
    n = 220
    ref = oracle.run_nonuniform(g, mats, n, sources=srcs, flux_monitors=mons)
    pg = rfx_b200.make_nonuniform_grid((0.014, 0.012), dz, 1e-3, cpml_layers=4)
    assert tuple(pg.shape) == tuple(g.shape)
    fms = [rfx_b200.init_flux_monitor(m[0], m[1], m[6], pg.shape, pg.dx, pg.dx, dft_total_steps=m[7],
                                      dft_window=m[8], dft_window_alpha=m[9], lo1=m[2], hi1=m[3], lo2=m[4], hi2=m[5])
           for m in mons]
    out = rfx_b200.run_nonuniform(pg, rfx_b200.MaterialArrays(*mats), n, sources=srcs, flux_monitors=fms)
    assert len(out["flux_monitors"]) == len(mons)
    for q, (fm, acc) in enumerate(zip(out["flux_monitors"], ref.flux)):
        got = np.stack([fm.e1_dft, fm.e2_dft, fm.h1_dft, fm.h2_dft])
        e = np.linalg.norm(got - acc) / np.linalg.norm(acc)
        sp = rfx_b200.flux_spectrum(fm)
        sp_ref = rfx_b200.flux_spectrum(fm._replace(e1_dft=acc[0], e2_dft=acc[1], h1_dft=acc[2], h2_dft=acc[3]))
        print("graded monitor", q, "relL2", e, "flux", sp, "oracle", sp_ref)
        assert e < 1e-4
        assert np.allclose(sp, sp_ref, rtol=1e-3, atol=1e-3 * np.abs(sp_ref).max())


@pytest.mark.gpu
def test_run_until_decay_flux_matches_a_plain_run(cuda):
    """run_until_decay replays check intervals from the flux kernel tables at
    their step offset: the monitors equal those of a plain run of the same
    length."""
    import rfx_b200
    g, mats, srcs, mons = _scene()
    long = 900
    pg = rfx_b200.Grid(freq_max=10e9, domain=(0.030, 0.022, 0.020), dx=1e-3, cpml_layers=6)
    sl = [rfx_b200.SourceSpec(*s[:4], np.concatenate([s[4], np.zeros(long - len(s[4]), np.float32)])) for s in srcs]
    fms = [rfx_b200.init_flux_monitor(m[0], m[1], m[6], pg.shape, pg.dx, pg.dx, lo1=m[2], hi1=m[3], lo2=m[4],
                                      hi2=m[5]) for m in mons[:2]]
    m = rfx_b200.MaterialArrays(*mats)
    r1 = rfx_b200.run_until_decay(pg, m, decay_by=1e-2, check_interval=40, min_steps=80, max_steps=long,
                                  boundary="cpml", pec_axes="", sources=sl, flux_monitors=fms)
    steps = int(r1.state.step)
    assert steps < long
    r2 = rfx_b200.run(pg, m, steps, boundary="cpml", pec_axes="", sources=sl, flux_monitors=fms)
    for a, b in zip(r1.flux_monitors, r2.flux_monitors):
        for name in ("e1_dft", "e2_dft", "h1_dft", "h2_dft"):
            x, y = getattr(a, name), getattr(b, name)
            assert np.linalg.norm(x - y) <= 1e-6 * np.linalg.norm(y), name
