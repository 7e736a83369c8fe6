"""CPU tests of the oracle itself: pinned against the reference's golden
vector and restated physics gates of the reference's own test suite."""

import os

import numpy as np
import pytest

import oracle
from oracle.port import GOLDEN_FREQS, GOLDEN_STEPS, golden_port_scenario, s11_from_vi, vi_dft
from tests.scenarios import c1_readme, medium_uniform, rel_l2, small_nonuniform, small_uniform

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_reproduces_reference_golden_s11():
    """tests/test_lumped_rlc_ad.py:138-152 of the reference: S11 of a CPML-6
    lumped-port forward run equals golden_forward_no_rlc_s11.npy within
    rtol 1e-5, atol 1e-6."""
    golden = np.load(os.path.join(GOLDEN, "forward_no_rlc_s11.npy"))
    grid, mats, idx, wave = golden_port_scenario()
    assert grid.shape == (28, 28, 28) and idx == (13, 13, 13)
    r = oracle.run_uniform(grid, mats, GOLDEN_STEPS, boundary="cpml", pec_axes="",
                           sources=[(*idx, "ez", wave)], vi_ports=[(*idx, "ez")], dtype=np.float32)
    v, i = vi_dft(r.vi[:, 0, :], grid.dt, GOLDEN_FREQS)
    s11 = s11_from_vi(v, i)
    np.testing.assert_allclose(s11, golden, rtol=1e-5, atol=1e-6)


def test_grid_geometry_matches_reference_configs():
    """Shapes and dt quoted for the benchmark configurations (rfx/grid.py)."""
    g = oracle.make_uniform_grid((0.14, 0.06, 0.05), 2e-3, cpml_layers=8)
    assert g.shape == (87, 47, 42)
    assert abs(g.dt - 3.8131e-12) / 3.8131e-12 < 1e-4
    g2 = oracle.make_uniform_grid((0.256, 0.256, 0.256), 1e-3, cpml_layers=10)
    assert g2.shape == (277, 277, 277)
    g4 = oracle.make_uniform_grid((0.1, 0.06, 0.024), 0.5e-3, cpml_layers=10)
    assert g4.shape == (221, 141, 69)
    dz = np.full(96, 0.3e-3)
    g3 = oracle.make_nonuniform_grid((0.096, 0.096), dz, 0.5e-3, cpml_layers=12)
    assert g3.shape == (217, 217, 121)


def test_nonuniform_tables_collapse_on_uniform_profile():
    """rfx/nonuniform.py:207-212: on a uniform mesh both metrics are 1/d
    (inv_d_h ends in 0)."""
    e, h = oracle.profile_to_inv_arrays(np.full(10, 1e-3))
    np.testing.assert_allclose(e, 1e3, rtol=1e-6)
    np.testing.assert_allclose(h[:-1], 1e3, rtol=1e-6)
    assert h[-1] == 0.0


def test_cpml_profile_quirks():
    """rfx/boundaries/cpml.py:101-171: order 3, R=1e-15, alpha = 0.05 (1-rho)
    unscaled, the innermost layer has sigma = 0 and c = 0."""
    p = oracle.cpml_profile(8, 3.8e-12, 2e-3)
    assert p.sigma[-1] == 0.0 and p.c[-1] == 0.0
    assert np.all(np.diff(p.sigma) < 0)
    eta = np.sqrt(oracle.MU_0 / oracle.EPS_0)
    smax = -np.log(1e-15) * 4 / (2 * eta * 8 * 2e-3)
    assert abs(p.sigma[0] - smax) / smax < 1e-6
    assert abs(p.alpha[0]) < 1e-12 and abs(p.alpha[-1] - 0.05) < 1e-7


def _reflection_db(n_layers, n_steps=160):
    """Peak deviation of a CPML run from a clean free-space run whose walls are
    too far to echo within the window (tests/test_cpml.py:43-110, scaled)."""
    f0, freq_max = 2e9, 5e9
    dx = oracle.C0 / freq_max / 20.0
    dt = dx / (oracle.C0 * np.sqrt(3.0)) * 0.99
    ref_extent = 1.15 * n_steps * dt * oracle.C0
    gr = oracle.make_uniform_grid((ref_extent,) * 3, dx, cpml_layers=0)
    gc = oracle.make_uniform_grid((0.06,) * 3, dx, cpml_layers=n_layers)
    out = []
    for g, bnd in ((gr, "pec"), (gc, "cpml")):
        c = (g.nx // 2, g.ny // 2, g.nz // 2)
        w = oracle.gaussian_pulse(np.arange(n_steps, dtype=np.float32) * np.float32(g.dt), f0, 0.5)
        mats = tuple(np.full(g.shape, v, np.float32) for v in (1.0, 0.0, 1.0))
        r = oracle.run_uniform(g, mats, n_steps, boundary=bnd, pec_axes="xyz" if bnd == "pec" else "",
                               sources=[(*c, "ez", w.astype(np.float32))], probes=[(c[0] + 3, c[1], c[2], "ez")])
        out.append(r.time_series[:, 0].astype(np.float64))
    ref, cp = out
    return 20 * np.log10(np.max(np.abs(cp - ref)) / np.max(np.abs(ref)))


@pytest.mark.slow
def test_oracle_cpml_reflection_gate():
    """tests/test_cpml.py:130-184: an 8-layer CPML stays below -55 dB and a
    2-layer one does not."""
    assert _reflection_db(8) < -55
    assert _reflection_db(2) > _reflection_db(8)


def test_oracle_running_dft_matches_post_hoc_dft():
    """tests/test_dft_probes.py:20-72: the running DFT of a plane equals the
    post-hoc DFT of the probe series at the (n+1) dt time stamp."""
    sc = small_uniform(n_steps=200)
    i, j, k = 20, 18, 13
    sc.probes = [(i, j, k, "ez")]
    freqs = np.array([10e9, 15e9], np.float32)
    sc.dft = [(2, k, "ez", freqs)]
    r = sc.run_oracle(np.float64)
    ts = r.time_series[:, 0]
    t = (np.arange(sc.n_steps) + 1) * sc.ogrid.dt
    post = (ts[None, :] * np.exp(-2j * np.pi * freqs[:, None].astype(np.float64) * t[None, :])).sum(1) * sc.ogrid.dt
    run = r.dft_planes[0][:, i, j]
    np.testing.assert_allclose(np.abs(run), np.abs(post), rtol=1e-2)
    assert np.max(np.abs(np.angle(run / post))) < 0.1


def test_oracle_nonuniform_reduces_to_uniform():
    """tests/test_nonuniform_uniform_end_to_end_reduction.py: a graded grid with
    a constant profile reproduces the uniform lane away from the extra
    bounding node (same dt, sources, probes)."""
    dx = 1e-3
    n = 14
    gnu = oracle.make_nonuniform_grid((n * dx, n * dx), np.full(n, dx), dx, cpml_layers=0)
    gu = oracle.UniformGrid(gnu.nx, gnu.ny, gnu.nz, dx, gnu.dt, 0, (0,) * 6)
    mats = tuple(np.full(gnu.shape, v, np.float32) for v in (1.0, 0.0, 1.0))
    w = oracle.gaussian_pulse(np.arange(80, dtype=np.float32) * np.float32(gnu.dt), 60e9, 0.8).astype(np.float32)
    src = [(7, 7, 7, "ez", w)]
    prb = [(9, 7, 7, "ez"), (7, 9, 8, "ex")]
    a = oracle.run_nonuniform(gnu, mats, 80, sources=src, probes=prb, dtype=np.float64)
    b = oracle.run_uniform(gu, mats, 80, boundary="pec", pec_axes="xyz", sources=src, probes=prb, dtype=np.float64)
    # the graded lane zeroes the H term of the last (duplicate) cell; probes far
    # from that face agree until its influence arrives, up to the float32
    # rounding of the graded lane's 1/d tables
    assert rel_l2(a.time_series[:20], b.time_series[:20]) < 1e-6


@pytest.mark.parametrize("build", [small_uniform, small_nonuniform, medium_uniform])
def test_oracle_matches_committed_fixture(build):
    """The oracle is deterministic against its committed fixtures."""
    sc = build()
    ref = np.load(os.path.join(GOLDEN, f"oracle_{sc.name}.npz"))
    r = sc.run_oracle(np.float64)
    np.testing.assert_allclose(r.time_series, ref["ts_f64"], rtol=0, atol=0)
    for q, acc in enumerate(r.dft_planes):
        np.testing.assert_allclose(acc, ref[f"dft{q}_f64"], rtol=0, atol=0)


def test_oracle_fp32_vs_fp64_close():
    """FP32 drift of the restatement against its FP64 twin on the small
    scenarios stays far below the 1e-4 parity tolerance."""
    for build in (small_uniform, small_nonuniform, medium_uniform):
        ref = np.load(os.path.join(GOLDEN, f"oracle_{build().name}.npz"))
        assert rel_l2(ref["ts_f32"], ref["ts_f64"]) < 3e-5
