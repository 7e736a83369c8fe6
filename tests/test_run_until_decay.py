"""run_until_decay (rfx/simulation.py:2198-2700) on the CUDA path against the
oracle's restatement: the same stop step and probe traces within the parity
tolerance, for the absorbing-boundary energy stop and the closed-boundary
point-field stop.  The oracle side also runs on CPU as a check of the
restatement itself (the energy stop fires well before max_steps)."""

import numpy as np
import pytest

import oracle
from tests.scenarios import rel_l2

TOL = 1e-4


def _scene(boundary):
    dx = 1e-3
    g = oracle.make_uniform_grid((0.024, 0.020, 0.018), dx, cpml_layers=6 if boundary == "cpml" else 0,
                                 cpml_axes="xyz" if boundary == "cpml" else "")
    rng = np.random.default_rng(4)
    eps = np.ones(g.shape, np.float32)
    eps[8:16, 8:14, 8:12] = np.float32(rng.uniform(2.0, 4.0))
    sig = np.zeros(g.shape, np.float32)
    if boundary == "pec":
        sig[:] = np.float32(0.02)     # a lossy cavity, so the point field decays
    mats = (eps, sig, np.ones(g.shape, np.float32))
    src = (g.nx // 2 - 3, g.ny // 2, g.nz // 2)
    w = oracle.j_source_waveform(g, src, mats, 4000, f0=15e9, bandwidth=0.8)
    probes = [(g.nx // 2 + 4, g.ny // 2, g.nz // 2, "ez"), (g.nx // 2, g.ny // 2 + 3, g.nz // 2, "hy")]
    return g, mats, [(*src, "ez", w)], probes


KW = dict(decay_by=1e-3, check_interval=50, min_steps=100, max_steps=4000, decay_energy_consecutive=2)


def _oracle(boundary):
    g, mats, srcs, probes = _scene(boundary)
    mon = (g.nx // 2, g.ny // 2, g.nz // 2, "ez")
    return oracle.run_until_decay_uniform(g, mats, boundary=boundary, sources=srcs, probes=probes, monitor=mon, **KW)


@pytest.mark.slow
@pytest.mark.parametrize("boundary", ["cpml", "pec"])
def test_oracle_run_until_decay_stops(boundary):
    res, steps = _oracle(boundary)
    print(boundary, "oracle stopped after", steps, "steps")
    assert KW["min_steps"] <= steps < KW["max_steps"]
    assert (steps - 1) % KW["check_interval"] == 0
    assert res.time_series.shape[0] == steps


@pytest.mark.gpu
@pytest.mark.parametrize("boundary", ["cpml", "pec"])
def test_run_until_decay_matches_oracle(cuda, boundary):
    import rfx_b200
    g, mats, srcs, probes = _scene(boundary)
    res, steps = _oracle(boundary)
    pg = rfx_b200.Grid(freq_max=10e9, domain=(0.024, 0.020, 0.018), dx=1e-3,
                       cpml_layers=6 if boundary == "cpml" else 0, cpml_axes="xyz" if boundary == "cpml" else "")
    assert tuple(pg.shape) == tuple(g.shape)
    out = rfx_b200.run_until_decay(pg, rfx_b200.MaterialArrays(*mats), boundary=boundary,
                                   sources=[rfx_b200.SourceSpec(*s) for s in srcs],
                                   probes=[rfx_b200.ProbeSpec(*p) for p in probes], **KW)
    n = out.time_series.shape[0]
    print(boundary, "CUDA stopped after", n, "steps; oracle", steps)
    assert n == steps
    for p in range(len(probes)):
        e = rel_l2(out.time_series[:, p], res.time_series[:, p])
        print(boundary, "probe", p, "relL2", e)
        assert e < TOL


FLUX_BOX = ((0.004, 0.004, 0.004), (0.020, 0.016, 0.014))


def _oracle_flux():
    g, mats, srcs, probes = _scene("cpml")
    idx = [tuple(int(round(c / 1e-3)) + 6 for c in corner) for corner in FLUX_BOX]
    box = (idx[0][0], idx[1][0], idx[0][1], idx[1][1], idx[0][2], idx[1][2])
    return oracle.run_until_decay_uniform(g, mats, boundary="cpml", sources=srcs, probes=probes, flux_box=box,
                                          flux_env_checks=4, **KW)


@pytest.mark.slow
def test_oracle_radiated_flux_stop():
    """The radiated-flux stop (rfx/simulation.py:2513-2540, 2580-2600) fires
    on a check step after min_steps."""
    res, steps = _oracle_flux()
    print("oracle radiated-flux stop after", steps, "steps")
    assert KW["min_steps"] <= steps < KW["max_steps"]
    assert (steps - 1) % KW["check_interval"] == 0


@pytest.mark.gpu
def test_radiated_flux_stop_matches_oracle(cuda):
    import rfx_b200
    g, mats, srcs, probes = _scene("cpml")
    res, steps = _oracle_flux()
    pg = rfx_b200.Grid(freq_max=10e9, domain=(0.024, 0.020, 0.018), dx=1e-3, cpml_layers=6)
    out = rfx_b200.run_until_decay(pg, rfx_b200.MaterialArrays(*mats), boundary="cpml",
                                   sources=[rfx_b200.SourceSpec(*s) for s in srcs],
                                   probes=[rfx_b200.ProbeSpec(*p) for p in probes], radiated_flux_box=FLUX_BOX,
                                   flux_env_checks=4, **KW)
    n = out.time_series.shape[0]
    print("radiated-flux stop: CUDA after", n, "steps; oracle", steps)
    assert n == steps
    for p in range(len(probes)):
        assert rel_l2(out.time_series[:, p], res.time_series[:, p]) < TOL


# ---------------------------------------------------------------------------
# graded lane: rfx.nonuniform.run_nonuniform_until_decay (rfx/nonuniform.py:1988-2260)

GDZ = 1e-3 * np.array([1.0, 0.9, 0.75, 0.6, 0.5, 0.5, 0.6, 0.75, 0.9, 1.0, 1.0, 1.0, 0.8, 0.7, 0.8, 1.0])
GKW = dict(decay_by=1e-3, check_interval=50, min_steps=100, max_steps=3000, decay_energy_consecutive=2)
GFLUX_BOX = ((0.004, 0.004, 0.003), (0.018, 0.016, 0.010))


def _graded_scene():
    dx = 1e-3
    g = oracle.make_nonuniform_grid((0.022, 0.020), GDZ, dx, cpml_layers=6)
    eps = np.ones(g.shape, np.float32)
    eps[10:18, 9:15, 8:13] = np.float32(2.5)
    mats = (eps, np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    t = np.arange(GKW["max_steps"], dtype=np.float32) * np.float32(g.dt)
    w = (oracle.gaussian_pulse(t, 20e9, 0.8) * 50.0).astype(np.float32)
    src = [(g.nx // 2 - 2, g.ny // 2, g.nz // 2, "ez", w)]
    probes = [(g.nx // 2 + 3, g.ny // 2, g.nz // 2, "ez"), (g.nx // 2, g.ny // 2 + 2, g.nz // 2 - 1, "hx")]
    return g, mats, src, probes


def _product_graded_grid():
    import rfx_b200
    return rfx_b200.make_nonuniform_grid((0.022, 0.020), GDZ, 1e-3, cpml_layers=6)


def test_graded_position_to_index():
    """Nearest interior cell edge per axis plus the low pad
    (rfx/nonuniform.py:477-524); with uniform x/y cells it reduces to
    round(pos / dx) + pad, and on z it follows the graded edges."""
    from rfx_b200.nonuniform import position_to_index
    g = _product_graded_grid()
    assert position_to_index(g, (0.0, 0.0, 0.0)) == (6, 6, 6)
    assert position_to_index(g, (0.0104, 0.0196, 0.0)) == (6 + 10, 6 + 20, 6)
    edges = np.insert(np.cumsum(GDZ), 0, 0.0)
    for q in (3, 7, 12):
        assert position_to_index(g, (0.0, 0.0, edges[q] + 1e-6))[2] == 6 + q


def _oracle_graded(flux):
    g, mats, srcs, probes = _graded_scene()
    box = None
    if flux:
        from rfx_b200.nonuniform import position_to_index
        pg = _product_graded_grid()
        lo, hi = (position_to_index(pg, c) for c in GFLUX_BOX)
        box = (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])
    return oracle.run_until_decay_nonuniform(g, mats, sources=srcs, probes=probes, flux_box=box, **GKW)


@pytest.mark.slow
@pytest.mark.parametrize("flux", [False, True])
def test_oracle_graded_run_until_decay_stops(flux):
    res, steps, checks = _oracle_graded(flux)
    print("graded", "flux" if flux else "energy", "stop: oracle after", steps, "steps")
    assert GKW["min_steps"] <= steps < GKW["max_steps"]
    assert steps % GKW["check_interval"] == 0          # checks after k * interval steps
    assert res.time_series.shape[0] == steps
    if not flux:
        assert checks[-1][0] == steps and all(u >= 0 for _, u, _ in checks)
        assert all(u < GKW["decay_by"] * p for _, u, p in checks[-2:])


@pytest.mark.gpu
@pytest.mark.parametrize("flux", [False, True])
def test_graded_run_until_decay_matches_oracle(cuda, flux):
    import rfx_b200
    g, mats, srcs, probes = _graded_scene()
    res, steps, checks = _oracle_graded(flux)
    pg = _product_graded_grid()
    assert tuple(pg.shape) == tuple(g.shape)
    out = rfx_b200.run_nonuniform_until_decay(pg, rfx_b200.MaterialArrays(*mats), sources=srcs, probes=probes,
                                              radiated_flux_box=GFLUX_BOX if flux else None, **GKW)
    n = out["time_series"].shape[0]
    print("graded", "flux" if flux else "energy", "stop: CUDA after", n, "steps; oracle", steps)
    assert n == steps and out["state"].step == steps
    for p in range(len(probes)):
        assert rel_l2(out["time_series"][:, p], res.time_series[:, p]) < TOL
    if not flux:
        assert len(out["decay_checks"]) == len(checks)
        for (s1, u1, p1), (s2, u2, p2) in zip(out["decay_checks"], checks):
            assert s1 == s2 and abs(u1 - u2) <= 1e-3 * p2


def test_graded_run_until_decay_rejects_bad_arguments():
    """The reference's argument checks (rfx/nonuniform.py:2096-2100) and the
    features outside this path, raised before any device work."""
    import rfx_b200
    g, mats, srcs, probes = _graded_scene()
    pg = _product_graded_grid()
    m = rfx_b200.MaterialArrays(*mats)
    with pytest.raises(ValueError, match="check_interval"):
        rfx_b200.run_nonuniform_until_decay(pg, m, check_interval=0, sources=srcs)
    with pytest.raises(ValueError, match="max_steps"):
        rfx_b200.run_nonuniform_until_decay(pg, m, max_steps=0, sources=srcs)
    with pytest.raises(NotImplementedError):
        rfx_b200.run_nonuniform_until_decay(pg, m, debye=((1.0,), (1e-9,)), sources=srcs)


def test_static_remnant_advisory_on_cap_hit():
    """rfx/simulation.py:2145-2197: after an energy cap-hit, an interior
    energy that is almost all electric (a static source-charge remnant) draws
    the advisory warning; an equipartitioned (radiating) field does not."""
    import warnings

    import rfx_b200
    from rfx_b200.simulation import warn_static_remnant_cap_hit
    g = rfx_b200.Grid(freq_max=10e9, domain=(0.01, 0.01, 0.01), dx=1e-3, cpml_layers=4)
    shape = tuple(g.shape)
    mats = rfx_b200.MaterialArrays(np.ones(shape, np.float32), np.zeros(shape, np.float32), np.ones(shape, np.float32))
    rng = np.random.default_rng(0)
    e = [rng.standard_normal(shape).astype(np.float32) for _ in range(3)]
    eta = float(np.sqrt(rfx_b200.grid.MU_0 / rfx_b200.grid.EPS_0))
    static = e + [np.zeros(shape, np.float32)] * 3
    with pytest.warns(UserWarning, match="static charge remnant"):
        assert warn_static_remnant_cap_hit(static, mats, g)
    radiating = e + [(rng.standard_normal(shape) / eta).astype(np.float32) for _ in range(3)]
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        assert not warn_static_remnant_cap_hit(radiating, mats, g)
    # cells inside the CPML pads do not count
    pads_only = [np.zeros(shape, np.float32) for _ in range(6)]
    pads_only[0][0, 0, 0] = 1.0
    assert not warn_static_remnant_cap_hit(pads_only, mats, g)
