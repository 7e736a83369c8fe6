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
