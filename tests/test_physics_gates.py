"""Physics gates of the reference's own test suite, restated on this path.

CPML energy decay (rfx tests/test_cpml.py:110-157): a differentiated-Gaussian
pulse (2 GHz, bandwidth 0.5) is injected into Ez at the centre of a 12 cm
vacuum cube with CPML 15 for 200 steps; 500 source-free steps later the
electromagnetic energy must have dropped by more than 20 dB.  Checked on the
oracle (CPU) and on the CUDA path (GPU), which must also agree with each
other on the two energies.
"""

import numpy as np
import pytest

import oracle

EPS_0 = 8.854187817e-12
MU_0 = 1.2566370614e-6
N_SRC, N_FREE = 200, 500


def _energy(f):
    return float(0.5 * EPS_0 * sum(np.sum(np.asarray(f[c], np.float64) ** 2) for c in ("ex", "ey", "ez")) +
                 0.5 * MU_0 * sum(np.sum(np.asarray(f[c], np.float64) ** 2) for c in ("hx", "hy", "hz")))


def _setup():
    dx = (299792458.0 / 3e9) / 20.0
    g = oracle.make_uniform_grid((0.12, 0.12, 0.12), dx, cpml_layers=15)
    c = (g.nx // 2, g.ny // 2, g.nz // 2)
    t = np.arange(N_SRC + N_FREE, dtype=np.float32) * np.float32(g.dt)
    w = oracle.gaussian_pulse(t, 2e9, 0.5).astype(np.float32)
    w[N_SRC:] = 0.0
    mats = (np.ones(g.shape, np.float32), np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    return g, c, w, mats, dx


def _oracle_energies():
    g, c, w, mats, _ = _setup()
    out = []
    for n in (N_SRC, N_SRC + N_FREE):
        r = oracle.run_uniform(g, mats, n, boundary="cpml", pec_axes="", sources=[(*c, "ez", w[:n])])
        out.append(_energy(r.state))
    return out


@pytest.mark.slow
def test_oracle_cpml_energy_decay():
    e0, e1 = _oracle_energies()
    db = 10 * np.log10(e1 / e0)
    print("oracle energy decay", db, "dB")
    assert db < -20


@pytest.mark.gpu
def test_cuda_cpml_energy_decay(cuda):
    import rfx_b200
    g, c, w, mats, dx = _setup()
    pg = rfx_b200.Grid(freq_max=3e9, domain=(0.12, 0.12, 0.12), cpml_layers=15)
    assert tuple(pg.shape) == tuple(g.shape)
    es = []
    for n in (N_SRC, N_SRC + N_FREE):
        r = rfx_b200.run(pg, rfx_b200.MaterialArrays(*mats), n, boundary="cpml", pec_axes="",
                         sources=[rfx_b200.SourceSpec(*c, "ez", w[:n])])
        es.append(_energy({k: getattr(r.state, k) for k in ("ex", "ey", "ez", "hx", "hy", "hz")}))
    db = 10 * np.log10(es[1] / es[0])
    ref = _oracle_energies()
    print("CUDA energy decay", db, "dB; energies", es, "oracle", ref)
    assert db < -20
    # energies agree with the oracle's float32 run to a small part of the
    # injected energy (the residual after absorption is 32 dB down, so its
    # own relative difference reflects float32 rounding of the CPML)
    assert abs(es[0] - ref[0]) <= 1e-4 * ref[0]
    assert abs(es[1] - ref[1]) <= 1e-5 * ref[0]
