"""Physics gates of the reference's own test suite, restated on this path.

CPML energy decay (rfx tests/test_cpml.py:110-157): a differentiated-Gaussian
pulse (2 GHz, bandwidth 0.5) is injected into Ez at the centre of a 12 cm
vacuum cube with CPML 15 for 200 steps; 500 source-free steps later the
electromagnetic energy must have dropped by more than 20 dB.  Checked on the
oracle (CPU) and on the CUDA path (GPU), which must also agree with each
other on the two energies.

Numerical dispersion (rfx tests/test_numerical_dispersion_oracle.py:60-78):
the reference measures the phase velocity of a TFSF plane wave (a source
outside this path) and requires it to follow the analytic Yee dispersion
relation within 0.3 % while the Yee value itself lies more than 0.3 % below
the continuum.  Restated with this path's own features: the resonance of
the lowest x-uniform Ex mode of a PEC cavity (2 x 9 x 7 cells at 1 mm, a
short soft-source pulse, one probe, 8192 steps) obeys the discrete Yee
relation sin(w dt / 2) = c dt sqrt(sum sin^2(k dx / 2) / dx^2) with
k = pi / ((n - 1) dx) exactly; it is measured from the probe spectrum (Hann
window, parabolic peak interpolation) and gated like the reference: within
0.3 % of Yee, and Yee as well as the measurement more than 0.3 % below the
continuum value (0.38 % here, the discriminating part).
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


C0 = 299792458.0
CAV = (9, 7)          # (ny, nz): PEC cavity of 8 x 6 cells across y, z
CAV_DX = 1e-3
CAV_STEPS = 8192


def _cavity_inputs():
    ny, nz = CAV
    g = oracle.make_uniform_grid((CAV_DX, (ny - 1) * CAV_DX, (nz - 1) * CAV_DX), CAV_DX, cpml_layers=0)
    n = np.arange(CAV_STEPS)
    w = np.exp(-((n - 30) / 6.0) ** 2).astype(np.float32)
    mats = (np.ones(g.shape, np.float32), np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    return g, w, mats


def _cavity_frequencies(dt):
    ny, nz = CAV
    ky, kz = np.pi / ((ny - 1) * CAV_DX), np.pi / ((nz - 1) * CAV_DX)
    s = C0 * dt * np.sqrt(np.sin(ky * CAV_DX / 2) ** 2 + np.sin(kz * CAV_DX / 2) ** 2) / CAV_DX
    return np.arcsin(s) / (np.pi * dt), C0 / (2 * np.pi) * np.hypot(ky, kz)


def _peak_frequency(x, dt, f_guess):
    x = np.asarray(x, np.float64)[200:]       # free oscillation after the pulse
    pad = 16 * len(x)
    X = np.abs(np.fft.rfft(x * np.hanning(len(x)), n=pad))
    f = np.fft.rfftfreq(pad, dt)
    k0 = int(np.argmax(np.where((f > 0.9 * f_guess) & (f < 1.1 * f_guess), X, 0.0)))
    a, b, c = np.log(X[k0 - 1:k0 + 2])
    return (k0 + 0.5 * (a - c) / (a - 2 * b + c)) * (f[1] - f[0])


def _dispersion_gate(f_meas, dt, label):
    f_yee, f_cont = _cavity_frequencies(dt)
    print(f"{label}: resonance {f_meas / 1e9:.6f} GHz, Yee {f_yee / 1e9:.6f}, continuum {f_cont / 1e9:.6f}; "
          f"vs Yee {(f_meas - f_yee) / f_yee:.2e}, below continuum {1 - f_meas / f_cont:.2e}")
    assert f_yee < f_cont * (1 - 3e-3)                  # the Yee deficit is real at this resolution
    assert abs(f_meas - f_yee) / f_yee < 3e-3           # the step obeys its own discrete dispersion
    assert f_meas < f_cont * (1 - 3e-3)                 # and is not dispersion-free


def test_oracle_cavity_resonance_follows_yee_dispersion():
    g, w, mats = _cavity_inputs()
    r = oracle.run_uniform(g, mats, CAV_STEPS, boundary="pec", sources=[(0, 3, 2, "ex", w)],
                           probes=[(0, 5, 4, "ex")], dtype=np.float32)
    f_yee, _ = _cavity_frequencies(g.dt)
    f = _peak_frequency(r.time_series[:, 0], g.dt, f_yee)
    _dispersion_gate(f, g.dt, "oracle")
    assert abs(f - f_yee) / f_yee < 1e-6


@pytest.mark.gpu
def test_cuda_cavity_resonance_follows_yee_dispersion(cuda):
    import rfx_b200
    g, w, mats = _cavity_inputs()
    ny, nz = CAV
    pg = rfx_b200.Grid(freq_max=10e9, domain=(CAV_DX, (ny - 1) * CAV_DX, (nz - 1) * CAV_DX), dx=CAV_DX,
                       cpml_layers=0)
    assert tuple(pg.shape) == tuple(g.shape) and pg.dt == g.dt
    r = rfx_b200.run(pg, rfx_b200.MaterialArrays(*mats), CAV_STEPS, boundary="pec",
                     sources=[rfx_b200.SourceSpec(0, 3, 2, "ex", w)], probes=[rfx_b200.ProbeSpec(0, 5, 4, "ex")])
    f_yee, _ = _cavity_frequencies(g.dt)
    f = _peak_frequency(np.asarray(r.time_series)[:, 0], g.dt, f_yee)
    _dispersion_gate(f, g.dt, "CUDA")
    assert abs(f - f_yee) / f_yee < 1e-6
