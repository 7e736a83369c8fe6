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


def _cuda_reflection_db(n_layers, n_steps=160):
    """The CPML reflection measurement of the oracle gate
    (tests/test_cpml.py:43-110 as restated in tests/test_oracle.py) through
    ``rfx_b200.run``: peak deviation of an n-layer CPML run from a free-space
    run whose PEC walls are too far to echo within the window."""
    import rfx_b200
    f0, freq_max = 2e9, 5e9
    dx = oracle.C0 / freq_max / 20.0
    dt = dx / (oracle.C0 * np.sqrt(3.0)) * 0.99
    ref_extent = 1.15 * n_steps * dt * oracle.C0
    out = []
    for extent, layers, bnd in ((ref_extent, 0, "pec"), (0.06, n_layers, "cpml")):
        og = oracle.make_uniform_grid((extent,) * 3, dx, cpml_layers=layers)
        g = rfx_b200.Grid(freq_max=freq_max, domain=(extent,) * 3, dx=dx, cpml_layers=layers)
        assert tuple(g.shape) == tuple(og.shape)
        c = (g.nx // 2, g.ny // 2, g.nz // 2)
        w = oracle.gaussian_pulse(np.arange(n_steps, dtype=np.float32) * np.float32(og.dt), f0, 0.5)
        mats = rfx_b200.MaterialArrays(*(np.full(g.shape, v, np.float32) for v in (1.0, 0.0, 1.0)))
        r = rfx_b200.run(g, mats, n_steps, boundary=bnd, pec_axes="xyz" if bnd == "pec" else "",
                         sources=[rfx_b200.SourceSpec(*c, "ez", w.astype(np.float32))],
                         probes=[rfx_b200.ProbeSpec(c[0] + 3, c[1], c[2], "ez")])
        out.append(np.asarray(r.time_series)[:, 0].astype(np.float64))
    ref, cp = out
    return 20 * np.log10(np.max(np.abs(cp - ref)) / np.max(np.abs(ref)))


@pytest.mark.gpu
def test_cuda_cpml_reflection_gate(cuda):
    """tests/test_cpml.py:130-184 on the CUDA path: an 8-layer CPML stays
    below -55 dB and a 2-layer one reflects more."""
    db8, db2 = _cuda_reflection_db(8), _cuda_reflection_db(2)
    print(f"CUDA CPML reflection: 8 layers {db8:.1f} dB, 2 layers {db2:.1f} dB")
    assert db8 < -55
    assert db2 > db8


@pytest.mark.gpu
def test_cuda_nonuniform_reduces_to_uniform(cuda):
    """tests/test_nonuniform_uniform_end_to_end_reduction.py on the CUDA path:
    a graded grid with a constant profile reproduces the uniform lane (PEC
    faces, same dt, sources and probes) until the graded lane's extra
    bounding cell can influence the probes."""
    import rfx_b200
    dx, n, steps = 1e-3, 14, 80
    gnu = rfx_b200.make_nonuniform_grid((n * dx, n * dx), np.full(n, dx), dx, cpml_layers=0)
    nx, ny, nz = (int(v) for v in gnu.shape)
    gu = rfx_b200.Grid(freq_max=10e9, domain=((nx - 1) * dx, (ny - 1) * dx, (nz - 1) * dx), dx=dx, cpml_layers=0)
    assert tuple(gu.shape) == (nx, ny, nz) and abs(gu.dt - gnu.dt) <= 1e-9 * gnu.dt
    mats = rfx_b200.MaterialArrays(*(np.full((nx, ny, nz), v, np.float32) for v in (1.0, 0.0, 1.0)))
    w = oracle.gaussian_pulse(np.arange(steps, dtype=np.float32) * np.float32(gnu.dt), 60e9, 0.8).astype(np.float32)
    prb = [(9, 7, 7, "ez"), (7, 9, 8, "ex")]
    a = rfx_b200.run_nonuniform(gnu, mats, steps, sources=[(7, 7, 7, "ez", w)], probes=prb)["time_series"]
    b = rfx_b200.run(gu, mats, steps, boundary="pec", pec_axes="xyz", sources=[rfx_b200.SourceSpec(7, 7, 7, "ez", w)],
                     probes=[rfx_b200.ProbeSpec(*p) for p in prb]).time_series
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    e = float(np.linalg.norm(a[:20] - b[:20]) / np.linalg.norm(b[:20]))
    print(f"CUDA graded-to-uniform reduction, first 20 steps: relL2 {e:.2e}")
    assert e < 1e-5 and np.abs(b[:20]).max() > 0


# Graded lane: the same x-uniform Ex cavity mode with a graded z spacing.  Its
# discrete frequency follows from the eigenvalues of the graded second
# difference the lane applies: with the H metric ih[k] = 1/d[k] and the E
# metric ie[k] = 2/(d[k-1] + d[k]) of rfx/nonuniform.py:187-224,
#   (A_z e)[k] = -ie[k] (ih[k] (e[k+1] - e[k]) - ih[k-1] (e[k] - e[k-1])),
# e = 0 on the PEC faces, and the leapfrog gives
#   sin^2(w dt / 2) = dt^2 / (eps0 mu0) (lambda_y + lambda_z) / 4,
# lambda_y = (2 / dy)^2 sin^2(pi / (2 (ny - 1))), lambda_z the lowest
# eigenvalue of A_z.  Nothing here comes from the time stepping itself, so a
# grading error in either lane moves the measured resonance off it.
GCAV_NYI = 8
GCAV_DZ = 0.4e-3 * 1.15 ** np.arange(9)     # 0.40 .. 1.22 mm, adjacent ratio 1.15


def _graded_cavity_inputs():
    g = oracle.make_nonuniform_grid((CAV_DX, GCAV_NYI * CAV_DX), GCAV_DZ, CAV_DX, cpml_layers=0)
    n = np.arange(CAV_STEPS)
    w = np.exp(-((n - 30) / 6.0) ** 2).astype(np.float32)
    mats = (np.ones(g.shape, np.float32), np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    return g, w, mats


def _graded_cavity_frequency(g):
    from oracle.fdtd import EPS_0 as E0, MU_0 as M0
    ie = np.asarray(g.inv_dz, np.float64)
    ih = np.asarray(g.inv_dz_h, np.float64)
    nz = g.nz
    m = nz - 2                                   # interior E nodes k = 1 .. nz-2
    A = np.zeros((m, m))
    for r, k in enumerate(range(1, nz - 1)):
        A[r, r] = ie[k] * (ih[k] + ih[k - 1])
        if k + 1 <= nz - 2:
            A[r, r + 1] = -ie[k] * ih[k]
        if k - 1 >= 1:
            A[r, r - 1] = -ie[k] * ih[k - 1]
    lam_z = float(np.min(np.real(np.linalg.eigvals(A))))
    ny = g.ny
    lam_y = (2.0 / float(g.dy) * np.sin(np.pi / (2 * (ny - 1)))) ** 2
    s = g.dt * np.sqrt((lam_y + lam_z) / (E0 * M0)) / 2.0
    return np.arcsin(s) / (np.pi * g.dt)


def test_oracle_graded_cavity_resonance_matches_graded_operator():
    g, w, mats = _graded_cavity_inputs()
    assert g.shape == (2, GCAV_NYI + 1, len(GCAV_DZ) + 1)
    f_pred = _graded_cavity_frequency(g)
    r = oracle.run_nonuniform(g, mats, CAV_STEPS, sources=[(0, 3, 2, "ex", w)], probes=[(0, 5, 4, "ex")],
                              dtype=np.float32)
    f = _peak_frequency(r.time_series[:, 0], g.dt, f_pred)
    print(f"oracle graded cavity: {f / 1e9:.7f} GHz, graded operator {f_pred / 1e9:.7f}, "
          f"rel {(f - f_pred) / f_pred:.2e}")
    assert abs(f - f_pred) / f_pred < 1e-6


@pytest.mark.gpu
def test_cuda_graded_cavity_resonance_matches_graded_operator(cuda):
    import rfx_b200
    g, w, mats = _graded_cavity_inputs()
    pg = rfx_b200.make_nonuniform_grid((CAV_DX, GCAV_NYI * CAV_DX), GCAV_DZ, CAV_DX, cpml_layers=0)
    assert tuple(pg.shape) == tuple(g.shape) and pg.dt == g.dt
    f_pred = _graded_cavity_frequency(g)
    r = rfx_b200.run_nonuniform(pg, rfx_b200.MaterialArrays(*mats), CAV_STEPS, sources=[(0, 3, 2, "ex", w)],
                                probes=[(0, 5, 4, "ex")])
    f = _peak_frequency(np.asarray(r["time_series"])[:, 0], g.dt, f_pred)
    print(f"CUDA graded cavity: {f / 1e9:.7f} GHz, graded operator {f_pred / 1e9:.7f}, "
          f"rel {(f - f_pred) / f_pred:.2e}")
    assert abs(f - f_pred) / f_pred < 1e-6
