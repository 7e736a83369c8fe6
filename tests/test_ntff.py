"""NTFF Huygens-box accumulation (rfx/farfield.py:208-313) and the far-field
transform that reads it (rfx/farfield.py:393-556, 780-802).

CPU: the oracle's Kahan complex64 running DFT on the six faces against a
float64 post-hoc DFT of the same face fields, with the E factor at t = n dt
and the H factor half a step later; and the reference's short-dipole gates
(rfx tests/test_farfield.py:108-180: sin(theta) pattern, small E_phi in the
E-plane, directivity 1.76 +- 0.75 dBi) on oracle NTFF data.

GPU: the CUDA accumulation against the oracle on the uniform and graded
lanes, the device far-field transform against the NumPy restatement, the
dipole gates through the product API, and run_until_decay's chunked NTFF
against one uninterrupted run.
"""

import numpy as np
import pytest

import oracle
from oracle import fdtd
from oracle import farfield as off


def rel_l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _small_case():
    g = oracle.make_uniform_grid((0.012, 0.014, 0.013), 1e-3, cpml_layers=4)
    c = (g.nx // 2, g.ny // 2 + 1, g.nz // 2)
    n = 140
    t = np.arange(n, dtype=np.float32) * np.float32(g.dt)
    w = oracle.gaussian_pulse(t, 30e9, 0.5).astype(np.float32)
    mats = (np.ones(g.shape, np.float32), np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    box = (6, g.nx - 6, 5, g.ny - 6, 6, g.nz - 5, np.array([25e9, 31e9, 40e9], np.float32))
    return g, mats, [(*c, "ez", w), (c[0] - 2, c[1], c[2] + 1, "ex", 0.5 * w)], n, box


def test_oracle_ntff_matches_posthoc_dft():
    g, mats, srcs, n, box = _small_case()
    st = fdtd._Stepper(g, mats, dtype=np.float32, nonuniform=False, cpml_axes="xyz", pec_axes="",
                       pec_mask=None)
    i0, i1, j0, j1, k0, k1, freqs = box
    rec = {name: [] for name in oracle.NTFF_FACES}
    lo, hi = (i0, j0, k0), (i1, j1, k1)

    def record(step, F):
        for q, name in enumerate(oracle.NTFF_FACES):
            ax = q // 2
            sl = [slice(i0, i1), slice(j0, j1), slice(k0, k1)]
            sl[ax] = hi[ax] if q & 1 else lo[ax]
            rec[name].append(np.stack([np.asarray(F[c][tuple(sl)], np.float64)
                                       for c in fdtd._NTFF_COMPONENTS[ax]], -1))
        return False

    r = fdtd._run(st, n, srcs, (), (), (), 1, probes_before_dft=True, dx_vi=g.dx, stop=record, ntff=box)
    dt = float(np.float32(g.dt))
    f = np.asarray(freqs, np.float64)
    tt = np.arange(n, dtype=np.float64) * dt
    ke = np.exp(-2j * np.pi * f[:, None] * tt[None, :]) * dt            # (n_f, n)
    kh = np.exp(-2j * np.pi * f[:, None] * (tt[None, :] + 0.5 * dt)) * dt
    for name in oracle.NTFF_FACES:
        v = np.stack(rec[name])                                          # (n, n1, n2, 4)
        ref = np.concatenate([np.einsum("fn,nabc->fabc", ke, v[..., :2]),
                              np.einsum("fn,nabc->fabc", kh, v[..., 2:])], -1)
        got = r.ntff[name]
        assert got.dtype == np.complex64 and got.shape == ref.shape
        assert np.linalg.norm(ref) > 0
        e = rel_l2(got, ref)
        print(name, "Kahan complex64 vs float64 post-hoc DFT relL2", e)
        assert e < 2e-5, name
        # the residuals stay at the rounding level of the sums
        assert np.max(np.abs(r.ntff["c_" + name])) <= 1e-5 * np.max(np.abs(got))


def _dipole_grid():
    dx = (299792458.0 / 5e9) / 20.0
    return oracle.make_uniform_grid((0.03, 0.03, 0.03), dx, cpml_layers=8), dx


def _dipole_checks(Et, Ep, theta, phi, D):
    # rfx tests/test_farfield.py:108-141: sin(theta) pattern in the E-plane
    e = np.abs(Et[0, :, 0])
    en = e / e.max()
    peak = theta[int(np.argmax(en))]
    assert abs(peak - np.pi / 2) < np.pi / 6
    pole = (theta < np.radians(20)) | (theta > np.radians(160))
    assert np.max(en[pole]) < 0.5
    # :144-154: E_phi small in the E-plane
    assert np.max(np.abs(Ep[0, :, 0])) / e.max() < 0.3
    # :157-180: short-dipole directivity 1.76 +- 0.75 dBi
    assert abs(D - 1.76) < 0.75


def _dipole_oracle(n_steps=200):
    g, dx = _dipole_grid()
    c = (g.nx // 2, g.ny // 2, g.nz // 2)
    t = np.arange(n_steps, dtype=np.float32) * np.float32(g.dt)
    w = oracle.gaussian_pulse(t, 3e9, 0.5).astype(np.float32)
    lo = int(round(0.004 / dx)) + 8
    hi = int(round(0.026 / dx)) + 8
    box = (lo, hi, lo, hi, lo, hi, np.array([3e9], np.float32))
    mats = (np.ones(g.shape, np.float32), np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    r = oracle.run_uniform(g, mats, n_steps, boundary="cpml", pec_axes="", sources=[(*c, "ez", w)], ntff=box)
    return g, dx, box, r


def test_oracle_dipole_far_field_gates():
    g, dx, box, r = _dipole_oracle()
    theta = np.linspace(0.01, np.pi - 0.01, 37)
    phi = np.linspace(0.0, 2 * np.pi, 24, endpoint=False)
    Et, Ep = off.compute_far_field(r.ntff, box, dx, (8, 8, 8), theta, phi)
    D = float(off.directivity(Et, Ep, theta, phi)[0])
    print("oracle short-dipole directivity", D, "dBi")
    _dipole_checks(Et, Ep, theta, phi, D)


# ---------------------------------------------------------------- GPU


def _device_ntff_data(r):
    return {name: getattr(r.ntff_data, name) for name in oracle.NTFF_FACES}


@pytest.mark.gpu
def test_ntff_matches_oracle(cuda):
    import rfx_b200
    g, mats, srcs, n, box = _small_case()
    ref = oracle.run_uniform(g, mats, n, boundary="cpml", pec_axes="", sources=srcs, ntff=box)
    pg = rfx_b200.Grid(freq_max=5e9, domain=(0.012, 0.014, 0.013), dx=1e-3, cpml_layers=4)
    assert tuple(pg.shape) == tuple(g.shape)
    nb = rfx_b200.NTFFBox(*box)
    r = rfx_b200.run(pg, rfx_b200.MaterialArrays(*mats), n, boundary="cpml", pec_axes="",
                     sources=[rfx_b200.SourceSpec(*s) for s in srcs], ntff=nb)
    assert r.ntff_box == nb
    for name in oracle.NTFF_FACES:
        got = getattr(r.ntff_data, name)
        assert got.dtype == np.complex64 and got.shape == ref.ntff[name].shape
        e = rel_l2(got, ref.ntff[name])
        print(name, "relL2", e)
        assert e < 1e-4, name


@pytest.mark.gpu
def test_ntff_graded_lane_matches_oracle(cuda):
    """run_nonuniform(ntff_box, ntff_data) on a graded z axis: the CUDA
    accumulation against the oracle's (E factor at t = n dt on both lanes)."""
    import rfx_b200
    dz = np.concatenate([np.full(8, 1e-3), np.linspace(1e-3, 0.6e-3, 6), np.full(8, 0.6e-3)])
    og = oracle.make_nonuniform_grid((0.012, 0.011), dz, 1e-3, cpml_layers=4)
    pg = rfx_b200.make_nonuniform_grid((0.012, 0.011), dz, 1e-3, cpml_layers=4)
    assert tuple(pg.shape) == tuple(og.shape)
    n = 120
    t = np.arange(n, dtype=np.float32) * np.float32(og.dt)
    w = oracle.gaussian_pulse(t, 30e9, 0.5).astype(np.float32)
    c = (og.nx // 2, og.ny // 2, og.nz // 2)
    mats = (np.ones(og.shape, np.float32), np.zeros(og.shape, np.float32), np.ones(og.shape, np.float32))
    box = (5, og.nx - 5, 5, og.ny - 6, 5, og.nz - 5, np.array([28e9, 36e9], np.float32))
    ref = oracle.run_nonuniform(og, mats, n, sources=[(*c, "ez", w)], ntff=box)
    nb = rfx_b200.NTFFBox(*box)
    out = rfx_b200.run_nonuniform(pg, rfx_b200.MaterialArrays(*mats), n, sources=[(*c, "ez", w)], ntff_box=nb,
                                  ntff_data=rfx_b200.init_ntff_data(nb))
    for name in oracle.NTFF_FACES:
        e = rel_l2(getattr(out["ntff_data"], name), ref.ntff[name])
        print(name, "relL2", e)
        assert e < 1e-4, name
    # without ntff_data the box is ignored, as in the reference
    out2 = rfx_b200.run_nonuniform(pg, rfx_b200.MaterialArrays(*mats), 4, sources=[(*c, "ez", w)], ntff_box=nb)
    assert "ntff_data" not in out2


@pytest.mark.gpu
def test_device_far_field_and_dipole_gates(cuda):
    import rfx_b200
    pg = rfx_b200.Grid(freq_max=5e9, domain=(0.03, 0.03, 0.03), cpml_layers=8)
    n = 200
    src = rfx_b200.make_source(pg, (0.015, 0.015, 0.015), "ez", rfx_b200.GaussianPulse(f0=3e9, bandwidth=0.5), n)
    box = rfx_b200.make_ntff_box(pg, (0.004,) * 3, (0.026,) * 3, [3e9])
    mats = rfx_b200.MaterialArrays(*(np.ones(pg.shape, np.float32), np.zeros(pg.shape, np.float32),
                                     np.ones(pg.shape, np.float32)))
    r = rfx_b200.run(pg, mats, n, boundary="cpml", sources=[src], ntff=box)
    theta = np.linspace(0.01, np.pi - 0.01, 37)
    phi = np.linspace(0.0, 2 * np.pi, 24, endpoint=False)
    ff = rfx_b200.compute_far_field(r.ntff_data, r.ntff_box, r.grid, theta, phi)
    Et, Ep = off.compute_far_field(_device_ntff_data(r), tuple(box[:6]) + (box.freqs,), pg.dx, (8, 8, 8),
                                   theta, phi)
    assert rel_l2(ff.E_theta, Et) < 1e-10 and rel_l2(ff.E_phi, Ep) < 1e-10
    D = float(rfx_b200.directivity(ff)[0])
    assert abs(D - float(off.directivity(Et, Ep, theta, phi)[0])) < 1e-9
    print("CUDA short-dipole directivity", D, "dBi")
    _dipole_checks(ff.E_theta, ff.E_phi, theta, phi, D)
    pat = rfx_b200.radiation_pattern(ff)
    assert pat.shape == ff.E_theta.shape and abs(pat.max()) < 1e-9


@pytest.mark.gpu
def test_run_until_decay_ntff_matches_a_plain_run(cuda):
    import rfx_b200
    g, mats, srcs, n, box = _small_case()
    pg = rfx_b200.Grid(freq_max=5e9, domain=(0.012, 0.014, 0.013), dx=1e-3, cpml_layers=4)
    long = 600
    srcs_l = [rfx_b200.SourceSpec(*s[:4], np.concatenate([s[4], np.zeros(long - n, np.float32)])) for s in srcs]
    nb = rfx_b200.NTFFBox(*box)
    m = rfx_b200.MaterialArrays(*mats)
    r1 = rfx_b200.run_until_decay(pg, m, decay_by=1e-2, check_interval=25, min_steps=50, max_steps=long,
                                  boundary="cpml", pec_axes="", sources=srcs_l, ntff=nb)
    steps = int(r1.state.step)
    assert steps < long
    r2 = rfx_b200.run(pg, m, steps, boundary="cpml", pec_axes="", sources=srcs_l, ntff=nb)
    for name in oracle.NTFF_FACES:
        a, b = getattr(r1.ntff_data, name), getattr(r2.ntff_data, name)
        assert rel_l2(a, b) < 1e-6, name


@pytest.mark.gpu
def test_monitors_in_a_batch_match_single_plans(cuda):
    """Two plans of different shapes, each with a DFT plane, a flux monitor and
    an NTFF box, advanced as one batch (one launch per step and kernel for
    both): every accumulator matches the plan advanced on its own."""
    import torch
    import rfx_b200
    from rfx_b200.engine import Batch
    from rfx_b200.simulation import prepare_device_run

    def scene(domain, seed, box, ff, fflux):
        g = rfx_b200.Grid(freq_max=20e9, domain=domain, dx=1e-3, cpml_layers=4)
        n = 90
        t = np.arange(n, dtype=np.float32) * np.float32(g.dt)
        w = rfx_b200.GaussianPulse(f0=28e9, bandwidth=0.5)(t).astype(np.float32)
        c = (g.nx // 2, g.ny // 2, g.nz // 2)
        eps = (1.0 + np.random.default_rng(seed).random(g.shape)).astype(np.float32)
        mats = rfx_b200.MaterialArrays(eps, np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
        planes = [rfx_b200.init_dft_plane_probe(1, c[1] - 2, "ex", ff, g.shape)]
        mons = [rfx_b200.init_flux_monitor(2, c[2] + 3, fflux, g.shape, g.dx, g.dx, lo1=3, hi1=g.nx - 3)]
        kw = dict(cpml_axes="xyz", pec_axes="", sources=[(*c, "ez", w)], probes=[(c[0], c[1] + 1, c[2], "ey")],
                  dft_planes=planes, pec_mask=None, dft_time_offset=1, flux_monitors=mons,
                  ntff_box=rfx_b200.NTFFBox(*box))
        return g, mats, n, kw

    scenes = [scene((0.012, 0.014, 0.011), 1, (4, 9, 5, 11, 4, 10, np.array([25e9, 30e9], np.float32)),
                    [24e9, 29e9, 33e9], [26e9]),
              scene((0.016, 0.010, 0.013), 2, (5, 13, 4, 8, 5, 11, np.array([27e9], np.float32)),
                    [26e9], [24e9, 31e9])]

    def outputs(r):
        return ([a.cpu().numpy() for a in r.dft_accs] + [a.cpu().numpy() for a in r.flux_accs] +
                [r.ntff[0].cpu().numpy(), r.probe_out.cpu().numpy()] + [f.cpu().numpy() for f in r.plan.store_fields()])

    single = []
    for g, mats, n, kw in scenes:
        r = prepare_device_run(g, mats, n, **kw)
        try:
            r.plan.advance(0, n, r.src_table, r.probe_out, r.dft_accs, r.dft_phases, r.flux_accs, r.flux_kernels,
                           r.ntff)
            single.append(outputs(r))
        finally:
            r.plan.close()
    runs = [prepare_device_run(g, mats, n, **kw) for g, mats, n, kw in scenes]
    try:
        b = Batch([r.plan for r in runs])
        try:
            b.advance(0, scenes[0][2], [dict(src_table=r.src_table, probe_out=r.probe_out, dft_accs=r.dft_accs,
                                             dft_phases=r.dft_phases, flux_accs=r.flux_accs,
                                             flux_kernels=r.flux_kernels, ntff=r.ntff) for r in runs])
            b.check_device()
        finally:
            b.close()
        for r, ref in zip(runs, single):
            for q, (x, y) in enumerate(zip(outputs(r), ref)):
                assert np.linalg.norm(y) > 0, q
                assert rel_l2(x, y) < 1e-5, q
    finally:
        for r in runs:
            r.plan.close()
    torch.cuda.synchronize()
