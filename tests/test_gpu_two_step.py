"""Temporal blocking: forward passes of two time steps (launch configuration
``fwd_depth = 2``) give the one-step results bit for bit.

A two-step pass advances the CPML-free interior tiles from step n to n+2 on
the two-step kernel (one read of E^n, H^{n-1/2}, ca/cb with a two-cell halo,
the intermediate state in shared memory) while the CPML tiles and the tiles
near sources, probes, faces and the gradient region take two one-step
launches through an intermediate field buffer.  Every cell is computed with
the same rounding sequence either way, so the fields, probe traces, DFT
planes and -- through the batched sweep -- objectives and gradients must be
identical, not merely close:

* the uniform CPML grid of the 277^3 configuration at 117^3 (8 probes, a
  source, a z-plane DFT through two-step tiles), from random fields in every
  cell, over odd and even step counts and cut into chunks of odd lengths;
* the reference's own PEC benchmark (no CPML, PEC faces) at 129^3, and grids
  mixing CPML, PEC and open faces by axis (the guarded path of the tiles
  whose cells reach a face);
* a graded-z grid with CPML and a PEC sheet (the spacing tables of the
  non-uniform lane, the PEC edge mask in both steps of a pass);
* a DFT plane, a flux monitor and an NTFF box through two-step tiles (the
  observers read each pass's intermediate state);
* the batched sweep (history recording, adjoint gradients);
* a saved and restored state blob and checkpoints taken mid-run.
"""

import numpy as np
import pytest
import torch

from oracle.fdtd import COMPONENTS
from rfx_b200 import workloads
from tests.test_gpu_fullsize import _advance, _device, _random_fields

pytestmark = pytest.mark.gpu


def _fields(r):
    return [f.cpu().numpy().copy() for f in r.plan.store_fields()]


def _run(r, n, init, depth, chunks=1):
    r.plan.set_launch_config(fwd_depth=depth)
    ts, planes = _advance(r, n, init=init, chunks=chunks)
    return ts, planes, _fields(r)


def _same(a, b, label):
    (ts1, pl1, f1), (ts2, pl2, f2) = a, b
    for c, x, y in zip(COMPONENTS, f1, f2):
        assert np.array_equal(x, y), (label, c, float(np.abs(x - y).max()))
    assert np.array_equal(ts1, ts2), label
    assert len(pl1) == len(pl2)
    for x, y in zip(pl1, pl2):
        assert np.array_equal(x, y), label


def _check_two_step_available(r):
    cur, lim = r.plan.launch_config()
    assert cur["fwd_depth"] == 1 and lim["fwd_depth"] == 2


@pytest.mark.parametrize("n", [36, 37])
def test_two_step_uniform_cpml_grid_equals_one_step(cuda, n):
    g, eps, sig, src, probes, dft = workloads.large_uniform(n_steps=n, n_interior=96)
    r = _device(g, eps, sig, n, src, probes, dft, "uniform")
    try:
        _check_two_step_available(r)
        init = _random_fields(g.shape, 5)
        one = _run(r, n, init, 1)
        two = _run(r, n, init, 2)
        _same(one, two, "uniform")
        assert np.abs(two[0]).max() > 0 and np.abs(two[1][0]).max() > 0
        # advances of odd lengths: a pass never straddles two calls
        _same(one, _run(r, n, init, 2, chunks=5), "uniform, chunked")
        launches = r.plan.step_launches()[0]
        assert launches == 5   # per pass: two-step tiles + two launches of each one-step list
    finally:
        r.plan.close()


def test_two_step_pec_cube_equals_one_step(cuda):
    from rfx_b200.simulation import MaterialArrays, prepare_device_run
    n = 41
    g, eps, sig, src, prb = workloads.pec_uniform(n_cells=128, n_steps=n)
    mats = MaterialArrays(eps, sig, np.ones_like(eps))
    r = prepare_device_run(g, mats, n, cpml_axes="", pec_axes="xyz", sources=[tuple(src)], probes=[(*prb, "ez")],
                           dft_planes=[], pec_mask=None, dft_time_offset=1)
    try:
        _check_two_step_available(r)
        init = _random_fields(g.shape, 6)
        _same(_run(r, n, init, 1), _run(r, n, init, 2), "pec cube")
    finally:
        r.plan.close()


@pytest.mark.parametrize("cpml_axes,pec_axes", [("z", "x"), ("xy", ""), ("", "yz"), ("", "")])
def test_two_step_mixed_faces_equal_one_step(cuda, cpml_axes, pec_axes):
    """Axes with CPML, with PEC faces and open (zero guards only): the tiles
    whose cells reach a PEC or open face take the guarded path."""
    from rfx_b200.simulation import MaterialArrays, init_dft_plane_probe, prepare_device_run
    n = 29
    g, eps, sig, src, probes, dft = workloads.large_uniform(n_steps=n, n_interior=80)
    planes = [init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in dft]
    r = prepare_device_run(g, MaterialArrays(eps, sig, np.ones_like(eps)), n, cpml_axes=cpml_axes,
                           pec_axes=pec_axes, sources=src, probes=[p[:4] for p in probes], dft_planes=planes,
                           pec_mask=None, dft_time_offset=1)
    try:
        _check_two_step_available(r)
        init = _random_fields(g.shape, 10)
        _same(_run(r, n, init, 1), _run(r, n, init, 2), f"cpml {cpml_axes!r}, pec {pec_axes!r}")
    finally:
        r.plan.close()


def test_two_step_observers_equal_one_step(cuda):
    """A DFT plane, a flux monitor and an NTFF box whose planes pass through
    two-step tiles: their accumulators read the intermediate state of every
    pass (stored by those tiles) and match one step per pass bit for bit,
    over an odd step count (a pass of two and a last single step)."""
    import rfx_b200
    from rfx_b200.simulation import prepare_device_run
    g = rfx_b200.Grid(freq_max=20e9, domain=(0.08, 0.08, 0.08), dx=1e-3, cpml_layers=4)
    n = 51
    t = np.arange(n, dtype=np.float32) * np.float32(g.dt)
    w = rfx_b200.GaussianPulse(f0=28e9, bandwidth=0.5)(t).astype(np.float32)
    c = (g.nx // 2, g.ny // 2, g.nz // 2)
    eps = (1.0 + np.random.default_rng(4).random(g.shape)).astype(np.float32)
    mats = rfx_b200.MaterialArrays(eps, np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    planes = [rfx_b200.init_dft_plane_probe(1, c[1] - 13, "ex", [24e9, 29e9], g.shape)]
    mons = [rfx_b200.init_flux_monitor(2, c[2] + 13, [26e9], g.shape, g.dx, g.dx, lo1=3, hi1=g.nx - 3)]
    box = (20, g.nx - 20, 22, g.ny - 22, 18, g.nz - 18, np.array([25e9, 30e9], np.float32))
    r = prepare_device_run(g, mats, n, cpml_axes="xyz", pec_axes="", sources=[(*c, "ez", w)],
                           probes=[(c[0], c[1] + 1, c[2], "ey")], dft_planes=planes, pec_mask=None,
                           dft_time_offset=1, flux_monitors=mons, ntff_box=rfx_b200.NTFFBox(*box))

    def run(depth):
        p = r.plan
        p.set_launch_config(fwd_depth=depth)
        p.reset()
        for a in list(r.dft_accs) + list(r.flux_accs) + [r.ntff[0], r.ntff[1]]:   # (NTFF: sums, residuals)
            a.zero_()
        p.advance(0, n, r.src_table, r.probe_out, r.dft_accs, r.dft_phases, r.flux_accs, r.flux_kernels, r.ntff)
        torch.cuda.synchronize()
        p.check_device()
        return ([a.cpu().numpy().copy() for a in r.dft_accs] + [a.cpu().numpy().copy() for a in r.flux_accs] +
                [r.ntff[0].cpu().numpy().copy(), r.probe_out.cpu().numpy().copy()] + _fields(r))

    try:
        _check_two_step_available(r)
        one, two = run(1), run(2)
        for q, (x, y) in enumerate(zip(one, two)):
            assert np.abs(x).max() > 0, q
            assert np.array_equal(x, y), q
    finally:
        r.plan.close()


def test_two_step_graded_grid_equals_one_step(cuda):
    from rfx_b200.grid import make_nonuniform_grid
    n = 30
    rng = np.random.default_rng(7)
    dx = 0.5e-3
    dz = workloads.graded_dz(3)[:72]
    g = make_nonuniform_grid((100 * dx, 100 * dx), dz, dx, cpml_layers=10)
    eps = rng.uniform(1.0, 4.0, g.shape).astype(np.float32)
    sig = rng.uniform(0.0, 0.02, g.shape).astype(np.float32)
    c = (g.nx // 2, g.ny // 2, g.nz // 2)
    src = [(*c, "ez", rng.standard_normal(n).astype(np.float32))]
    probes = [(c[0] + 7, c[1] - 5, c[2], "ez")]
    dft = [(2, c[2] + 11, "ex", np.linspace(10e9, 30e9, 4).astype(np.float32))]
    # a PEC sheet with a hole, through the two-step tiles (edge mask)
    pec = np.zeros(g.shape, bool)
    pec[15:g.nx - 15, 12:g.ny - 12, c[2] - 6] = True
    pec[40:60, 40:60, c[2] - 6] = False
    r = _device(g, eps, sig, n, src, probes, dft, "graded", pec=pec)
    try:
        _check_two_step_available(r)
        init = _random_fields(g.shape, 8)
        _same(_run(r, n, init, 1), _run(r, n, init, 2), "graded")
    finally:
        r.plan.close()


def test_two_step_state_blob_and_checkpoints(cuda):
    g, eps, sig, src, probes, dft = workloads.large_uniform(n_steps=40, n_interior=96)
    r = _device(g, eps, sig, 40, src, probes, [], "uniform")
    p = r.plan
    try:
        init = _random_fields(g.shape, 9)
        ref = _run(r, 40, init, 1)[2]
        # 18 steps (nine passes: the fields' parity flips, the psi's does
        # not), save, 22 more; then restore and redo the 22 on one-step
        # launches, and from a checkpoint on two-step passes again
        p.set_launch_config(fwd_depth=2)
        p.reset()
        p.load_fields([init[c] for c in COMPONENTS])
        p.advance(0, 18, r.src_table, r.probe_out)
        blob = p.save_state()
        p.checkpoint_reserve(1)
        p.checkpoint_save(0)
        p.advance(18, 22, r.src_table, r.probe_out)
        torch.cuda.synchronize()
        p.check_device()
        for x, y in zip(_fields(r), ref):
            assert np.array_equal(x, y)
        p.set_launch_config(fwd_depth=1)
        p.restore_state(blob)
        p.advance(18, 22, r.src_table, r.probe_out)
        for x, y in zip(_fields(r), ref):
            assert np.array_equal(x, y)
        p.set_launch_config(fwd_depth=2)
        p.checkpoint_load(0)
        p.advance(18, 22, r.src_table, r.probe_out)
        torch.cuda.synchronize()
        for x, y in zip(_fields(r), ref):
            assert np.array_equal(x, y)
    finally:
        p.close()


def test_two_step_batched_sweep_equals_one_step(cuda):
    from rfx_b200.batch import Sweep
    insts = workloads.batched_sweep(seed=5, n_inst=3, n_steps=90, n_lo=96, n_hi=120)
    sw = Sweep(insts, 90, device=torch.device("cuda", 0), batched=True)
    try:
        cur, lim = sw.batch.launch_config()
        assert lim["fwd_depth"] == 2
        J1, g1 = sw.run()
        J1 = np.array([float(j) for j in J1])
        g1 = [x.detach().cpu().numpy().copy() for x in g1]
        sw.batch.set_launch_config(fwd_depth=2)
        J2, g2 = sw.run()
        sw.check_device()
        assert np.array_equal(J1, np.array([float(j) for j in J2]))
        for a, b in zip(g1, g2):
            assert np.array_equal(a, b.detach().cpu().numpy())
        with pytest.raises(Exception):
            sw.batch.set_launch_config(fwd_depth=2, fwd_persist=1)
    finally:
        sw.close()
