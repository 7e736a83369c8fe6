"""Parity at the configurations' full sizes: the 277^3 uniform grid, the
217 x 217 x 121 graded grid with its PEC sheet, the 221 x 141 x 69 adjoint
grid and the batched sweep's instances.

The float32 oracle finishes only a few steps of these grids in seconds, so
each is checked two ways:

1. directly against the oracle over a few steps started from seeded random
   fields in every cell (E ~ N(0, 1), H ~ N(0, 1) / 377 ohm), so that every
   cell's coefficients, the CPML slabs, the PEC faces and the PEC sheet act
   from the first step; 1e-4 relative L2 per field component, probe trace
   and DFT plane;
2. over the configuration's full step count through properties that hold
   at any size: superposition in the source table (the step is linear, so
   ts(w1 + w2) = ts(w1) + ts(w2), DFT planes alike), an advance cut into
   chunks equal to one advance bit for bit, the adjoint's exact transpose
   (<g, ts(w)> = <dJ/dw, w>), checkpoint-every-64 with a ragged last segment
   equal to the single-pass history bit for bit, and the batched sweep
   equal to its simulations run one at a time.
"""

import numpy as np
import pytest
import torch

import oracle
from oracle.fdtd import COMPONENTS
from tests.scenarios import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4
ETA0 = 376.730313668


def _random_fields(shape, seed):
    rng = np.random.default_rng(seed)
    return {c: (rng.standard_normal(shape) / (1.0 if c[0] == "e" else ETA0)).astype(np.float32)
            for c in COMPONENTS}


def _device(g, eps, sig, n, src, probes, dft, lane, pec=None):
    from rfx_b200.grid import face_pads
    from rfx_b200.simulation import MaterialArrays, init_dft_plane_probe, prepare_device_run
    planes = [init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in dft]
    if lane == "uniform":
        axes, offset = "xyz", 1
    else:
        pads = face_pads(g)
        axes = "".join(a for a, (lo, hi) in zip("xyz", (pads[0:2], pads[2:4], pads[4:6])) if lo + hi > 0)
        offset = 0
    return prepare_device_run(g, MaterialArrays(eps, sig, np.ones_like(eps)), n, cpml_axes=axes, pec_axes="xyz",
                              sources=src, probes=[p[:4] for p in probes], dft_planes=planes, pec_mask=pec,
                              dft_time_offset=offset)


def _advance(r, n, table=None, init=None, chunks=1):
    p = r.plan
    p.reset()
    for a in r.dft_accs:
        a.zero_()
    if table is not None:
        r.src_table.copy_(table)
    if init is not None:
        p.load_fields([init[c] for c in COMPONENTS])
    cuts = np.linspace(0, n, chunks + 1).astype(int)
    for a, b in zip(cuts[:-1], cuts[1:]):
        p.advance(int(a), int(b - a), r.src_table, r.probe_out, r.dft_accs, r.dft_phases)
    torch.cuda.synchronize()
    p.check_device()
    ts = r.probe_out.cpu().numpy().copy() if r.probe_out is not None else np.zeros((n, 0), np.float32)
    return ts, [a.cpu().numpy().copy() for a in r.dft_accs]


def _compare_with_oracle(label, r, ref, n, init):
    ts, planes = _advance(r, n, init=init)
    fields = [f.cpu().numpy() for f in r.plan.store_fields()]
    for c, f in zip(COMPONENTS, fields):
        e = rel_l2(f, ref.state[c])
        print(f"{label} {c}: relL2 vs oracle f32 {e:.2e}")
        assert e < TOL, c
    for q in range(ts.shape[1]):
        e = rel_l2(ts[:, q], ref.time_series[:, q])
        assert e < TOL, q
    for q, acc in enumerate(planes):
        e = rel_l2(acc, ref.dft_planes[q])
        print(f"{label} dft {q}: relL2 vs oracle f32 {e:.2e}")
        assert e < TOL


def _superposition(label, r, n):
    w1 = r.src_table.clone()
    rng = np.random.default_rng(11)
    w2 = torch.from_numpy(rng.standard_normal(tuple(w1.shape)).astype(np.float32)).to(w1.device)
    w2 *= float(w1.square().mean().sqrt()) / float(w2.square().mean().sqrt())
    a_ts, a_pl = _advance(r, n, w1)
    b_ts, b_pl = _advance(r, n, w2)
    c_ts, c_pl = _advance(r, n, w1 + w2)
    e = rel_l2(a_ts + b_ts, c_ts)
    print(f"{label}: superposition of the probe traces over {n} steps, relL2 {e:.2e}")
    assert e < TOL
    assert np.abs(c_ts).max() > 0
    for q, (x, y, z) in enumerate(zip(a_pl, b_pl, c_pl)):
        e = rel_l2(x + y, z)
        print(f"{label}: superposition of DFT plane {q}, relL2 {e:.2e}")
        assert e < TOL
    # the same run cut into uneven chunks (graph replays of other lengths)
    d_ts, d_pl = _advance(r, n, w1, chunks=7)
    assert np.array_equal(d_ts, a_ts)
    for x, y in zip(d_pl, a_pl):
        assert np.array_equal(x, y)
    r.src_table.copy_(w1)


def test_large_uniform_full_size(cuda):
    """277^3, CPML 10, 32 seeded boxes, 8 probes, z-plane DFT at 16
    frequencies: 3 steps against the oracle from random fields, then the full
    4000 steps through superposition and chunking."""
    from rfx_b200 import workloads
    n_or, n_full = 3, 4000
    g, eps, sig, src, probes, dft = workloads.large_uniform(n_steps=n_full)
    assert tuple(g.shape) == (277, 277, 277)
    og = oracle.make_uniform_grid(g.domain, g.dx, cpml_layers=g.cpml_layers)
    assert tuple(og.shape) == tuple(g.shape) and og.dt == g.dt
    init = _random_fields(g.shape, 1)
    src_or = [(i, j, k, c, w[:n_or]) for (i, j, k, c, w) in src]
    ref = oracle.run_uniform(og, (eps, sig, np.ones_like(eps)), n_or, boundary="cpml", sources=src_or,
                             probes=probes, dft_planes=dft, dtype=np.float32, init_fields=init)
    r = _device(g, eps, sig, n_or, src_or, probes, dft, "uniform")
    try:
        _compare_with_oracle("large_uniform", r, ref, n_or, init)
    finally:
        r.plan.close()
    del ref
    r = _device(g, eps, sig, n_full, src, probes, dft, "uniform")
    try:
        _superposition("large_uniform", r, n_full)
    finally:
        r.plan.close()


def test_graded_full_size(cuda):
    """217 x 217 x 121 graded grid, CPML 12, PEC sheet, substrate, 4 probes,
    DFT plane at 8 frequencies: 6 steps against the oracle from random fields,
    then the full 6000 steps through superposition and chunking."""
    from rfx_b200 import workloads
    n_or, n_full = 6, 6000
    g, eps, sig, pec, src, probes, dft = workloads.graded(n_steps=n_full)
    assert tuple(g.shape) == (217, 217, 121)
    dx = 0.5e-3
    og = oracle.make_nonuniform_grid((192 * dx, 192 * dx), workloads.graded_dz(0), dx, cpml_layers=12)
    assert tuple(og.shape) == tuple(g.shape)
    init = _random_fields(g.shape, 2)
    src_or = [(i, j, k, c, np.asarray(w)[:n_or]) for (i, j, k, c, w) in src]
    ref = oracle.run_nonuniform(og, (eps, sig, np.ones_like(eps)), n_or, sources=src_or, probes=probes,
                                dft_planes=dft, pec_mask=pec, dtype=np.float32, init_fields=init)
    r = _device(g, eps, sig, n_or, src_or, probes, dft, "nonuniform", pec)
    try:
        _compare_with_oracle("graded", r, ref, n_or, init)
    finally:
        r.plan.close()
    r = _device(g, eps, sig, n_full, src, probes, dft, "nonuniform", pec)
    try:
        _superposition("graded", r, n_full)
    finally:
        r.plan.close()


def test_adjoint_config_full_size(cuda):
    """221 x 141 x 69, CPML 10, 64 x 64 x 2 design region, 3000 steps: the
    forward against the oracle for 8 steps from random fields; the reverse
    sweep over all 3000 steps is the exact transpose of the forward (<g, ts>
    reproduced through the source-table gradient), and checkpoint-every-64
    (46 full segments and a ragged one of 56) gives the single-pass history's
    probe traces and gradients bit for bit."""
    from rfx_b200 import MaterialArrays, workloads
    from rfx_b200.adjoint import AdjointRunner
    n_or, n_full = 8, 3000
    g, eps, sig, src, probes, box, freqs = workloads.adjoint_region(n_steps=n_full)
    assert tuple(g.shape) == (221, 141, 69)
    og = oracle.make_uniform_grid(g.domain, g.dx, cpml_layers=g.cpml_layers)
    init = _random_fields(g.shape, 3)
    src_or = [(i, j, k, c, w[:n_or]) for (i, j, k, c, w) in src]
    ref = oracle.run_uniform(og, (eps, sig, np.ones_like(eps)), n_or, boundary="cpml", sources=src_or,
                             probes=probes, dtype=np.float32, init_fields=init)
    r = _device(g, eps, sig, n_or, src_or, probes, [], "uniform")
    try:
        _compare_with_oracle("adjoint_region", r, ref, n_or, init)
    finally:
        r.plan.close()

    mats = MaterialArrays(eps, sig, np.ones_like(eps))
    kw = dict(sources=src, probes=probes, box=box, boundary="cpml", cpml_axes="xyz", pec_axes="xyz")
    a = AdjointRunner(g, mats, n_full, mode="history", **kw)
    b = AdjointRunner(g, mats, n_full, mode="segments", checkpoint_every=64, **kw)
    try:
        ts = a.forward()
        # cotangent g = ts: J = |ts|^2 has no cancellation, so the relative
        # error of J measures the transpose
        g_ts = ts.detach().clone().contiguous()
        J = float(ts.double().square().sum())
        _, src_adj = a.backward(g_ts)
        J_adj = float((src_adj.double() * a.src_table.double()).sum())
        print(f"adjoint_region full size, g = ts: J {J:.6e}, via the reverse sweep {J_adj:.6e}, "
              f"rel {abs(J - J_adj) / J:.2e}")
        assert abs(J - J_adj) <= 2e-5 * J
        # a random cotangent: J sums 12,000 terms of both signs, so the error
        # is bounded against |g| |ts| (the dot-product test's scale)
        gvec = torch.from_numpy(np.random.default_rng(5).standard_normal(tuple(ts.shape)).astype(np.float32)).cuda()
        J = float((gvec.double() * ts.double()).sum())
        grad_a, src_adj = a.backward(gvec)
        J_adj = float((src_adj.double() * a.src_table.double()).sum())
        scale = float(gvec.double().norm() * ts.double().norm())
        print(f"adjoint_region full size, random g: J {J:.6e}, via the reverse sweep {J_adj:.6e}, "
              f"|dJ| / (|g| |ts|) {abs(J - J_adj) / scale:.2e}")
        assert abs(J - J_adj) <= 1e-5 * scale
        tb = b.forward()
        grad_b, src_b = b.backward(gvec)
        assert torch.equal(ts, tb)
        assert torch.equal(grad_a, grad_b)
        assert torch.equal(src_adj, src_b)
        assert float(grad_a.abs().max()) > 0
    finally:
        a.close()
        b.close()


def test_sweep_instances_full_size_batched_equals_single(cuda):
    """Eight of the batched sweep's instances at their full sizes ((n+17)^3,
    n ~ U{64..160}, seed 0) over the full 2000 steps, forward + objective +
    adjoint: the batched launch gives every instance's objective and
    gradient as the instance run alone."""
    from rfx_b200.batch import Sweep
    from rfx_b200.workloads import batched_sweep
    insts = batched_sweep(seed=0, n_inst=64, n_steps=2000)[:8]
    a = Sweep(insts, 2000, device=torch.device("cuda", 0), batched=True)
    b = Sweep(insts, 2000, device=torch.device("cuda", 0), batched=False)
    try:
        Ja, ga = a.run()
        Jb, gb = b.run()
        a.check_device()
        b.check_device()
        for x, y, u, v in zip(Ja, Jb, ga, gb):
            assert abs(float(x) - float(y)) <= 1e-6 * abs(float(y))
            ua, vb = u.cpu().numpy(), v.cpu().numpy()
            e = rel_l2(ua, vb)
            print(f"sweep instance {u.shape}: J {float(x):.6e} / {float(y):.6e}, gradient relL2 {e:.2e}")
            assert e <= 1e-5 and np.abs(ua).max() > 0 and float(y) > 0
    finally:
        a.close()
        b.close()
