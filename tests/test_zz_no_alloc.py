"""``rfxb_forward_noalloc`` (forward steps in the library's fixed device
array, no allocation) against ``rfxb_forward`` on a freshly reset plan, both
through the C ABI.  Collected last so that it also runs after every other GPU
test in the same process; one test also runs it in a fresh process whose first
library call is this entry point (no plan created before it)."""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from tests.scenarios import rel_l2, small_uniform

TOL = 1e-4


def _spec(sc, pec_axes="xyz"):
    from rfx_b200.cpml import build_cpml
    from rfx_b200.engine import PlanSpec
    from rfx_b200.grid import spacing_tables
    g = sc.product_grid()
    return PlanSpec(shape=tuple(int(v) for v in g.shape), dt=float(g.dt), tables=spacing_tables(g),
                    cpml=build_cpml(g, "xyz"), pec_axes=pec_axes,
                    sources=[(i, j, k, c) for (i, j, k, c, _w) in sc.sources],
                    probes=[(i, j, k, c, False) for (i, j, k, c) in sc.probes]), g


def _case(seed, n_total, field_scale):
    """A small CPML scene (materials of the given seed), its source table
    over n_total steps and seeded initial fields."""
    import torch
    sc = small_uniform(n_steps=n_total, seed=seed)
    spec, _ = _spec(sc)
    tab = np.stack([w[:n_total] for (*_c, w) in sc.sources], axis=-1).astype(np.float32)
    rng = np.random.default_rng(100 + seed)
    f0 = [(field_scale * rng.standard_normal(spec.shape)).astype(np.float32) for _ in range(6)]
    return sc, spec, torch.from_numpy(np.ascontiguousarray(tab)).cuda(), f0


def _via_plan(spec, sc, src, f0, step0, n_steps, n_total):
    """rfxb_forward on a new plan (zero psi) through the C ABI."""
    import torch
    from rfx_b200 import _lib
    from rfx_b200.engine import Plan
    plan = Plan(spec)
    plan.set_materials(sc.materials[0], sc.materials[1])
    plan.reset()
    fields = [torch.from_numpy(f).cuda() for f in f0]
    probe = torch.zeros((n_total, len(spec.probes)), device="cuda", dtype=torch.float32)
    io, keep = plan.step_io(src, probe)
    arr = (C.c_void_p * 6)(*[t.data_ptr() for t in fields])
    _lib.check(_lib.load().rfxb_forward(plan.handle, C.byref(io), arr, step0, n_steps,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream)), "rfxb_forward")
    torch.cuda.synchronize()
    plan.check_device()
    plan.close()
    del keep
    return [f.cpu().numpy() for f in fields], probe.cpu().numpy()


def _via_noalloc(spec, sc, src, f0, step0, n_steps, n_total):
    import torch
    from rfx_b200.noalloc import forward_noalloc
    eps = torch.from_numpy(sc.materials[0]).cuda()
    sig = torch.from_numpy(sc.materials[1]).cuda()
    fields = [torch.from_numpy(f).cuda() for f in f0]
    probe = torch.zeros((n_total, len(spec.probes)), device="cuda", dtype=torch.float32)
    forward_noalloc(spec, eps, sig, fields, src, probe, step0, n_steps)
    torch.cuda.synchronize()
    return [f.cpu().numpy() for f in fields], probe.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_plan_forward_two_calls(cuda):
    """Two no-alloc calls in a row on different scenes, initial fields and
    step ranges, each within 1e-4 relative L2 of the plan path (fields and
    probe series)."""
    cases = [(1, 0, 90, 0.0), (5, 30, 70, 1e-3)]
    for seed, step0, n, scale in cases:
        n_total = step0 + n
        sc, spec, src, f0 = _case(seed, n_total, scale)
        ref_f, ref_p = _via_plan(spec, sc, src, f0, step0, n, n_total)
        got_f, got_p = _via_noalloc(spec, sc, src, f0, step0, n, n_total)
        for c, (a, b) in enumerate(zip(got_f, ref_f)):
            assert np.isfinite(a).all()
            e = rel_l2(a, b)
            assert e < TOL, (seed, c, e)
        assert float(np.abs(ref_p[step0:]).max()) > 0.0
        e = rel_l2(got_p[step0:], ref_p[step0:])
        assert e < TOL, (seed, "probes", e)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_grid(cuda):
    """A grid whose internal state exceeds the fixed array is refused with
    RFXB_E_NOMEM before any work is queued."""
    import torch
    from rfx_b200.engine import PlanSpec
    from rfx_b200.noalloc import forward_noalloc
    n = 128
    spec = PlanSpec(shape=(n, n, n), dt=1e-12, tables=tuple(np.full(n, 1e3, np.float32) for _ in range(6)))
    eps = torch.ones((n, n, n), device="cuda")
    sig = torch.zeros((n, n, n), device="cuda")
    fields = [torch.zeros((n, n, n), device="cuda") for _ in range(6)]
    with pytest.raises(RuntimeError, match=r"code -\d+\).*64 MiB"):
        forward_noalloc(spec, eps, sig, fields, None, None, 0, 4)


def _compare(seed, step0, n, scale, noalloc_first):
    """One scene through both paths; returns the worst relative L2 over the
    fields and the probe series."""
    n_total = step0 + n
    sc, spec, src, f0 = _case(seed, n_total, scale)
    if noalloc_first:
        got_f, got_p = _via_noalloc(spec, sc, src, f0, step0, n, n_total)
        ref_f, ref_p = _via_plan(spec, sc, src, f0, step0, n, n_total)
    else:
        ref_f, ref_p = _via_plan(spec, sc, src, f0, step0, n, n_total)
        got_f, got_p = _via_noalloc(spec, sc, src, f0, step0, n, n_total)
    assert all(np.isfinite(a).all() for a in got_f)
    assert float(np.abs(ref_p[step0:]).max()) > 0.0
    errs = [rel_l2(a, b) for a, b in zip(got_f, ref_f)] + [rel_l2(got_p[step0:], ref_p[step0:])]
    return max(errs)


def fresh_process_main():
    """Entry of the fresh-process test: the no-alloc call is the first thing
    the library does on the device (it does its own per-device set-up, the
    kernel's shared-memory opt-in included), then the plan path, twice."""
    import torch
    torch.cuda.set_device(0)
    worst = max(_compare(3, 0, 60, 0.0, True), _compare(4, 10, 50, 1e-3, True))
    print(f"fresh-process worst relL2 {worst:.3e}")
    if not worst < TOL:
        raise SystemExit(f"no-alloc path disagrees with the plan path: {worst:.3e}")


@pytest.mark.gpu
def test_noalloc_first_call_in_a_fresh_process(cuda):
    """In a new process, with no plan created first, the no-alloc entry point
    agrees with the plan path within 1e-4 relative L2 on two calls in a row."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", "from tests.test_zz_no_alloc import fresh_process_main; "
                        "fresh_process_main()"], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process worst relL2" in r.stdout


@pytest.mark.gpu
def test_noalloc_refused_on_a_capturing_stream(cuda):
    """A call made while its stream is capturing a CUDA graph is refused with
    RFXB_E_INVALID (each call uploads host tables that live only during the
    call), and the capture itself stays usable."""
    import torch
    sc, spec, src, f0 = _case(2, 20, 0.0)
    eps = torch.from_numpy(sc.materials[0]).cuda()
    sig = torch.from_numpy(sc.materials[1]).cuda()
    fields = [torch.from_numpy(f).cuda() for f in f0]
    probe = torch.zeros((20, len(spec.probes)), device="cuda", dtype=torch.float32)
    from rfx_b200.noalloc import forward_noalloc
    forward_noalloc(spec, eps, sig, fields, src, probe, 0, 2)   # set-up outside any capture
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    err = None
    with torch.cuda.stream(side):
        g.capture_begin()
        try:
            forward_noalloc(spec, eps, sig, fields, src, probe, 0, 2)
        except RuntimeError as e:
            err = str(e)
        finally:
            g.capture_end()
    torch.cuda.synchronize()
    assert err is not None and "capturing" in err, err
    # the device is still usable afterwards
    forward_noalloc(spec, eps, sig, fields, src, probe, 0, 2)
    torch.cuda.synchronize()
    assert all(torch.isfinite(f).all().item() for f in fields)
