"""The step kernels' work lists, on CPU (no device: ``rfxb_debug_work_lists``
runs the host-side split and balancing of ``rfxb_capi.cu``).

Every list a batch launches for one step must update each (tile, x plane)
of every plan exactly once -- a missed plane leaves stale fields, a doubled
one races with itself -- and the CPML-free kernels may only be given tiles
and planes whose update needs no CPML term:

* forward: all tiles on one kernel (0), or CPML-free (1) + staged-psi (2);
  a CPML-free forward item's cells (rows y0-1 .. y0+7, columns z0-1 ..
  z0+31) reach no y / z slab and its planes lie in ncp+1 .. nx-ncp-1;
* reverse: CPML-free (3) + CPML (4), or CPML-free (3) + y-slab (5) + the
  rest (6); a reverse CPML-free item's rows y0-1 .. y0+8 and columns z0-1 ..
  z0+32 reach no slab and its planes lie in ncp+1 .. nx-ncp-2; a variant-4
  item (6) reaches no y slab;
* two-step passes: two-step tiles (7) + one-step CPML-free work (8) + one-step
  CPML work (9); every cell a two-step item computes (rows y0-2 .. y0+8,
  columns z0-2 .. z0+32, planes xa-2 .. xb) lies out of the slabs, an item
  whose cells reach a grid face or guard takes the guarded path, and an item
  stores its intermediate state wherever one-step work reads it.
"""

import ctypes as C

import numpy as np
import pytest

from rfx_b200 import _lib

TY, TZ = 8, 32


def _lists(plans, which, resident=444):
    lib = _lib.load()
    dims = (C.c_int32 * (5 * len(plans)))(*[int(v) for p in plans for v in p])
    n = C.c_int32()
    rc = lib.rfxb_debug_work_lists(len(plans), dims, resident, which, None, 0, C.byref(n))
    assert rc == 0, _lib.load().rfxb_last_error()
    out = (C.c_int32 * max(1, 5 * n.value))()
    assert lib.rfxb_debug_work_lists(len(plans), dims, resident, which, out, n.value, C.byref(n)) == 0
    return np.frombuffer(out, np.int32)[: 5 * n.value].reshape(-1, 5).copy()


def _coverage(plans, items):
    """Count of updates per (plan, y tile, z tile, x plane)."""
    cov = [np.zeros(((p[1] + TY - 1) // TY, (p[2] + TZ - 1) // TZ, p[0]), np.int32) for p in plans]
    for q, y0, z0, xa, xb in items:
        assert y0 % TY == 0 and z0 % TZ == 0
        assert 0 <= xa < xb <= plans[q][0]
        cov[q][y0 // TY, z0 // TZ, xa:xb] += 1
    return cov


def _reaches(lo, hi, n, ncp):
    """Rows (or columns) lo .. hi include a cell of a CPML slab of width ncp."""
    return lo < ncp or hi >= n - ncp


def _random_plans(rng, k):
    plans = []
    for _ in range(k):
        ncp = int(rng.choice([0, 4, 8, 10, 12]))
        axes = int(rng.integers(0, 8)) if ncp else 0
        lo = 2 * ncp + 6
        plans.append((int(rng.integers(lo, lo + 90)), int(rng.integers(lo, lo + 90)), int(rng.integers(lo, lo + 90)),
                      ncp, axes))
    return plans


CASES = [
    [(87, 47, 42, 8, 7)],                   # README quick start grid
    [(81, 81, 81, 8, 7), (177, 177, 177, 8, 7), (100, 37, 140, 8, 3)],
    [(221, 141, 69, 10, 7)],                # adjoint configuration
    [(40, 40, 40, 0, 0), (30, 31, 33, 12, 6)],
]


@pytest.mark.parametrize("case", range(len(CASES) + 6))
@pytest.mark.parametrize("resident", [148, 592])
def test_work_lists_cover_each_plane_once(case, resident):
    plans = CASES[case] if case < len(CASES) else _random_plans(np.random.default_rng(case), 4)
    groups = {"all": [0], "fwd split": [1, 2], "rev split": [3, 4], "rev lite": [3, 5, 6], "two-step": [7, 8, 9]}
    for name, ids in groups.items():
        items = np.concatenate([_lists(plans, w, resident) for w in ids])
        items[:, 0] &= 0xFFFF   # the two-step list's intermediate-store flags
        for q, c in enumerate(_coverage(plans, items)):
            assert c.min() == 1 and c.max() == 1, (name, plans[q])


@pytest.mark.parametrize("case", range(len(CASES) + 6))
def test_cpml_free_lists_touch_no_slab(case):
    plans = CASES[case] if case < len(CASES) else _random_plans(np.random.default_rng(100 + case), 4)
    for q, y0, z0, xa, xb in _lists(plans, 1):
        nx, ny, nz, ncp, ax = plans[q]
        if not ncp or not ax:
            continue
        assert not ((ax & 2) and _reaches(y0 - 1, y0 + TY - 1, ny, ncp))
        assert not ((ax & 4) and _reaches(z0 - 1, z0 + TZ - 1, nz, ncp))
        if ax & 1:
            assert xa >= ncp + 1 and xb <= nx - ncp
    for q, y0, z0, xa, xb in _lists(plans, 3):
        nx, ny, nz, ncp, ax = plans[q]
        if not ncp or not ax:
            continue
        assert not ((ax & 2) and _reaches(y0 - 1, y0 + TY, ny, ncp))
        assert not ((ax & 4) and _reaches(z0 - 1, z0 + TZ, nz, ncp))
        if ax & 1:
            assert xa >= ncp + 1 and xb <= nx - ncp - 1
    for q, y0, z0, xa, xb in _lists(plans, 6):
        nx, ny, nz, ncp, ax = plans[q]
        assert not ((ax & 2) and _reaches(y0 - 1, y0 + TY, ny, ncp))


def _two_step_column(plan, y0, z0):
    """0: tile column (y0, z0) runs one-step work in a two-step pass; 1: it
    runs on the two-step kernel's interior path; 2: on its guarded path (cells
    reach a grid face) -- for a plan without sources, probes or gradient
    region."""
    nx, ny, nz, ncp, ax = plan
    ax = ax if ncp else 0
    if not (0 <= y0 < ny and 0 <= z0 < nz):
        return 0
    if ax & 2 and (y0 - 2 < ncp or y0 + TY > ny - ncp - 1):
        return 0
    if ax & 4 and (z0 - 2 < ncp or z0 + TZ > nz - ncp - 1):
        return 0
    inner = y0 - 1 >= 1 and y0 + TY <= ny - 2 and z0 - 1 >= 1 and z0 + TZ <= nz - 2
    return 1 if inner else 2


def _two_step_xrange(plan):
    nx, ny, nz, ncp, ax = plan
    ncpx = ncp if (ncp and ax & 1) else 0
    return (ncpx + 1, nx - ncpx - 1) if ncpx else (0, nx)


TWO_STEP_CASES = CASES + [[(129, 129, 129, 0, 0)], [(117, 117, 117, 10, 7), (90, 200, 75, 8, 7)],
                          [(100, 90, 77, 10, 5), (64, 64, 64, 8, 1)]]


@pytest.mark.parametrize("case", range(len(TWO_STEP_CASES) + 4))
def test_two_step_tiles_stay_clear_and_store_what_one_step_work_reads(case):
    plans = (TWO_STEP_CASES[case] if case < len(TWO_STEP_CASES)
             else _random_plans(np.random.default_rng(200 + case), 4))
    items = _lists(plans, 7)
    cols = set()
    for code, y0, z0, xa, xb in items:
        q, mid = code & 0xFFFF, code >> 16
        plan = plans[q]
        nx = plan[0]
        kind = _two_step_column(plan, y0, z0)
        assert kind > 0, (plan, y0, z0)
        lo, hi = _two_step_xrange(plan)
        assert lo <= xa < xb <= hi
        cols.add((q, y0, z0))
        # first / last plane of the column's two-step range: one-step work
        # continues beyond it and reads that plane's intermediate state
        assert bool(mid & 2) == (xa == lo and lo > 0) and bool(mid & 4) == (xb == hi and hi < nx)
        ring = all(_two_step_column(plan, y0 + dy * TY, z0 + dz * TZ) > 0 or
                   not (0 <= y0 + dy * TY < plan[1] and 0 <= z0 + dz * TZ < plan[2])
                   for dy in (-1, 0, 1) for dz in (-1, 0, 1))
        assert bool(mid & 1) == (not ring)
        # the guarded path wherever a computed cell reaches a face or a guard
        assert bool(mid & 8) == (kind == 2 or xa < 2 or xb > nx - 2)
    # a plan large enough for it has two-step tiles; the one-step CPML-free
    # work of a pass keeps the CPML-free kernel's bounds
    for q, plan in enumerate(plans):
        nx, ny, nz, ncp, ax = plan
        lo, hi = _two_step_xrange(plan)
        any_col = any(_two_step_column(plan, y0, z0) for y0 in range(0, ny, TY) for z0 in range(0, nz, TZ))
        assert any(qq == q for (qq, _, _) in cols) == (any_col and hi - lo >= 8)
    for q, y0, z0, xa, xb in _lists(plans, 8):
        nx, ny, nz, ncp, ax = plans[q]
        if not ncp or not ax:
            continue
        assert not ((ax & 2) and _reaches(y0 - 1, y0 + TY - 1, ny, ncp))
        assert not ((ax & 4) and _reaches(z0 - 1, z0 + TZ - 1, nz, ncp))
        if ax & 1:
            assert xa >= ncp + 1 and xb <= nx - ncp


def test_bad_arguments_are_rejected():
    lib = _lib.load()
    n = C.c_int32()
    dims = (C.c_int32 * 5)(1, 10, 10, 0, 0)
    invalid = -1   # RFXB_E_INVALID
    assert lib.rfxb_debug_work_lists(1, dims, 100, 0, None, 0, C.byref(n)) == invalid
    dims = (C.c_int32 * 5)(20, 20, 20, 4, 7)
    assert lib.rfxb_debug_work_lists(1, dims, 100, 10, None, 0, C.byref(n)) == invalid
    assert lib.rfxb_debug_work_lists(1, dims, 100, 0, None, 0, C.byref(n)) == 0 and n.value > 0
    small = (C.c_int32 * 5)()
    assert lib.rfxb_debug_work_lists(1, dims, 100, 0, small, 1, C.byref(n)) == invalid
