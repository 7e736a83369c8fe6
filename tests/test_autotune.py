"""Launch-configuration autotuner: the search and cache logic on CPU (a fake
plan/batch whose step time depends on its configuration), and on the GPU
that every launch configuration of a batched sweep computes the same
objective and gradient, batched and unbatched alike."""

import json

import numpy as np
import pytest

from rfx_b200 import autotune as at


class FakeTarget:
    """Stands in for a Plan / Batch: launch_config() / set_launch_config()."""

    def __init__(self, limits, current=None):
        self.limits = dict(limits)
        self.cur = dict(current or {"fwd_split": limits["fwd_split"], "fwd_order": 0,
                                    "adj_lite": limits["adj_lite"], "adj_order": 0})
        self.sets = 0

    def launch_config(self):
        return dict(self.cur), dict(self.limits)

    def set_launch_config(self, **f):
        for k, v in f.items():
            assert 0 <= v <= self.limits[k], (k, v)
        self.cur.update(f)
        self.sets += 1


FULL = {"fwd_split": 1, "fwd_order": 1, "adj_lite": 1, "adj_order": 5}


def _timer_for(target, fwd_ms, rev_ms):
    """A timer that reads the fake target's configuration: forward calls cost
    fwd_ms(config), reverse calls rev_ms(config)."""
    def timer(fn):
        return fn()
    calls = {"n": 0}

    def run_forward():
        calls["n"] += 1
        return fwd_ms(target.cur)

    def run_reverse():
        calls["n"] += 1
        return rev_ms(target.cur)
    return timer, run_forward, run_reverse, calls


def test_candidates_cover_the_limits():
    cur = {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0}
    f = at.forward_candidates(FULL, cur)
    assert f[0] == {"fwd_split": 1, "fwd_order": 0}
    assert sorted(map(lambda d: tuple(d.values()), f)) == [(0, 0), (1, 0), (1, 1)]
    r = at.reverse_candidates(FULL, cur)
    assert r[0] == {"adj_lite": 1, "adj_order": 0}
    assert len(r) == 6 + 2 and len({tuple(d.values()) for d in r}) == 8
    # no split and no variant 4: nothing to choose
    none = {"fwd_split": 0, "fwd_order": 0, "adj_lite": 0, "adj_order": 0}
    assert at.forward_candidates(none, none) == [{"fwd_split": 0, "fwd_order": 0}]
    assert at.reverse_candidates(none, none) == [{"adj_lite": 0, "adj_order": 0}]
    # a target with the persistent launches: three more forward candidates
    # (0, 1, 2 CPML-free-first CTAs per SM) and one more reverse candidate
    full_p = dict(FULL, fwd_persist=3, adj_persist=1)
    cur_p = {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0, "fwd_persist": 0, "adj_persist": 0}
    f = at.forward_candidates(full_p, cur_p)
    assert f[0] == {"fwd_split": 1, "fwd_order": 0, "fwd_persist": 0} and len(f) == 6
    assert {d["fwd_persist"] for d in f} == {0, 1, 2, 3}
    r = at.reverse_candidates(full_p, cur_p)
    assert r[0] == {"adj_lite": 1, "adj_order": 0, "adj_persist": 0} and len(r) == 9
    assert r[-1] == {"adj_lite": 1, "adj_order": 0, "adj_persist": 1}
    cur_p2 = dict(cur_p, fwd_persist=2, adj_persist=1)
    assert at.forward_candidates(full_p, cur_p2)[0] == {"fwd_split": 1, "fwd_order": 0, "fwd_persist": 2}
    assert at.reverse_candidates(full_p, cur_p2)[0] == {"adj_lite": 1, "adj_order": 0, "adj_persist": 1}
    # split reverse without variant 4: the two relative orders of 2 and 3
    lim = {"fwd_split": 0, "fwd_order": 0, "adj_lite": 0, "adj_order": 5}
    cur = {"fwd_split": 0, "fwd_order": 0, "adj_lite": 0, "adj_order": 4}   # (3, 4, 2): 3 before 2
    r = at.reverse_candidates(lim, cur)
    assert r == [{"adj_lite": 0, "adj_order": 1}, {"adj_lite": 0, "adj_order": 0}]


def test_depth_candidates_and_choice():
    """With two-step tiles (fwd_depth limit 2) the forward search adds one
    two-step candidate (no persistent launch) and keeps depth 1 unless two
    steps per pass are faster by more than the margin."""
    lim = dict(FULL, fwd_persist=3, adj_persist=1, fwd_depth=2)
    cur = {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0, "fwd_persist": 0, "adj_persist": 0,
           "fwd_depth": 1}
    f = at.forward_candidates(lim, cur)
    assert f[0] == {"fwd_split": 1, "fwd_order": 0, "fwd_persist": 0, "fwd_depth": 1} and len(f) == 7
    assert [d for d in f if d["fwd_depth"] == 2] == [{"fwd_split": 1, "fwd_order": 0, "fwd_persist": 0,
                                                       "fwd_depth": 2}]
    assert all(d["fwd_persist"] == 0 for d in f if d["fwd_depth"] == 2)
    # the current setting on two-step passes comes first
    f2 = at.forward_candidates(lim, dict(cur, fwd_depth=2))
    assert f2[0]["fwd_depth"] == 2 and len(f2) == 7
    for gain, want in ((0.3, 2), (0.005, 1)):
        t = FakeTarget(lim, dict(cur))
        fwd = lambda c, g=gain: 10.0 * (1.0 - g * (c.get("fwd_depth", 1) == 2))
        timer, rf, rr, _ = _timer_for(t, fwd, lambda c: 20.0)
        res = at.autotune(t, rf, rr, timer=timer, repeats=1)
        assert res.config["fwd_depth"] == want and t.cur["fwd_depth"] == want


def test_picks_the_fastest_configuration():
    t = FakeTarget(FULL)
    fwd = lambda c: 10.0 - 3.0 * (c["fwd_split"] == 1 and c["fwd_order"] == 1)
    rev = lambda c: 20.0 - 5.0 * (c["adj_lite"] == 1 and c["adj_order"] == 3)
    timer, rf, rr, _ = _timer_for(t, fwd, rev)
    res = at.autotune(t, rf, rr, timer=timer, repeats=1)
    assert res.config == {"fwd_split": 1, "fwd_order": 1, "adj_lite": 1, "adj_order": 3}
    assert t.cur == res.config
    assert min(res.forward_ms.values()) == 7.0 and min(res.reverse_ms.values()) == 15.0
    assert len(res.forward_ms) == 3 and len(res.reverse_ms) == 8


def test_l2_promotion_stage_times_the_whole_step():
    """With an l2_promo limit the tuner times every promotion on the forward
    and reverse runs together, after choosing the launches, current setting
    first, and keeps the fastest."""
    lim = dict(FULL, l2_promo=3)
    cur = {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0, "l2_promo": 2}
    t = FakeTarget(lim, cur)
    fwd = lambda c: 10.0 - (1.0 if c["l2_promo"] == 1 else 0.0)
    rev = lambda c: 20.0 - (2.0 if c["l2_promo"] == 1 else 0.0)
    timer, rf, rr, _ = _timer_for(t, fwd, rev)
    res = at.autotune(t, rf, rr, timer=timer, repeats=1)
    assert list(res.promo_ms)[0] == (("l2_promo", 2),) and len(res.promo_ms) == 4
    assert res.promo_ms[(("l2_promo", 1),)] == 27.0 and res.promo_ms[(("l2_promo", 2),)] == 30.0
    assert res.config["l2_promo"] == 1 and t.cur["l2_promo"] == 1


def test_noise_does_not_move_the_current_configuration():
    t = FakeTarget(FULL)
    # the alternatives are faster by 0.5 %, inside the 1 % margin
    fwd = lambda c: 10.0 if (c["fwd_split"], c["fwd_order"]) == (1, 0) else 9.95
    rev = lambda c: 20.0 if (c["adj_lite"], c["adj_order"]) == (1, 0) else 19.9
    timer, rf, rr, _ = _timer_for(t, fwd, rev)
    res = at.autotune(t, rf, rr, timer=timer, repeats=1)
    assert res.config == {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0}


def test_nothing_to_choose_runs_nothing():
    lim = {"fwd_split": 0, "fwd_order": 0, "adj_lite": 0, "adj_order": 0}
    t = FakeTarget(lim)
    timer, rf, rr, calls = _timer_for(t, lambda c: 1.0, lambda c: 1.0)
    res = at.autotune(t, rf, rr, timer=timer)
    assert calls["n"] == 0 and res.forward_ms == {} and res.reverse_ms == {}


def test_cache_by_signature(tmp_path, monkeypatch):
    monkeypatch.setattr(at, "_memory_cache", {})
    path = str(tmp_path / "tune.json")
    sig = {"device": "fake", "instances": [((30, 30, 30), "xyz", "")]}
    t = FakeTarget(FULL)
    fwd = lambda c: 5.0 if c["fwd_split"] == 0 else 9.0
    rev = lambda c: 5.0 if c["adj_order"] == 2 and c["adj_lite"] == 1 else 9.0
    timer, rf, rr, calls = _timer_for(t, fwd, rev)
    res = at.autotune(t, rf, rr, signature=sig, cache_path=path, timer=timer, repeats=1)
    assert not res.cached and res.config["fwd_split"] == 0 and res.config["adj_order"] == 2
    stored = json.load(open(path))
    assert list(stored.values()) == [res.config]
    # a new process (empty memory cache) and a fresh target: no timing, same choice
    monkeypatch.setattr(at, "_memory_cache", {})
    t2 = FakeTarget(FULL)
    timer2, rf2, rr2, calls2 = _timer_for(t2, fwd, rev)
    res2 = at.autotune(t2, rf2, rr2, signature=sig, cache_path=path, timer=timer2)
    assert res2.cached and calls2["n"] == 0 and t2.cur == res.config
    # another workload is tuned anew
    res3 = at.autotune(FakeTarget(FULL), rf2, rr2, signature={"device": "fake", "instances": []},
                       cache_path=path, timer=timer2, repeats=1)
    assert not res3.cached and len(json.load(open(path))) == 2


def test_launch_config_bindings_validate_fields():
    from rfx_b200 import engine

    class Lib:
        def __init__(self):
            self.cur = engine.RfxbLaunchConfig(1, 0, 1, 0)
            self.lim = engine.RfxbLaunchConfig(1, 1, 0, 5)

        def get(self, h, cur, lim):
            cur._obj.fwd_split, cur._obj.fwd_order, cur._obj.adj_lite, cur._obj.adj_order = (
                self.cur.fwd_split, self.cur.fwd_order, self.cur.adj_lite, self.cur.adj_order)
            lim._obj.fwd_split, lim._obj.fwd_order, lim._obj.adj_lite, lim._obj.adj_order = (
                self.lim.fwd_split, self.lim.fwd_order, self.lim.adj_lite, self.lim.adj_order)
            return 0

        def set(self, h, cfg):
            self.cur = engine.RfxbLaunchConfig(cfg._obj.fwd_split, cfg._obj.fwd_order, cfg._obj.adj_lite,
                                               cfg._obj.adj_order)
            return 0

    lib = Lib()
    lib.get.__func__.__name__ = "rfxb_batch_launch_config"
    cur, lim = engine._get_launch(lib.get, None)
    assert cur == {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0, "fwd_persist": 0, "adj_persist": 0,
                   "l2_promo": 0, "fwd_depth": 0}
    assert lim["adj_order"] == 5
    engine._set_launch(lib.get, lib.set, None, {"adj_order": 3})
    assert engine._get_launch(lib.get, None)[0]["adj_order"] == 3
    with pytest.raises(ValueError):
        engine._set_launch(lib.get, lib.set, None, {"tile": 2})


# ---------------------------------------------------------------------------
# GPU: every configuration computes the same sweep


def _small_sweep(batched):
    import torch
    from rfx_b200.batch import Sweep
    from rfx_b200.workloads import batched_sweep
    insts = batched_sweep(seed=3, n_inst=3, n_steps=120, n_lo=40, n_hi=72)
    return Sweep(insts, 120, device=torch.device("cuda", 0), batched=batched)


def _run(sw):
    Js, grads = sw.run()
    sw.check_device()
    return np.array([float(j) for j in Js]), [g.detach().cpu().numpy().copy() for g in grads]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
def test_every_launch_configuration_gives_the_same_sweep(cuda):
    sw = _small_sweep(True)
    try:
        J0, g0 = _run(sw)
        _, lim = sw.batch.launch_config()
        configs = [{"fwd_order": 1}, {"adj_order": 3}, {"adj_order": 5}]
        if lim["fwd_split"]:
            configs.append({"fwd_split": 0})
        if lim["adj_lite"]:
            configs.append({"adj_lite": 0, "adj_order": 1})
        assert lim["fwd_persist"] >= 1 and lim["adj_persist"] == 1
        # the persistent launches run the same kernel variants on the same
        # lists: bit-identical to the split launches
        configs += [{"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0, "fwd_persist": k,
                     "adj_persist": 1} for k in range(1, lim["fwd_persist"] + 1)]
        configs.append({"fwd_persist": 0, "adj_persist": 0})
        # the L2 promotion of the TMA boxes moves no value
        assert lim["l2_promo"] == 3
        configs += [{"l2_promo": v} for v in (0, 1, 3, 2)]
        # two steps per pass compute every cell with the same rounding
        configs += [{"fwd_depth": 2}, {"fwd_depth": 1}]
        for c in configs:
            if any(v > lim[k] for k, v in c.items()):
                continue
            sw.batch.set_launch_config(**c)
            J, g = _run(sw)
            order_only = (set(c) <= {"fwd_order", "adj_order", "l2_promo", "fwd_depth"}
                          or c.get("fwd_persist", 0) > 0 or c == {"fwd_persist": 0, "adj_persist": 0})
            for a, b in zip(g, g0):
                # the launch order cannot change a value; another kernel
                # variant on the same tiles may round differently
                assert _rel(a, b) <= (0.0 if order_only else 1e-6), c
            assert _rel(J, J0) <= (0.0 if order_only else 1e-6), c
        res = sw.autotune(trial_steps=16, repeats=1)
        cur, lim = sw.batch.launch_config()
        assert cur == res.config and all(0 <= cur[k] <= lim[k] for k in cur)
        J, g = _run(sw)
        for a, b in zip(g, g0):
            assert _rel(a, b) <= 1e-6
    finally:
        sw.close()


@pytest.mark.gpu
def test_batched_sweep_matches_single_plans(cuda):
    a, b = _small_sweep(True), _small_sweep(False)
    try:
        Ja, ga = _run(a)
        Jb, gb = _run(b)
        assert _rel(Ja, Jb) <= 1e-6
        for x, y in zip(ga, gb):
            assert _rel(x, y) <= 1e-5
            assert np.isfinite(x).all() and np.abs(x).max() > 0
    finally:
        a.close()
        b.close()


def test_l2_promotion_stage_accepts_runs_that_return_arrays():
    """The real runs return probe traces (arrays) or nothing; the whole-step
    closure of the promotion stage must not combine them."""
    lim = dict(FULL, l2_promo=3)
    t = FakeTarget(lim, {"fwd_split": 1, "fwd_order": 0, "adj_lite": 1, "adj_order": 0, "l2_promo": 2})
    calls = {"n": 0}

    def run_forward():
        calls["n"] += 1
        return np.zeros((4, 2))

    def run_reverse():
        calls["n"] += 1

    res = at.autotune(t, run_forward, run_reverse, timer=lambda fn: (fn(), 1.0)[1], repeats=1)
    assert len(res.promo_ms) == 4 and res.config["l2_promo"] == 2 and calls["n"] > 0
