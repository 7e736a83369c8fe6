"""Launch-configuration autotuner for plans and batched sweeps.

A plan or batch can launch its step kernels in several equivalent ways (the
``RfxbLaunchConfig`` fields of ``rfxb200.h``): the forward tiles split
between the CPML-free kernel and the staged-psi kernel on two streams or run
as one launch, which of the concurrent launches the captured graph hands to
the SMs first, whether the reverse step's CPML work without a y slab runs
on variant 4 or on variant 2, whether a persistent launch over device work
queues replaces the split launches, and the L2 promotion of the TMA boxes
(how much of a partly covered line a halo miss fetches; 64 B measured 1.6 %
faster than 128 B on the batched sweep and 2.8 % slower on a 513^3 PEC
grid).  Every setting computes the same steps; which
one is fastest depends on the workload (grid sizes, CPML share, number of
instances).  The autotuner times a few steps of each candidate with CUDA
events on the real workload, keeps the fastest, and caches the choice by a
workload signature (in memory, and in a JSON file when a path is given).

The reference has no counterpart: XLA schedules its scan body itself.
"""

from __future__ import annotations

import hashlib
import json
import os
from dataclasses import dataclass, field

# Reverse launch orders (rfxb200.h): permutations of (variant 4, variant 2,
# variant 3) by index.  Without variant 4 only the relative order of 2 and 3
# counts, so orders 0 (2 before 3) and 1 (3 before 2) represent all six.
REVERSE_ORDERS = ((4, 2, 3), (4, 3, 2), (2, 4, 3), (2, 3, 4), (3, 4, 2), (3, 2, 4))

_memory_cache: dict = {}


@dataclass
class TuneResult:
    """The chosen launch configuration and the measured milliseconds of
    every candidate (keyed by the candidate's fields as a tuple)."""
    config: dict
    forward_ms: dict = field(default_factory=dict)
    reverse_ms: dict = field(default_factory=dict)
    promo_ms: dict = field(default_factory=dict)
    cached: bool = False

    def as_json(self) -> dict:
        return {"config": self.config, "cached": self.cached,
                "forward_ms": {_key_str(k): v for k, v in self.forward_ms.items()},
                "reverse_ms": {_key_str(k): v for k, v in self.reverse_ms.items()},
                "l2_promo_ms": {_key_str(k): v for k, v in self.promo_ms.items()}}


def _key_str(k) -> str:
    return ",".join(f"{a}={b}" for a, b in k)


def forward_candidates(limits: dict, current: dict) -> list:
    """Forward settings to time: split with either launch order, the single
    launch, (where the target offers it) the persistent launch with 0, 1 or
    2 CPML-free-first CTAs per SM, and (where the target has two-step tiles)
    two-step passes, as far as the limits allow (the current setting first).
    The temporal-block depth is chosen here with the launches: 1 or 2 steps
    per pass over HBM."""
    c = []
    if limits["fwd_split"]:
        c += [{"fwd_split": 1, "fwd_order": 0}, {"fwd_split": 1, "fwd_order": 1}, {"fwd_split": 0, "fwd_order": 0}]
    else:
        c.append({"fwd_split": 0, "fwd_order": 0})
    cur = {"fwd_split": current["fwd_split"], "fwd_order": current["fwd_order"] if current["fwd_split"] else 0}
    np_ = limits.get("fwd_persist", 0)
    if np_:
        c = [dict(x, fwd_persist=0) for x in c]
        c += [{"fwd_split": 1, "fwd_order": 0, "fwd_persist": k} for k in range(1, np_ + 1)]
        k = current.get("fwd_persist", 0)
        cur = dict(cur, fwd_persist=k) if not k else {"fwd_split": 1, "fwd_order": 0, "fwd_persist": k}
    if limits.get("fwd_depth", 1) >= 2:
        # a two-step pass has its own lists; split and order only shape an
        # odd trailing step
        two = {"fwd_split": 1 if limits["fwd_split"] else 0, "fwd_order": 0}
        if np_:
            two["fwd_persist"] = 0
        two["fwd_depth"] = 2
        c = [dict(x, fwd_depth=1) for x in c] + [two]
        cur = dict(cur, fwd_depth=1) if (current.get("fwd_depth", 1) or 1) == 1 else two
    return [cur] + [x for x in c if x != cur]


def reverse_candidates(limits: dict, current: dict) -> list:
    """Reverse settings to time: every order with variant 4, and the two
    distinct orders without it, as far as the limits allow (the current
    setting first)."""
    c = []
    if limits["adj_order"] > 0:
        if limits["adj_lite"]:
            c += [{"adj_lite": 1, "adj_order": o} for o in range(len(REVERSE_ORDERS))]
        c += [{"adj_lite": 0, "adj_order": 0}, {"adj_lite": 0, "adj_order": 1}]
    else:
        c.append({"adj_lite": 0, "adj_order": 0})
    cur = {"adj_lite": current["adj_lite"], "adj_order": current["adj_order"]}
    if not cur["adj_lite"]:   # the representative of the current relative order of 2 and 3
        o = REVERSE_ORDERS[cur["adj_order"]]
        cur["adj_order"] = 0 if o.index(2) < o.index(3) else 1
    if limits.get("adj_persist", 0):
        # the persistent launch runs variants 2, 4 and 3 over all three lists
        c = [dict(x, adj_persist=0) for x in c] + [{"adj_lite": 1, "adj_order": 0, "adj_persist": 1}]
        cur = (dict(cur, adj_persist=0) if not current.get("adj_persist", 0)
               else {"adj_lite": 1, "adj_order": 0, "adj_persist": 1})
    if cur in c:
        c.remove(cur)
    elif limits["adj_order"] == 0:
        return c
    return [cur] + c


def pick(timings: dict, rel_margin: float = 0.01):
    """The fastest candidate, keeping the first (current) one unless another
    is faster by more than ``rel_margin`` (timing noise is not a reason to
    change)."""
    items = list(timings.items())
    first_k, first_t = items[0]
    best_k, best_t = min(items, key=lambda kv: kv[1])
    return best_k if best_t < first_t * (1.0 - rel_margin) else first_k


def cuda_timer(fn) -> float:
    """Milliseconds of ``fn()`` on the current stream, measured with CUDA events."""
    import torch
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    return float(a.elapsed_time(b))


def _time(fn, repeats, timer):
    fn()   # first call captures the step graphs of the new configuration
    return min(timer(fn) for _ in range(max(1, repeats)))


def _load_cache(path):
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def autotune(target, run_forward, run_reverse=None, *, signature=None, cache_path=None, repeats=2,
             timer=None, rel_margin=0.01) -> TuneResult:
    """Choose the launch configuration of ``target`` (a ``Plan`` or ``Batch``:
    anything with ``launch_config()`` and ``set_launch_config(**fields)``).

    ``run_forward()`` runs a few forward steps of the real workload and
    ``run_reverse()`` (optional) a few reverse steps; each is run once per
    candidate untimed (graph capture) and then ``repeats`` times timed, the
    minimum counting.  The forward fields are chosen first, then the reverse
    fields with the forward choice in place.  With a ``signature`` the choice
    is cached (and with ``cache_path`` stored as JSON) and reused without
    timing.  The target is left on the chosen configuration; its state after
    the trial steps is arbitrary, so the caller resets it before a real run.
    """
    timer = timer or cuda_timer
    key = None
    if signature is not None:
        key = hashlib.sha1(json.dumps(signature, sort_keys=True, default=str).encode()).hexdigest()
        hit = _memory_cache.get(key) or _load_cache(cache_path).get(key)
        if hit is not None:
            target.set_launch_config(**hit)
            _memory_cache[key] = dict(hit)
            return TuneResult(config=dict(hit), cached=True)
    current, limits = target.launch_config()
    res = TuneResult(config=dict(current))
    fc = forward_candidates(limits, current)
    if len(fc) > 1:
        for c in fc:
            target.set_launch_config(**c)
            res.forward_ms[tuple(sorted(c.items()))] = _time(run_forward, repeats, timer)
        best = dict(pick(res.forward_ms, rel_margin))
        target.set_launch_config(**best)
        res.config.update(best)
    rc = reverse_candidates(limits, current) if run_reverse is not None else []
    if len(rc) > 1:
        for c in rc:
            target.set_launch_config(**c)
            res.reverse_ms[tuple(sorted(c.items()))] = _time(run_reverse, repeats, timer)
        best = dict(pick(res.reverse_ms, rel_margin))
        target.set_launch_config(**best)
        res.config.update(best)
    # the L2 promotion of the TMA boxes, timed on the whole step (forward and
    # reverse together) with the chosen launches in place
    if limits.get("l2_promo", 0):
        cur_p = target.launch_config()[0]["l2_promo"]
        pc = [cur_p] + [v for v in range(limits["l2_promo"] + 1) if v != cur_p]

        def whole_step():
            a = run_forward()
            b = run_reverse() if run_reverse is not None else None
            # runs that report a time (stand-in timers) add up; real runs
            # return arrays or nothing and are timed with CUDA events
            if isinstance(a, (int, float)) and isinstance(b, (int, float, type(None))):
                return float(a) + float(b or 0.0)
            return None
        for v in pc:
            target.set_launch_config(l2_promo=v)
            res.promo_ms[(("l2_promo", v),)] = _time(whole_step, repeats, timer)
        best = dict(pick(res.promo_ms, rel_margin))
        target.set_launch_config(**best)
    res.config = target.launch_config()[0]
    if key is not None:
        _memory_cache[key] = dict(res.config)
        if cache_path:
            data = _load_cache(cache_path)
            data[key] = dict(res.config)
            tmp = cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, cache_path)
    return res
