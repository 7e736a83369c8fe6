"""Benchmark of the rfx time-stepping hot path on B200.

Workload (default, the configuration the metric names): a batched design
sweep -- 64 independent simulations of uneven size (n^3 interior, n ~ U{64..160}
seeded, CPML 8, +1 fence -> (n+17)^3 cells, 161 M cells in total for seed 0),
each with 8 seeded dielectric boxes, a 16x16x2 design region, an Ez 12 GHz
soft source and 4 Ez probes, 2000 time steps; one bench step = forward of all
64 (one step-kernel launch per time step for the whole batch) + per-instance
probe-DFT objective + hand-written adjoint sweep giving dJ/d eps_r over every
design region.  Metric: Mcell-steps/s = total cells x time steps / time,
counting forward+adjoint once.  Inputs are seeded synthetic data with the
configuration's shapes (the reference publishes no dataset).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N GPUs (``--gpus N``; launched under torchrun, or re-launched under it
by this script) the sweep has 64 x N instances drawn from seed 0 and each rank
takes a cell-balanced share (``rfx_b200.distributed.shard_instances``) of them:
independent instances, no data-path collective, weak scaling.  The time is
the max over ranks and ``value`` counts the cells of every rank's share.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import re
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s fwd+adjoint grad, batched vs single, 1 B200; % HBM roofline"
UNIT = "Mcell-steps/s"


def _sweep_cells(args, world=1):
    """Cells of the whole sweep at ``world`` GPUs."""
    from rfx_b200.workloads import batched_sweep_cells
    return batched_sweep_cells(seed=0, n_inst=args.instances * world)


def _workload_config(args, cells, world):
    """``cells``: all ranks' cells together."""
    n_all = args.instances * world
    return {"workload": f"batched_sweep: {n_all} instances (n+17)^3, n~U{{64..160}} seed 0, "
                        f"CPML 8, {args.time_steps} time steps, forward + probe-DFT objective + adjoint "
                        f"dJ/d eps_r over 16x16x2 regions",
            "instances_per_gpu": args.instances, "time_steps": args.time_steps,
            "cells_total": int(cells), "adjoint_mode": "history (design-region E^n and curl H recorded in HBM)",
            "l2": f"inputs larger than L2 (a step reads the fields and coefficients of {cells / world / 1e6:.1f} M "
                  f"cells per GPU, {cells / world * 32 / 1e9:.2f} GB)",
            "parallelism": (f"{n_all} independent instances sharded over {world} GPUs by cells "
                            f"(rfx_b200.distributed.shard_instances), no data-path collective"
                            if world > 1 else "independent instances x 1 GPU")}


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.1)

    def __enter__(self):
        if self.nv is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv is not None:
            self.t.join(timeout=2)

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU baselines (the oracle port; never part of the measured GPU path)
# ---------------------------------------------------------------------------

def _oracle_sample(args_tuple):
    """Forward + adjoint of one instance on the oracle for a few time steps."""
    q, n_time, seed, n_inst = args_tuple
    import oracle  # noqa: F401
    from oracle.adjoint import forward_adjoint
    from oracle.fdtd import make_uniform_grid
    from rfx_b200.workloads import batched_sweep
    inst = batched_sweep(seed=seed, n_inst=n_inst, n_steps=n_time)[q]
    g = inst.grid
    og = make_uniform_grid(g.domain, g.dx, cpml_layers=g.cpml_layers)
    assert og.shape == tuple(g.shape)
    mats = (inst.eps_r, inst.sigma, np.ones(g.shape, np.float32))
    freqs = inst.freqs
    dt = g.dt

    def obj_grad(ts):
        n = np.arange(ts.shape[0])
        ph = np.exp(-2j * np.pi * freqs[:, None] * n[None, :] * dt) * dt
        X = ph @ ts.astype(np.float64)
        return 2.0 * np.real(np.conj(X)[:, None, :] * ph[:, :, None]).sum(0)

    t0 = time.perf_counter()
    forward_adjoint(og, mats, n_time, boundary="cpml", pec_axes="", sources=inst.sources, probes=inst.probes,
                    box=inst.box, objective_grad=obj_grad, dtype=np.float32)
    dt_s = time.perf_counter() - t0
    return int(np.prod(g.shape)) * n_time, dt_s


def _smallest(n_inst, seed):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(64, 161, n_inst)
    return int(np.argmin(sizes)), int(sizes.min())


def cpu_baseline_port(args, n_workers=1, n_time=60):
    q, n = _smallest(args.instances, 0)
    jobs = [(q, n_time, 0, args.instances)] * n_workers
    t0 = time.perf_counter()
    if n_workers == 1:
        res = [_oracle_sample(jobs[0])]
    else:
        with mp.get_context("spawn").Pool(n_workers) as pool:
            res = pool.map(_oracle_sample, jobs)
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    return {"value": work / wall / 1e6, "unit": UNIT, "cores": n_workers, "kind": "port",
            "sample": f"{n_workers} x instance {q} of seed 0 ({n + 17}^3 cells), {n_time} time steps, forward + "
                      f"adjoint on the NumPy float32 oracle (the reference's own JAX solver is not installable "
                      f"here), timed on the host"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def _traffic_per_cell(kernel, key="small_case_dram_bytes_per_cell_per_step"):
    """DRAM bytes per cell and time step of a step kernel (all its launches
    of one step), measured by ncu on the 4-instance case of the same sweep
    (committed in profiles/<kernel>.md as ``key: value``) and scaled by cells
    to the workload; None if the summary has no such line."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.md")
    if not os.path.exists(path):
        return None
    m = re.search(re.escape(key) + r":\s*([0-9.eE+-]+)", open(path).read())
    return float(m.group(1)) if m else None


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from rfx_b200.batch import Sweep
    from rfx_b200.workloads import batched_sweep

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    if world > 1:
        from rfx_b200.distributed import shard_instances
        from rfx_b200.workloads import batched_sweep_instance_cells
        n_all = args.instances * world
        mine = shard_instances(batched_sweep_instance_cells(seed=0, n_inst=n_all), world)[rank]
        insts = batched_sweep(seed=0, n_inst=n_all, n_steps=args.time_steps, subset=mine)
    else:
        insts = batched_sweep(seed=0, n_inst=args.instances, n_steps=args.time_steps)
    sw = Sweep(insts, args.time_steps, device=dev, batched=True)
    cells = sw.cells()
    total_cells = cells
    if world > 1:
        tc = torch.tensor([float(cells)], device=dev, dtype=torch.float64)
        dist.all_reduce(tc, op=dist.ReduceOp.SUM)
        total_cells = int(tc.item())
    N = args.time_steps
    stream = torch.cuda.current_stream()
    # launch configuration chosen by the autotuner (trial steps of this
    # workload, before the warm-up; the first forward resets the state)
    launch = None
    if not args.no_autotune:
        tune = sw.autotune(trial_steps=min(32, N), repeats=2)
        launch = {"chosen_by": "rfx_b200.autotune (32 trial steps per candidate)", **tune.as_json()}
    else:
        launch = {"chosen_by": "defaults", "config": sw.batch.launch_config()[0]}

    def one_step():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sw.forward()
        e1.record(stream)
        _, gs = sw.objectives()
        e2.record(stream)
        sw.backward(gs)
        e3.record(stream)
        return e0, e1, e2, e3

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    events = []
    with ClockSampler(local_rank) as clk:
        t_host0 = time.perf_counter()
        for _ in range(args.steps):
            events.append(one_step())
        torch.cuda.synchronize()
        t_host = time.perf_counter() - t_host0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = sum(a.elapsed_time(d) for a, b, c, d in events)
    fwd_ms = sum(a.elapsed_time(b) for a, b, c, d in events)
    adj_ms = sum(c.elapsed_time(d) for a, b, c, d in events)
    t = torch.tensor([total_ms, fwd_ms, adj_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, fwd_ms, adj_ms = float(t[0]), float(t[1]), float(t[2])
    value = total_cells * N * args.steps / (total_ms / 1e3) / 1e6

    # rooflines of the two step kernels: algorithmic bytes per launch over the
    # average launch time (one launch per time step in each phase; the
    # backward phase also holds one adjoint-init launch per bench step)
    def roof(kernel, alg, ms, what, key="small_case_dram_bytes_per_cell_per_step"):
        step_s = ms / 1e3 / (N * args.steps)
        achieved = alg / step_s / 1e9
        tpc = _traffic_per_cell(kernel, key)
        return {"kernel": kernel, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(achieved / hbm_peak, 4),
                "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs, burst copy)",
                "traffic": (round(tpc * cells) if tpc else None), "algorithmic_bytes_per_step": int(alg),
                "share_of_step": round(ms / total_ms, 3), "what": what}

    roof_adj = roof("adj_step_kernel", sum(p.adjoint_algorithmic_bytes_per_step() for p in sw.plans), adj_ms,
                    "fused reverse step, batched over all instances: variant 2 on the tiles that reach a y slab, "
                    "variant 4 on the other CPML work, variant 3 on the plain tiles, three streams; one step = "
                    "the three launches")
    two_step = (sw.batch or sw.plans[0]).launch_config()[0].get("fwd_depth", 1) == 2
    if two_step:
        roof_fwd = roof("fwd_step_kernel", sum(p.algorithmic_bytes_per_step() for p in sw.plans), fwd_ms,
                        "forward in two-step passes, batched over all instances: fwd2_step_kernel advances the "
                        "tiles clear of CPML, sources, probes and the gradient region two steps per read of the "
                        "state, beside two launches of variant 2 (CPML tiles) and variant 1 (the other CPML-free "
                        "work) per pass; algorithmic bytes counted per step",
                        key="small_case_dram_bytes_per_cell_per_step_two_step")
    else:
        roof_fwd = roof("fwd_step_kernel", sum(p.algorithmic_bytes_per_step() for p in sw.plans), fwd_ms,
                        "fused forward step, batched over all instances: variant 2 on the CPML tiles and variant 1 "
                        "on the plain tiles, two streams; one step = both launches")
    roofline, roofline_other = (roof_adj, roof_fwd) if adj_ms >= fwd_ms else (roof_fwd, roof_adj)

    # single-instance comparison (each simulation launched on its own)
    single = None
    if rank == 0 and not args.no_single:
        sw1 = Sweep(insts, N, device=dev, batched=False)
        sw1.forward()
        _, gs = sw1.objectives()
        sw1.backward(gs)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sw1.forward()
        _, gs = sw1.objectives()
        sw1.backward(gs)
        b.record(stream)
        torch.cuda.synchronize()
        sms = a.elapsed_time(b)
        single_rate = cells * N / (sms / 1e3) / 1e6
        batched_rate = cells * N * args.steps / (total_ms / 1e3) / 1e6
        single = {"value": round(single_rate, 1), "unit": UNIT,
                  "what": f"same {args.instances} simulations, forward+adjoint launched one simulation at a time",
                  "batched_over_single": round(batched_rate / single_rate, 3)}
        sw1.close()

    # end to end through the public API with host buffers: upload every
    # instance's eps_r / sigma from pinned host memory, run, read J and grads back
    e2e = None
    if not args.no_e2e:
        host_eps = [torch.from_numpy(s.eps_r).pin_memory() for s in insts]
        host_sig = [torch.from_numpy(s.sigma).pin_memory() for s in insts]
        h2d = sum(x.numel() * 4 for x in host_eps) + sum(x.numel() * 4 for x in host_sig)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        d2h = 0
        a.record(stream)
        for _ in range(args.steps):
            sw.set_materials([x.to(dev, non_blocking=True) for x in host_eps],
                             [x.to(dev, non_blocking=True) for x in host_sig])
            Js, grads = sw.run()
            outs = [g.to("cpu", non_blocking=True) for g in grads] + [torch.stack(Js).to("cpu", non_blocking=True)]
            d2h = sum(o.numel() * o.element_size() for o in outs)
        b.record(stream)
        torch.cuda.synchronize()
        ems = a.elapsed_time(b)
        et = torch.tensor([ems], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e = {"value": round(total_cells * N * args.steps / (float(et[0]) / 1e3) / 1e6, 1), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "rfx_b200.batch.Sweep.set_materials + run (host pinned eps_r/sigma in, J and dJ/d eps_r out)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_port(args, n_workers=1, n_time=args.cpu_time_steps)

    # our kernels per bench step: N forward steps, one adjoint init per
    # simulation launch group, N reverse steps, each step as many step-kernel
    # launches as the library reports (CPML / plain split, variant 4; per
    # pass of two steps with two-step passes)
    fl, rl = sw.step_launches()
    cfg = (sw.batch or sw.plans[0]).launch_config()[0]
    launches = args.steps * (forward_launches(fl, cfg, N) + N * rl + (1 if sw.batch is not None else len(sw.plans)))
    sw.close()

    # the other configurations, each timed on its own full step count (one
    # GPU): large uniform, graded, adjoint with checkpoints every 64 steps
    secondary = None
    if rank == 0 and world == 1 and not args.no_secondary:
        secondary = {}
        for name, n_t in (("large_uniform", 4000), ("graded", 6000), ("adjoint_region", 3000),
                          ("pec_uniform", 1000)):
            sargs = argparse.Namespace(**vars(args))
            sargs.time_steps = n_t
            sargs.steps = 2
            sargs.warmup = max(3, min(args.warmup, 3))
            torch.cuda.empty_cache()
            sl = run_secondary(sargs, name, emit=False)
            secondary[name] = {k: sl[k] for k in ("metric", "value", "unit", "steps", "warmup", "ms_per_step",
                                                  "config", "roofline", "launch", "clocks", "e2e", "vs_baseline",
                                                  "baseline") if k in sl}
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 2), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": _workload_config(args, total_cells, world), "roofline": roofline,
                "roofline_other_kernel": roofline_other, "cpu_baseline": cpu,
                "e2e": e2e, "single": single, "gpu_launches": launches, "launch": launch,
                "clocks": clk.summary(), "host_wall_s_timed": round(t_host, 3), "secondary": secondary}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, rank, world):
    if rank != 0:
        return
    workers = max(1, min(len(os.sched_getaffinity(0)), 16))
    vals = []
    for _ in range(args.warmup):
        cpu_baseline_port(args, n_workers=workers, n_time=args.ref_time_steps)
    for _ in range(args.steps):
        vals.append(cpu_baseline_port(args, n_workers=workers, n_time=args.ref_time_steps))
    v = statistics.mean(x["value"] for x in vals)
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": _workload_config(args, _sweep_cells(args, world), world), "cpu_baseline": cb,
            "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference = NumPy float32 restatement of rfx's scan body and its transpose (oracle port); "
                    "rfx itself needs JAX, which is not installable offline here"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# secondary workloads (the other configurations, on request)
# ---------------------------------------------------------------------------

def run_secondary(args, which, emit=True):
    """One device-timed line for the large uniform, graded or adjoint
    configuration: each bench step runs the configuration's full step count.
    Prints it (``emit``) or returns it."""
    import torch

    from rfx_b200 import workloads
    from rfx_b200.grid import face_pads
    from rfx_b200.simulation import MaterialArrays, init_dft_plane_probe, prepare_device_run

    torch.cuda.set_device(0)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    N = args.time_steps
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    if which == "pec_uniform":
        return run_pec_uniform(args, emit, hbm_peak, peak_src)
    if which in ("large_uniform", "graded"):
        if which == "large_uniform":
            g, eps, sig, src, probes, dft = workloads.large_uniform(n_steps=N)
            pec, axes, offset = None, "xyz", 1
            desc = ("large_uniform: 256^3 interior dx 1 mm + CPML 10 -> 277^3, 32 seeded boxes, Ez pulse 10 GHz, "
                    "8 probes, z-plane DFT at 16 frequencies")
        else:
            g, eps, sig, pec, src, probes, dft = workloads.graded(n_steps=N)
            pads = face_pads(g)
            axes = "".join(a for a, (lo, hi) in zip("xyz", (pads[0:2], pads[2:4], pads[4:6])) if lo + hi > 0)
            offset = 0
            desc = ("graded: 192 x 192 x 96 cells, z graded 0.1-0.5 mm, CPML 12 -> 217 x 217 x 121, PEC sheet, "
                    "substrate, Ex pulse 20 GHz, 4 probes, DFT plane at 8 frequencies")
        planes = [init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in dft]
        mats = MaterialArrays(eps, sig, np.ones_like(eps))
        r = prepare_device_run(g, mats, N, cpml_axes=axes, pec_axes="xyz", sources=src,
                               probes=[p[:4] for p in probes], dft_planes=planes, pec_mask=pec,
                               dft_time_offset=offset)
        plan = r.plan
        cells = int(np.prod(g.shape))

        def one():
            plan.reset()
            for a in r.dft_accs:
                a.zero_()
            plan.advance(0, N, r.src_table, r.probe_out, r.dft_accs, r.dft_phases)

        dft_bytes = sum(32 * len(d.freqs) * int(np.prod(a.shape[1:])) for d, a in zip(planes, r.dft_accs))
        alg = plan.algorithmic_bytes_per_step() + dft_bytes
        metric = "Mcell-steps/s forward, 1 B200"
        kernel = "fwd_step_kernel + dft_kernel (whole step)"
    else:
        from rfx_b200.adjoint import AdjointRunner, probe_dft_objective
        g, eps, sig, src, probes, box, freqs = workloads.adjoint_region(n_steps=N)
        runner = AdjointRunner(g, MaterialArrays(eps, sig, np.ones_like(eps)), N, sources=src, probes=probes, box=box,
                               boundary="cpml", cpml_axes="xyz", pec_axes="xyz", mode="segments",
                               checkpoint_every=64)
        plan = runner.plan
        cells = int(np.prod(g.shape))
        desc = ("adjoint_region: 200 x 120 x 48 at 0.5 mm + CPML 10 -> 221 x 141 x 69, design 64 x 64 x 2, "
                "Ez pulse 15 GHz, 4 probes, objective over 5 frequencies, checkpoint every 64 steps")

        def one():
            ts = runner.forward()
            t = ts.detach().clone().requires_grad_(True)
            probe_dft_objective(t, freqs, float(g.dt)).backward()
            runner.backward(t.grad.to(torch.float32).contiguous())

        # forward + segment recompute + reverse step, each ~ one forward's bytes
        alg = 3 * plan.algorithmic_bytes_per_step()
        metric = "Mcell-steps/s fwd+adjoint grad (checkpoint every 64), 1 B200"
        kernel = "fwd_step_kernel x2 + adj_step_kernel (whole step)"
    # launch configuration of this plan chosen by the autotuner (trial runs
    # before the warm-up; every timed run starts from a reset state)
    launch = {"chosen_by": "defaults", "config": plan.launch_config()[0]}
    if not args.no_autotune:
        from rfx_b200.autotune import autotune
        if which == "adjoint_region":
            res = autotune(plan, lambda: runner.forward(), one, repeats=1)
            launch = {"chosen_by": "rfx_b200.autotune (whole forward / forward + adjoint runs per candidate)",
                      **res.as_json()}
        else:
            T = min(64, N)
            res = autotune(plan, lambda: plan.advance(0, T, r.src_table, r.probe_out, r.dft_accs, r.dft_phases),
                           None, repeats=2)
            launch = {"chosen_by": f"rfx_b200.autotune ({T} trial steps per candidate)", **res.as_json()}
    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        ev[0].record()
        for _ in range(args.steps):
            one()
        ev[1].record()
        torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1])
    variant = {"forward": plan.forward_variant(), "reverse": plan.adjoint_variant()}
    step_s = ms / 1e3 / (args.steps * N)
    achieved = alg / step_s / 1e9
    line = {"metric": metric, "value": round(cells * N * args.steps / (ms / 1e3) / 1e6, 1), "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": desc, "time_steps": N, "cells": cells, "kernel_variants": variant,
                       "l2": "inputs larger than L2"},
            "roofline": {"kernel": kernel, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4), "peak_source": peak_src,
                         "traffic": None, "algorithmic_bytes_per_step": int(alg)},
            "launch": launch, "clocks": clk.summary()}
    plan.close()
    if emit:
        print(json.dumps(line), flush=True)
    return line


PUBLISHED_GPU_MCELLS = 7309.0   # README.md:28 of the reference: RTX 4090, rfx.gpu.benchmark (PEC-only run())


def forward_launches(per_step, cfg, n):
    """Forward step-kernel launches of n steps.  ``per_step`` is the
    library's count (``step_launches()[0]``): launches of one step, or of one
    pass of two steps when two-step passes run (an odd last step then runs on
    the one-step launches: both lists, or one)."""
    if cfg.get("fwd_depth", 1) == 2:
        return (n // 2) * per_step + (n % 2) * (2 if cfg.get("fwd_split", 0) else 1)
    return n * per_step


def run_pec_uniform(args, emit, hbm_peak, peak_src):
    """The reference's own GPU benchmark on this path: rfx.gpu.benchmark
    (rfx/gpu.py:58-107) times run() on a PEC cube without CPML after a JIT
    warm-up and reports cells x steps / s; its README quotes 7,309 Mcells/s on
    an RTX 4090.  ``value`` is the device-timed step loop of the plan,
    ``e2e`` the whole public rfx_b200.run() call timed the reference's way
    (host arrays in, plan set-up, steps, probe trace out), and vs_baseline
    compares e2e with the published figure."""
    import torch

    import rfx_b200
    from rfx_b200 import workloads
    from rfx_b200.simulation import MaterialArrays, prepare_device_run

    N = args.time_steps
    g, eps, sig, src, prb = workloads.pec_uniform(n_cells=args.pec_cells, n_steps=N)
    mats = MaterialArrays(eps, sig, np.ones_like(eps))
    cells = int(np.prod(g.shape))
    r = prepare_device_run(g, mats, N, cpml_axes="", pec_axes="xyz", sources=[tuple(src)],
                           probes=[(*prb, "ez")], dft_planes=[], pec_mask=None, dft_time_offset=1)
    plan = r.plan

    def one():
        plan.reset()
        plan.advance(0, N, r.src_table, r.probe_out)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        ev[0].record()
        for _ in range(args.steps):
            one()
        ev[1].record()
        torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1])
    alg = plan.algorithmic_bytes_per_step()
    cfg = plan.launch_config()[0]
    launches = forward_launches(plan.step_launches()[0], cfg, N)
    plan.close()
    torch.cuda.empty_cache()
    # the reference's timing: the public run() call after a warm-up call
    e2e = None
    if not args.no_e2e:
        spec_src = rfx_b200.SourceSpec(*src)
        spec_prb = rfx_b200.ProbeSpec(*prb, "ez")
        rfx_b200.run(g, mats, N, boundary="pec", sources=[spec_src], probes=[spec_prb], return_state=False)
        walls = []
        for _ in range(3):   # the median of three calls (a call's set-up varies with the process's history)
            t0 = time.perf_counter()
            res = rfx_b200.run(g, mats, N, boundary="pec", sources=[spec_src], probes=[spec_prb], return_state=False)
            float(np.asarray(res.time_series)[-1, 0])
            walls.append(time.perf_counter() - t0)
        wall = sorted(walls)[1]
        e2e = {"value": round(cells * N / wall / 1e6, 1), "unit": "Mcells/s",
               "path": "rfx_b200.run(..., return_state=False), host eps_r/sigma in, probe trace out, plan set-up "
                       "included, median of three calls",
               "wall_s": round(wall, 3), "walls_s": [round(x, 3) for x in walls],
               "h2d_bytes_per_step": int(eps.nbytes + sig.nbytes + eps.nbytes), "d2h_bytes_per_step": int(4 * N)}
    step_s = ms / 1e3 / (args.steps * N)
    depth2 = cfg.get("fwd_depth", 1) == 2
    kernel = ("fwd2_step_kernel (two steps per pass; algorithmic bytes counted per step)"
              if depth2 else "fwd_step_kernel (CPML-free variant)")
    # DRAM bytes per cell-step of the 257^3 capture of the same scene
    tpc = _traffic_per_cell("fwd2_step_kernel", "pec_257_dram_bytes_per_cell_per_step_" +
                            ("two_step" if depth2 else "one_step"))
    line = {"metric": "Mcells/s (cell updates per second), PEC-only uniform run(): the reference's rfx.gpu.benchmark",
            "value": round(cells * N * args.steps / (ms / 1e3) / 1e6, 1), "unit": "Mcells/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2),
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": round(e2e["value"] / PUBLISHED_GPU_MCELLS, 3) if e2e else None,
            "baseline": {"value": PUBLISHED_GPU_MCELLS, "hardware": "RTX 4090", "source": "reference README.md:28"},
            "dtype": "f32", "data": "synthetic (vacuum)",
            "config": {"workload": f"pec_uniform: {g.shape[0]}^3 cells ({args.pec_cells} mm cube at dx 1 mm + fence), "
                                   f"PEC faces, no CPML, raw Ez field source GaussianPulse(5 GHz) and Ez probe at the "
                                   f"centre", "time_steps": N, "cells": cells, "gpu_launches_per_run": launches,
                       "launch": cfg, "l2": "inputs larger than L2"},
            "e2e": e2e,
            "roofline": {"kernel": kernel, "bound": "hbm",
                         "achieved": round(alg / step_s / 1e9, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(alg / step_s / 1e9 / hbm_peak, 4), "peak_source": peak_src,
                         "traffic": round(tpc * cells) if tpc else None,
                         "algorithmic_bytes_per_step": int(alg)},
            "clocks": clk.summary()}
    if emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--time-steps", type=int, default=2000)
    ap.add_argument("--cpu-time-steps", type=int, default=40)
    ap.add_argument("--pec-cells", type=int, default=512,
                    help="pec_uniform: cube edge in cells (512: the benchmark line; smaller for profiling)")
    ap.add_argument("--ref-time-steps", type=int, default=20)
    ap.add_argument("--no-single", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch configuration")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the large-uniform, graded and adjoint configurations in the default line")
    ap.add_argument("--workload", default="batched_sweep",
                    choices=["batched_sweep", "large_uniform", "graded", "adjoint_region", "pec_uniform"],
                    help="batched_sweep is the headline line; the others print a secondary forward (or "
                         "forward+adjoint) line for the other configurations")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: re-launch this command under torchrun
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        os.execv(sys.executable, [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                                  f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
                                  "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]])
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but {world} ranks were launched")
    if args.workload != "batched_sweep":
        if args.impl == "reference" or world > 1:
            raise SystemExit("secondary workloads run on our arm at one GPU only")
        if "--time-steps" not in sys.argv:
            args.time_steps = {"large_uniform": 4000, "graded": 6000, "adjoint_region": 3000,
                               "pec_uniform": 1000}[args.workload]
        run_secondary(args, args.workload)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
