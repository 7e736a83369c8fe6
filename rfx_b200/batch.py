"""Batched design sweep: many simulations of uneven grid sizes advanced
together, forward then adjoint, with one step-kernel launch per time step for
all of them.

The reference batches only equal-shape material sweeps (``jax.vmap`` of the
scan body, rfx/vmap_sweep.py:871-1017); a sweep over uneven grids is a Python
loop of ``forward`` + ``jax.grad`` calls.  Here every instance keeps its own
resident state and CPML, the work lists of all instances are concatenated
into one launch, and each instance's probe-DFT objective gradient comes from
the hand-written adjoint (``rfx_b200.adjoint``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from .adjoint import coefficient_derivatives, coefficient_derivatives_torch, probe_dft_objective
from .cpml import build_cpml
from .engine import Batch, Plan, PlanSpec, require_cuda
from .grid import spacing_tables


@dataclass
class SweepInstance:
    grid: object
    eps_r: np.ndarray
    sigma: np.ndarray
    sources: list            # (i, j, k, comp, waveform)
    probes: list             # (i, j, k, comp)
    box: tuple               # gradient region (i0, i1, j0, j1, k0, k1)
    freqs: np.ndarray        # objective frequencies
    cpml_axes: str = "xyz"
    pec_axes: str = ""


class Sweep:
    """Forward + adjoint of a list of instances with equal step counts."""

    def __init__(self, instances, n_steps, device=None, batched=True):
        self.device = require_cuda(device)
        self.n_steps = int(n_steps)
        self.inst = list(instances)
        self.plans = []
        self.io = []
        for s in self.inst:
            g = s.grid
            spec = PlanSpec(shape=tuple(g.shape), dt=float(g.dt), tables=spacing_tables(g),
                            cpml=build_cpml(g, s.cpml_axes), pec_axes=s.pec_axes,
                            sources=[tuple(x[:4]) for x in s.sources],
                            probes=[(i, j, k, c, False) for (i, j, k, c) in s.probes], grad_box=s.box)
            p = Plan(spec, self.device)
            p.set_materials(s.eps_r, s.sigma)
            tab = np.stack([np.asarray(x[4], np.float32)[: self.n_steps] for x in s.sources], axis=-1)
            src = torch.from_numpy(np.ascontiguousarray(tab)).to(self.device)
            ts = torch.zeros((self.n_steps, len(s.probes)), device=self.device, dtype=torch.float32)
            i0, i1, j0, j1, k0, k1 = s.box
            dca, dcb = coefficient_derivatives(s.eps_r[i0:i1, j0:j1, k0:k1], s.sigma[i0:i1, j0:j1, k0:k1],
                                               float(g.dt))
            nbox = (i1 - i0) * (j1 - j0) * (k1 - k0)
            self.io.append(dict(
                src=src, ts=ts,
                dca=torch.from_numpy(dca.astype(np.float32).ravel()).to(self.device),
                dcb=torch.from_numpy(dcb.astype(np.float32).ravel()).to(self.device),
                grad=torch.zeros(nbox, device=self.device, dtype=torch.float64)))
            self.plans.append(p)
        self.batched = batched
        self.batch = Batch(self.plans) if batched else None

    def set_materials(self, eps_list, sigma_list):
        """Replace every instance's eps_r / sigma (device or host arrays of the
        instance shape) and the coefficient derivatives over its region."""
        for q, (p, s, io) in enumerate(zip(self.plans, self.inst, self.io)):
            e = torch.as_tensor(eps_list[q], device=self.device, dtype=torch.float32)
            sg = torch.as_tensor(sigma_list[q], device=self.device, dtype=torch.float32)
            p.set_materials(e, sg)
            i0, i1, j0, j1, k0, k1 = s.box
            dca, dcb = coefficient_derivatives_torch(e[i0:i1, j0:j1, k0:k1], sg[i0:i1, j0:j1, k0:k1],
                                                     float(s.grid.dt))
            io["dca"] = dca.reshape(-1).contiguous()
            io["dcb"] = dcb.reshape(-1).contiguous()

    def cells(self) -> int:
        return int(sum(int(np.prod(s.grid.shape)) for s in self.inst))

    def forward(self):
        N = self.n_steps
        for p in self.plans:
            p.reset()
            p.record_history(0, N)
        if self.batched:
            self.batch.advance(0, N, [dict(src_table=io["src"], probe_out=io["ts"]) for io in self.io])
        else:
            for p, io in zip(self.plans, self.io):
                p.advance(0, N, io["src"], io["ts"])
        return [io["ts"] for io in self.io]

    def objectives(self):
        """Per-instance probe-DFT objective values and their cotangents."""
        Js, gs = [], []
        for s, io in zip(self.inst, self.io):
            t = io["ts"].detach().clone().requires_grad_(True)
            J = probe_dft_objective(t, s.freqs, float(s.grid.dt))
            J.backward()
            Js.append(J.detach())
            gs.append(t.grad.to(torch.float32).contiguous())
        return Js, gs

    def backward(self, gs):
        N = self.n_steps
        aios = []
        for io, g in zip(self.io, gs):
            io["grad"].zero_()
            aios.append(dict(g=g, grad=io["grad"], dca=io["dca"], dcb=io["dcb"], src_adj=None))
        if self.batched:
            self.batch.adjoint_begin(N, aios)
            self.batch.adjoint_advance(N, N, aios)
        else:
            for p, a in zip(self.plans, aios):
                p.adjoint_begin(N, **a)
                p.adjoint_advance(N, N, **a)
        return [io["grad"].view(tuple(b - a for a, b in zip(s.box[0::2], s.box[1::2])))
                for s, io in zip(self.inst, self.io)]

    def run(self):
        """Forward, objectives, adjoint: returns (J list, dJ/d eps_r list)."""
        self.forward()
        Js, gs = self.objectives()
        return Js, self.backward(gs)

    def signature(self):
        """What the fastest launch configuration depends on: the instances'
        grid shapes and CPML / PEC axes, batching, and the device."""
        dev = torch.cuda.get_device_name(self.device) if torch.cuda.is_available() else "cpu"
        return {"device": dev, "batched": self.batched,
                "instances": [(tuple(int(n) for n in s.grid.shape), s.cpml_axes, s.pec_axes) for s in self.inst]}

    def autotune(self, trial_steps=32, repeats=2, cache_path=None):
        """Pick the batch's launch configuration (``rfx_b200.autotune``) by
        timing ``trial_steps`` forward and reverse steps of this sweep per
        candidate.  The next ``forward`` resets the state the trials leave.
        Returns the ``TuneResult``; None for an unbatched sweep (each
        simulation keeps the default of its plan)."""
        from .autotune import autotune
        if not self.batched:
            return None
        T = max(1, min(int(trial_steps), self.n_steps))
        ios = [dict(src_table=io["src"], probe_out=io["ts"]) for io in self.io]
        zero_g = [torch.zeros_like(io["ts"]) for io in self.io]
        for p in self.plans:
            p.reset()
            p.record_history(0, T)

        def run_forward():
            self.batch.advance(0, T, ios)

        def run_reverse():
            aios = [dict(g=g, grad=io["grad"], dca=io["dca"], dcb=io["dcb"], src_adj=None)
                    for io, g in zip(self.io, zero_g)]
            self.batch.adjoint_begin(T, aios)
            self.batch.adjoint_advance(T, T, aios)

        run_forward()   # history of the trial steps for the reverse trials
        return autotune(self.batch, run_forward, run_reverse, signature=self.signature(), cache_path=cache_path,
                        repeats=repeats)

    def step_launches(self):
        """Step-kernel launches of one forward time step and one reverse
        time step of the whole sweep (every instance included)."""
        if self.batch is not None:
            return self.batch.step_launches()
        f = r = 0
        for p in self.plans:
            a, b = p.step_launches()
            f, r = f + a, r + b
        return f, r

    def check_device(self):
        """Synchronise and raise if a bounded wait inside a kernel ran out."""
        if self.batch is not None:
            self.batch.check_device()
        for p in self.plans:
            p.check_device()

    def close(self):
        if self.batch is not None:
            self.batch.close()
        for p in self.plans:
            p.close()
