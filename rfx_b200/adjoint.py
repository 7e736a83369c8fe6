"""Hand-written reverse-time adjoint: forward with history, then the
transposed step backwards in time.  Replaces ``jax.grad`` through the scan
(rfx/simulation.py:1972-2058 with ``checkpoint_segments``; rfx/nonuniform.py:
1755-1796 with ``checkpoint_every``) for gradients of objectives of the probe
traces, of running-DFT plane accumulators, of Poynting-flux monitors and of
the NTFF box (far-field objectives) with respect to eps_r over a region of
cells and to the source table.

Field history.  The gradient needs, at every step n and every cell of the
region, E^n and curl H^{n+1/2} (the factors of d E^{n+1} / d eps_r through
ca and cb).  In CPML slab cells the E-side correction ce (psi + (1/kappa-1)
curl) of rfx/boundaries/cpml.py:536-546 also depends on eps_r through
ce = dt / (eps_r eps0); since d ce / d eps_r = (ce / cb)^2 d cb / d eps_r,
the forward kernel records curl + (ce / cb)^2 corr in the curl slot, so the
region may reach into the absorber like the reference's.
When that history for all steps fits the HBM budget it is recorded during
the single forward pass and the adjoint runs straight through ("history"
mode: forward + adjoint, no recomputation).  Otherwise the forward pass
stores full-state checkpoints every K steps and the adjoint recomputes each
segment with history recording just before sweeping it backwards
("segments" mode: checkpoint-every-K with segment recompute, the ragged last
segment allowed).  Both give the same gradient.
"""

from __future__ import annotations

import numpy as np
import torch

from .cpml import build_cpml
from .engine import Plan, PlanSpec, require_cuda
from .farfield import face_views, init_ntff_data, ntff_descriptor, ntff_phase_table, pack_ntff
from .grid import EPS_0, spacing_tables
from .simulation import dft_phase_table, flux_kernel_table, tangential_edge_masks


def coefficient_derivatives(eps_r, sigma, dt):
    """d ca / d eps_r and d cb / d eps_r of rfx/core/yee.py:387-393 (float64).

    L = sigma dt / (2 eps0 eps_r), ca = (1 - L)/(1 + L), cb = dt / (eps0 eps_r (1 + L)):
    d ca = 2 L / (eps_r (1 + L)^2),  d cb = -dt eps0 / (eps0 eps_r + sigma dt / 2)^2.
    """
    e = np.asarray(eps_r, np.float64)
    s = np.asarray(sigma, np.float64)
    L = s * dt / (2.0 * EPS_0 * e)
    dca = 2.0 * L / (e * (1.0 + L) ** 2)
    dcb = -dt * EPS_0 / (EPS_0 * e + s * dt / 2.0) ** 2
    return dca, dcb


def coefficient_derivatives_torch(eps_r, sigma, dt):
    """Device twin of :func:`coefficient_derivatives` (float64 math, float32 out)."""
    e = eps_r.to(torch.float64)
    s = sigma.to(torch.float64)
    L = s * dt / (2.0 * EPS_0 * e)
    dca = 2.0 * L / (e * (1.0 + L) ** 2)
    dcb = -dt * EPS_0 / (EPS_0 * e + s * dt / 2.0) ** 2
    return dca.to(torch.float32), dcb.to(torch.float32)


class AdjointRunner:
    """One simulation with a gradient region ``box = (i0, i1, j0, j1, k0, k1)``."""

    def __init__(self, grid, materials, n_steps, *, sources, probes, box, boundary="cpml", cpml_axes="xyz",
                 pec_axes="", pec_mask=None, checkpoint_every=None, mode="auto",
                 history_budget_bytes=8 << 30, dft_planes=None, dft_time_offset=1, ntff=None, flux_monitors=None,
                 device=None, _plan=None):
        """``dft_planes``: ``DFTPlaneProbe`` values accumulated by the forward
        pass (sample time (n + dft_time_offset) dt: 1 on the uniform lane, 0 on
        the graded one; it also selects the flux monitors' sample times);
        ``ntff``: an ``NTFFBox`` and ``flux_monitors``: ``FluxMonitor`` values
        accumulated by the forward pass.
        Their accumulators can carry cotangents."""
        self.device = require_cuda(device)
        self.grid = grid
        self.n_steps = int(n_steps)
        self.box = tuple(int(v) for v in box)
        i0, i1, j0, j1, k0, k1 = self.box
        self.box_shape = (i1 - i0, j1 - j0, k1 - k0)
        n = int(grid.cpml_layers)
        use_cpml = boundary == "cpml" and n > 0 and bool(cpml_axes)
        shape = tuple(int(v) for v in grid.shape)
        self.sources = [tuple(s[:4]) for s in sources]
        self.src_waves = [np.asarray(s[4], np.float32) for s in sources]
        self.probes = [tuple(p[:4]) for p in probes]
        self.dft_planes = list(dft_planes or [])
        self.ntff = ntff
        self.flux_monitors = list(flux_monitors or [])
        spec = PlanSpec(shape=shape, dt=float(grid.dt), tables=spacing_tables(grid),
                        cpml=build_cpml(grid, cpml_axes if use_cpml else "",
                                        noop_faces=set(getattr(grid, "pec_faces", None) or ())) if use_cpml else None,
                        pec_axes=pec_axes, sources=self.sources,
                        probes=[(i, j, k, c, False) for (i, j, k, c) in self.probes], grad_box=self.box,
                        dft=[(d.axis, d.index, d.component, len(d.freqs)) for d in self.dft_planes],
                        ntff=ntff_descriptor(ntff) if ntff is not None else None,
                        flux=[(m.axis, m.index, m.lo1, m.hi1, m.lo2, m.hi2, len(m.freqs)) for m in self.flux_monitors])
        self.plan = _plan or Plan(spec, self.device)
        self.eps = torch.as_tensor(np.asarray(materials.eps_r, np.float32)).to(self.device).contiguous()
        self.sigma = torch.as_tensor(np.asarray(materials.sigma, np.float32)).to(self.device).contiguous()
        mu = getattr(materials, "mu_r", None)
        self.mu = None if mu is None else torch.as_tensor(np.asarray(mu, np.float32)).to(self.device)
        self.emask = tangential_edge_masks(pec_mask) if pec_mask is not None else None
        hcells = int(np.prod(self.box_shape))
        hist_bytes = 24 * hcells * self.n_steps
        if mode == "auto":
            mode = "history" if (checkpoint_every is None and hist_bytes <= history_budget_bytes) else "segments"
        self.mode = mode
        self.K = int(checkpoint_every or 64)
        if self.mode == "segments":
            self.plan.checkpoint_reserve((self.n_steps + self.K - 1) // self.K)
        tab = np.stack(self.src_waves, axis=-1)[: self.n_steps] if self.src_waves else np.zeros((self.n_steps, 0))
        self.src_table = torch.from_numpy(np.ascontiguousarray(tab, np.float32)).to(self.device)
        self.dft_phases = [torch.from_numpy(dft_phase_table(d.freqs, self.n_steps, grid.dt, dft_time_offset))
                           .to(self.device) for d in self.dft_planes]
        self.dft_accs = []
        self.ntff_phase = (torch.from_numpy(ntff_phase_table(ntff.freqs, self.n_steps, grid.dt)).to(self.device)
                           if ntff is not None else None)
        self.ntff_faces = []
        self.flux_kernels = [torch.from_numpy(flux_kernel_table(m, self.n_steps, grid.dt, dft_time_offset))
                             .to(self.device) for m in self.flux_monitors]
        self.flux_accs = []
        self._dirty = True

    # materials ------------------------------------------------------------
    def set_box_eps(self, eps_box):
        i0, i1, j0, j1, k0, k1 = self.box
        self.eps[i0:i1, j0:j1, k0:k1] = torch.as_tensor(eps_box, dtype=torch.float32, device=self.device)
        self._dirty = True

    def _sync_materials(self):
        if self._dirty:
            self.plan.set_materials(self.eps, self.sigma, self.mu, self.emask)
            self._dirty = False

    # passes ---------------------------------------------------------------
    def forward(self, src_table=None):
        """Run the forward pass; returns the probe traces (n_steps, n_probes)
        (the DFT-plane accumulators are left in ``dft_accs``)."""
        self._sync_materials()
        if src_table is not None:
            self.src_table = src_table.detach().to(self.device, torch.float32).contiguous()
        p, N = self.plan, self.n_steps
        p.reset()
        ts = torch.zeros((N, len(self.probes)), device=self.device, dtype=torch.float32)
        st = self.src_table if self.sources else None
        accs = [torch.zeros(d.accumulator.shape, device=self.device, dtype=torch.complex64) for d in self.dft_planes]
        dk = dict(dft_accs=accs, dft_phases=self.dft_phases) if accs else {}
        if self.ntff is not None:
            nacc, ncmp = pack_ntff(init_ntff_data(self.ntff), self.device)
            dk["ntff"] = (nacc, ncmp, self.ntff_phase)
        faccs = [torch.zeros((4,) + tuple(np.shape(m.e1_dft)), device=self.device, dtype=torch.complex128)
                 for m in self.flux_monitors]
        if faccs:
            dk.update(flux_accs=faccs, flux_kernels=self.flux_kernels)
        if self.mode == "history":
            p.record_history(0, N)
            p.advance(0, N, st, ts, **dk)
        else:
            for q, s0 in enumerate(range(0, N, self.K)):
                p.checkpoint_save(q)
                p.advance(s0, min(self.K, N - s0), st, ts, **dk)
        self.dft_accs = accs
        self.ntff_faces = face_views(dk["ntff"][0], self.ntff) if self.ntff is not None else []
        self.flux_accs = faccs
        p.check_device()
        self.ts = ts
        return ts

    def backward(self, g_ts, want_source_grad=True, g_dft=None, g_ntff=None, g_flux=None):
        """Adjoint sweep for probe cotangents ``g_ts`` (n_steps, n_probes; may
        be None), DFT-plane cotangents ``g_dft`` (per plane a complex
        (n_freqs, n1, n2) array dJ/dRe + i dJ/dIm, or None) and NTFF
        cotangents ``g_ntff`` (the six faces x_lo .. z_hi, each like its
        accumulator, or None), flux cotangents ``g_flux`` (per monitor a
        complex (4, n_freqs, n1, n2) array for E1 E2 H1 H2, or None).

        Returns (dJ/d eps_r over the box as float64, dJ/d source table)."""
        p, N = self.plan, self.n_steps
        i0, i1, j0, j1, k0, k1 = self.box
        dca, dcb = coefficient_derivatives(self.eps[i0:i1, j0:j1, k0:k1].cpu().numpy(),
                                           self.sigma[i0:i1, j0:j1, k0:k1].cpu().numpy(), float(self.grid.dt))
        dca = torch.from_numpy(dca.astype(np.float32).ravel()).to(self.device)
        dcb = torch.from_numpy(dcb.astype(np.float32).ravel()).to(self.device)
        grad = torch.zeros(int(np.prod(self.box_shape)), device=self.device, dtype=torch.float64)
        if g_ts is None:
            g_ts = torch.zeros((N, len(self.probes)), device=self.device, dtype=torch.float32)
        g = g_ts.detach().to(self.device, torch.float32).contiguous()
        src_adj = (torch.zeros((N, len(self.sources)), device=self.device, dtype=torch.float32)
                   if (want_source_grad and self.sources) else None)
        kw = dict(g=g, grad=grad, dca=dca, dcb=dcb, src_adj=src_adj)
        if g_dft is not None and any(c is not None for c in g_dft):
            if len(g_dft) != len(self.dft_planes):
                raise ValueError("one DFT-plane cotangent (or None) per DFT plane")
            cots = [None if c is None else torch.as_tensor(c).to(self.device, torch.complex64).contiguous()
                    for c in g_dft]
            for c, d in zip(cots, self.dft_planes):
                if c is not None and tuple(c.shape) != tuple(d.accumulator.shape):
                    raise ValueError(f"DFT-plane cotangent of shape {tuple(c.shape)}, accumulator "
                                     f"{tuple(d.accumulator.shape)}")
            kw.update(dft_cots=cots, dft_phases=self.dft_phases)
        if g_ntff is not None and any(c is not None for c in g_ntff):
            if self.ntff is None or len(g_ntff) != 6:
                raise ValueError("NTFF cotangents need the runner's NTFF box and one entry per face")
            parts = []
            for c, f in zip(g_ntff, self.ntff_faces):
                c = torch.zeros_like(f) if c is None else torch.as_tensor(c).to(self.device, torch.complex64)
                if tuple(c.shape) != tuple(f.shape):
                    raise ValueError(f"NTFF face cotangent of shape {tuple(c.shape)}, face {tuple(f.shape)}")
                parts.append(c.reshape(-1))
            kw.update(ntff=(torch.cat(parts).contiguous(), self.ntff_phase))
        if g_flux is not None and any(c is not None for c in g_flux):
            if len(g_flux) != len(self.flux_monitors):
                raise ValueError("one flux cotangent (or None) per flux monitor")
            fc = [None if c is None else torch.as_tensor(c).to(self.device, torch.complex128).contiguous()
                  for c in g_flux]
            kw.update(flux_cots=fc, flux_kernels=self.flux_kernels)
        p.adjoint_begin(N, **kw)
        st = self.src_table if self.sources else None
        if self.mode == "history":
            p.adjoint_advance(N, N, **kw)
        else:
            starts = list(range(0, N, self.K))
            for q in reversed(range(len(starts))):
                s0 = starts[q]
                L = min(self.K, N - s0)
                p.checkpoint_load(q)
                p.record_history(s0, L)
                p.advance(s0, L, st, None)
                p.adjoint_advance(s0 + L, L, **kw)
        p.check_device()
        return grad.view(self.box_shape), src_adj

    def close(self):
        self.plan.close()


class FDTDFunction(torch.autograd.Function):
    """Probe traces (and, when the runner has them, the complex64 DFT-plane
    accumulators, the six NTFF face accumulators x_lo .. z_hi and the
    complex128 flux-monitor accumulators (4, n_freqs, n1, n2) as further
    outputs) as a differentiable function of eps_r
    over the runner's box and of the source table: the
    ``torch.autograd.Function`` face of the hand-written adjoint."""

    @staticmethod
    def forward(ctx, eps_box, src_table, runner):
        runner.set_box_eps(eps_box.detach())
        ts = runner.forward(src_table.detach() if src_table is not None else None)
        ctx.runner = runner
        ctx.has_src = src_table is not None
        if runner.dft_planes or runner.ntff is not None or runner.flux_monitors:
            return (ts.clone(), *[a.clone() for a in runner.dft_accs], *[f.clone() for f in runner.ntff_faces],
                    *[a.clone() for a in runner.flux_accs])
        return ts.clone()

    @staticmethod
    def backward(ctx, g_ts, *g_rest):
        r = ctx.runner
        nd, nn = len(r.dft_planes), len(r.ntff_faces)
        g_dft, g_ntff, g_flux = list(g_rest[:nd]), list(g_rest[nd:nd + nn]), list(g_rest[nd + nn:])
        grad, src_adj = r.backward(g_ts, want_source_grad=ctx.has_src, g_dft=g_dft or None, g_ntff=g_ntff or None,
                                   g_flux=g_flux or None)
        return grad.to(torch.float32), (src_adj if ctx.has_src else None), None


def probe_dft_objective(ts, freqs, dt):
    """Sum over frequencies and probes of |sum_n ts[n, p] exp(-j 2 pi f n dt) dt|^2
    (the objective of the adjoint benchmark configuration)."""
    n = torch.arange(ts.shape[0], device=ts.device, dtype=torch.float64)
    f = torch.as_tensor(np.asarray(freqs, np.float64), device=ts.device)
    ph = torch.exp(-2j * np.pi * f[:, None] * n[None, :] * dt) * dt   # (nf, N)
    X = ph.to(torch.complex128) @ ts.to(torch.complex128)             # (nf, np)
    return (X.real ** 2 + X.imag ** 2).sum()
