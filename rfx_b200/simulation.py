"""Drop-in ``run()`` for the uniform lane, backed by the CUDA step kernel.

Mirrors ``rfx.simulation.run`` (rfx/simulation.py:1686-2138): the same
arguments for the features on this path, the same source / probe / DFT-plane
specs, the same ``SimResult`` fields, and the same errors for bad
``checkpoint_segments``.  The whole ``jax.lax.scan`` (rfx/simulation.py:1977)
runs as one resident device simulation; features outside this path
(dispersion, TFSF, NTFF, waveguide ports, conformal PEC, periodic axes, ...)
raise ``NotImplementedError`` instead of silently changing the physics.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch

from .cpml import build_cpml
from .engine import Plan, PlanSpec, require_cuda
from .farfield import init_ntff_data, ntff_descriptor, ntff_phase_table, pack_ntff, unpack_ntff
from .grid import EPS_0, MU_0, face_pads, spacing_tables
from .sources import SourceSpec  # noqa: F401  (re-export: the reference's spec type)


class MaterialArrays(NamedTuple):
    """rfx/core/yee.py:31-39."""
    eps_r: np.ndarray
    sigma: np.ndarray
    mu_r: np.ndarray


class FDTDState(NamedTuple):
    """rfx/core/yee.py:16-28 (final fields of a run)."""
    ex: np.ndarray
    ey: np.ndarray
    ez: np.ndarray
    hx: np.ndarray
    hy: np.ndarray
    hz: np.ndarray
    step: int


class ProbeSpec(NamedTuple):
    """rfx/simulation.py:75-80."""
    i: int
    j: int
    k: int
    component: str


class LumpedPortSParamSpec(NamedTuple):
    """rfx/simulation.py:102-132: V/I DFT at a single-cell lumped port."""
    i: int
    j: int
    k: int
    component: str
    freqs: np.ndarray
    impedance: float


class DFTPlaneProbe(NamedTuple):
    """rfx/probes/probes.py:379-405."""
    accumulator: np.ndarray
    freqs: np.ndarray
    component: str
    axis: int
    index: int
    total_steps: int = 0
    window: str = "rect"
    window_alpha: float = 0.25


class FluxMonitor(NamedTuple):
    """Poynting-flux DFT accumulators of a plane region
    (rfx/probes/probes.py:476-506); accumulators are complex128."""
    e1_dft: np.ndarray
    e2_dft: np.ndarray
    h1_dft: np.ndarray
    h2_dft: np.ndarray
    freqs: np.ndarray
    axis: int
    index: int
    dA: np.ndarray
    total_steps: int
    window: str
    window_alpha: float
    lo1: int = 0
    hi1: int = -1
    lo2: int = 0
    hi2: int = -1


def init_flux_monitor(axis, index, freqs, grid_shape, d1, d2, dft_total_steps=0, dft_window="rect",
                      dft_window_alpha=0.25, lo1=0, hi1=-1, lo2=0, hi2=-1) -> FluxMonitor:
    """rfx/probes/probes.py:515-579: a flux monitor on plane ``index`` of
    ``axis`` over [lo1, hi1) x [lo2, hi2) of the tangential axes (-1: full
    extent), area weight dA = d1 d2 (scalars or per-cell arrays)."""
    full1 = grid_shape[1] if axis == 0 else grid_shape[0]
    full2 = grid_shape[1] if axis == 2 else grid_shape[2]
    hi1 = full1 if hi1 < 0 else hi1
    hi2 = full2 if hi2 < 0 else hi2
    n1, n2, nf = hi1 - lo1, hi2 - lo2, len(freqs)
    zeros = np.zeros((nf, n1, n2), np.complex128)
    w1 = np.asarray(d1, np.float32)
    w2 = np.asarray(d2, np.float32)
    if w1.ndim > 0:
        w1 = w1[lo1:hi1]
    if w2.ndim > 0:
        w2 = w2[lo2:hi2]
    dA = np.reshape(w1, (-1, 1)) * np.reshape(w2, (1, -1))
    return FluxMonitor(zeros, zeros.copy(), zeros.copy(), zeros.copy(), np.asarray(freqs), int(axis), int(index),
                       dA, int(dft_total_steps), dft_window, float(dft_window_alpha), lo1, hi1, lo2, hi2)


def flux_spectrum(mon: FluxMonitor, *, exact_f64: bool = False) -> np.ndarray:
    """rfx/probes/probes.py:613-680: the integral of Re(E x H*) . n dA per
    frequency (positive: power flowing towards +axis).  The accumulators are
    complex128 here, so both paths evaluate in float64."""
    e1, e2 = np.asarray(mon.e1_dft, np.complex128), np.asarray(mon.e2_dft, np.complex128)
    h1, h2 = np.asarray(mon.h1_dft, np.complex128), np.asarray(mon.h2_dft, np.complex128)
    integrand = e1 * np.conj(h2) - e2 * np.conj(h1)
    return np.real(np.sum(integrand * np.asarray(mon.dA, np.float64), axis=(-2, -1)))


def dft_window_weight(step, total_steps, window, alpha):
    """rfx/core/dft_utils.py:8-50, float32 arithmetic."""
    if total_steps <= 1 or window == "rect":
        return np.float32(1.0)
    x = np.float32(step) / np.float32(max(total_steps - 1, 1))
    if window == "hann" or (window == "tukey" and alpha >= 1.0):
        return np.float32(0.5) * (np.float32(1.0) - np.cos(np.float32(2.0 * np.pi) * x))
    if window == "tukey":
        a = float(alpha)
        if a <= 0.0:
            return np.float32(1.0)
        if x < a / 2.0:
            return np.float32(0.5) * (np.float32(1.0) + np.cos(np.float32(np.pi) * (np.float32(2.0) * x / np.float32(a)
                                                                                    - np.float32(1.0))))
        if x <= 1.0 - a / 2.0:
            return np.float32(1.0)
        return np.float32(0.5) * (np.float32(1.0) + np.cos(np.float32(np.pi) * (
            np.float32(2.0) * x / np.float32(a) - np.float32(2.0 / a) + np.float32(1.0))))
    raise ValueError(f"unknown DFT window {window!r}")


def flux_kernel_table(mon: FluxMonitor, n_steps, dt, time_offset=1):
    """(n_steps, 2, n_freqs) complex128 step factors of a flux monitor: E
    sampled at t, H at t - dt/2, times dt and the window weight.  Uniform lane
    (time_offset 1, rfx/simulation.py:1590-1642): t = (n+1) dt in float64 and
    the weight of step n+1.  Graded lane (time_offset 0, rfx/nonuniform.py:
    1483-1520): t = f32(n) * dt rounded to float32, the weight of step n."""
    f = np.asarray(mon.freqs, np.float64)
    steps = np.arange(time_offset, time_offset + n_steps)
    if time_offset == 1:
        t = steps.astype(np.float64) * float(dt)
    else:
        t = (steps.astype(np.float32) * np.float32(dt)).astype(np.float64)
    w = np.array([dft_window_weight(n, mon.total_steps, mon.window, mon.window_alpha) for n in steps], np.float64)
    out = np.empty((n_steps, 2, len(f)), np.complex128)
    out[:, 0, :] = np.exp(-1j * 2.0 * np.pi * f[None, :] * t[:, None]) * float(dt) * w[:, None]
    out[:, 1, :] = np.exp(-1j * 2.0 * np.pi * f[None, :] * (t[:, None] - float(dt) * 0.5)) * float(dt) * w[:, None]
    return out


class SimResult(NamedTuple):
    """rfx/simulation.py:135-178 (fields on this path)."""
    state: FDTDState | None
    time_series: np.ndarray
    ntff_data: object = None
    dft_planes: tuple | None = None
    flux_monitors: tuple | None = None
    waveguide_ports: tuple | None = None
    wire_port_sparams: tuple | None = None
    lumped_port_sparams: tuple | None = None
    snapshots: dict | None = None
    ntff_box: object = None
    grid: object = None
    wire_refplane_sparams: tuple | None = None


def init_dft_plane_probe(axis, index, component, freqs, grid_shape, dft_total_steps=0,
                         dft_window="rect", dft_window_alpha=0.25) -> DFTPlaneProbe:
    """rfx/probes/probes.py:408-449 (complex64 accumulator)."""
    if axis == 0:
        plane = (grid_shape[1], grid_shape[2])
    elif axis == 1:
        plane = (grid_shape[0], grid_shape[2])
    else:
        plane = (grid_shape[0], grid_shape[1])
    freqs = np.asarray(freqs, np.float32)
    return DFTPlaneProbe(np.zeros((len(freqs),) + plane, np.complex64), freqs, component, int(axis),
                         int(index), int(dft_total_steps), dft_window, float(dft_window_alpha))


def tangential_edge_masks(cell_mask):
    """Per-component tangential edge masks of a PEC cell mask on non-periodic
    3-D axes (rfx/boundaries/pec.py:90-176), packed as bits 1/2/4."""
    m = np.asarray(cell_mask, dtype=bool)
    bits = np.zeros(m.shape, np.uint8)
    for ax in range(3):
        nb = np.zeros_like(m)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(1, None)
        hi[ax] = slice(0, -1)
        nb[tuple(lo)] |= m[tuple(hi)]
        nb[tuple(hi)] |= m[tuple(lo)]
        bits |= ((m & nb).astype(np.uint8) << ax)
    return bits


def dft_phase_table(freqs, n_steps, dt, time_offset):
    """(n_steps, n_freqs, 2) float32 of ``(cos, sin)(-2 pi f t) * dt``.

    The sample time follows the reference: ``t = (n + 1) dt`` on the uniform
    lane (rfx/simulation.py:1574) and ``n dt`` on the graded lane
    (rfx/nonuniform.py:1461), with the float32 phase argument
    ``f32(-2 pi f) * f32(t)`` of those lines.
    """
    fr = np.asarray(freqs, np.float32)
    w = (fr * np.float32(-2.0 * np.pi)).astype(np.float32)
    t = np.arange(time_offset, time_offset + n_steps, dtype=np.float32) * np.float32(dt)
    arg = (t[:, None] * w[None, :]).astype(np.float32).astype(np.float64)
    out = np.empty((n_steps, len(fr), 2), np.float32)
    out[..., 0] = np.cos(arg) * dt
    out[..., 1] = np.sin(arg) * dt
    return out


def _vi_probes(spec: LumpedPortSParamSpec):
    """Probe cells whose pre-source samples give the port V and I
    (rfx/simulation.py:1480-1500)."""
    i, j, k, c = spec.i, spec.j, spec.k, spec.component
    if c == "ez":
        h = [(i, j, k, "hy", 1.0), (i - 1, j, k, "hy", -1.0), (i, j, k, "hx", -1.0), (i, j - 1, k, "hx", 1.0)]
    elif c == "ex":
        h = [(i, j, k, "hz", 1.0), (i, j - 1, k, "hz", -1.0), (i, j, k, "hy", -1.0), (i, j, k - 1, "hy", 1.0)]
    else:
        h = [(i, j, k, "hx", 1.0), (i, j, k - 1, "hx", -1.0), (i, j, k, "hz", -1.0), (i - 1, j, k, "hz", 1.0)]
    return [(i, j, k, c, -1.0)] + h


def _unsupported(**kw):
    bad = [k for k, v in kw.items() if v not in (None, False, (), [], 0, "")]
    if bad:
        raise NotImplementedError(
            "rfx_b200 runs the Yee/CPML/source/probe/DFT-plane scan body only; these features are outside that "
            "path: " + ", ".join(sorted(bad)))


def _to_np(a, dtype=np.float32):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.asarray(a, dtype=dtype)


class DeviceRun(NamedTuple):
    """A prepared device run: the plan with materials set and state reset,
    and the device tables its steps read and write."""
    plan: object
    src_table: object          # (n_steps, n_src) float32 or None
    probe_out: object          # (n_steps, n_probe) float32 or None
    dft_accs: list             # complex64 accumulators per DFT plane
    dft_phases: list           # (n_steps, n_f) phase tables per plane
    probes: list               # probe tuples (user probes first, then port V/I probes)
    vi_rows: list              # per lumped port: [(probe row, sign), ...]
    flux_accs: tuple = ()      # complex128 (4, n_f, n1, n2) per flux monitor
    flux_kernels: tuple = ()   # complex128 (n_steps, 2, n_f) per flux monitor
    ntff: tuple | None = None  # NTFF box: (sums, Kahan residuals, (n_steps, 2, n_f) phase table)


def prepare_device_run(grid, materials, n_steps, *, cpml_axes, pec_axes, sources, probes, dft_planes, pec_mask,
                       dft_time_offset, lumped_specs=(), kappa_max=None, noop_faces=(), flux_monitors=(),
                       ntff_box=None, ntff_data=None, device=None) -> DeviceRun:
    """``dft_time_offset`` (1 uniform lane, 0 graded lane) also selects the
    flux monitors' sample times."""
    """Build the plan of one simulation and upload its inputs (the set-up half
    of ``run_device``); the caller owns the plan and closes it."""
    dev = require_cuda(device)
    shape = tuple(int(v) for v in grid.shape)
    n_steps = int(n_steps)
    srcs = [(int(s[0]), int(s[1]), int(s[2]), s[3], s[4]) for s in sources]
    prb = [(int(p[0]), int(p[1]), int(p[2]), p[3], False) for p in probes]
    vi_rows = []
    for spec in lumped_specs:
        rows = []
        for (i, j, k, c, sgn) in _vi_probes(spec):
            rows.append((len(prb), sgn))
            prb.append((i, j, k, c, True))
        vi_rows.append(rows)
    cp = build_cpml(grid, cpml_axes, kappa_max=kappa_max, noop_faces=noop_faces) if cpml_axes else None
    plan = Plan(PlanSpec(shape=shape, dt=float(grid.dt), tables=spacing_tables(grid), cpml=cp,
                         pec_axes=pec_axes, sources=[s[:4] for s in srcs], probes=prb,
                         dft=[(d.axis, d.index, d.component, len(d.freqs)) for d in dft_planes],
                         flux=[(m.axis, m.index, m.lo1, m.hi1, m.lo2, m.hi2, len(m.freqs)) for m in flux_monitors],
                         ntff=ntff_descriptor(ntff_box) if ntff_box is not None else None),
                dev)
    try:
        em = tangential_edge_masks(_to_np(pec_mask, bool)) if pec_mask is not None else None
        mu = getattr(materials, "mu_r", None)
        plan.set_materials(_to_np(materials.eps_r), _to_np(materials.sigma),
                           None if mu is None else _to_np(mu), em)
        plan.reset()
        src_table = None
        if srcs:
            tab = np.stack([_to_np(s[4])[:n_steps] for s in srcs], axis=-1)
            if tab.shape[0] < n_steps:
                raise ValueError("source waveform shorter than n_steps")
            src_table = torch.from_numpy(np.ascontiguousarray(tab, np.float32)).to(dev)
        probe_out = torch.zeros((n_steps, len(prb)), device=dev, dtype=torch.float32) if prb else None
        accs, phases = [], []
        for d in dft_planes:
            accs.append(torch.from_numpy(np.ascontiguousarray(np.asarray(d.accumulator, np.complex64))).to(dev))
            phases.append(torch.from_numpy(dft_phase_table(d.freqs, n_steps, grid.dt, dft_time_offset)).to(dev))
        faccs, fkerns = [], []
        for m in flux_monitors:
            faccs.append(torch.from_numpy(np.stack([np.asarray(a, np.complex128) for a in
                                                    (m.e1_dft, m.e2_dft, m.h1_dft, m.h2_dft)])).to(dev).contiguous())
            fkerns.append(torch.from_numpy(flux_kernel_table(m, n_steps, grid.dt, dft_time_offset)).to(dev))
        ntff = None
        if ntff_box is not None:
            acc, cmp = pack_ntff(ntff_data if ntff_data is not None else init_ntff_data(ntff_box), dev)
            ntff = (acc, cmp, torch.from_numpy(ntff_phase_table(ntff_box.freqs, n_steps, grid.dt)).to(dev))
    except BaseException:
        plan.close()
        raise
    return DeviceRun(plan, src_table, probe_out, accs, phases, prb, vi_rows, faccs, fkerns, ntff)


def run_device(grid, materials, n_steps, *, cpml_axes, pec_axes, sources, probes, dft_planes, pec_mask,
               dft_time_offset, lumped_specs=(), return_state=True, report_every=None, report_label="",
               kappa_max=None, noop_faces=(), flux_monitors=(), ntff_box=None, ntff_data=None, device=None):
    """Shared driver of the uniform and graded lanes.  Returns (time series,
    DFT planes, lumped-port results, state, flux monitors, NTFF data or None)."""
    n_steps = int(n_steps)
    flux_monitors = list(flux_monitors)
    r = prepare_device_run(grid, materials, n_steps, cpml_axes=cpml_axes, pec_axes=pec_axes, sources=sources,
                           probes=probes, dft_planes=dft_planes, pec_mask=pec_mask, dft_time_offset=dft_time_offset,
                           lumped_specs=lumped_specs, kappa_max=kappa_max, noop_faces=noop_faces,
                           flux_monitors=flux_monitors, ntff_box=ntff_box, ntff_data=ntff_data, device=device)
    plan, probe_out, accs = r.plan, r.probe_out, r.dft_accs
    try:
        chunk = int(report_every) if report_every else n_steps
        done = 0
        while done < n_steps:
            k = min(chunk, n_steps - done)
            plan.advance(done, k, r.src_table, probe_out, accs, r.dft_phases, r.flux_accs, r.flux_kernels, r.ntff)
            done += k
            if report_every:
                torch.cuda.current_stream().synchronize()
                print(f"[PROGRESS] {report_label} step {done}/{n_steps}", flush=True)
        plan.check_device()
        ts_all = probe_out.cpu().numpy() if probe_out is not None else np.zeros((n_steps, 0), np.float32)
        ts = ts_all[:, :len(probes)]
        out_planes = tuple(d._replace(accumulator=a.cpu().numpy()) for d, a in zip(dft_planes, accs))
        lumped = None
        if lumped_specs:
            lumped = []
            for spec, rows in zip(lumped_specs, r.vi_rows):
                dx = float(grid.dx)
                v = ts_all[:, rows[0][0]].astype(np.float64) * rows[0][1] * dx
                iv = sum(ts_all[:, q].astype(np.float64) * sg for q, sg in rows[1:]) * dx
                lumped.append((spec, _vi_dft(v, iv, spec.freqs, float(grid.dt))))
            lumped = tuple(lumped)
        state = None
        if return_state:
            f = [t.cpu().numpy() for t in plan.store_fields()]
            state = FDTDState(*f, step=n_steps)
        out_flux = []
        for m, a in zip(flux_monitors, r.flux_accs):
            a = a.cpu().numpy()
            out_flux.append(m._replace(e1_dft=a[0], e2_dft=a[1], h1_dft=a[2], h2_dft=a[3]))
        ntff_out = unpack_ntff(ntff_box, r.ntff[0], r.ntff[1]) if ntff_box is not None else None
        return ts, out_planes, lumped, state, tuple(out_flux), ntff_out
    finally:
        plan.close()


def _vi_dft(v, i, freqs, dt):
    """Port V/I DFT with the reference's sample time ``n dt``
    (rfx/simulation.py:1447, 1480-1500), summed in float64."""
    n = np.arange(len(v), dtype=np.float64)
    ph = np.exp(-1j * 2.0 * np.pi * np.asarray(freqs, np.float64)[:, None] * (n[None, :] * dt)) * dt
    return ((ph @ v).astype(np.complex64), (ph @ i).astype(np.complex64))


def run(grid, materials, n_steps, *, boundary="pec", cpml_axes="xyz", pec_axes=None, periodic=None, debye=None,
        lorentz=None, tfsf=None, sources=None, probes=None, dft_planes=None, flux_monitors=None,
        waveguide_ports=None, ntff=None, snapshot=None, checkpoint=False, checkpoint_segments=None,
        aniso_eps=None, aniso_inv_eps=None, aniso_inv_eps_smooth=False, pec_mask=None, pec_occupancy=None,
        conformal_weights=None, wire_port_sparams=None, lumped_port_sparams=None, wire_refplane_sparams=None,
        lumped_rlc=None, kerr_chi3=None, field_dtype=None, return_state=True, mag_sources=None,
        stencil_order=2, report_every=None, report_label="", sheet_impedance=None, device=None) -> SimResult:
    """Uniform-grid scan (rfx/simulation.py:1686).  Step order per
    rfx/simulation.py:1255-1685: H, CPML-H, E, CPML-E, PEC faces, PEC mask,
    soft sources, probes, NTFF box (an ``NTFFBox``), DFT planes at
    ``t = (n+1) dt``, flux monitors."""
    _unsupported(debye=debye, lorentz=lorentz, tfsf=tfsf,
                 waveguide_ports=waveguide_ports, snapshot=snapshot, aniso_eps=aniso_eps,
                 aniso_inv_eps=aniso_inv_eps, pec_occupancy=pec_occupancy, conformal_weights=conformal_weights,
                 wire_port_sparams=wire_port_sparams, wire_refplane_sparams=wire_refplane_sparams,
                 lumped_rlc=lumped_rlc, kerr_chi3=kerr_chi3, mag_sources=mag_sources,
                 sheet_impedance=sheet_impedance)
    if periodic is not None and any(periodic):
        raise NotImplementedError("periodic axes are outside this path")
    if stencil_order != 2:
        raise NotImplementedError("only the (2,2) Yee stencil is on this path")
    if field_dtype not in (None, np.float32, "float32", torch.float32):
        raise NotImplementedError("fields are float32 on this path")
    if checkpoint_segments is not None:
        K = int(checkpoint_segments)
        if K < 1:
            raise ValueError(f"checkpoint_segments must be ≥ 1, got {checkpoint_segments}")
        if n_steps % K != 0:
            raise ValueError(f"checkpoint_segments={K} does not divide n_steps={n_steps}; pick a divisor")
        if report_every is not None:
            raise NotImplementedError("report_every is not supported together with checkpoint_segments")
    if pec_axes is None:
        pec_axes = "xyz"
    use_cpml = boundary == "cpml" and int(grid.cpml_layers) > 0
    if boundary not in ("pec", "cpml"):
        raise NotImplementedError(f"boundary={boundary!r} is outside this path")
    srcs = [(s.i, s.j, s.k, s.component, s.waveform) for s in (sources or [])]
    prbs = [(p.i, p.j, p.k, p.component) for p in (probes or [])]
    ts, planes, lumped, state, flux, ntff_data = run_device(
        grid, materials, n_steps, cpml_axes=cpml_axes if use_cpml else "", pec_axes=pec_axes, sources=srcs,
        probes=prbs, dft_planes=list(dft_planes or []), pec_mask=pec_mask, dft_time_offset=1,
        lumped_specs=list(lumped_port_sparams or []), return_state=return_state, report_every=report_every,
        report_label=report_label, noop_faces=set(getattr(grid, "pec_faces", None) or ()),
        flux_monitors=list(flux_monitors or []), ntff_box=ntff, device=device)
    return SimResult(state=state, time_series=ts, ntff_data=ntff_data, dft_planes=planes if dft_planes else None,
                     flux_monitors=flux if flux_monitors else None, lumped_port_sparams=lumped, ntff_box=ntff,
                     grid=grid)


def run_until_decay(grid, materials, *, decay_by=1e-3, check_interval=50, min_steps=100, max_steps=50_000,
                    decay_energy_consecutive=2, radiated_flux_box=None, flux_env_checks=4, monitor_component="ez",
                    monitor_position=None, boundary="pec", cpml_axes="xyz", pec_axes=None, periodic=None,
                    debye=None, lorentz=None, tfsf=None, sources=None, probes=None, dft_planes=None,
                    flux_monitors=None, waveguide_ports=None, ntff=None, snapshot=None, checkpoint=False,
                    aniso_eps=None, aniso_inv_eps=None, aniso_inv_eps_smooth=False, pec_mask=None,
                    pec_occupancy=None, conformal_weights=None, wire_port_sparams=None, lumped_port_sparams=None,
                    lumped_rlc=None, kerr_chi3=None, field_dtype=None, return_state=True, mag_sources=None,
                    checkpoint_segments=None, stencil_order=2, report_every=None, report_label="",
                    sheet_impedance=None, device=None) -> SimResult:
    """Run until the field energy decays (rfx/simulation.py:2198-2700).

    Absorbing boundary: every ``check_interval`` steps (once ``min_steps`` are
    done) the interior energy U = sum(E^2 + H^2) over the non-CPML slice is
    reduced on the device (float64 accumulation); the run stops after
    ``decay_energy_consecutive`` consecutive checks with U < decay_by * peak U.
    With ``radiated_flux_box`` = ((x0, y0, z0), (x1, y1, z1)) on an absorbing
    boundary the stop uses the net outgoing Poynting flux through that box
    instead (rfx/simulation.py:2513-2540, 2580-2600): computed on the device
    at every check step from the first, its |value| enveloped by the maximum
    over the last ``flux_env_checks`` checks, and ``decay_energy_consecutive``
    checks (once ``min_steps`` are done) with the envelope below decay_by
    times its running peak stop the run.
    Closed boundary: the squared field ``monitor_component`` at
    ``monitor_position`` (default: the domain centre) keeps a running peak
    over every step, and a check step with value^2 < decay_by * peak stops.
    The steps run between checks are replayed as one captured chunk."""
    _unsupported(debye=debye, lorentz=lorentz, tfsf=tfsf,
                 waveguide_ports=waveguide_ports, aniso_eps=aniso_eps, aniso_inv_eps=aniso_inv_eps,
                 pec_occupancy=pec_occupancy, conformal_weights=conformal_weights,
                 wire_port_sparams=wire_port_sparams, lumped_port_sparams=lumped_port_sparams,
                 lumped_rlc=lumped_rlc, kerr_chi3=kerr_chi3, mag_sources=mag_sources,
                 sheet_impedance=sheet_impedance)
    if checkpoint_segments is not None:
        raise NotImplementedError("checkpoint_segments is not supported by run_until_decay "
                                  "(rfx/simulation.py:2289-2294)")
    if periodic is not None and any(periodic):
        raise NotImplementedError("periodic axes are outside this path")
    if stencil_order != 2:
        raise NotImplementedError("only the (2,2) Yee stencil is on this path")
    if boundary not in ("pec", "cpml"):
        raise NotImplementedError(f"boundary={boundary!r} is outside this path")
    if check_interval < 1 or max_steps < 1:
        raise ValueError("check_interval and max_steps must be >= 1")
    if pec_axes is None:
        pec_axes = "xyz"
    absorbing = boundary == "cpml"
    use_cpml = absorbing and int(grid.cpml_layers) > 0
    srcs = [(s.i, s.j, s.k, s.component, s.waveform) for s in (sources or [])]
    for s in srcs:
        if np.asarray(s[4]).shape[0] < max_steps:
            raise ValueError("source waveforms must cover max_steps")
    prbs = [(p.i, p.j, p.k, p.component) for p in (probes or [])]
    n_user = len(prbs)
    if not absorbing:
        if monitor_position is None:
            mon = (grid.nx // 2, grid.ny // 2, grid.nz // 2)
        else:
            mon = tuple(grid.position_to_index(monitor_position))
        prbs.append((*mon, monitor_component))
    planes = list(dft_planes or [])
    r = prepare_device_run(grid, materials, max_steps, cpml_axes=cpml_axes if use_cpml else "", pec_axes=pec_axes,
                           sources=srcs, probes=prbs, dft_planes=planes, pec_mask=pec_mask, dft_time_offset=1,
                           noop_faces=set(getattr(grid, "pec_faces", None) or ()), ntff_box=ntff,
                           flux_monitors=list(flux_monitors or []), device=device)
    plan = r.plan
    try:
        box = (grid.pad_x_lo, grid.nx - grid.pad_x_hi, grid.pad_y_lo, grid.ny - grid.pad_y_hi,
               grid.pad_z_lo, grid.nz - grid.pad_z_hi)
        energy = torch.empty((), device=plan.device, dtype=torch.float64)
        peak_u, below, peak_sq = 0.0, 0, 0.0
        flux_stop = radiated_flux_box is not None and absorbing
        if flux_stop:
            lo = grid.position_to_index(radiated_flux_box[0])
            hi = grid.position_to_index(radiated_flux_box[1])
            fbox = (min(lo[0], hi[0]), max(lo[0], hi[0]), min(lo[1], hi[1]), max(lo[1], hi[1]),
                    min(lo[2], hi[2]), max(lo[2], hi[2]))
            peak_flux, flux_hist = 0.0, []
        # first check step: the flux stop tracks its peak from step 0, the
        # other stops only check once min_steps are done
        n_check = 0 if flux_stop else -(-(max(min_steps, 1) - 1) // check_interval) * check_interval
        done = 0
        fired = False
        while done < max_steps:
            target = min(n_check + 1, max_steps)
            # steps done .. target-1, relative to the tables' row `done` (the
            # captured chunk is then reused for every later check interval)
            plan.advance(0, target - done,
                         r.src_table[done:] if r.src_table is not None else None,
                         r.probe_out[done:] if r.probe_out is not None else None,
                         r.dft_accs, [ph[done:] for ph in r.dft_phases], r.flux_accs,
                         [k[done:] for k in r.flux_kernels],
                         ntff=(r.ntff[0], r.ntff[1], r.ntff[2][done:]) if r.ntff is not None else None)
            first, done = done, target
            if done - 1 != n_check:
                break
            if flux_stop:
                flux_hist.append(abs(float(plan.box_flux(fbox, energy).item())))
                env = max(flux_hist[-flux_env_checks:])
                peak_flux = max(peak_flux, env)
                if done >= min_steps and peak_flux > 0.0 and env < decay_by * peak_flux:
                    below += 1
                    if below >= decay_energy_consecutive:
                        break
                else:
                    below = 0
            elif absorbing:
                u = float(plan.box_energy(box, energy).item())
                peak_u = max(peak_u, u)
                if u < decay_by * peak_u:
                    below += 1
                    if below >= decay_energy_consecutive:
                        fired = True
                        break
                else:
                    below = 0
            else:
                v = r.probe_out[first:done, -1].double().cpu().numpy()
                peak_sq = max(peak_sq, float(np.max(v * v)))
                if peak_sq > 0.0 and float(v[-1]) ** 2 < decay_by * peak_sq:
                    break
            n_check += check_interval
        plan.check_device()
        ts = r.probe_out[:done, :n_user].cpu().numpy() if r.probe_out is not None else np.zeros((done, 0),
                                                                                               np.float32)
        out_planes = tuple(d._replace(accumulator=a.cpu().numpy()) for d, a in zip(planes, r.dft_accs))
        state = None
        fields = None
        if return_state or (absorbing and not flux_stop and not fired):
            fields = [t.cpu().numpy() for t in plan.store_fields()]
        if absorbing and not flux_stop and not fired:
            warn_static_remnant_cap_hit(fields, materials, grid)
        if return_state:
            state = FDTDState(*fields, step=done)
        ntff_data = unpack_ntff(ntff, r.ntff[0], r.ntff[1]) if ntff is not None else None
        flux = None
        if flux_monitors:
            flux = []
            for m, a in zip(flux_monitors, r.flux_accs):
                a = a.cpu().numpy()
                flux.append(m._replace(e1_dft=a[0], e2_dft=a[1], h1_dft=a[2], h2_dft=a[3]))
            flux = tuple(flux)
        return SimResult(state=state, time_series=ts, ntff_data=ntff_data,
                         dft_planes=out_planes if planes else None, flux_monitors=flux, ntff_box=ntff, grid=grid)
    finally:
        plan.close()


def warn_static_remnant_cap_hit(fields, materials, grid) -> bool:
    """The measured post-run advisory of rfx/simulation.py:2145-2197 (issue
    #388), used by both lanes' decay loops when max_steps was reached and the
    interior-energy criterion never fired.

    A soft current source can leave a static charge remnant whose electric
    self-energy neither radiates nor is absorbed, so the interior energy stays
    above decay_by * peak.  A radiating field splits its energy roughly evenly
    between E and H; the remnant is electric only.  When the magnetic share of
    the final interior energy (0.5 eps |E|^2 vs 0.5 mu |H|^2 over the cells
    inside the CPML pads) is below 1e-2 this warns (UserWarning) and returns
    True."""
    import warnings
    ex, ey, ez, hx, hy, hz = (np.asarray(f, np.float64) for f in fields)
    nx, ny, nz = ex.shape
    sl = (slice(grid.pad_x_lo, nx - grid.pad_x_hi), slice(grid.pad_y_lo, ny - grid.pad_y_hi),
          slice(grid.pad_z_lo, nz - grid.pad_z_hi))
    eps = np.asarray(materials.eps_r, np.float64)[sl]
    mu = getattr(materials, "mu_r", None)
    mu = np.asarray(mu, np.float64)[sl] if mu is not None and np.ndim(mu) > 0 else 1.0
    u_e = 0.5 * EPS_0 * float(np.sum(eps * (ex[sl] ** 2 + ey[sl] ** 2 + ez[sl] ** 2)))
    u_h = 0.5 * MU_0 * float(np.sum(mu * (hx[sl] ** 2 + hy[sl] ** 2 + hz[sl] ** 2)))
    tot = u_e + u_h
    if tot <= 0.0:
        return False
    h_share = u_h / tot
    if h_share >= 1e-2:
        return False
    warnings.warn(
        f"run_until_decay reached max_steps without the interior-energy criterion firing, and "
        f"{100.0 * (1.0 - h_share):.1f}% of the final interior energy is electric (magnetic share "
        f"{h_share:.1e}): a static charge remnant of the soft source is holding the interior energy "
        f"above decay_by * peak while the radiating field has settled.  Stop on the radiated flux "
        f"instead (radiated_flux_box=((x0, y0, z0), (x1, y1, z1)) around the radiator), lower the "
        f"source's DC content, or run a fixed n_steps.", UserWarning, stacklevel=3)
    return True


def extract_lumped_s11(v_dft, i_dft, z0=50.0):
    """rfx/probes/probes.py:1240-1274."""
    denom = v_dft - z0 * i_dft
    safe = np.where(np.abs(denom) > 0.0, denom, np.ones_like(denom))
    return (v_dft + z0 * i_dft) / safe
