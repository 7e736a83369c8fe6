"""Drop-in ``run_nonuniform()`` for the graded lane.

Mirrors ``rfx.nonuniform.run_nonuniform`` (rfx/nonuniform.py:1589-1804) for
the features on this path: the same source tuples ``(i, j, k, comp, wave)``,
probe tuples ``(i, j, k, comp)``, DFT planes and PEC mask, and the same
result dict keys.  Step order per rfx/nonuniform.py:1256-1568: H, CPML-H,
E, CPML-E, PEC on every axis, PEC mask, sources, DFT planes at ``t = n dt``,
NTFF box (``ntff_box`` with its initial ``ntff_data``), flux monitors
(E at t = n dt rounded to float32, H half a step earlier), probes.  ``checkpoint_every`` and ``n_warmup`` only shape the reference's
AD tape and do not change forward values; they are validated and accepted.
"""

from __future__ import annotations

import numpy as np

from .grid import face_pads
from .simulation import _unsupported, run_device


def run_nonuniform(grid, materials, n_steps, *, pec_mask=None, pec_occupancy=None, sources=None, probes=None,
                   wire_ports=None, s_param_freqs=None, debye=None, lorentz=None, pec_faces=None, pmc_faces=None,
                   dft_planes=None, rlc_metas=(), rlc_states=(), ntff_box=None, ntff_data=None,
                   waveguide_ports=None, tfsf=None, flux_monitors=None, checkpoint=False, emit_time_series=True,
                   checkpoint_every=None, n_warmup=0, aniso_eps=None, sheet_impedance=None, device=None) -> dict:
    _unsupported(pec_occupancy=pec_occupancy, wire_ports=wire_ports, debye=debye, lorentz=lorentz,
                 pmc_faces=pmc_faces, rlc_metas=rlc_metas, waveguide_ports=waveguide_ports,
                 tfsf=tfsf, aniso_eps=aniso_eps, sheet_impedance=sheet_impedance)
    if n_warmup and n_warmup >= n_steps:
        raise ValueError(f"n_warmup ({n_warmup}) must be < n_steps ({n_steps})")
    pads = face_pads(grid)
    axes = "".join(a for a, (lo, hi) in zip("xyz", (pads[0:2], pads[2:4], pads[4:6])) if lo + hi > 0)
    use_cpml = int(grid.cpml_layers) > 0
    srcs = [tuple(s) for s in (sources or [])]
    prbs = [tuple(p) for p in (probes or [])]
    if ntff_box is None or ntff_data is None:   # both or neither (rfx/nonuniform.py:1046)
        ntff_box = ntff_data = None
    ts, planes, _, state, flux, ntff_out = run_device(
        grid, materials, n_steps, cpml_axes=axes if use_cpml else "", pec_axes="xyz", sources=srcs,
        probes=prbs, dft_planes=list(dft_planes or []), pec_mask=pec_mask, dft_time_offset=0,
        return_state=True, noop_faces=set(pec_faces or ()), flux_monitors=list(flux_monitors or []),
        ntff_box=ntff_box, ntff_data=ntff_data, device=device)
    out = {"state": state, "time_series": ts if emit_time_series else None, "dt": grid.dt}
    if dft_planes:
        out["dft_planes"] = planes
    if flux_monitors:
        out["flux_monitors"] = flux
    if ntff_box is not None:
        out["ntff_data"] = ntff_out
    return out


def _interior_edges(d_full, pad_lo, pad_hi):
    """Cell-edge positions of the interior cells of a padded graded axis, 0
    at the first interior face (rfx/nonuniform.py:155-168, 425-438: the
    array is lo pad, interior, hi pad, bounding-node duplicate)."""
    d = np.asarray(d_full, np.float64)
    interior = d[pad_lo:len(d) - pad_hi - 1]
    return np.insert(np.cumsum(interior), 0, 0.0)


def position_to_index(grid, pos):
    """Physical (x, y, z) to graded-grid indices (rfx/nonuniform.py:477-524):
    the nearest interior cell edge on each axis, offset by the low pad."""
    pads = face_pads(grid)
    out = []
    for d, lo, hi, p in ((grid.dx_arr, pads[0], pads[1], pos[0]), (grid.dy_arr, pads[2], pads[3], pos[1]),
                         (grid.dz, pads[4], pads[5], pos[2])):
        edges = _interior_edges(d, lo, hi)
        out.append(int(np.argmin(np.abs(edges - float(p)))) + lo)
    return tuple(out)


def run_nonuniform_until_decay(grid, materials, *, decay_by=1e-3, check_interval=50, min_steps=100,
                               max_steps=50_000, decay_energy_consecutive=2, radiated_flux_box=None,
                               flux_env_checks=4, pec_mask=None, pec_occupancy=None, sources=None, probes=None,
                               wire_ports=None, s_param_freqs=None, debye=None, lorentz=None, pec_faces=None,
                               pmc_faces=None, dft_planes=None, rlc_metas=(), rlc_states=(), ntff_box=None,
                               ntff_data=None, waveguide_ports=None, tfsf=None, flux_monitors=None,
                               emit_time_series=True, aniso_eps=None, sheet_impedance=None, device=None) -> dict:
    """Graded-lane run until the interior energy decays
    (rfx/nonuniform.py:1988-2260).

    Chunks of ``check_interval`` steps (the last one shorter, so exactly
    ``max_steps`` bound the run) are replayed from captured graphs; after each
    chunk, once ``min_steps`` steps are done, the interior energy
    U = sum((Ex^2 + ... + Hz^2) dx[i] dy[j] dz[k]) over the non-CPML cells is
    reduced on the device (float64 accumulation), its running peak updated
    before the compare, and ``decay_energy_consecutive`` consecutive checks
    with U < decay_by * peak stop the run (``decay_by = 0`` never stops).
    With ``radiated_flux_box`` = ((x0, y0, z0), (x1, y1, z1)) the stop uses
    the net outgoing co-located Poynting flux through that box instead: its
    |value| after every chunk from the first, enveloped by the maximum of the
    last ``flux_env_checks`` checks, against decay_by times the envelope's
    running peak once ``min_steps`` are done.  Returns the ``run_nonuniform``
    dict plus ``decay_checks``, one ``(steps, U, peak U)`` per energy check.
    """
    import torch

    from .farfield import unpack_ntff
    from .simulation import FDTDState, prepare_device_run
    _unsupported(pec_occupancy=pec_occupancy, wire_ports=wire_ports, debye=debye, lorentz=lorentz,
                 pmc_faces=pmc_faces, rlc_metas=rlc_metas, waveguide_ports=waveguide_ports,
                 tfsf=tfsf, aniso_eps=aniso_eps, sheet_impedance=sheet_impedance)
    if check_interval < 1:
        raise ValueError(f"check_interval must be >= 1, got {check_interval}")
    if max_steps < 1:
        raise ValueError(f"max_steps must be >= 1, got {max_steps}")
    pads = face_pads(grid)
    axes = "".join(a for a, (lo, hi) in zip("xyz", (pads[0:2], pads[2:4], pads[4:6])) if lo + hi > 0)
    use_cpml = int(grid.cpml_layers) > 0
    # source tables padded with zeros / cut to max_steps (rfx/nonuniform.py:2113-2120)
    srcs = []
    for s in (sources or []):
        w = np.asarray(s[4], np.float32)[:max_steps]
        if w.shape[0] < max_steps:
            w = np.concatenate([w, np.zeros(max_steps - w.shape[0], np.float32)])
        srcs.append((int(s[0]), int(s[1]), int(s[2]), s[3], w))
    prbs = [tuple(p) for p in (probes or [])]
    if ntff_box is None or ntff_data is None:
        ntff_box = ntff_data = None
    planes = list(dft_planes or [])
    flux_monitors = list(flux_monitors or [])
    r = prepare_device_run(grid, materials, max_steps, cpml_axes=axes if use_cpml else "", pec_axes="xyz",
                           sources=srcs, probes=prbs, dft_planes=planes, pec_mask=pec_mask, dft_time_offset=0,
                           noop_faces=set(pec_faces or ()), flux_monitors=flux_monitors, ntff_box=ntff_box,
                           ntff_data=ntff_data, device=device)
    plan = r.plan
    try:
        box = (pads[0], grid.nx - pads[1], pads[2], grid.ny - pads[3], pads[4], grid.nz - pads[5])
        dev = plan.device
        wx, wy, wz = (torch.as_tensor(np.asarray(a, np.float64), device=dev)
                      for a in (grid.dx_arr, grid.dy_arr, grid.dz))
        scratch = torch.empty((), device=dev, dtype=torch.float64)
        flux_stop = radiated_flux_box is not None
        if flux_stop:
            lo = position_to_index(grid, radiated_flux_box[0])
            hi = position_to_index(grid, radiated_flux_box[1])
            fbox = (min(lo[0], hi[0]), max(lo[0], hi[0]), min(lo[1], hi[1]), max(lo[1], hi[1]),
                    min(lo[2], hi[2]), max(lo[2], hi[2]))
        peak_u, below, peak_flux, flux_hist, checks = 0.0, 0, 0.0, [], []
        done = 0
        fired = False
        while done < max_steps:
            k = min(int(check_interval), max_steps - done)
            plan.advance(0, k,
                         r.src_table[done:] if r.src_table is not None else None,
                         r.probe_out[done:] if r.probe_out is not None else None,
                         r.dft_accs, [ph[done:] for ph in r.dft_phases], r.flux_accs,
                         [q[done:] for q in r.flux_kernels],
                         ntff=(r.ntff[0], r.ntff[1], r.ntff[2][done:]) if r.ntff is not None else None)
            done += k
            if flux_stop:
                flux_hist.append(abs(float(plan.box_flux(fbox, scratch).item())))
                env = max(flux_hist[-flux_env_checks:])
                peak_flux = max(peak_flux, env)
                if done >= min_steps and peak_flux > 0.0 and env < decay_by * peak_flux:
                    below += 1
                    if below >= decay_energy_consecutive:
                        break
                else:
                    below = 0
            elif done >= min_steps:
                u = float(plan.box_energy_weighted(box, wx, wy, wz, scratch).item())
                peak_u = max(peak_u, u)
                checks.append((done, u, peak_u))
                if u < decay_by * peak_u:
                    below += 1
                    if below >= decay_energy_consecutive:
                        fired = True
                        break
                else:
                    below = 0
        plan.check_device()
        ts = r.probe_out[:done].cpu().numpy() if r.probe_out is not None else np.zeros((done, 0), np.float32)
        fields = [t.cpu().numpy() for t in plan.store_fields()]
        if not flux_stop and not fired:   # rfx/nonuniform.py:2234-2242
            from .simulation import warn_static_remnant_cap_hit
            warn_static_remnant_cap_hit(fields, materials, grid)
        state = FDTDState(*fields, step=done)
        out = {"state": state, "time_series": ts if emit_time_series else None, "dt": grid.dt,
               "decay_checks": checks}
        if planes:
            out["dft_planes"] = tuple(d._replace(accumulator=a.cpu().numpy()) for d, a in zip(planes, r.dft_accs))
        if flux_monitors:
            flux = []
            for m, a in zip(flux_monitors, r.flux_accs):
                a = a.cpu().numpy()
                flux.append(m._replace(e1_dft=a[0], e2_dft=a[1], h1_dft=a[2], h2_dft=a[3]))
            out["flux_monitors"] = tuple(flux)
        if ntff_box is not None:
            out["ntff_data"] = unpack_ntff(ntff_box, r.ntff[0], r.ntff[1])
        return out
    finally:
        plan.close()
