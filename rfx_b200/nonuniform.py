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
