"""Python face of ``rfxb_forward_noalloc``: forward steps without any device
allocation by the library.

For callers whose host program cannot let a library call cudaMalloc (its own
allocator owns device memory, or an allocation's device-wide synchronisation
is not acceptable inside its loop): the caller passes every buffer (materials,
fields in/out, source table, probe output) and the library uses a fixed 64 MiB
device array of its own for the internal state.  Grids larger than that state
(about 0.8 M cells) are rejected; use :class:`rfx_b200.engine.Plan` for them.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import RfxbDesc, RfxbStepIO, check
from .engine import COMP, PROBE_PRESOURCE, PlanSpec, axes_mask, require_cuda


def _desc(spec: PlanSpec):
    """RfxbDesc of a spec (no DFT planes, no gradient region) and the host
    arrays it points into."""
    nx, ny, nz = (int(v) for v in spec.shape)
    tabs = [np.ascontiguousarray(t, dtype=np.float32) for t in spec.tables]
    keep = list(tabs)
    d = RfxbDesc()
    d.nx, d.ny, d.nz = nx, ny, nz
    d.dt = float(spec.dt)
    fp = [t.ctypes.data_as(_lib.c_float_p) for t in tabs]
    d.inv_xe_host, d.inv_xh_host, d.inv_ye_host, d.inv_yh_host, d.inv_ze_host, d.inv_zh_host = fp
    cp = spec.cpml
    if cp is not None and cp.layers > 0 and cp.axes:
        arrs = [np.ascontiguousarray(a, np.float32).reshape(6, cp.layers) for a in (cp.b, cp.c, cp.kappa)]
        keep += arrs
        d.cpml_layers = int(cp.layers)
        d.cpml_axes = axes_mask(cp.axes)
        d.cpml_b_host, d.cpml_c_host, d.cpml_kappa_host = [a.ctypes.data_as(_lib.c_float_p) for a in arrs]
        for f in range(6):
            d.cpml_cell[f] = float(cp.cell[f])
    d.pec_axes = axes_mask(spec.pec_axes)
    def comp(c):
        return COMP[c] if isinstance(c, str) else int(c)

    src = np.ascontiguousarray(np.array([[i, j, k, comp(c)] for (i, j, k, c) in spec.sources],
                                        dtype=np.int32).reshape(-1, 4))
    prb = np.ascontiguousarray(np.array([[i, j, k, comp(c) | (PROBE_PRESOURCE if pre else 0)]
                                         for (i, j, k, c, pre) in spec.probes], dtype=np.int32).reshape(-1, 4))
    keep += [src, prb]
    d.n_src = len(src)
    d.src_cells_host = src.ctypes.data_as(_lib.c_int32_p)
    d.n_probe = len(prb)
    d.probe_cells_host = prb.ctypes.data_as(_lib.c_int32_p)
    d.n_dft = 0
    return d, keep


def forward_noalloc(spec: PlanSpec, eps_r, sigma, fields, src_table=None, probe_out=None, step0=0, n_steps=0):
    """Advance ``fields`` (six device tensors ex..hz, reference layout,
    updated in place) by ``n_steps`` steps of the simulation ``spec``.
    ``eps_r``/``sigma`` are device tensors of the grid shape; ``src_table``
    (n_total, n_src) and ``probe_out`` (n_total, n_probe) device tensors are
    indexed by global step.  Starts from zero CPML psi."""
    dev = require_cuda()
    lib = _lib.load()
    d, keep = _desc(spec)
    e = torch.as_tensor(eps_r, dtype=torch.float32, device=dev).contiguous()
    s = torch.as_tensor(sigma, dtype=torch.float32, device=dev).contiguous()
    for f in fields:
        if f.dtype != torch.float32 or not f.is_cuda or not f.is_contiguous():
            raise ValueError("fields must be contiguous float32 CUDA tensors")
    arr = (C.c_void_p * 6)(*[f.data_ptr() for f in fields])
    io = RfxbStepIO()
    io.src_wave_dev = src_table.data_ptr() if src_table is not None else None
    io.probe_out_dev = probe_out.data_ptr() if probe_out is not None else None
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.rfxb_forward_noalloc(C.byref(d), C.c_void_p(e.data_ptr()), C.c_void_p(s.data_ptr()), arr,
                                   C.byref(io), int(step0), int(n_steps), stream), "rfxb_forward_noalloc")
    del keep
