"""Plan objects: the Python face of one (or a batch of) device simulations.

A :class:`Plan` wraps ``RfxbPlan`` from the C ABI.  It takes host-side
setup (spacing tables, CPML profiles, monitor cells) once, keeps the
simulation state resident in HBM, and advances it with the fused step
kernel.  Device buffers the caller owns (materials, source tables, probe
outputs, DFT accumulators, adjoint tables) are torch tensors.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import RfxbAdjointIO, RfxbDesc, RfxbDftDesc, RfxbLaunchConfig, RfxbStepIO, check

COMP = {"ex": 0, "ey": 1, "ez": 2, "hx": 3, "hy": 4, "hz": 5}
PROBE_PRESOURCE = 16
AXES = {"x": 1, "y": 2, "z": 4}


def axes_mask(axes: str) -> int:
    m = 0
    for a in axes or "":
        m |= AXES[a]
    return m


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("rfx_b200 runs on a CUDA device only (no CPU fallback); no GPU is visible")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if dev.type != "cuda":
        raise RuntimeError(f"rfx_b200 needs a CUDA device, got {dev}")
    return dev


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


_LAUNCH_FIELDS = ("fwd_split", "fwd_order", "adj_lite", "adj_order", "fwd_persist", "adj_persist", "l2_promo",
                  "fwd_depth")


def _get_launch(getter, h):
    cur, lim = RfxbLaunchConfig(), RfxbLaunchConfig()
    check(getter(h, C.byref(cur), C.byref(lim)), getter.__name__)
    return ({f: int(getattr(cur, f)) for f in _LAUNCH_FIELDS}, {f: int(getattr(lim, f)) for f in _LAUNCH_FIELDS})


def _set_launch(getter, setter, h, fields):
    unknown = set(fields) - set(_LAUNCH_FIELDS)
    if unknown:
        raise ValueError(f"unknown launch configuration fields {sorted(unknown)}")
    cur, _ = _get_launch(getter, h)
    cur.update({k: int(v) for k, v in fields.items()})
    check(setter(h, C.byref(RfxbLaunchConfig(**cur))), setter.__name__)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_lib.c_float_p)


def _dptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


@dataclass
class CPMLSetup:
    """Per-face float32 CPML profiles (faces x_lo, x_hi, y_lo, y_hi, z_lo, z_hi)."""
    layers: int
    axes: str
    b: np.ndarray        # (6, layers)
    c: np.ndarray
    kappa: np.ndarray
    cell: tuple          # 6 boundary cell sizes


@dataclass
class PlanSpec:
    shape: tuple
    dt: float
    tables: tuple                     # (xe, xh, ye, yh, ze, zh) float32
    cpml: CPMLSetup | None = None
    pec_axes: str = ""
    sources: list = field(default_factory=list)   # (i, j, k, comp)
    probes: list = field(default_factory=list)    # (i, j, k, comp, presource)
    dft: list = field(default_factory=list)       # (axis, index, comp, n_freqs)
    grad_box: tuple | None = None                 # (i0, i1, j0, j1, k0, k1)
    flux: list = field(default_factory=list)      # (axis, index, lo1, hi1, lo2, hi2, n_freqs)
    ntff: tuple | None = None                     # (i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, n_freqs)


class Plan:
    """One resident simulation on the current CUDA device."""

    def __init__(self, spec: PlanSpec, device=None):
        self.device = require_cuda(device)
        self.spec = spec
        lib = _lib.load()
        nx, ny, nz = (int(v) for v in spec.shape)
        self.shape = (nx, ny, nz)
        tabs = [np.ascontiguousarray(t, dtype=np.float32) for t in spec.tables]
        for t, n in zip(tabs, (nx, nx, ny, ny, nz, nz)):
            if t.shape != (n,):
                raise ValueError(f"spacing table of length {t.shape} does not match axis length {n}")
        self._keep = list(tabs)
        d = RfxbDesc()
        d.nx, d.ny, d.nz = nx, ny, nz
        d.dt = float(spec.dt)
        (d.inv_xe_host, d.inv_xh_host, d.inv_ye_host, d.inv_yh_host,
         d.inv_ze_host, d.inv_zh_host) = [_fptr(t) for t in tabs]
        cp = spec.cpml
        if cp is not None and cp.layers > 0 and cp.axes:
            b = np.ascontiguousarray(cp.b, np.float32).reshape(6, cp.layers)
            c = np.ascontiguousarray(cp.c, np.float32).reshape(6, cp.layers)
            k = np.ascontiguousarray(cp.kappa, np.float32).reshape(6, cp.layers)
            self._keep += [b, c, k]
            d.cpml_layers = int(cp.layers)
            d.cpml_axes = axes_mask(cp.axes)
            d.cpml_b_host, d.cpml_c_host, d.cpml_kappa_host = _fptr(b), _fptr(c), _fptr(k)
            for f in range(6):
                d.cpml_cell[f] = float(cp.cell[f])
        else:
            d.cpml_layers = 0
            d.cpml_axes = 0
        d.pec_axes = axes_mask(spec.pec_axes)
        src = np.array([[i, j, k, COMP[cmp] if isinstance(cmp, str) else int(cmp)]
                        for (i, j, k, cmp) in spec.sources], dtype=np.int32).reshape(-1, 4)
        prb = np.array([[i, j, k, (COMP[cmp] if isinstance(cmp, str) else int(cmp))
                         | (PROBE_PRESOURCE if pre else 0)]
                        for (i, j, k, cmp, pre) in spec.probes], dtype=np.int32).reshape(-1, 4)
        src = np.ascontiguousarray(src)
        prb = np.ascontiguousarray(prb)
        self._keep += [src, prb]
        for a in src:
            if a[3] > 2:
                raise ValueError("soft sources drive E components only")
        d.n_src = len(src)
        d.src_cells_host = src.ctypes.data_as(_lib.c_int32_p)
        d.n_probe = len(prb)
        d.probe_cells_host = prb.ctypes.data_as(_lib.c_int32_p)
        dft_arr = (RfxbDftDesc * max(1, len(spec.dft)))()
        for q, (axis, index, comp, nf) in enumerate(spec.dft):
            dft_arr[q].axis = int(axis)
            dft_arr[q].index = int(index)
            dft_arr[q].component = COMP[comp] if isinstance(comp, str) else int(comp)
            dft_arr[q].n_freqs = int(nf)
        self._keep.append(dft_arr)
        d.n_dft = len(spec.dft)
        d.dft_host = C.cast(dft_arr, C.POINTER(RfxbDftDesc))
        gb = spec.grad_box or (0, 0, 0, 0, 0, 0)
        for q in range(6):
            d.grad_box[q] = int(gb[q])
        flux_arr = (_lib.RfxbFluxDesc * max(1, len(spec.flux)))()
        for q, fdesc in enumerate(spec.flux):
            for name, v in zip(("axis", "index", "lo1", "hi1", "lo2", "hi2", "n_freqs"), fdesc):
                setattr(flux_arr[q], name, int(v))
        self._keep.append(flux_arr)
        d.n_flux = len(spec.flux)
        d.flux_host = C.cast(flux_arr, C.POINTER(_lib.RfxbFluxDesc))
        if spec.ntff is not None:
            box = _lib.RfxbNtffDesc(*(int(v) for v in spec.ntff))
            self._keep.append(box)
            d.ntff_host = C.pointer(box)
        self.n_src = len(src)
        self.n_probe = len(prb)
        self.dft = list(spec.dft)
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(lib.rfxb_plan_create(C.byref(d), C.byref(self._h)), "rfxb_plan_create")
        self._lib = lib

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        # rfxb_plan_destroy synchronises the current device before freeing:
        # make that the plan's own device
        if getattr(self, "_h", None) and self._h.value:
            with torch.cuda.device(self.device):
                self._lib.rfxb_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def psi_entries(self) -> int:
        """CPML psi entries, E and H side, over all absorbing faces."""
        cp = self.spec.cpml
        if cp is None or cp.layers <= 0:
            return 0
        nx, ny, nz = self.shape
        cross = {"x": ny * nz, "y": nx * nz, "z": nx * ny}
        return sum(2 * 2 * 2 * cp.layers * cross[a] for a in cp.axes)

    def algorithmic_bytes_per_step(self) -> int:
        """Bytes one forward step must move at minimum: six fields read and
        written (48 B/cell), the ca/cb coefficients (8 B/cell), every psi entry
        read and written (8 B)."""
        nx, ny, nz = self.shape
        return 56 * nx * ny * nz + 8 * self.psi_entries()

    def adjoint_algorithmic_bytes_per_step(self) -> int:
        """Bytes one reverse step must move at minimum: the forward's (six
        adjoint fields read and written, ca/cb, adjoint psi read and written)
        plus, over the gradient region, the recorded history (6 floats) read
        and the float64 gradient read and written."""
        gb = self.spec.grad_box
        box = 0
        if gb:
            i0, i1, j0, j1, k0, k1 = gb
            box = max(0, i1 - i0) * max(0, j1 - j0) * max(0, k1 - k0)
        return self.algorithmic_bytes_per_step() + (24 + 16) * box

    def device_bytes(self) -> int:
        return int(self._lib.rfxb_plan_device_bytes(self._h))

    def box_energy(self, box, out=None):
        """Device scalar (float64 tensor) of sum(E^2 + H^2) over ``box`` =
        (i0, i1, j0, j1, k0, k1) of the current state, in stream order."""
        if out is None:
            out = torch.empty((), device=self.device, dtype=torch.float64)
        b = (C.c_int * 6)(*[int(v) for v in box])
        check(self._lib.rfxb_plan_box_energy(self._h, b, C.c_void_p(out.data_ptr()), _stream()),
              "rfxb_plan_box_energy")
        return out

    def box_energy_weighted(self, box, wx, wy, wz, out=None):
        """As ``box_energy`` with cell (i, j, k) weighted by wx[i] wy[j] wz[k]
        (float64 device tensors of length nx, ny, nz)."""
        if out is None:
            out = torch.empty((), device=self.device, dtype=torch.float64)
        ws = [w.to(device=self.device, dtype=torch.float64).contiguous() for w in (wx, wy, wz)]
        for w, n in zip(ws, self.shape):
            if w.numel() != n:
                raise ValueError("weight tables must have lengths nx, ny, nz")
        b = (C.c_int * 6)(*[int(v) for v in box])
        check(self._lib.rfxb_plan_box_energy_weighted(self._h, b, *[C.c_void_p(w.data_ptr()) for w in ws],
                                                      C.c_void_p(out.data_ptr()), _stream()),
              "rfxb_plan_box_energy_weighted")
        return out

    def box_flux(self, box, out=None):
        """Device scalar (float64 tensor) of the net outgoing co-located
        Poynting flux through the faces of ``box`` = (i0, i1, j0, j1, k0, k1)
        (face planes i0, i1, ...; tangential ranges half-open)."""
        if out is None:
            out = torch.empty((), device=self.device, dtype=torch.float64)
        b = (C.c_int * 6)(*[int(v) for v in box])
        check(self._lib.rfxb_plan_box_flux(self._h, b, C.c_void_p(out.data_ptr()), _stream()), "rfxb_plan_box_flux")
        return out

    def forward_variant(self) -> int:
        """0 generic step kernel, 1 TMA staging without CPML, 2 TMA staging
        with TMA-staged CPML psi."""
        return int(self._lib.rfxb_plan_forward_variant(self._h))

    def adjoint_variant(self) -> int:
        """0 cp.async staging, 1 TMA staging, 2 TMA staging with TMA-staged
        adjoint psi; -1 before the first adjoint advance."""
        return int(self._lib.rfxb_plan_adjoint_variant(self._h))

    def step_launches(self):
        """(step-kernel launches per forward step, per reverse step; -1
        before the first adjoint advance)."""
        f, r = C.c_int(), C.c_int()
        check(self._lib.rfxb_plan_step_launches(self._h, C.byref(f), C.byref(r)), "rfxb_plan_step_launches")
        return f.value, r.value

    def launch_config(self):
        """(current, limits) launch configuration dicts (``rfxb200.h``
        ``RfxbLaunchConfig``: fwd_split, fwd_order, adj_lite, adj_order)."""
        return _get_launch(self._lib.rfxb_plan_launch_config, self._h)

    def set_launch_config(self, **fields):
        """Change some launch-configuration fields (the rest keep their
        value); synchronises the device and drops the cached step graphs."""
        _set_launch(self._lib.rfxb_plan_launch_config, self._lib.rfxb_plan_set_launch_config, self._h, fields)

    # -- state ---------------------------------------------------------------
    def _dev(self, a, dtype=torch.float32):
        t = torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a)
        return t.to(device=self.device, dtype=dtype).contiguous()

    def set_materials(self, eps_r, sigma, mu_r=None, edge_mask=None):
        e = self._dev(eps_r)
        s = self._dev(sigma)
        if tuple(e.shape) != self.shape or tuple(s.shape) != self.shape:
            raise ValueError(f"material arrays must have shape {self.shape}")
        m = None
        if mu_r is not None:
            m = self._dev(mu_r)
            if bool((m == 1.0).all()):
                m = None
        em = self._dev(edge_mask, torch.uint8) if edge_mask is not None else None
        self._mat = (e, s, m, em)
        check(self._lib.rfxb_plan_set_materials(self._h, _dptr(e), _dptr(s), _dptr(m), _dptr(em), _stream()),
              "rfxb_plan_set_materials")

    def reset(self):
        check(self._lib.rfxb_plan_reset(self._h, _stream()), "rfxb_plan_reset")

    def load_fields(self, fields):
        ts = [self._dev(f) for f in fields]
        arr = (C.c_void_p * 6)(*[t.data_ptr() for t in ts])
        check(self._lib.rfxb_plan_load_fields(self._h, arr, _stream()), "rfxb_plan_load_fields")
        torch.cuda.current_stream().synchronize()

    def store_fields(self):
        out = [torch.empty(self.shape, device=self.device, dtype=torch.float32) for _ in range(6)]
        arr = (C.c_void_p * 6)(*[t.data_ptr() for t in out])
        check(self._lib.rfxb_plan_store_fields(self._h, arr, _stream()), "rfxb_plan_store_fields")
        return out

    # -- stepping ------------------------------------------------------------
    @staticmethod
    def step_io(src_table=None, probe_out=None, dft_accs=None, dft_phases=None, flux_accs=None, flux_kernels=None,
                ntff=None):
        """``ntff``: (running sums, Kahan residuals, phase table) device
        tensors of the NTFF box (layout in ``rfx_b200.simulation.NTFFData``)."""
        io = RfxbStepIO()
        io.src_wave_dev = src_table.data_ptr() if src_table is not None else None
        io.probe_out_dev = probe_out.data_ptr() if probe_out is not None else None
        keep = []
        if dft_accs:
            acc = (C.c_void_p * len(dft_accs))(*[a.data_ptr() for a in dft_accs])
            ph = (C.c_void_p * len(dft_phases))(*[p.data_ptr() for p in dft_phases])
            io.dft_acc_dev = C.cast(acc, C.POINTER(C.c_void_p))
            io.dft_phase_dev = C.cast(ph, C.POINTER(C.c_void_p))
            keep += [acc, ph]
        if flux_accs:
            acc = (C.c_void_p * len(flux_accs))(*[a.data_ptr() for a in flux_accs])
            kn = (C.c_void_p * len(flux_kernels))(*[k.data_ptr() for k in flux_kernels])
            io.flux_acc_dev = C.cast(acc, C.POINTER(C.c_void_p))
            io.flux_kernel_dev = C.cast(kn, C.POINTER(C.c_void_p))
            keep += [acc, kn]
        if ntff is not None:
            acc, cmp, ph = ntff
            io.ntff_acc_dev, io.ntff_cmp_dev, io.ntff_phase_dev = acc.data_ptr(), cmp.data_ptr(), ph.data_ptr()
        return io, keep

    def advance(self, step0, n_steps, src_table=None, probe_out=None, dft_accs=None, dft_phases=None,
                flux_accs=None, flux_kernels=None, ntff=None):
        io, keep = self.step_io(src_table, probe_out, dft_accs, dft_phases, flux_accs, flux_kernels, ntff)
        check(self._lib.rfxb_plan_advance(self._h, C.byref(io), int(step0), int(n_steps), _stream()),
              "rfxb_plan_advance")
        del keep

    def record_history(self, step0, n_steps):
        check(self._lib.rfxb_plan_record_history(self._h, int(step0), int(n_steps)), "rfxb_plan_record_history")

    def check_device(self):
        """Synchronise and raise if a bounded wait inside a kernel ran out."""
        check(self._lib.rfxb_plan_device_status(self._h, _stream()), "rfxb_plan_device_status")

    def save_state(self):
        """The plan's resumable state (fields, psi, DFT Kahan residuals) as a
        host uint8 array (``rfxb_plan_save_state``)."""
        n = int(self._lib.rfxb_plan_state_bytes(self._h))
        if n < 0:
            check(n, "rfxb_plan_state_bytes")
        out = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        check(self._lib.rfxb_plan_save_state(self._h, out.data_ptr(), _stream()), "rfxb_plan_save_state")
        torch.cuda.current_stream().synchronize()
        return out.numpy().copy()

    def restore_state(self, blob):
        """Load a blob of :meth:`save_state` (same shape and set-up)."""
        src = torch.from_numpy(np.ascontiguousarray(blob, np.uint8)).pin_memory()
        check(self._lib.rfxb_plan_restore_state(self._h, src.data_ptr(), _stream()), "rfxb_plan_restore_state")
        torch.cuda.current_stream().synchronize()

    def checkpoint_reserve(self, n):
        check(self._lib.rfxb_plan_checkpoint_reserve(self._h, int(n)), "rfxb_plan_checkpoint_reserve")

    def checkpoint_save(self, slot):
        check(self._lib.rfxb_plan_checkpoint_save(self._h, int(slot), _stream()), "rfxb_plan_checkpoint_save")

    def checkpoint_load(self, slot):
        check(self._lib.rfxb_plan_checkpoint_load(self._h, int(slot), _stream()), "rfxb_plan_checkpoint_load")

    # -- adjoint -------------------------------------------------------------
    @staticmethod
    def adjoint_io(g=None, grad=None, dca=None, dcb=None, src_adj=None, dft_cots=None, dft_phases=None,
                   ntff=None, flux_cots=None, flux_kernels=None):
        """``dft_cots``: per DFT plane a complex64 cotangent (n_freqs, n1, n2)
        or None; ``dft_phases``: the phase tables the forward used; ``ntff``:
        (flat complex64 cotangent of the NTFF faces, the forward's NTFF phase
        table) or None; ``flux_cots``: per flux monitor a complex128 cotangent
        (4, n_freqs, n1, n2) or None, with the forward's ``flux_kernels``."""
        a = RfxbAdjointIO()
        a.g_dev = g.data_ptr() if g is not None else None
        a.grad_dev = grad.data_ptr() if grad is not None else None
        a.dca_dev = dca.data_ptr() if dca is not None else None
        a.dcb_dev = dcb.data_ptr() if dcb is not None else None
        a.src_adj_dev = src_adj.data_ptr() if src_adj is not None else None
        if dft_cots is not None and any(c is not None for c in dft_cots):
            cot = (C.c_void_p * len(dft_cots))(*[c.data_ptr() if c is not None else None for c in dft_cots])
            ph = (C.c_void_p * len(dft_phases))(*[t.data_ptr() for t in dft_phases])
            a.dft_cot_dev = C.cast(cot, C.POINTER(C.c_void_p))
            a.dft_phase_dev = C.cast(ph, C.POINTER(C.c_void_p))
            a._keep = (cot, ph)   # the pointer arrays live as long as the struct
        if ntff is not None:
            a.ntff_cot_dev, a.ntff_phase_dev = ntff[0].data_ptr(), ntff[1].data_ptr()
        if flux_cots is not None and any(c is not None for c in flux_cots):
            fc = (C.c_void_p * len(flux_cots))(*[c.data_ptr() if c is not None else None for c in flux_cots])
            fk = (C.c_void_p * len(flux_kernels))(*[t.data_ptr() for t in flux_kernels])
            a.flux_cot_dev = C.cast(fc, C.POINTER(C.c_void_p))
            a.flux_kernel_dev = C.cast(fk, C.POINTER(C.c_void_p))
            a._keep_flux = (fc, fk)
        return a

    def adjoint_begin(self, n_total, **kw):
        a = self.adjoint_io(**kw)
        check(self._lib.rfxb_plan_adjoint_begin(self._h, C.byref(a), int(n_total), _stream()),
              "rfxb_plan_adjoint_begin")

    def adjoint_advance(self, step_hi, n_steps, **kw):
        a = self.adjoint_io(**kw)
        check(self._lib.rfxb_plan_adjoint_advance(self._h, C.byref(a), int(step_hi), int(n_steps), _stream()),
              "rfxb_plan_adjoint_advance")


class Batch:
    """Several plans advanced together: one launch per step for all of them."""

    def __init__(self, plans):
        self.plans = list(plans)
        lib = _lib.load()
        arr = (C.c_void_p * len(self.plans))(*[p.handle.value for p in self.plans])
        self._h = C.c_void_p()
        check(lib.rfxb_batch_create(arr, len(self.plans), C.byref(self._h)), "rfxb_batch_create")
        self._lib = lib

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            with torch.cuda.device(self.plans[0].device):
                self._lib.rfxb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, step0, n_steps, ios):
        """``ios``: one dict per plan with keys of :meth:`Plan.step_io`."""
        arr = (RfxbStepIO * len(self.plans))()
        keep = []
        for q, kw in enumerate(ios):
            io, k = Plan.step_io(**kw)
            arr[q] = io
            keep += k
        check(self._lib.rfxb_batch_advance(self._h, arr, int(step0), int(n_steps), _stream()), "rfxb_batch_advance")
        del keep

    def record_history(self, step0, n_steps):
        check(self._lib.rfxb_batch_record_history(self._h, int(step0), int(n_steps)), "rfxb_batch_record_history")

    def check_device(self):
        check(self._lib.rfxb_batch_device_status(self._h, _stream()), "rfxb_batch_device_status")

    def step_launches(self):
        """(step-kernel launches per forward step, per reverse step)."""
        f, r = C.c_int(), C.c_int()
        check(self._lib.rfxb_batch_step_launches(self._h, C.byref(f), C.byref(r)), "rfxb_batch_step_launches")
        return f.value, r.value

    def launch_config(self):
        """(current, limits) launch configuration dicts, as ``Plan.launch_config``."""
        return _get_launch(self._lib.rfxb_batch_launch_config, self._h)

    def set_launch_config(self, **fields):
        """As ``Plan.set_launch_config``, for the whole batch."""
        _set_launch(self._lib.rfxb_batch_launch_config, self._lib.rfxb_batch_set_launch_config, self._h, fields)

    def adjoint_begin(self, n_total, aios):
        ios = [Plan.adjoint_io(**kw) for kw in aios]   # keeps the pointer arrays alive for the call
        arr = (RfxbAdjointIO * len(self.plans))(*ios)
        check(self._lib.rfxb_batch_adjoint_begin(self._h, arr, int(n_total), _stream()), "rfxb_batch_adjoint_begin")
        del ios

    def adjoint_advance(self, step_hi, n_steps, aios):
        ios = [Plan.adjoint_io(**kw) for kw in aios]
        arr = (RfxbAdjointIO * len(self.plans))(*ios)
        check(self._lib.rfxb_batch_adjoint_advance(self._h, arr, int(step_hi), int(n_steps), _stream()),
              "rfxb_batch_adjoint_advance")
        del ios
