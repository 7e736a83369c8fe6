"""JAX face of the CUDA path: XLA FFI custom calls and a ``jax.custom_vjp``.

The reference runs its time stepping as the body of a ``jax.lax.scan``
(rfx/simulation.py:1958-1977) inside ``Simulation.forward`` under ``jax.jit``
(rfx/api/_execute.py:1534) and differentiates it with ``jax.grad``.  This
module is the drop-in for that seam: the scan becomes one custom call per
direction, registered with XLA through ``jax.ffi`` (handlers in
``rfx_b200/csrc/ffi/rfxb_ffi.cc``, built by ``rfx_b200.build.build_ffi``
where jaxlib's FFI headers exist), and ``probe_traces`` pairs the recording
forward with the hand-written adjoint as a ``jax.custom_vjp`` -- the JAX twin
of ``rfx_b200.adjoint.FDTDFunction``.

Importing this module needs ``jax``; everything else in ``rfx_b200`` works
without it.  There is no fallback: without the built FFI library the calls
raise.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

import jax
import jax.numpy as jnp

from .adjoint import coefficient_derivatives
from .build import FFI_LIB
from .cpml import build_cpml
from .engine import Plan, PlanSpec
from .grid import EPS_0, spacing_tables

_TARGETS = ("rfxb_ffi_forward", "rfxb_ffi_forward_record", "rfxb_ffi_adjoint")
_SYMBOLS = ("RfxbFfiForward", "RfxbFfiForwardRecord", "RfxbFfiAdjoint")
_registered = False


def register():
    """Load ``librfxb200_ffi.so`` and register its handlers for the CUDA
    platform (once per process)."""
    global _registered
    if _registered:
        return
    if not os.path.exists(FFI_LIB):
        raise RuntimeError(f"{FFI_LIB} is not built: run rfx_b200.build.build_ffi() with jaxlib installed")
    lib = C.CDLL(FFI_LIB)
    for name, sym in zip(_TARGETS, _SYMBOLS):
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(lib, sym)), platform="CUDA")
    _registered = True


class JaxFDTD:
    """One simulation whose scan is an XLA custom call.

    ``grid``, ``materials`` (base eps_r / sigma of the whole grid), ``sources``
    ((i, j, k, comp, waveform)), ``probes`` ((i, j, k, comp)) and the gradient
    region ``box`` follow ``rfx_b200.adjoint.AdjointRunner``.  The plan holds
    the forward history between the forward and backward halves of
    ``probe_traces``, so one instance serves one differentiation at a time."""

    def __init__(self, grid, materials, n_steps, *, sources, probes, box, boundary="cpml", cpml_axes="xyz",
                 pec_axes=""):
        register()
        self.n_steps = int(n_steps)
        self.box = tuple(int(v) for v in box)
        shape = tuple(int(v) for v in grid.shape)
        use_cpml = boundary == "cpml" and int(grid.cpml_layers) > 0 and bool(cpml_axes)
        self.sources = [tuple(s[:4]) for s in sources]
        self.probes = [tuple(p[:4]) for p in probes]
        spec = PlanSpec(shape=shape, dt=float(grid.dt), tables=spacing_tables(grid),
                        cpml=build_cpml(grid, cpml_axes) if use_cpml else None, pec_axes=pec_axes,
                        sources=self.sources, probes=[(i, j, k, c, False) for (i, j, k, c) in self.probes],
                        grad_box=self.box)
        self.plan = Plan(spec)
        self.dt = float(grid.dt)
        self.eps = jnp.asarray(np.asarray(materials.eps_r, np.float32))
        self.sigma = jnp.asarray(np.asarray(materials.sigma, np.float32))
        tab = (np.stack([np.asarray(s[4], np.float32) for s in sources], axis=-1)[: self.n_steps]
               if sources else np.zeros((self.n_steps, 0), np.float32))
        self.src_table = jnp.asarray(np.ascontiguousarray(tab))
        self._attrs = dict(plan=np.int64(self.plan.handle.value), n_steps=np.int64(self.n_steps))
        fshape = jax.ShapeDtypeStruct(shape, jnp.float32)
        self._fwd_types = (jax.ShapeDtypeStruct((self.n_steps, len(self.probes)), jnp.float32),) + (fshape,) * 6
        i0, i1, j0, j1, k0, k1 = self.box
        self._box_shape = (i1 - i0, j1 - j0, k1 - k0)
        self._adj_types = (jax.ShapeDtypeStruct(self._box_shape, jnp.float64),
                           jax.ShapeDtypeStruct((self.n_steps, len(self.sources)), jnp.float32))
        self.probe_traces = self._make_vjp()

    def _eps_full(self, eps_box):
        i0, i1, j0, j1, k0, k1 = self.box
        return self.eps.at[i0:i1, j0:j1, k0:k1].set(eps_box.astype(jnp.float32))

    def forward(self, eps_r=None, src_table=None):
        """Probe traces (n_steps, n_probes) and the six final fields."""
        out = jax.ffi.ffi_call("rfxb_ffi_forward", self._fwd_types)(
            self.eps if eps_r is None else eps_r, self.sigma,
            self.src_table if src_table is None else src_table, **self._attrs)
        return out[0], out[1:]

    def _coef_derivs(self, eps_box):
        """d ca / d eps_r and d cb / d eps_r over the region
        (rfx/core/yee.py:387-393; the same formula as coefficient_derivatives)."""
        i0, i1, j0, j1, k0, k1 = self.box
        e = eps_box.astype(jnp.float32)
        s = self.sigma[i0:i1, j0:j1, k0:k1]
        L = s * self.dt / (2.0 * EPS_0 * e)
        dca = 2.0 * L / (e * (1.0 + L) ** 2)
        dcb = -self.dt * EPS_0 / (EPS_0 * e + s * self.dt / 2.0) ** 2
        return dca.astype(jnp.float32), dcb.astype(jnp.float32)

    def _make_vjp(self):
        @jax.custom_vjp
        def traces(eps_box, src_table):
            return self.forward(self._eps_full(eps_box), src_table)[0]

        def fwd(eps_box, src_table):
            out = jax.ffi.ffi_call("rfxb_ffi_forward_record", self._fwd_types)(
                self._eps_full(eps_box), self.sigma, src_table, **self._attrs)
            return out[0], eps_box

        def bwd(eps_box, g):
            dca, dcb = self._coef_derivs(eps_box)
            grad, src_adj = jax.ffi.ffi_call("rfxb_ffi_adjoint", self._adj_types)(
                g.astype(jnp.float32), dca, dcb, **self._attrs)
            return grad.astype(eps_box.dtype), src_adj

        traces.defvjp(fwd, bwd)
        return traces

    def close(self):
        self.plan.close()


__all__ = ["JaxFDTD", "register", "coefficient_derivatives"]
