"""State files: the reference's HDF5 helpers and a resumable plan state.

``save_state`` / ``load_state`` / ``save_snapshots`` / ``load_snapshots`` /
``save_materials`` / ``load_materials`` follow rfx/checkpoint.py:33-186: the
same HDF5 groups, datasets and attributes, and the same ``ImportError`` when
h5py is missing (as it is in this image).

``save_plan_state`` / ``load_plan_state`` write and read the complete
resumable state of a device plan -- fields, CPML psi and the DFT Kahan
residuals, as the C ABI's ``rfxb_plan_save_state`` blob -- plus the step, in
a NumPy ``.npz`` file, so a long run or sweep restarts bit for bit.  The
reference's HDF5 state holds the fields and the step only; a CPML run resumed
from it restarts its psi at zero.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

try:
    import h5py
except ImportError:
    h5py = None

from .simulation import FDTDState, MaterialArrays

_COMPONENTS = ("ex", "ey", "ez", "hx", "hy", "hz")


def _require_h5py():
    """rfx/checkpoint.py:26-31."""
    if h5py is None:
        raise ImportError("h5py is required for checkpoint save/load. Install with: pip install h5py")


def _grid_attrs(g, grid):
    g.attrs["shape"] = list(grid.shape)
    g.attrs["dx"] = grid.dx
    g.attrs["dt"] = grid.dt
    g.attrs["freq_max"] = getattr(grid, "freq_max", 0.0)
    g.attrs["mode"] = getattr(grid, "mode", "3d")


def save_state(path, state: FDTDState, grid=None) -> None:
    """rfx/checkpoint.py:33-62: group ``state`` with the six fields and a
    ``step`` attribute; group ``grid`` with shape, dx, dt, freq_max, mode,
    cpml_layers."""
    _require_h5py()
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with h5py.File(path, "w") as f:
        grp = f.create_group("state")
        for name in _COMPONENTS:
            grp.create_dataset(name, data=np.asarray(getattr(state, name)))
        grp.attrs["step"] = int(state.step)
        if grid is not None:
            g = f.create_group("grid")
            _grid_attrs(g, grid)
            g.attrs["cpml_layers"] = grid.cpml_layers


def load_state(path):
    """rfx/checkpoint.py:65-97: (FDTDState, grid metadata dict)."""
    _require_h5py()
    with h5py.File(Path(path), "r") as f:
        grp = f["state"]
        fields = {name: np.asarray(grp[name][:]) for name in _COMPONENTS}
        state = FDTDState(**fields, step=int(grp.attrs.get("step", 0)))
        meta = {}
        if "grid" in f:
            meta = {k: f["grid"].attrs[k] for k in f["grid"].attrs}
            if "shape" in meta:
                meta["shape"] = tuple(meta["shape"])
    return state, meta


def save_snapshots(path, snapshots: dict, grid=None, dt: float | None = None) -> None:
    """rfx/checkpoint.py:100-135."""
    _require_h5py()
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with h5py.File(path, "w") as f:
        grp = f.create_group("snapshots")
        for name, arr in snapshots.items():
            grp.create_dataset(name, data=np.asarray(arr))
        if dt is not None:
            grp.attrs["dt"] = dt
            grp.attrs["n_steps"] = next(iter(snapshots.values())).shape[0]
        if grid is not None:
            _grid_attrs(f.create_group("grid"), grid)


def load_snapshots(path):
    """rfx/checkpoint.py:138-161: (snapshots dict, metadata dict)."""
    _require_h5py()
    with h5py.File(Path(path), "r") as f:
        grp = f["snapshots"]
        snaps = {name: np.asarray(grp[name][:]) for name in grp}
        meta = dict(grp.attrs)
        if "grid" in f:
            meta.update({k: f["grid"].attrs[k] for k in f["grid"].attrs})
            if "shape" in meta:
                meta["shape"] = tuple(meta["shape"])
    return snaps, meta


def save_materials(path, materials: MaterialArrays) -> None:
    """rfx/checkpoint.py:164-174."""
    _require_h5py()
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with h5py.File(path, "w") as f:
        grp = f.create_group("materials")
        for name in ("eps_r", "sigma", "mu_r"):
            grp.create_dataset(name, data=np.asarray(getattr(materials, name)))


def load_materials(path) -> MaterialArrays:
    """rfx/checkpoint.py:177-186."""
    _require_h5py()
    with h5py.File(Path(path), "r") as f:
        grp = f["materials"]
        return MaterialArrays(eps_r=np.asarray(grp["eps_r"][:]), sigma=np.asarray(grp["sigma"][:]),
                              mu_r=np.asarray(grp["mu_r"][:]))


def save_plan_state(path, plan, step: int, grid=None) -> None:
    """Write ``plan``'s resumable device state after ``step`` steps."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    meta = {"step": int(step), "shape": list(plan.shape)}
    if grid is not None:
        meta.update(dx=float(grid.dx), dt=float(grid.dt), cpml_layers=int(grid.cpml_layers))
    with open(path, "wb") as fh:
        np.savez(fh, blob=plan.save_state(), meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))


def load_plan_state(path, plan) -> tuple[int, dict]:
    """Restore a state file of :func:`save_plan_state` into ``plan`` (same
    shape, CPML and DFT set-up; else the C ABI's shape error).  Returns
    (step, metadata); the caller continues with ``advance(step, ...)``."""
    with np.load(Path(path), allow_pickle=False) as z:
        blob = z["blob"]
        meta = json.loads(bytes(z["meta"]).decode())
    if tuple(meta["shape"]) != tuple(plan.shape):
        raise ValueError(f"state file holds a {tuple(meta['shape'])} grid, the plan is {tuple(plan.shape)}")
    plan.restore_state(blob)
    return int(meta["step"]), meta
