"""Near-to-far-field (NTFF) Huygens box: types, device buffers and the
far-field transform (rfx/farfield.py).

The running DFT of the tangential E and H on the box's six faces is
accumulated on the device once per step by ``ntff_kernel``
(``rfx_b200/csrc/rfxb_reduce.cu``), in complex64 with Kahan residuals as
rfx/farfield.py:208-313 does.  The accumulators live in one flat device
buffer per run (faces x_lo, x_hi, y_lo, y_hi, z_lo, z_hi back to back, each
(n_freqs, n1, n2, 4)); ``NTFFData`` returns them in the reference's layout.

``far_field`` is the post-run transform of rfx/farfield.py:393-556 (surface
currents J = n x H, M = -n x E, radiation vectors N and L, far-field E_theta /
E_phi) on torch tensors in complex128, one complex matrix product per face
and frequency, differentiable with respect to the face accumulators (with
``directivity_torch`` and the NTFF outputs of ``rfx_b200.adjoint.FDTDFunction``
it gives far-field objectives a gradient through the hand-written adjoint);
``compute_far_field`` wraps it with the reference's NumPy interface.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch

from .grid import C0, EPS_0, MU_0

ETA_0 = float(np.sqrt(MU_0 / EPS_0))
FACES = ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")


class NTFFBox(NamedTuple):
    """rfx/farfield.py:32-79: face planes i_lo, i_hi (x), j_lo, j_hi (y),
    k_lo, k_hi (z); each face covers [lo, hi) of its tangential axes."""
    i_lo: int
    i_hi: int
    j_lo: int
    j_hi: int
    k_lo: int
    k_hi: int
    freqs: np.ndarray
    cpml_lo_x: int = 0
    cpml_hi_x: int = 0
    cpml_lo_y: int = 0
    cpml_hi_y: int = 0
    cpml_lo_z: int = 0
    cpml_hi_z: int = 0

    @classmethod
    def from_grid(cls, grid, *, i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, freqs):
        """rfx/farfield.py:55-79: per-face CPML thicknesses from the grid."""
        fl = getattr(grid, "face_layers", None)
        if fl is None:
            n = int(getattr(grid, "cpml_layers", 0) or 0)
            fl = {f: n for f in FACES}
        return cls(i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, freqs, int(fl["x_lo"]), int(fl["x_hi"]), int(fl["y_lo"]),
                   int(fl["y_hi"]), int(fl["z_lo"]), int(fl["z_hi"]))


class NTFFData(NamedTuple):
    """rfx/farfield.py:81-104: complex64 running sums per face, shape
    (n_freqs, n1, n2, 4) (x faces: ey ez hy hz; y faces: ex ez hx hz; z faces:
    ex ey hx hy), and the Kahan residuals ``c_*`` of the same shape."""
    x_lo: np.ndarray
    x_hi: np.ndarray
    y_lo: np.ndarray
    y_hi: np.ndarray
    z_lo: np.ndarray
    z_hi: np.ndarray
    c_x_lo: np.ndarray = None
    c_x_hi: np.ndarray = None
    c_y_lo: np.ndarray = None
    c_y_hi: np.ndarray = None
    c_z_lo: np.ndarray = None
    c_z_hi: np.ndarray = None


class FarFieldResult(NamedTuple):
    """rfx/farfield.py:107-124."""
    E_theta: np.ndarray
    E_phi: np.ndarray
    theta: np.ndarray
    phi: np.ndarray
    freqs: np.ndarray


def make_ntff_box(grid, corner_lo, corner_hi, freqs) -> NTFFBox:
    """rfx/farfield.py:127-141: a box from physical corners."""
    lo = grid.position_to_index(corner_lo)
    hi = grid.position_to_index(corner_hi)
    return NTFFBox(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], np.asarray(freqs, np.float32))


def face_shapes(box: NTFFBox):
    """(n1, n2) of the six faces in ``FACES`` order."""
    ni, nj, nk = box.i_hi - box.i_lo, box.j_hi - box.j_lo, box.k_hi - box.k_lo
    return [(nj, nk), (nj, nk), (ni, nk), (ni, nk), (ni, nj), (ni, nj)]


def init_ntff_data(box: NTFFBox, field_dtype=np.float32) -> NTFFData:
    """rfx/farfield.py:164-205: zeroed complex64 sums and residuals."""
    if np.dtype(field_dtype) != np.float32:
        raise NotImplementedError("fields are float32 on this path")
    nf = len(box.freqs)
    z = [np.zeros((nf, a, b, 4), np.complex64) for (a, b) in face_shapes(box)]
    return NTFFData(*z, *[np.zeros_like(a) for a in z])


def ntff_descriptor(box: NTFFBox):
    """(i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, n_freqs) of the plan descriptor."""
    return (int(box.i_lo), int(box.i_hi), int(box.j_lo), int(box.j_hi), int(box.k_lo), int(box.k_hi),
            len(box.freqs))


def ntff_phase_table(freqs, n_steps, dt, step0=0):
    """(n_steps, 2, n_freqs) complex64 step factors of rfx/farfield.py:230-244
    for steps step0 .. step0 + n_steps - 1, in its float32 arithmetic:
    t = f32(n) * f32(dt), omega = f32(2 pi) * f32(f), E factor
    exp(-1j f32(omega t)) * dt, H factor the same at f32(t + dt/2)."""
    d = np.float32(dt)
    n = np.arange(step0, step0 + n_steps, dtype=np.float32)
    t = n * d
    om = np.float32(2 * np.pi) * np.asarray(freqs, np.float32)
    out = np.empty((n_steps, 2, len(om)), np.complex64)
    for q, tt in enumerate((t, (t + d * np.float32(0.5)).astype(np.float32))):
        a = (tt[:, None] * om[None, :]).astype(np.float32).astype(np.float64)
        out[:, q, :].real = np.cos(a).astype(np.float32) * d
        out[:, q, :].imag = (-np.sin(a)).astype(np.float32) * d
    return out


def face_views(flat, box: NTFFBox):
    """The six (n_freqs, n1, n2, 4) face views of a flat NTFF buffer."""
    nf = len(box.freqs)
    out, o = [], 0
    for (n1, n2) in face_shapes(box):
        m = nf * n1 * n2 * 4
        out.append(flat[o:o + m].view(nf, n1, n2, 4))
        o += m
    return out


def pack_ntff(data: NTFFData, device):
    """Flat device buffers (sums, residuals) of an ``NTFFData``."""
    def flat(arrs):
        return torch.from_numpy(np.concatenate([np.ascontiguousarray(a, np.complex64).reshape(-1)
                                                for a in arrs])).to(device)
    res = [getattr(data, "c_" + f) for f in FACES]
    res = [np.zeros_like(np.asarray(getattr(data, f))) if r is None else r for f, r in zip(FACES, res)]
    return flat([getattr(data, f) for f in FACES]), flat(res)


def unpack_ntff(box: NTFFBox, acc, cmp) -> NTFFData:
    """``NTFFData`` of the flat device buffers."""
    nf = len(box.freqs)
    a, c = acc.cpu().numpy(), cmp.cpu().numpy()
    outs, res, o = [], [], 0
    for (n1, n2) in face_shapes(box):
        m = nf * n1 * n2 * 4
        outs.append(a[o:o + m].reshape(nf, n1, n2, 4))
        res.append(c[o:o + m].reshape(nf, n1, n2, 4))
        o += m
    return NTFFData(*outs, *res)


def _currents(f, axis, sign):
    """J = n x H, M = -n x E of the stored tangential components
    (rfx/farfield.py:316-341); f is (..., 4), results (..., 3)."""
    s = float(sign)
    f0, f1, f2, f3 = f[..., 0], f[..., 1], f[..., 2], f[..., 3]
    z = torch.zeros_like(f0)
    if axis == 0:
        J = torch.stack([z, -s * f3, s * f2], -1)
        M = torch.stack([z, s * f1, -s * f0], -1)
    elif axis == 1:
        J = torch.stack([s * f3, z, -s * f2], -1)
        M = torch.stack([-s * f1, z, s * f0], -1)
    else:
        J = torch.stack([-s * f3, s * f2, z], -1)
        M = torch.stack([s * f1, -s * f0, z], -1)
    return J, M


def _face_positions(grid, box, axis, idx, r1, r2, z_edges, lo):
    """(n1, n2, 3) cell positions of a face (rfx/farfield.py:344-390)."""
    dx = float(grid.dx)
    dy = float(getattr(grid, "dy", dx))
    cx, cy, cz = lo

    def zpos(k):
        return z_edges[k] if z_edges is not None else (k - cz) * dx

    if axis == 0:
        y = (np.arange(*r1) - cy) * dy
        z = np.array([zpos(k) for k in range(*r2)], np.float64)
        Y, Z = np.meshgrid(y, z, indexing="ij")
        X = np.full_like(Y, (idx - cx) * dx)
    elif axis == 1:
        x = (np.arange(*r1) - cx) * dx
        z = np.array([zpos(k) for k in range(*r2)], np.float64)
        X, Z = np.meshgrid(x, z, indexing="ij")
        Y = np.full_like(X, (idx - cy) * dy)
    else:
        x = (np.arange(*r1) - cx) * dx
        y = (np.arange(*r2) - cy) * dy
        X, Y = np.meshgrid(x, y, indexing="ij")
        Z = np.full_like(X, zpos(idx))
    return np.stack([X, Y, Z], -1)


def far_field(faces, box: NTFFBox, grid, theta, phi, chunk_cells: int = 1 << 14):
    """rfx/farfield.py:393-556 on torch tensors: ``faces`` = the six NTFF face
    tensors (x_lo .. z_hi, complex, (n_freqs, n1, n2, 4), all on one CUDA
    device).  Returns (E_theta, E_phi), complex128 (n_freqs, n_theta, n_phi),
    differentiable with respect to the faces: for every face, frequency and
    observation direction the radiation vectors N = sum J exp(jk r.r') dS and
    L = sum M exp(jk r.r') dS (a complex matrix product over face cells,
    ``chunk_cells`` cells at a time), projected onto theta / phi.  Graded
    grids (a ``dz`` table) use the z edge positions and per-cell dS of the
    reference."""
    dev = faces[0].device
    theta = np.asarray(theta, np.float64)
    phi = np.asarray(phi, np.float64)
    freqs = np.asarray(box.freqs, np.float64)
    nf = len(freqs)
    k_arr = 2 * np.pi * freqs / C0
    dx = float(grid.dx)
    dy = float(getattr(grid, "dy", dx))
    dz_arr = getattr(grid, "dz", None)
    legacy = int(getattr(grid, "cpml_layers", 0) or 0)
    lo = (box.cpml_lo_x or legacy, box.cpml_lo_y or legacy, box.cpml_lo_z or legacy)
    z_edges = None
    if dz_arr is not None:
        z_edges = np.concatenate([[0.0], np.cumsum(np.asarray(dz_arr, np.float64))])
        z_edges = z_edges - z_edges[lo[2]]
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    sth, cth, sph, cph = np.sin(TH), np.cos(TH), np.sin(PH), np.cos(PH)
    r_hat = np.stack([sth * cph, sth * sph, cth], -1).reshape(-1, 3)
    th_hat = np.stack([cth * cph, cth * sph, -sth], -1).reshape(-1, 3)
    ph_hat = np.stack([-sph, cph, np.zeros_like(sth)], -1).reshape(-1, 3)
    n_dir = r_hat.shape[0]
    r_d = torch.from_numpy(r_hat).to(dev)
    N = torch.zeros((nf, n_dir, 3), dtype=torch.complex128, device=dev)
    L = torch.zeros_like(N)
    i0, i1, j0, j1, k0, k1 = box.i_lo, box.i_hi, box.j_lo, box.j_hi, box.k_lo, box.k_hi
    specs = [(0, -1, i0, (j0, j1), (k0, k1)), (0, 1, i1, (j0, j1), (k0, k1)),
             (1, -1, j0, (i0, i1), (k0, k1)), (1, 1, j1, (i0, i1), (k0, k1)),
             (2, -1, k0, (i0, i1), (j0, j1)), (2, 1, k1, (i0, i1), (j0, j1))]
    for fd, (axis, sign, idx, r1, r2) in zip(faces, specs):
        fd = fd.to(torch.complex128)
        n1, n2 = fd.shape[1], fd.shape[2]
        if n1 == 0 or n2 == 0:
            continue
        pos = torch.from_numpy(_face_positions(grid, box, axis, idx, r1, r2, z_edges, lo).reshape(-1, 3)).to(dev)
        J, M = _currents(fd.reshape(nf, -1, 4), axis, sign)
        if dz_arr is not None and axis in (0, 1):
            dS = (dy if axis == 0 else dx) * np.asarray(dz_arr[r2[0]:r2[1]], np.float64)
            dS = torch.from_numpy(np.tile(dS, n1)).to(dev)[None, :, None]
        else:
            dS = dx * dy
        J = J * dS
        M = M * dS
        nc = pos.shape[0]
        for c0 in range(0, nc, chunk_cells):
            c1 = min(nc, c0 + chunk_cells)
            dot = r_d @ pos[c0:c1].T                               # (n_dir, cells)
            Nc, Lc = [], []
            for fi in range(nf):
                ph = torch.polar(torch.ones_like(dot), float(k_arr[fi]) * dot)
                Nc.append(ph @ J[fi, c0:c1])
                Lc.append(ph @ M[fi, c0:c1])
            N = N + torch.stack(Nc)
            L = L + torch.stack(Lc)
    th_d = torch.from_numpy(th_hat).to(dev).to(torch.complex128)
    ph_d = torch.from_numpy(ph_hat).to(dev).to(torch.complex128)
    N_th, N_ph = (N * th_d).sum(-1), (N * ph_d).sum(-1)
    L_th, L_ph = (L * th_d).sum(-1), (L * ph_d).sum(-1)
    jk = torch.from_numpy(1j * k_arr).to(dev)[:, None]
    E_th = -jk / (4 * np.pi) * (L_ph + ETA_0 * N_th)
    E_ph = jk / (4 * np.pi) * (L_th - ETA_0 * N_ph)
    return E_th.reshape(nf, len(theta), len(phi)), E_ph.reshape(nf, len(theta), len(phi))


def compute_far_field(ntff_data: NTFFData, box: NTFFBox, grid, theta, phi, device=None,
                      chunk_cells: int = 1 << 14) -> FarFieldResult:
    """rfx/farfield.py:393-556 on the device (``far_field`` on the faces of
    an ``NTFFData``), returned as NumPy arrays like the reference's."""
    from .engine import require_cuda
    dev = require_cuda(device)
    faces = [torch.as_tensor(np.asarray(getattr(ntff_data, name)), device=dev) for name in FACES]
    E_th, E_ph = far_field(faces, box, grid, theta, phi, chunk_cells)
    return FarFieldResult(E_th.cpu().numpy(), E_ph.cpu().numpy(), np.asarray(theta, np.float64),
                          np.asarray(phi, np.float64), np.asarray(box.freqs, np.float64))


def directivity_torch(E_theta, E_phi, theta, phi):
    """``directivity`` (rfx/farfield.py:780-802) as a linear ratio
    4 pi U / P_rad on torch tensors, per frequency and direction
    (n_freqs, n_theta, n_phi), differentiable: the objective of far-field
    inverse design (rfx/optimize_objectives.py maximize_directivity takes its
    logarithm at a target direction)."""
    p = E_theta.real ** 2 + E_theta.imag ** 2 + E_phi.real ** 2 + E_phi.imag ** 2
    th = np.asarray(theta, np.float64)
    ph = np.asarray(phi, np.float64)
    dth = np.gradient(th) if len(th) > 1 else np.array([np.pi])
    dph = np.gradient(ph) if len(ph) > 1 else np.array([2 * np.pi])
    w = torch.from_numpy(np.sin(th)[:, None] * dth[:, None] * dph[None, :]).to(p.device)
    prad = (p * w[None]).sum(dim=(1, 2))
    return 4 * np.pi * p / prad[:, None, None]


def radiation_pattern(ff: FarFieldResult) -> np.ndarray:
    """rfx/farfield.py:769-777: normalised pattern in dB."""
    p = np.abs(ff.E_theta) ** 2 + np.abs(ff.E_phi) ** 2
    peak = np.max(p, axis=(1, 2), keepdims=True)
    return 10 * np.log10(np.maximum(p / np.where(peak > 0, peak, 1.0), 1e-10))


def directivity(ff: FarFieldResult) -> np.ndarray:
    """rfx/farfield.py:780-802: D = 4 pi U_max / P_rad in dBi per frequency,
    P_rad by the gradient-weighted sum over theta and phi."""
    p = np.abs(ff.E_theta) ** 2 + np.abs(ff.E_phi) ** 2
    dth = np.gradient(ff.theta) if len(ff.theta) > 1 else np.array([np.pi])
    dph = np.gradient(ff.phi) if len(ff.phi) > 1 else np.array([2 * np.pi])
    prad = np.sum(p * np.sin(ff.theta)[None, :, None] * dth[None, :, None] * dph[None, None, :], axis=(1, 2))
    umax = np.max(p, axis=(1, 2))
    d = 4 * np.pi * umax / np.where(prad > 0, prad, 1.0)
    return 10 * np.log10(np.maximum(d, 1e-10))
