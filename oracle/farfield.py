"""Far-field transform of NTFF Huygens-box data -- TEST INFRASTRUCTURE ONLY.

NumPy float64 restatement of rfx/farfield.py:316-556 (surface currents, face
positions, radiation vectors, far-field E_theta / E_phi) and :780-802
(directivity), used by the tests to check the device transform and to run the
reference's dipole pattern and directivity gates (rfx tests/test_farfield.py)
on NTFF data from the oracle and from the CUDA path.

``data`` is a dict of the six faces {"x_lo": (n_f, n1, n2, 4), ...} and
``box`` = (i_lo, i_hi, j_lo, j_hi, k_lo, k_hi, freqs).
"""

import numpy as np

from .fdtd import C0, EPS_0, MU_0, NTFF_FACES

ETA_0 = float(np.sqrt(MU_0 / EPS_0))


def surface_currents(f, axis, sign):
    """rfx/farfield.py:316-341: J = n x H, M = -n x E of (..., 4) tangential
    components [E1, E2, H1, H2]."""
    s = sign
    f0, f1, f2, f3 = (f[..., q] for q in range(4))
    z = np.zeros_like(f0)
    if axis == 0:
        return np.stack([z, -s * f3, s * f2], -1), np.stack([z, s * f1, -s * f0], -1)
    if axis == 1:
        return np.stack([s * f3, z, -s * f2], -1), np.stack([-s * f1, z, s * f0], -1)
    return np.stack([-s * f3, s * f2, z], -1), np.stack([s * f1, -s * f0, z], -1)


def compute_far_field(data, box, dx, cpml_lo, theta, phi, dz=None, dy=None):
    """rfx/farfield.py:393-556 for a grid of cell sizes ``dx``, ``dy`` (default
    dx) and a graded ``dz`` table (default uniform dx), origin at the inner edge of the low CPML faces
    ``cpml_lo`` = (x, y, z).  Returns (E_theta, E_phi) of shape
    (n_f, n_theta, n_phi)."""
    i0, i1, j0, j1, k0, k1, freqs = box
    dy = dx if dy is None else dy
    freqs = np.asarray(freqs, np.float64)
    kk = 2 * np.pi * freqs / C0
    cx, cy, cz = cpml_lo
    z_edges = None
    if dz is not None:
        z_edges = np.concatenate([[0.0], np.cumsum(np.asarray(dz, np.float64))])
        z_edges = z_edges - z_edges[cz]

    def zpos(k):
        return z_edges[k] if z_edges is not None else (k - cz) * dx

    TH, PH = np.meshgrid(np.asarray(theta, np.float64), np.asarray(phi, np.float64), indexing="ij")
    r = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)], -1).reshape(-1, 3)
    th = np.stack([np.cos(TH) * np.cos(PH), np.cos(TH) * np.sin(PH), -np.sin(TH)], -1).reshape(-1, 3)
    ph = np.stack([-np.sin(PH), np.cos(PH), np.zeros_like(TH)], -1).reshape(-1, 3)
    nf = len(freqs)
    N = np.zeros((nf, r.shape[0], 3), np.complex128)
    L = np.zeros_like(N)
    faces = [(0, -1, i0, (j0, j1), (k0, k1)), (0, 1, i1, (j0, j1), (k0, k1)),
             (1, -1, j0, (i0, i1), (k0, k1)), (1, 1, j1, (i0, i1), (k0, k1)),
             (2, -1, k0, (i0, i1), (j0, j1)), (2, 1, k1, (i0, i1), (j0, j1))]
    for name, (axis, sign, idx, ra, rb) in zip(NTFF_FACES, faces):
        f = np.asarray(data[name], np.complex128)
        n1, n2 = f.shape[1], f.shape[2]
        if n1 == 0 or n2 == 0:
            continue
        a = np.arange(*ra)
        b = np.arange(*rb)
        A, B = np.meshgrid(a, b, indexing="ij")
        if axis == 0:
            pos = np.stack([np.full(A.shape, (idx - cx) * dx), (A - cy) * dy,
                            np.vectorize(zpos)(B).astype(np.float64)], -1)
        elif axis == 1:
            pos = np.stack([(A - cx) * dx, np.full(A.shape, (idx - cy) * dy),
                            np.vectorize(zpos)(B).astype(np.float64)], -1)
        else:
            pos = np.stack([(A - cx) * dx, (B - cy) * dy, np.full(A.shape, zpos(idx), np.float64)], -1)
        pos = pos.reshape(-1, 3)
        J, M = surface_currents(f.reshape(nf, -1, 4), axis, sign)
        if dz is not None and axis in (0, 1):
            dS = np.tile((dy if axis == 0 else dx) * np.asarray(dz[rb[0]:rb[1]], np.float64), n1)[:, None]
        else:
            dS = dx * dy
        dot = r @ pos.T
        for q in range(nf):
            e = np.exp(1j * kk[q] * dot)
            N[q] += e @ (J[q] * dS)
            L[q] += e @ (M[q] * dS)
    Nth, Nph = np.sum(N * th[None], -1), np.sum(N * ph[None], -1)
    Lth, Lph = np.sum(L * th[None], -1), np.sum(L * ph[None], -1)
    jk = 1j * kk[:, None]
    Et = -jk / (4 * np.pi) * (Lph + ETA_0 * Nth)
    Ep = jk / (4 * np.pi) * (Lth - ETA_0 * Nph)
    shp = (nf, len(theta), len(phi))
    return Et.reshape(shp), Ep.reshape(shp)


def directivity(E_theta, E_phi, theta, phi):
    """rfx/farfield.py:780-802: D = 4 pi U_max / P_rad in dBi per frequency."""
    p = np.abs(E_theta) ** 2 + np.abs(E_phi) ** 2
    dth = np.gradient(theta) if len(theta) > 1 else np.array([np.pi])
    dph = np.gradient(phi) if len(phi) > 1 else np.array([2 * np.pi])
    prad = np.sum(p * np.sin(theta)[None, :, None] * dth[None, :, None] * dph[None, None, :], axis=(1, 2))
    d = 4 * np.pi * np.max(p, axis=(1, 2)) / np.where(prad > 0, prad, 1.0)
    return 10 * np.log10(np.maximum(d, 1e-10))
