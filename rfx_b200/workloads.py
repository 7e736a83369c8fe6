"""Seeded synthetic inputs of the benchmark configurations.

The reference publishes no dataset for this path; these builders generate the
shapes, sizes and value distributions the configurations name, from a seed.

  large_uniform   256^3 interior, dx 1 mm, CPML 10 -> (277)^3; 32 boxes, edge
                  8-64 cells, eps_r ~ U[1,10], sigma ~ U[0,0.05]; Ez pulse
                  f0 10 GHz bw 0.8 at the centre; 8 probes; z-plane DFT at 16
                  frequencies in 5-15 GHz.
  graded          192 x 192 x 96 cells, x/y 0.5 mm, z graded 0.1-0.5 mm (ratio
                  <= 1.2), CPML 12; PEC sheet at z-index 10 (+pad); substrate
                  eps_r ~ U[2,4.5] over 8 z cells; Ex pulse f0 20 GHz; 4 probes;
                  DFT plane at 8 frequencies.
  adjoint_region  200 x 120 x 48 at 0.5 mm, CPML 10; design 64 x 64 x 2 with
                  rho ~ U[0,1], eps_r = 1 + 3.4 rho; Ez pulse 15 GHz; 4 probes;
                  objective over 5 frequencies.
  batched_sweep   64 instances, n ~ U{64..160} per instance (cubic), CPML 8
                  (+1 fence) -> (n+17)^3; 8 boxes eps_r ~ U[1,8]; 16 x 16 x 2
                  design region; Ez pulse 12 GHz; 4 probes; objective over 3
                  frequencies.
"""

from __future__ import annotations

import numpy as np

from .batch import SweepInstance
from .grid import Grid, make_nonuniform_grid
from .sources import GaussianPulse, _cell_cb, _times


class _Mats:
    def __init__(self, eps_r, sigma):
        self.eps_r, self.sigma = eps_r, sigma


def _boxes(rng, shape, n, eps_lo, eps_hi, sig_hi, margin, size_lo, size_hi, build=True):
    """``n`` seeded boxes; with ``build=False`` only the random draws are made
    (the stream advances exactly as when building) and (None, None) returned."""
    eps = np.ones(shape, np.float32) if build else None
    sig = np.zeros(shape, np.float32) if build else None
    for _ in range(n):
        sz = [int(min(rng.integers(size_lo, size_hi + 1), shape[a] - 2 * margin - 1)) for a in range(3)]
        lo = [int(rng.integers(margin, max(margin + 1, shape[a] - margin - sz[a]))) for a in range(3)]
        sl = tuple(slice(lo[a], lo[a] + sz[a]) for a in range(3))
        v = np.float32(rng.uniform(eps_lo, eps_hi))
        if build:
            eps[sl] = v
        if sig_hi > 0:
            w = np.float32(rng.uniform(0.0, sig_hi))
            if build:
                sig[sl] = w
    return eps, sig


def j_wave(grid, idx, eps, sig, n_steps, f0, bw=0.8):
    cb = _cell_cb(_Mats(eps, sig), idx, grid.dt)
    return (cb * GaussianPulse(f0, bw)(_times(n_steps, grid.dt))).astype(np.float32)


def large_uniform(seed=0, n_steps=4000, n_interior=256):
    rng = np.random.default_rng(seed)
    dx = 1e-3
    g = Grid(freq_max=15e9, domain=(n_interior * dx,) * 3, dx=dx, cpml_layers=10)
    eps, sig = _boxes(rng, g.shape, 32, 1.0, 10.0, 0.05, 10, 8, 64)
    c = tuple(s // 2 for s in g.shape)
    src = [(*c, "ez", j_wave(g, c, eps, sig, n_steps, 10e9))]
    probes = [(int(rng.integers(20, g.nx - 20)), int(rng.integers(20, g.ny - 20)),
               int(rng.integers(20, g.nz - 20)), "ez") for _ in range(8)]
    dft = [(2, c[2], "ez", np.linspace(5e9, 15e9, 16).astype(np.float32))]
    return g, eps, sig, src, probes, dft


def _graded_dz(rng):
    dz = [float(rng.uniform(1e-4, 5e-4))]
    for _ in range(95):
        dz.append(min(5e-4, max(1e-4, dz[-1] * float(rng.uniform(1 / 1.2, 1.2)))))
    return np.asarray(dz)


def graded_dz(seed=0):
    """The 96-cell z profile of ``graded(seed)`` (its first draws)."""
    return _graded_dz(np.random.default_rng(seed))


def graded(seed=0, n_steps=6000):
    rng = np.random.default_rng(seed)
    dx = 0.5e-3
    dz = _graded_dz(rng)
    g = make_nonuniform_grid((192 * dx, 192 * dx), dz, dx, cpml_layers=12)
    shape = g.shape
    eps = np.ones(shape, np.float32)
    sig = np.zeros(shape, np.float32)
    kz = 12 + 10
    eps[:, :, kz + 1:kz + 9] = np.float32(rng.uniform(2.0, 4.5))
    pec = np.zeros(shape, bool)
    pec[:, :, kz] = True
    from .sources import make_current_source
    mats = _Mats(eps, sig)
    src = [make_current_source(g, (g.nx // 2, g.ny // 2, kz + 4), "ex", GaussianPulse(20e9, 0.8), n_steps, mats)]
    probes = [(int(rng.integers(20, g.nx - 20)), int(rng.integers(20, g.ny - 20)), kz + 4, "ex") for _ in range(4)]
    dft = [(2, kz + 4, "ex", np.linspace(10e9, 30e9, 8).astype(np.float32))]
    return g, eps, sig, pec, src, probes, dft


def pec_uniform(n_cells=512, n_steps=1000):
    """The reference's own GPU throughput benchmark (rfx/gpu.py:58-107, the
    figure quoted in its README): a PEC-bounded vacuum cube with no CPML,
    dx = 1 mm, a raw Ez field source GaussianPulse(f0 = 5 GHz) and an Ez probe
    at the centre, run() for n_steps.  The published grid size is not stated;
    n_cells = 512 fills a B200 (513^3 cells with the +1 fence)."""
    from .sources import make_source
    dx = 1e-3
    g = Grid(freq_max=10e9, domain=(n_cells * dx,) * 3, dx=dx, cpml_layers=0)
    eps = np.ones(g.shape, np.float32)
    sig = np.zeros(g.shape, np.float32)
    centre = tuple(n_cells * dx / 2 for _ in range(3))
    src = make_source(g, centre, "ez", GaussianPulse(5e9), n_steps)
    prb = g.position_to_index(centre)
    return g, eps, sig, src, prb


def adjoint_region(seed=0, n_steps=3000):
    rng = np.random.default_rng(seed)
    dx = 0.5e-3
    g = Grid(freq_max=20e9, domain=(200 * dx, 120 * dx, 48 * dx), dx=dx, cpml_layers=10)
    shape = g.shape
    eps = np.ones(shape, np.float32)
    sig = np.zeros(shape, np.float32)
    i0 = (shape[0] - 64) // 2
    j0 = (shape[1] - 64) // 2
    k0 = shape[2] // 2
    box = (i0, i0 + 64, j0, j0 + 64, k0, k0 + 2)
    rho = rng.uniform(0.0, 1.0, (64, 64, 2))
    eps[i0:i0 + 64, j0:j0 + 64, k0:k0 + 2] = (1.0 + 3.4 * rho).astype(np.float32)
    s = (20, shape[1] // 2, k0)
    src = [(*s, "ez", j_wave(g, s, eps, sig, n_steps, 15e9))]
    probes = [(shape[0] - 25, shape[1] // 2 + d, k0, "ez") for d in (-20, -7, 7, 20)]
    freqs = np.linspace(12e9, 18e9, 5)
    return g, eps, sig, src, probes, box, freqs


def batched_sweep_instance_cells(seed=0, n_inst=64, n_lo=64, n_hi=160):
    """Per-instance cell counts of ``batched_sweep(seed, n_inst, ...)``
    without building its material arrays (same size draw, same grids)."""
    sizes = np.random.default_rng(seed).integers(n_lo, n_hi + 1, n_inst)
    dx = 0.5e-3
    out = []
    for n in sizes:
        g = Grid(freq_max=20e9, domain=(int(n) * dx,) * 3, dx=dx, cpml_layers=8)
        out.append(int(g.nx * g.ny * g.nz))
    return out


def batched_sweep_cells(seed=0, n_inst=64, n_lo=64, n_hi=160):
    """Total cell count of ``batched_sweep(seed, n_inst, ...)``."""
    return int(sum(batched_sweep_instance_cells(seed, n_inst, n_lo, n_hi)))


def batched_sweep(seed=0, n_inst=64, n_steps=2000, n_lo=64, n_hi=160, subset=None):
    """The sweep's instances; with ``subset`` (instance indices) only those
    are built, from the same random stream (a rank's share of a sweep that is
    sharded over GPUs)."""
    rng = np.random.default_rng(seed)
    dx = 0.5e-3
    out = []
    sizes = rng.integers(n_lo, n_hi + 1, n_inst)
    keep = set(range(n_inst)) if subset is None else set(int(q) for q in subset)
    for q in range(n_inst):
        n = int(sizes[q])
        g = Grid(freq_max=20e9, domain=(n * dx,) * 3, dx=dx, cpml_layers=8)
        build = q in keep
        eps, sig = _boxes(rng, g.shape, 8, 1.0, 8.0, 0.0, 10, 4, max(5, n // 4), build=build)
        c = g.nx // 2
        box = (c - 8, c + 8, c - 8, c + 8, c, c + 2)
        rho = rng.uniform(0, 1, (16, 16, 2)).astype(np.float32)
        if not build:
            continue
        eps[box[0]:box[1], box[2]:box[3], box[4]:box[5]] = 1.0 + 3.4 * rho
        s = (10, c, c)
        src = [(*s, "ez", j_wave(g, s, eps, sig, n_steps, 12e9))]
        probes = [(g.nx - 12, c + d, c, "ez") for d in (-6, -2, 2, 6)]
        out.append(SweepInstance(grid=g, eps_r=eps, sigma=sig, sources=src, probes=probes, box=box,
                                 freqs=np.array([10e9, 12e9, 14e9])))
    return out
