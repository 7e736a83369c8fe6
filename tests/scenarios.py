"""Seeded scenarios shared by the oracle tests, the GPU parity tests and the
golden-fixture generator.  Each builds its inputs once (numpy) and can run
them through the CPU oracle or through ``rfx_b200``."""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

import oracle


@dataclass
class Scenario:
    name: str
    lane: str                      # "uniform" | "nonuniform"
    ogrid: object                  # oracle grid
    materials: tuple               # (eps_r, sigma, mu_r) float32
    n_steps: int
    sources: list                  # (i, j, k, comp, waveform)
    probes: list                   # (i, j, k, comp)
    dft: list = field(default_factory=list)     # (axis, index, comp, freqs)
    pec_mask: np.ndarray | None = None
    boundary: str = "cpml"
    pec_axes: str | None = None
    dz_profile: np.ndarray | None = None
    domain: tuple | None = None
    dx: float | None = None

    def run_oracle(self, dtype=np.float32, exact_materials=False):
        if self.lane == "uniform":
            return oracle.run_uniform(self.ogrid, self.materials, self.n_steps, boundary=self.boundary,
                                      pec_axes=self.pec_axes, sources=self.sources, probes=self.probes,
                                      dft_planes=self.dft, pec_mask=self.pec_mask, dtype=dtype,
                                      exact_materials=exact_materials)
        return oracle.run_nonuniform(self.ogrid, self.materials, self.n_steps, sources=self.sources,
                                     probes=self.probes, dft_planes=self.dft, pec_mask=self.pec_mask, dtype=dtype,
                                     exact_materials=exact_materials)

    def product_grid(self):
        import rfx_b200
        if self.lane == "uniform":
            return rfx_b200.Grid(freq_max=10e9, domain=self.domain, dx=self.dx, cpml_layers=self.ogrid.cpml_layers)
        return rfx_b200.make_nonuniform_grid(self.domain, self.dz_profile, self.dx,
                                             cpml_layers=self.ogrid.cpml_layers)

    def run_product(self):
        """Returns (time_series, [dft accumulators], final fields dict)."""
        import rfx_b200
        g = self.product_grid()
        assert tuple(g.shape) == tuple(self.ogrid.shape)
        mats = rfx_b200.MaterialArrays(*self.materials)
        if self.lane == "uniform":
            srcs = [rfx_b200.SourceSpec(i, j, k, c, w) for (i, j, k, c, w) in self.sources]
            prbs = [rfx_b200.ProbeSpec(i, j, k, c) for (i, j, k, c) in self.probes]
            dfts = [rfx_b200.init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in self.dft]
            r = rfx_b200.run(g, mats, self.n_steps, boundary=self.boundary, pec_axes=self.pec_axes,
                             sources=srcs, probes=prbs, dft_planes=dfts or None, pec_mask=self.pec_mask)
            planes = [p.accumulator for p in (r.dft_planes or ())]
            st = r.state
        else:
            dfts = [rfx_b200.init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in self.dft]
            r = rfx_b200.run_nonuniform(g, mats, self.n_steps, sources=self.sources, probes=self.probes,
                                        dft_planes=dfts or None, pec_mask=self.pec_mask)
            planes = [p.accumulator for p in r.get("dft_planes", ())]
            st = r["state"]
            r = type("R", (), {"time_series": r["time_series"]})
        fields = {c: getattr(st, c) for c in ("ex", "ey", "ez", "hx", "hy", "hz")}
        return r.time_series, planes, fields


def _boxes(rng, shape, n_boxes, eps_hi, sig_hi, lo_pad, size_lo, size_hi):
    eps = np.ones(shape, np.float32)
    sig = np.zeros(shape, np.float32)
    for _ in range(n_boxes):
        sz = rng.integers(size_lo, size_hi + 1, 3)
        lo = [int(rng.integers(lo_pad, max(lo_pad + 1, shape[a] - lo_pad - sz[a]))) for a in range(3)]
        sl = tuple(slice(lo[a], lo[a] + sz[a]) for a in range(3))
        eps[sl] = np.float32(rng.uniform(1.0, eps_hi))
        sig[sl] = np.float32(rng.uniform(0.0, sig_hi))
    return eps, sig


def c1_readme(n_steps=1200):
    """README quick start: domain (0.14, 0.06, 0.05) m, dx 2 mm, CPML 8, a
    dielectric box eps_r 2.2 sigma 0.01, Ez GaussianPulse(3 GHz, 0.8) at
    (0.03, 0.03, 0.025), Ez probe at (0.11, 0.03, 0.025); rfx run() (PEC pass
    on every axis, as run() defaults)."""
    dx = 2e-3
    g = oracle.make_uniform_grid((0.14, 0.06, 0.05), dx, cpml_layers=8)
    shape = g.shape
    eps = np.ones(shape, np.float32)
    sig = np.zeros(shape, np.float32)
    mu = np.ones(shape, np.float32)
    # Box((0.07, 0.018, 0.018), (0.09, 0.042, 0.032)): half-open [lo, hi) over
    # float32 node coordinates (rfx/geometry/csg.py:61-69, 235-307)
    masks = []
    for ax, (lo, hi) in enumerate(((0.07, 0.09), (0.018, 0.042), (0.018, 0.032))):
        coords = (np.arange(shape[ax], dtype=np.int32) - g.pads[2 * ax]).astype(np.float32) * np.float32(dx)
        masks.append((coords >= np.float32(lo)) & (coords < np.float32(hi)))
    box = masks[0][:, None, None] & masks[1][None, :, None] & masks[2][None, None, :]
    eps[box] = np.float32(2.2)
    sig[box] = np.float32(0.01)
    src = g.position_to_index((0.03, 0.03, 0.025))
    prb = g.position_to_index((0.11, 0.03, 0.025))
    w = oracle.j_source_waveform(g, src, (eps, sig, mu), n_steps, f0=3e9, bandwidth=0.8)
    return Scenario("c1_readme", "uniform", g, (eps, sig, mu), n_steps, [(*src, "ez", w)], [(*prb, "ez")],
                    domain=(0.14, 0.06, 0.05), dx=dx)


def small_uniform(n_steps=240, seed=1):
    """Small lossy dielectric scene with every uniform-lane feature: CPML 6,
    PEC faces, 3 boxes, two sources, E and H probes, a z DFT plane and an x
    DFT plane, and a thin PEC sheet."""
    rng = np.random.default_rng(seed)
    dx = 1e-3
    domain = (0.030, 0.024, 0.020)
    g = oracle.make_uniform_grid(domain, dx, cpml_layers=6)
    shape = g.shape
    eps, sig = _boxes(rng, shape, 3, 6.0, 0.05, 6, 3, 8)
    mu = np.ones(shape, np.float32)
    pec = np.zeros(shape, bool)
    pec[20:26, 14:20, 15] = True
    mats = (eps, sig, mu)
    s1 = (12, 13, 13)
    s2 = (24, 10, 9)
    w1 = oracle.j_source_waveform(g, s1, mats, n_steps, f0=12e9, bandwidth=0.8)
    w2 = oracle.j_source_waveform(g, s2, mats, n_steps, f0=20e9, bandwidth=0.5, amplitude=0.5)
    probes = [(30, 16, 12, "ez"), (10, 20, 18, "hy"), (25, 10, 9, "ex"), (18, 18, 7, "hz")]
    freqs = np.linspace(8e9, 20e9, 3).astype(np.float32)
    dft = [(2, 13, "ez", freqs), (0, 22, "hy", freqs[:2])]
    return Scenario("small_uniform", "uniform", g, mats, n_steps, [(*s1, "ez", w1), (*s2, "ey", w2)], probes,
                    dft, pec_mask=pec, domain=domain, dx=dx)


def medium_uniform(n_steps=200, seed=3):
    """small_uniform's feature set on a grid long enough in y and z (44 x 76
    cells across, CPML 6) that no 8 x 32 tile reaches both slabs of an axis,
    so the forward step stages its CPML psi by TMA."""
    rng = np.random.default_rng(seed)
    dx = 1e-3
    domain = (0.028, 0.032, 0.064)
    g = oracle.make_uniform_grid(domain, dx, cpml_layers=6)
    shape = g.shape
    eps, sig = _boxes(rng, shape, 4, 6.0, 0.05, 6, 3, 10)
    mu = np.ones(shape, np.float32)
    pec = np.zeros(shape, bool)
    pec[18:24, 14:22, 40] = True
    mats = (eps, sig, mu)
    s1 = (12, 13, 30)
    s2 = (24, 30, 50)
    w1 = oracle.j_source_waveform(g, s1, mats, n_steps, f0=12e9, bandwidth=0.8)
    w2 = oracle.j_source_waveform(g, s2, mats, n_steps, f0=20e9, bandwidth=0.5, amplitude=0.5)
    probes = [(30, 16, 60, "ez"), (22, 41, 48, "hy"), (25, 10, 70, "ex"), (18, 40, 33, "hz")]
    freqs = np.linspace(8e9, 20e9, 3).astype(np.float32)
    dft = [(2, 66, "ez", freqs), (1, 5, "hx", freqs[:2])]
    return Scenario("medium_uniform", "uniform", g, mats, n_steps, [(*s1, "ez", w1), (*s2, "ey", w2)], probes,
                    dft, pec_mask=pec, domain=domain, dx=dx)


def graded_dz(rng, n, lo=1e-4, hi=5e-4, max_ratio=1.2):
    """Seeded smooth grading within [lo, hi] with adjacent ratio <= max_ratio."""
    d = [float(rng.uniform(lo, hi))]
    for _ in range(n - 1):
        r = float(rng.uniform(1.0 / max_ratio, max_ratio))
        d.append(min(hi, max(lo, d[-1] * r)))
    return np.asarray(d)


def small_nonuniform(n_steps=240, seed=2):
    """Graded z with CPML 6, a PEC ground sheet, a substrate and an Ex
    current source, E/H probes and a z DFT plane."""
    rng = np.random.default_rng(seed)
    dx = 5e-4
    domain = (0.012, 0.010)
    dz = graded_dz(rng, 16)
    g = oracle.make_nonuniform_grid(domain, dz, dx, cpml_layers=6)
    shape = g.shape
    eps = np.ones(shape, np.float32)
    sig = np.zeros(shape, np.float32)
    mu = np.ones(shape, np.float32)
    eps[:, :, 9:13] = np.float32(rng.uniform(2.0, 4.5))
    pec = np.zeros(shape, bool)
    pec[:, :, 8] = True
    mats = (eps, sig, mu)
    src = (16, 13, 11)
    w = oracle.current_source_waveform(g, src, "ex", mats, n_steps, f0=60e9, bandwidth=0.8)
    probes = [(20, 12, 12, "ex"), (10, 16, 14, "ez"), (14, 10, 10, "hy")]
    freqs = np.linspace(40e9, 80e9, 4).astype(np.float32)
    dft = [(2, 12, "ex", freqs)]
    return Scenario("small_nonuniform", "nonuniform", g, mats, n_steps, [(*src, "ex", w)], probes, dft,
                    pec_mask=pec, dz_profile=dz, domain=domain, dx=dx)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
