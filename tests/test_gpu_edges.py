"""Edge cases of the forward step against the float32 oracle, each started
from seeded random fields in every cell:

* tile tails: ny = 4 * 8 + 1 and nz = 2 * 32 + 1, so the last y tile holds
  one row and the last z tile one column, with CPML on every axis;
* more than 32 sources and probes (the kernels match the first 32 per column
  by bit mask and the rest by a scan), two sources on the same cell and
  component (both added, in order), probes on H components;
* the smallest grids the descriptor accepts (2^3 and 3^3, PEC faces only),
  with no sources and no probes;
* an advance of zero steps changes nothing.
"""

import numpy as np
import pytest
import torch

import oracle
from oracle.fdtd import COMPONENTS
from tests.test_gpu_fullsize import _advance, _compare_with_oracle, _random_fields

pytestmark = pytest.mark.gpu


def _grid(domain, dx, cpml):
    import rfx_b200
    og = oracle.make_uniform_grid(domain, dx, cpml_layers=cpml)
    g = rfx_b200.Grid(freq_max=10e9, domain=domain, dx=dx, cpml_layers=cpml)
    assert tuple(g.shape) == tuple(og.shape) and g.dt == og.dt
    return og, g


def _device(g, mats, n, src, probes, dft, cpml_axes):
    from rfx_b200.simulation import MaterialArrays, init_dft_plane_probe, prepare_device_run
    planes = [init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in dft]
    return prepare_device_run(g, MaterialArrays(*mats), n, cpml_axes=cpml_axes, pec_axes="xyz", sources=src,
                              probes=probes, dft_planes=planes, pec_mask=None, dft_time_offset=1)


def _materials(shape, rng):
    eps = (1.0 + 5.0 * rng.random(shape)).astype(np.float32)
    sig = (0.02 * rng.random(shape)).astype(np.float32)
    return eps, sig, np.ones(shape, np.float32)


def test_tile_tails_and_many_monitors(cuda):
    og, g = _grid((13e-3, 16e-3, 48e-3), 1e-3, 8)
    assert tuple(g.shape) == (30, 33, 65)
    n = 40
    rng = np.random.default_rng(21)
    mats = _materials(g.shape, rng)
    comps_e = ("ex", "ey", "ez")
    cells = [(int(rng.integers(1, g.nx - 1)), int(rng.integers(1, g.ny - 1)), int(rng.integers(1, g.nz - 1)))
             for _ in range(38)]
    cells += [(g.nx - 2, g.ny - 1, g.nz - 1), (1, g.ny - 1, 64)]   # in the one-row / one-column tail tiles
    src = [(i, j, k, comps_e[q % 3], (rng.standard_normal(n) * 5.0).astype(np.float32))
           for q, (i, j, k) in enumerate(cells)]
    src.append((*cells[0], src[0][3], (rng.standard_normal(n) * 5.0).astype(np.float32)))   # same cell, same comp
    assert len(src) == 41
    probes = [(int(rng.integers(0, g.nx)), int(rng.integers(0, g.ny)), int(rng.integers(0, g.nz)),
               COMPONENTS[q % 6]) for q in range(37)]
    probes += [(i, j, k, c) for (i, j, k, c, _) in src[:3]]
    dft = [(2, 64, "ez", np.array([8e9, 11e9], np.float32)), (1, 32, "hx", np.array([9e9], np.float32))]
    init = _random_fields(g.shape, 22)
    ref = oracle.run_uniform(og, mats, n, boundary="cpml", sources=src, probes=probes, dft_planes=dft,
                             dtype=np.float32, init_fields=init)
    r = _device(g, mats, n, src, probes, dft, "xyz")
    try:
        _compare_with_oracle("tails", r, ref, n, init)
    finally:
        r.plan.close()


@pytest.mark.parametrize("n_int", [1, 2])
def test_smallest_grids(cuda, n_int):
    og, g = _grid((n_int * 1e-3,) * 3, 1e-3, 0)
    assert tuple(g.shape) == (n_int + 1,) * 3
    rng = np.random.default_rng(30 + n_int)
    mats = _materials(g.shape, rng)
    init = _random_fields(g.shape, 40 + n_int)
    n = 12
    ref = oracle.run_uniform(og, mats, n, boundary="pec", dtype=np.float32, init_fields=init)
    r = _device(g, mats, n, [], [], [], "")
    try:
        _advance(r, n, init=init)
        fields = [f.cpu().numpy() for f in r.plan.store_fields()]
        for c, f in zip(COMPONENTS, fields):
            np.testing.assert_allclose(f, ref.state[c], rtol=1e-5, atol=1e-6 * float(np.abs(ref.state[c]).max()))
    finally:
        r.plan.close()


def test_zero_step_advance_changes_nothing(cuda):
    og, g = _grid((12e-3, 10e-3, 9e-3), 1e-3, 4)
    rng = np.random.default_rng(50)
    mats = _materials(g.shape, rng)
    src = [(5, 5, 5, "ez", np.ones(20, np.float32))]
    r = _device(g, mats, 20, src, [(6, 6, 6, "ez")], [], "xyz")
    try:
        init = _random_fields(g.shape, 51)
        r.plan.reset()
        r.plan.load_fields([init[c] for c in COMPONENTS])
        r.plan.advance(0, 0, r.src_table, r.probe_out)
        r.plan.advance(7, 0, r.src_table, r.probe_out)
        torch.cuda.synchronize()
        for c, f in zip(COMPONENTS, r.plan.store_fields()):
            assert np.array_equal(f.cpu().numpy(), init[c])
        assert float(r.probe_out.abs().max()) == 0.0
    finally:
        r.plan.close()
