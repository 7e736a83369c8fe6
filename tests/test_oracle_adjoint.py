"""CPU tests of the oracle's reverse-mode gradient (the checker of the CUDA
adjoint): exact transpose and agreement with float64 finite differences."""

import numpy as np
import pytest

from oracle.adjoint import forward_adjoint
from tests.scenarios import small_nonuniform, small_uniform

CASES = [(small_uniform, (14, 20, 14, 20, 12, 14)), (small_nonuniform, (12, 18, 12, 18, 11, 13))]


def _fa(sc, box, G):
    return forward_adjoint(sc.ogrid, sc.materials, sc.n_steps, nonuniform=sc.lane == "nonuniform",
                           boundary=sc.boundary, pec_axes=sc.pec_axes, sources=sc.sources, probes=sc.probes,
                           pec_mask=sc.pec_mask, box=box, objective_grad=lambda ts: G)


@pytest.mark.parametrize("build,box", CASES)
def test_oracle_adjoint_is_exact_transpose(build, box):
    """J = <G, ts(w)> is linear in the source table: the adjoint's dJ/dw
    reproduces J (CPML, PEC faces and the PEC edge mask included)."""
    sc = build(n_steps=100)
    G = np.random.default_rng(0).standard_normal((sc.n_steps, len(sc.probes)))
    ts, grad, sadj = _fa(sc, box, G)
    J = float((G * ts).sum())
    Jt = sum(float((sadj[:, s] * sc.sources[s][4][:sc.n_steps]).sum()) for s in range(len(sc.sources)))
    assert abs(J - Jt) <= 1e-12 * abs(J)


@pytest.mark.parametrize("build,box", CASES)
def test_oracle_gradient_matches_finite_differences(build, box):
    sc = build(n_steps=100)
    rng = np.random.default_rng(1)
    G = rng.standard_normal((sc.n_steps, len(sc.probes)))
    _, grad, _ = _fa(sc, box, G)
    i0, i1, j0, j1, k0, k1 = box
    d = rng.standard_normal(grad.shape)
    h = 1e-4

    def J_of(eps):
        s2 = sc.__class__(**{**sc.__dict__, "materials": (eps, sc.materials[1], sc.materials[2])})
        return float((G * s2.run_oracle(np.float64, exact_materials=True).time_series).sum())

    ep = sc.materials[0].astype(np.float64).copy()
    em = ep.copy()
    ep[i0:i1, j0:j1, k0:k1] += h * d
    em[i0:i1, j0:j1, k0:k1] -= h * d
    fd = (J_of(ep) - J_of(em)) / (2 * h)
    ad = float((grad * d).sum())
    assert abs(ad - fd) <= 1e-5 * abs(fd)


@pytest.mark.parametrize("build", [small_uniform, small_nonuniform])
def test_oracle_gradient_inside_cpml_matches_finite_differences(build):
    """A region that reaches into the absorber (the x lo slab, both y slabs
    across the full transverse extent, the z hi slab and their corners): the
    CPML-E coefficient ce = dt/(eps_r eps0) of rfx/boundaries/cpml.py:536-546
    depends on eps_r there, and the gradient includes that term."""
    sc = build(n_steps=100)
    nx, ny, nz = sc.ogrid.shape
    n = sc.ogrid.cpml_layers
    box = (n - 4, n + 3, 0, ny, nz - n - 2, nz)
    rng = np.random.default_rng(2)
    G = rng.standard_normal((sc.n_steps, len(sc.probes)))
    _, grad, _ = _fa(sc, box, G)
    i0, i1, j0, j1, k0, k1 = box
    d = rng.standard_normal(grad.shape)
    h = 1e-4

    def J_of(eps):
        s2 = sc.__class__(**{**sc.__dict__, "materials": (eps, sc.materials[1], sc.materials[2])})
        return float((G * s2.run_oracle(np.float64, exact_materials=True).time_series).sum())

    ep = sc.materials[0].astype(np.float64).copy()
    em = ep.copy()
    ep[i0:i1, j0:j1, k0:k1] += h * d
    em[i0:i1, j0:j1, k0:k1] -= h * d
    fd = (J_of(ep) - J_of(em)) / (2 * h)
    ad = float((grad * d).sum())
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)
