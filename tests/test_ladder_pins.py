"""The adjoint pinned to the reference's own ``jax.grad``.

The reference holds two gradient witnesses computed by its JAX solver in
float32 (tests/fixtures/gradient_dx_ladder/, copied to tests/golden/; scenes
rebuilt in tests/ladder.py):

* a scalar slab eps_r whose mask spans the whole transverse extent, CPML pads
  included, at lambda/dx = 20, 30, 40, 60: J0, J(eps +- h) and
  grad_ad = dJ/d eps_slab from ``jax.grad``;
* a per-cell eps_r block at lambda/dx = 20, 30, 40: J0 and |dJ/d eps_r| of
  every cell from ``jax.grad``.

The oracle (CPU) is checked at the coarsest rung of each; the CUDA forward
and hand-written adjoint at every rung.  Bars: J within 1e-4 relative, the
slab gradient within 1e-3 relative, the per-cell gradients within 1e-3 of the
largest cell's magnitude (the smallest cells sit four orders of magnitude
below it, at the float32 resolution of the sum).
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.ladder import block_fixture, ladder_scene, oracle_J, oracle_forward_adjoint, slab_fixture

TOL_J = 1e-4
TOL_GRAD = 1e-3
TOL_CELL = 1e-3


def test_oracle_matches_reference_slab_ladder():
    """lambda/20 slab: J0, J(eps +- 0.04) and the slab gradient of the oracle
    against the reference's float32 JAX run."""
    r = slab_fixture()[0]
    sc = ladder_scene("slab", r["lambda_over_dx"])
    J0, grad = oracle_forward_adjoint(sc, r["eps0"])
    h = r["fd_step_abs"]
    Jp, Jm = oracle_J(sc, r["eps0"] + h), oracle_J(sc, r["eps0"] - h)
    errs = {"J0": abs(J0 / r["J0"] - 1), "J_plus": abs(Jp / r["J_plus"] - 1),
            "J_minus": abs(Jm / r["J_minus"] - 1), "grad_ad": abs(grad.sum() / r["grad_ad"] - 1)}
    print(f"oracle {r['rung']}: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert errs["J0"] < TOL_J and errs["J_plus"] < TOL_J and errs["J_minus"] < TOL_J
    assert errs["grad_ad"] < TOL_GRAD


def test_oracle_matches_reference_per_cell_gradients():
    """lambda/20 block: J0 and |dJ/d eps_r| of each of the 64 cells."""
    r = block_fixture()[0]
    sc = ladder_scene("block", r["lambda_over_dx"])
    J0, grad = oracle_forward_adjoint(sc, r["eps_block"])
    ref = np.asarray(r["per_cell_grad_abs"])
    got = np.abs(grad).ravel()
    cell = float(np.max(np.abs(got - ref)) / ref.max())
    print(f"oracle block {r['rung']}: J0 {abs(J0 / r['J0'] - 1):.2e}, per-cell {cell:.2e}")
    assert abs(J0 / r["J0"] - 1) < TOL_J
    assert cell < TOL_CELL


def _cuda_J_grad(sc, eps_value, want_grad=True):
    import torch

    import rfx_b200
    from rfx_b200.adjoint import AdjointRunner
    g = rfx_b200.Grid(freq_max=10e9, domain=sc.domain, dx=sc.dx, cpml_layers=8)
    assert tuple(g.shape) == tuple(sc.grid.shape)
    mats = sc.materials(eps_value)
    w = sc.source_wave(mats)
    run = AdjointRunner(g, rfx_b200.MaterialArrays(*mats), sc.n_steps, sources=[(*sc.src, "ez", w)],
                        probes=[(*sc.prb, "ez")], box=sc.box, boundary="cpml", cpml_axes="xyz", pec_axes="")
    ts = run.forward()[:, 0].detach().cpu().numpy()
    J, dJ = sc.objective(ts)
    grad = None
    if want_grad:
        gt = torch.from_numpy(dJ[:, None].astype(np.float32)).cuda()
        grad, _ = run.backward(gt, want_source_grad=False)
        grad = grad.detach().cpu().numpy().astype(np.float64)
    run.plan.close()
    return J, grad


@pytest.mark.gpu
def test_cuda_adjoint_matches_reference_slab_ladder(cuda):
    """Every rung of the slab ladder through the CUDA forward and adjoint:
    J0, J(eps +- h) and the slab gradient (cells in the y and z CPML slabs
    included) against the reference's jax.grad."""
    worst = {}
    for r in slab_fixture():
        sc = ladder_scene("slab", r["lambda_over_dx"])
        J0, grad = _cuda_J_grad(sc, r["eps0"])
        h = r["fd_step_abs"]
        Jp, _ = _cuda_J_grad(sc, r["eps0"] + h, want_grad=False)
        Jm, _ = _cuda_J_grad(sc, r["eps0"] - h, want_grad=False)
        errs = {"J0": abs(J0 / r["J0"] - 1), "J_plus": abs(Jp / r["J_plus"] - 1),
                "J_minus": abs(Jm / r["J_minus"] - 1), "grad_ad": abs(grad.sum() / r["grad_ad"] - 1),
                "vs_ref_fd": abs(grad.sum() / r["grad_fd"] - 1)}
        print(f"cuda slab {r['rung']} {tuple(r['grid_shape'])} x {r['n_steps']}: "
              + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
        for k, v in errs.items():
            worst[k] = max(worst.get(k, 0.0), v)
    assert worst["J0"] < TOL_J and worst["J_plus"] < TOL_J and worst["J_minus"] < TOL_J
    assert worst["grad_ad"] < TOL_GRAD


@pytest.mark.gpu
def test_cuda_adjoint_matches_reference_per_cell_gradients(cuda):
    """Every rung of the block ladder: J0 and the per-cell |dJ/d eps_r|."""
    for r in block_fixture():
        sc = ladder_scene("block", r["lambda_over_dx"])
        J0, grad = _cuda_J_grad(sc, r["eps_block"])
        ref = np.asarray(r["per_cell_grad_abs"])
        got = np.abs(grad).ravel()
        cell = float(np.max(np.abs(got - ref)) / ref.max())
        med = float(np.median(np.abs(got - ref) / ref))
        print(f"cuda block {r['rung']} {r['design_shape']}: J0 {abs(J0 / r['J0'] - 1):.2e}, "
              f"per-cell max {cell:.2e} (median relative {med:.2e})")
        assert abs(J0 / r["J0"] - 1) < TOL_J
        assert cell < TOL_CELL
