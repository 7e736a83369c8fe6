"""The XLA FFI face.  jax is not installed everywhere this suite runs: the
build recipe must then skip the handlers cleanly; where jax and a GPU exist,
the custom-call forward and the custom_vjp gradient agree with the torch face
of the same kernels."""

import os
import re

import numpy as np
import pytest

from rfx_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_ffi_source_binds_the_c_abi():
    """The handler source registers the three targets the Python side
    names, and calls only entry points the header declares."""
    src = open(build.FFI_SRC).read()
    for sym in ("RfxbFfiForward", "RfxbFfiForwardRecord", "RfxbFfiAdjoint"):
        assert re.search(rf"XLA_FFI_DEFINE_HANDLER_SYMBOL\(\s*{sym}\b", src), sym
    header = open(os.path.join(ROOT, "include", "rfxb200.h")).read()
    for name in set(re.findall(r"\b(rfxb_[a-z_]+)\(", src)):
        assert re.search(rf"\b{name}\s*\(", header), name


def test_build_recipe_skips_without_jaxlib_headers():
    if build.ffi_include_dir() is not None:
        pytest.skip("jaxlib FFI headers present: the handlers are built instead")
    assert build.build_ffi() is None


@pytest.mark.gpu
def test_jax_custom_vjp_matches_torch_adjoint(cuda):
    jax = pytest.importorskip("jax")
    import jax.numpy as jnp

    if build.build_ffi() is None:
        pytest.skip("jaxlib FFI headers not installed")
    import torch

    from rfx_b200.adjoint import AdjointRunner
    from rfx_b200.jax_ffi import JaxFDTD
    from tests.scenarios import small_uniform

    sc = small_uniform(n_steps=120)
    g = sc.product_grid()
    box = (14, 20, 14, 20, 12, 14)
    import rfx_b200
    mats = rfx_b200.MaterialArrays(*sc.materials)
    kw = dict(sources=sc.sources, probes=sc.probes, box=box, boundary="cpml", cpml_axes="xyz", pec_axes="xyz")
    G = np.random.default_rng(0).standard_normal((sc.n_steps, len(sc.probes))).astype(np.float32)
    run = AdjointRunner(g, mats, sc.n_steps, **kw)
    ts = run.forward().cpu().numpy()
    grad_t, _ = run.backward(torch.from_numpy(G).cuda())
    jf = JaxFDTD(g, mats, sc.n_steps, **kw)
    eps_box = jnp.asarray(sc.materials[0][14:20, 14:20, 12:14])
    ts_j = np.asarray(jf.probe_traces(eps_box, jf.src_table))
    assert np.linalg.norm(ts_j - ts) <= 1e-6 * np.linalg.norm(ts)
    gj = jax.grad(lambda e: jnp.sum(jf.probe_traces(e, jf.src_table) * G))(eps_box)
    gt = grad_t.cpu().numpy().reshape(gj.shape)
    assert np.linalg.norm(np.asarray(gj, np.float64) - gt) <= 1e-5 * np.linalg.norm(gt)
