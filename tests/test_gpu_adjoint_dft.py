"""GPU tests of the adjoint with DFT-plane, NTFF and flux objectives (the
transposes of the running DFT, rfx/simulation.py:1574-1588 and rfx/nonuniform.py:
1458-1472, and of the NTFF box, rfx/farfield.py:208-313, which the reference
differentiates with jax.grad through the scan).

1. Exact transpose: a DFT accumulator is linear in the source table, so for
   J = sum Re(conj(G) acc) (plus <g, ts> of the probes) the source adjoint
   must reproduce J.  The planes of the uniform scene cross a source cell
   (the cotangent feeds the source adjoint there) and a PEC sheet whose edge
   mask zeroes the sampled component (the cotangent is dropped there).
2. dJ/d eps_r of J = sum |acc|^2 against central finite differences of the
   float64 oracle along three seeded directions (tolerance 1e-3 relative).
3. The torch.autograd face returns the accumulators as outputs and accepts
   their gradients.
4. NTFF: the exact transpose for a face objective, and the directivity at
   one direction (through the differentiable device far-field transform)
   against float64 finite differences of the oracle.
5. Flux monitors (rfx/simulation.py:1590-1642): the exact transpose, and the
   power through two planes (one windowed) against float64 finite
   differences.
"""

import numpy as np
import pytest
import torch

import oracle  # noqa: F401
from tests.scenarios import small_nonuniform, small_uniform

pytestmark = pytest.mark.gpu


def _planes(sc):
    extra = [(2, 15, "ex", sc.dft[0][3])] if sc.lane == "uniform" else []   # crosses the PEC sheet
    return list(sc.dft) + extra


def _runner(sc, box, planes, mode="history", K=None):
    import rfx_b200
    from rfx_b200.adjoint import AdjointRunner
    g = sc.product_grid()
    mats = rfx_b200.MaterialArrays(*sc.materials)
    if sc.lane == "nonuniform":
        pads = (g.pad_x_lo + g.pad_x_hi, g.pad_y_lo + g.pad_y_hi, g.pad_z_lo + g.pad_z_hi)
        axes, pec_axes = "".join(a for a, p in zip("xyz", pads) if p > 0), "xyz"
    else:
        axes, pec_axes = "xyz", (sc.pec_axes if sc.pec_axes is not None else "xyz")
    dfts = [rfx_b200.init_dft_plane_probe(a, ix, c, f, g.shape) for (a, ix, c, f) in planes]
    return AdjointRunner(g, mats, sc.n_steps, sources=sc.sources, probes=sc.probes, box=box, boundary=sc.boundary,
                         cpml_axes=axes, pec_axes=pec_axes, pec_mask=sc.pec_mask, mode=mode, checkpoint_every=K,
                         dft_planes=dfts, dft_time_offset=1 if sc.lane == "uniform" else 0)


@pytest.mark.parametrize("build,box", [(small_uniform, (14, 18, 14, 18, 12, 14)),
                                       (small_nonuniform, (12, 16, 12, 16, 11, 13))])
@pytest.mark.parametrize("mode", ["history", "segments"])
def test_dft_adjoint_is_exact_transpose(cuda, build, box, mode):
    sc = build(n_steps=150)
    planes = _planes(sc)
    r = _runner(sc, box, planes, mode=mode, K=64)
    ts = r.forward()
    rng = np.random.default_rng(9)
    G = [torch.from_numpy((rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)).astype(np.complex64))
         .cuda() for a in r.dft_accs]
    g = torch.from_numpy(rng.standard_normal(ts.shape).astype(np.float32)).cuda()
    J_dft = sum(float((Gq.real.double() * a.real.double() + Gq.imag.double() * a.imag.double()).sum())
                for Gq, a in zip(G, r.dft_accs))
    J_prb = float((g.double() * ts.double()).sum())
    _, s1 = r.backward(None, g_dft=G)
    _, s2 = r.backward(g, g_dft=G)
    J1 = float((s1.double() * r.src_table.double()).sum())
    J2 = float((s2.double() * r.src_table.double()).sum())
    print(sc.name, mode, "J_dft", J_dft, "via adjoint", J1, "| J_dft + J_probe", J_dft + J_prb, "via adjoint", J2)
    assert abs(J1 - J_dft) <= 2e-5 * abs(J_dft)
    assert abs(J2 - (J_dft + J_prb)) <= 2e-5 * abs(J_dft + J_prb)
    r.close()


def _oracle_dft_J(sc, eps_full, planes):
    mats = (eps_full, sc.materials[1], sc.materials[2])
    kw = dict(sources=sc.sources, probes=sc.probes, dft_planes=planes, pec_mask=sc.pec_mask, dtype=np.float64,
              exact_materials=True)
    if sc.lane == "uniform":
        r = oracle.run_uniform(sc.ogrid, mats, sc.n_steps, boundary=sc.boundary, pec_axes=sc.pec_axes, **kw)
    else:
        r = oracle.run_nonuniform(sc.ogrid, mats, sc.n_steps, **kw)
    return float(sum(np.sum(np.abs(a) ** 2) for a in r.dft_planes))


@pytest.mark.parametrize("build,box", [(small_uniform, (14, 20, 14, 20, 12, 14)),
                                       (small_nonuniform, (12, 18, 12, 18, 11, 13))])
def test_dft_gradient_matches_fp64_finite_differences(cuda, build, box):
    sc = build(n_steps=160)
    planes = _planes(sc)
    r = _runner(sc, box, planes)
    r.forward()
    grad, _ = r.backward(None, g_dft=[2 * a for a in r.dft_accs])   # d|a|^2 = 2 Re(conj(a) da)
    grad = grad.cpu().numpy()
    i0, i1, j0, j1, k0, k1 = box
    rng = np.random.default_rng(13)
    for _ in range(3):
        d = rng.standard_normal((i1 - i0, j1 - j0, k1 - k0))
        h = 1e-3
        ep = sc.materials[0].astype(np.float64).copy()
        em = ep.copy()
        ep[i0:i1, j0:j1, k0:k1] += h * d
        em[i0:i1, j0:j1, k0:k1] -= h * d
        fd = (_oracle_dft_J(sc, ep, planes) - _oracle_dft_J(sc, em, planes)) / (2 * h)
        ad = float(np.sum(grad * d))
        print(sc.name, "directional AD", ad, "FD64", fd, "rel", abs(ad - fd) / abs(fd))
        assert abs(ad - fd) <= 1e-3 * abs(fd)
    r.close()


def test_autograd_function_with_dft_outputs(cuda):
    from rfx_b200.adjoint import FDTDFunction
    sc = small_uniform(n_steps=120)
    box = (14, 18, 14, 18, 12, 14)
    r = _runner(sc, box, _planes(sc))
    eps_box = torch.tensor(sc.materials[0][14:18, 14:18, 12:14], device="cuda", requires_grad=True)
    src = r.src_table.clone().requires_grad_(True)
    ts, *accs = FDTDFunction.apply(eps_box, src, r)
    assert len(accs) == 3 and all(a.dtype == torch.complex64 for a in accs)
    J = sum((a.abs() ** 2).sum() for a in accs) + ts.square().sum()
    J.backward()
    ge, gs = eps_box.grad, src.grad
    assert torch.isfinite(ge).all() and float(ge.abs().sum()) > 0
    # the same gradients from the runner directly
    g2, s2 = r.backward(2 * ts.detach(), g_dft=[2 * a.detach() for a in accs])
    assert torch.allclose(ge.double(), g2, rtol=1e-6, atol=0)
    assert torch.allclose(gs, s2, rtol=1e-6, atol=0)
    r.close()


# ---------------------------------------------------------------- NTFF box
# The box of the uniform scene: its x_lo face passes through the ez source
# (12, 13, 13) and its z_hi face lies on the PEC sheet (k = 15), whose edge
# mask zeroes ex / ey there.
_NTFF_BOX = (12, 30, 9, 26, 10, 15)
_NTFF_FREQS = np.array([12e9, 15e9], np.float32)


def _ntff_runner(sc, box, mode="history", K=None):
    import rfx_b200
    from rfx_b200.adjoint import AdjointRunner
    g = sc.product_grid()
    nb = rfx_b200.NTFFBox(*_NTFF_BOX, _NTFF_FREQS, *(sc.ogrid.cpml_layers,) * 6)
    return AdjointRunner(g, rfx_b200.MaterialArrays(*sc.materials), sc.n_steps, sources=sc.sources,
                         probes=sc.probes, box=box, boundary=sc.boundary, cpml_axes="xyz",
                         pec_axes=sc.pec_axes if sc.pec_axes is not None else "xyz", pec_mask=sc.pec_mask,
                         mode=mode, checkpoint_every=K, ntff=nb), nb


@pytest.mark.parametrize("mode", ["history", "segments"])
def test_ntff_adjoint_is_exact_transpose(cuda, mode):
    sc = small_uniform(n_steps=150)
    r, _ = _ntff_runner(sc, (14, 18, 14, 18, 12, 14), mode=mode, K=64)
    r.forward()
    rng = np.random.default_rng(21)
    G = [torch.from_numpy((rng.standard_normal(f.shape) + 1j * rng.standard_normal(f.shape)).astype(np.complex64))
         .cuda() for f in r.ntff_faces]
    J = sum(float((Gq.real.double() * f.real.double() + Gq.imag.double() * f.imag.double()).sum())
            for Gq, f in zip(G, r.ntff_faces))
    _, s1 = r.backward(None, g_ntff=G)
    J1 = float((s1.double() * r.src_table.double()).sum())
    print(mode, "J_ntff", J, "via adjoint", J1)
    assert abs(J1 - J) <= 2e-5 * abs(J)
    r.close()


def _oracle_directivity(sc, eps_full, theta, phi, it, ip):
    from oracle import farfield as off
    mats = (eps_full, sc.materials[1], sc.materials[2])
    r = oracle.run_uniform(sc.ogrid, mats, sc.n_steps, boundary=sc.boundary, pec_axes=sc.pec_axes,
                           sources=sc.sources, probes=sc.probes, pec_mask=sc.pec_mask, dtype=np.float64,
                           exact_materials=True, ntff=(*_NTFF_BOX, _NTFF_FREQS))
    n = sc.ogrid.cpml_layers
    Et, Ep = off.compute_far_field(r.ntff, (*_NTFF_BOX, _NTFF_FREQS), sc.ogrid.dx, (n, n, n), theta, phi)
    p = np.abs(Et) ** 2 + np.abs(Ep) ** 2
    dth, dph = np.gradient(theta), np.gradient(phi)
    prad = np.sum(p * np.sin(theta)[None, :, None] * dth[None, :, None] * dph[None, None, :], axis=(1, 2))
    return float(np.sum(4 * np.pi * p[:, it, ip] / prad))


def test_directivity_gradient_matches_fp64_finite_differences(cuda):
    """The far-field objective of rfx's directivity optimisation, restated:
    J = sum over the NTFF frequencies of the directivity (4 pi U / P_rad) at
    one direction, through the device far-field transform and the NTFF
    outputs of FDTDFunction (rfx tests/test_directivity_gradient.py checks
    the same path through jax.grad for a nonzero, finite value)."""
    import rfx_b200
    from rfx_b200.adjoint import FDTDFunction
    sc = small_uniform(n_steps=160)
    box = (14, 20, 14, 20, 12, 14)
    r, nb = _ntff_runner(sc, box)
    theta = np.linspace(0.05, np.pi - 0.05, 19)
    phi = np.linspace(0.0, 2 * np.pi, 12, endpoint=False)
    it, ip = 9, 0
    g = sc.product_grid()
    eps_box = torch.tensor(sc.materials[0][box[0]:box[1], box[2]:box[3], box[4]:box[5]], device="cuda",
                           requires_grad=True)
    ts, *faces = FDTDFunction.apply(eps_box, None, r)
    Et, Ep = rfx_b200.far_field(faces, nb, g, theta, phi)
    J = rfx_b200.directivity_torch(Et, Ep, theta, phi)[:, it, ip].sum()
    J.backward()
    grad = eps_box.grad.double().cpu().numpy()
    J0 = _oracle_directivity(sc, sc.materials[0].astype(np.float64), theta, phi, it, ip)
    Jv = float(J.detach())
    print("directivity objective CUDA", Jv, "oracle f64", J0)
    assert abs(Jv - J0) <= 1e-4 * abs(J0)
    i0, i1, j0, j1, k0, k1 = box
    rng = np.random.default_rng(17)
    for _ in range(3):
        d = rng.standard_normal((i1 - i0, j1 - j0, k1 - k0))
        h = 1e-3
        ep = sc.materials[0].astype(np.float64).copy()
        em = ep.copy()
        ep[i0:i1, j0:j1, k0:k1] += h * d
        em[i0:i1, j0:j1, k0:k1] -= h * d
        fd = (_oracle_directivity(sc, ep, theta, phi, it, ip) - _oracle_directivity(sc, em, theta, phi, it, ip)) / (2 * h)
        ad = float(np.sum(grad * d))
        print("directivity directional AD", ad, "FD64", fd, "rel", abs(ad - fd) / abs(fd))
        assert abs(ad - fd) <= 1e-3 * abs(fd)
    r.close()


# ---------------------------------------------------------- flux monitors
def _flux_mons(sc):
    f = np.array([10e9, 14e9, 18e9])
    nx, ny, nz = sc.ogrid.shape
    # an x plane through the ez source (12, 13, 13), a windowed z plane on the PEC sheet (k = 15)
    return [(0, 12, 6, ny - 6, 6, nz - 6, f, 0, "rect", 0.25),
            (2, 15, 6, nx - 6, 6, ny - 6, f[:2], sc.n_steps, "hann", 0.25)]


def _flux_runner(sc, box, mode="history", K=None):
    import rfx_b200
    from rfx_b200.adjoint import AdjointRunner
    g = sc.product_grid()
    fms = [rfx_b200.init_flux_monitor(m[0], m[1], m[6], g.shape, g.dx, g.dx, dft_total_steps=m[7], dft_window=m[8],
                                      dft_window_alpha=m[9], lo1=m[2], hi1=m[3], lo2=m[4], hi2=m[5])
           for m in _flux_mons(sc)]
    return AdjointRunner(g, rfx_b200.MaterialArrays(*sc.materials), sc.n_steps, sources=sc.sources,
                         probes=sc.probes, box=box, boundary=sc.boundary, cpml_axes="xyz",
                         pec_axes=sc.pec_axes if sc.pec_axes is not None else "xyz", pec_mask=sc.pec_mask,
                         mode=mode, checkpoint_every=K, flux_monitors=fms), fms


@pytest.mark.parametrize("mode", ["history", "segments"])
def test_flux_adjoint_is_exact_transpose(cuda, mode):
    sc = small_uniform(n_steps=150)
    r, _ = _flux_runner(sc, (14, 18, 14, 18, 12, 14), mode=mode, K=64)
    r.forward()
    rng = np.random.default_rng(23)
    G = [torch.from_numpy(rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)).cuda()
         for a in r.flux_accs]
    J = sum(float((Gq.real * a.real + Gq.imag * a.imag).sum()) for Gq, a in zip(G, r.flux_accs))
    _, s1 = r.backward(None, g_flux=G)
    J1 = float((s1.double() * r.src_table.double()).sum())
    print(mode, "J_flux", J, "via adjoint", J1)
    assert abs(J1 - J) <= 2e-5 * abs(J)
    r.close()


def _power(acc, dA):
    """flux_spectrum of a (4, n_f, n1, n2) accumulator, summed over frequency."""
    e1, e2, h1, h2 = acc[0], acc[1], acc[2], acc[3]
    return ((e1 * h2.conj() - e2 * h1.conj()).real * dA).sum()


def test_flux_gradient_matches_fp64_finite_differences(cuda):
    from rfx_b200.adjoint import FDTDFunction
    sc = small_uniform(n_steps=160)
    box = (14, 20, 14, 20, 12, 14)
    r, fms = _flux_runner(sc, box)
    mons = _flux_mons(sc)
    eps_box = torch.tensor(sc.materials[0][box[0]:box[1], box[2]:box[3], box[4]:box[5]], device="cuda",
                           requires_grad=True)
    ts, *accs = FDTDFunction.apply(eps_box, None, r)
    assert len(accs) == 2 and accs[0].dtype == torch.complex128
    dA = [torch.as_tensor(np.asarray(m.dA, np.float64), device="cuda") for m in fms]
    J = sum(_power(a, d) for a, d in zip(accs, dA))
    J.backward()
    grad = eps_box.grad.double().cpu().numpy()

    def oracle_J(eps_full):
        mats = (eps_full, sc.materials[1], sc.materials[2])
        o = oracle.run_uniform(sc.ogrid, mats, sc.n_steps, boundary=sc.boundary, pec_axes=sc.pec_axes,
                               sources=sc.sources, probes=sc.probes, pec_mask=sc.pec_mask, dtype=np.float64,
                               exact_materials=True, flux_monitors=mons)
        return float(sum(_power(torch.from_numpy(a), torch.from_numpy(np.asarray(m.dA, np.float64)))
                         for a, m in zip(o.flux, fms)))

    J0 = oracle_J(sc.materials[0].astype(np.float64))
    Jv = float(J.detach())
    print("flux objective CUDA", Jv, "oracle f64", J0)
    assert abs(Jv - J0) <= 1e-4 * abs(J0)
    i0, i1, j0, j1, k0, k1 = box
    rng = np.random.default_rng(19)
    for _ in range(3):
        d = rng.standard_normal((i1 - i0, j1 - j0, k1 - k0))
        h = 1e-3
        ep = sc.materials[0].astype(np.float64).copy()
        em = ep.copy()
        ep[i0:i1, j0:j1, k0:k1] += h * d
        em[i0:i1, j0:j1, k0:k1] -= h * d
        fd = (oracle_J(ep) - oracle_J(em)) / (2 * h)
        ad = float(np.sum(grad * d))
        print("flux directional AD", ad, "FD64", fd, "rel", abs(ad - fd) / abs(fd))
        assert abs(ad - fd) <= 1e-3 * abs(fd)
    r.close()
