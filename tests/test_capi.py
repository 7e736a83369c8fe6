"""CPU checks of the C ABI boundary and the host-side setup (no GPU work)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
import rfx_b200
from rfx_b200 import _lib
from rfx_b200.cpml import build_cpml
from rfx_b200.grid import spacing_tables

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rfxb200.h")


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "rfxb200.h")).read()
    return set(re.findall(r"^\s*(?:[A-Za-z_][A-Za-z0-9_ \*]*?)\b(rfxb_[a-z0-9_]+)\s*\(", txt, re.M))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in sorted(declared):
        assert hasattr(lib, name), f"{name} declared in include/rfxb200.h but not exported"
    assert declared == set(_lib.SIGNATURES), "ctypes signature table and header disagree"
    assert lib.rfxb_version() >= 10000


def test_struct_layout_matches_header(tmp_path):
    """ctypes mirrors of the header structs have the sizes and field offsets
    the C compiler gives them (the header compiled with gcc here)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    structs = {
        "RfxbDftDesc": _lib.RfxbDftDesc, "RfxbFluxDesc": _lib.RfxbFluxDesc, "RfxbNtffDesc": _lib.RfxbNtffDesc,
        "RfxbDesc": _lib.RfxbDesc,
        "RfxbStepIO": _lib.RfxbStepIO, "RfxbAdjointIO": _lib.RfxbAdjointIO,
        "RfxbLaunchConfig": _lib.RfxbLaunchConfig,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                                text=True).stdout.split("\n") if line)
    for name, cls in structs.items():
        assert int(out[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(out[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def _desc(shape=(10, 10, 10), **over):
    d = _lib.RfxbDesc()
    d.nx, d.ny, d.nz = shape
    d.dt = 1e-12
    tabs = [np.ones(n, np.float32) for n in (shape[0], shape[0], shape[1], shape[1], shape[2], shape[2])]
    (d.inv_xe_host, d.inv_xh_host, d.inv_ye_host, d.inv_yh_host, d.inv_ze_host,
     d.inv_zh_host) = [t.ctypes.data_as(_lib.c_float_p) for t in tabs]
    for k, v in over.items():
        setattr(d, k, v)
    return d, tabs


@pytest.mark.parametrize("field,value,code", [
    ("nx", 1, -2), ("dt", 0.0, -1), ("dt", -1.0, -1), ("cpml_layers", -1, -1),
])
def test_plan_create_rejects_bad_descriptor_before_touching_the_device(field, value, code):
    """Host-side validation returns an error code and a message; no kernel
    runs, no allocation happens (the checks precede any CUDA call)."""
    lib = _lib.load()
    d, keep = _desc(**{field: value})
    h = C.c_void_p()
    rc = lib.rfxb_plan_create(C.byref(d), C.byref(h))
    assert rc == code
    assert h.value is None
    assert lib.rfxb_last_error().decode()


def test_plan_create_rejects_out_of_range_monitors():
    lib = _lib.load()
    src = np.array([[0, 0, 99, 2]], np.int32)
    d, keep = _desc(n_src=1, src_cells_host=src.ctypes.data_as(_lib.c_int32_p))
    h = C.c_void_p()
    assert lib.rfxb_plan_create(C.byref(d), C.byref(h)) == -1
    assert "source" in lib.rfxb_last_error().decode()
    prb = np.array([[1, 1, 1, 7]], np.int32)
    d, keep = _desc(n_probe=1, probe_cells_host=prb.ctypes.data_as(_lib.c_int32_p))
    assert lib.rfxb_plan_create(C.byref(d), C.byref(h)) == -1
    assert "probe" in lib.rfxb_last_error().decode()
    # an NTFF face plane must lie inside the grid (i_hi is a plane index)
    for box in ((2, 10, 2, 8, 2, 8, 1), (5, 5, 2, 8, 2, 8, 1), (2, 8, 2, 8, 2, 8, 0)):
        nb = _lib.RfxbNtffDesc(*box)
        d, keep = _desc(ntff_host=C.pointer(nb))
        assert lib.rfxb_plan_create(C.byref(d), C.byref(h)) == -1
        assert "NTFF" in lib.rfxb_last_error().decode()
        assert h.value is None


def test_cpml_overlap_rejected():
    lib = _lib.load()
    b = np.ones((6, 8), np.float32)
    d, keep = _desc(shape=(10, 40, 40), cpml_layers=8, cpml_axes=7,
                    cpml_b_host=b.ctypes.data_as(_lib.c_float_p), cpml_c_host=b.ctypes.data_as(_lib.c_float_p),
                    cpml_kappa_host=b.ctypes.data_as(_lib.c_float_p))
    h = C.c_void_p()
    assert lib.rfxb_plan_create(C.byref(d), C.byref(h)) == -2


def test_host_cpml_tables_match_oracle():
    og = oracle.make_uniform_grid((0.14, 0.06, 0.05), 2e-3, cpml_layers=8)
    pg = rfx_b200.Grid(freq_max=5e9, domain=(0.14, 0.06, 0.05), dx=2e-3, cpml_layers=8)
    assert pg.shape == og.shape and pg.dt == og.dt
    cp = build_cpml(pg, "xyz")
    ref = oracle.build_cpml(og)
    for f, face in enumerate(("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")):
        b, c, k, d = ref[face]
        np.testing.assert_array_equal(cp.b[f], b)
        np.testing.assert_array_equal(cp.c[f], c)
        np.testing.assert_array_equal(cp.kappa[f], k)
        assert cp.cell[f] == d


def test_host_graded_tables_match_oracle():
    dz = np.linspace(1e-4, 5e-4, 20)
    og = oracle.make_nonuniform_grid((0.01, 0.008), dz, 5e-4, cpml_layers=6)
    pg = rfx_b200.make_nonuniform_grid((0.01, 0.008), dz, 5e-4, cpml_layers=6)
    assert pg.shape == og.shape and pg.dt == og.dt
    tabs = spacing_tables(pg)
    for t, name in zip(tabs, ("inv_dx", "inv_dx_h", "inv_dy", "inv_dy_h", "inv_dz", "inv_dz_h")):
        np.testing.assert_array_equal(t, getattr(og, name))
    cp = build_cpml(pg, "xyz")
    ref = oracle.build_cpml(og)
    for f, face in enumerate(("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")):
        np.testing.assert_array_equal(cp.b[f], ref[face][0])
        assert cp.cell[f] == ref[face][3]


def test_host_waveforms_match_oracle():
    og = oracle.make_uniform_grid((0.14, 0.06, 0.05), 2e-3, cpml_layers=8)
    pg = rfx_b200.Grid(freq_max=5e9, domain=(0.14, 0.06, 0.05), dx=2e-3, cpml_layers=8)
    shape = og.shape
    eps = np.full(shape, 2.2, np.float32)
    sig = np.full(shape, 0.01, np.float32)
    mats = rfx_b200.MaterialArrays(eps, sig, np.ones(shape, np.float32))
    s = rfx_b200.make_j_source(pg, (0.03, 0.03, 0.025), "ez", rfx_b200.GaussianPulse(3e9, 0.8), 500, mats)
    w = oracle.j_source_waveform(og, (s.i, s.j, s.k), (eps, sig, None), 500, 3e9, 0.8)
    np.testing.assert_array_equal(s.waveform, w)


def test_edge_mask_bits_match_oracle():
    rng = np.random.default_rng(0)
    m = rng.random((9, 8, 7)) > 0.7
    bits = rfx_b200.simulation.tangential_edge_masks(m)
    ref = oracle.tangential_edge_masks(m)
    for ax in range(3):
        np.testing.assert_array_equal(((bits >> ax) & 1).astype(bool), ref[ax])


def test_unsupported_features_raise():
    g = rfx_b200.Grid(freq_max=5e9, domain=(0.01, 0.01, 0.01), dx=1e-3, cpml_layers=2)
    mats = rfx_b200.MaterialArrays(*(np.ones(g.shape, np.float32),) * 3)
    with pytest.raises(NotImplementedError):
        rfx_b200.run(g, mats, 10, debye=object())
    with pytest.raises(NotImplementedError):
        rfx_b200.run(g, mats, 10, periodic=(True, False, False))
    with pytest.raises(ValueError):
        rfx_b200.run(g, mats, 10, checkpoint_segments=3)


@pytest.mark.parametrize("n_src,n_probe,null_src,null_prb", [
    (-1, 0, False, False), (0, -2, False, False), (1, 0, True, False), (0, 1, False, True),
])
def test_negative_counts_and_null_tables_rejected(n_src, n_probe, null_src, null_prb):
    """Negative source / probe counts, and a null cell table with a positive
    count, are refused with RFXB_E_INVALID by plan creation and by the no-alloc
    forward entry point, before any CUDA call (so on a host without a GPU)."""
    lib = _lib.load()
    src = np.array([[1, 1, 1, 2]], np.int32)
    prb = np.array([[2, 2, 2, 2]], np.int32)
    over = dict(n_src=n_src, n_probe=n_probe)
    if not null_src:
        over["src_cells_host"] = src.ctypes.data_as(_lib.c_int32_p)
    if not null_prb:
        over["probe_cells_host"] = prb.ctypes.data_as(_lib.c_int32_p)
    d, keep = _desc(**over)
    h = C.c_void_p()
    assert lib.rfxb_plan_create(C.byref(d), C.byref(h)) == -1
    assert h.value is None
    assert "count" in lib.rfxb_last_error().decode()
    # placeholder device addresses: the arguments are refused before any use
    fake = C.c_void_p(0x1000)
    fields = (C.c_void_p * 6)(*([0x1000] * 6))
    rc = lib.rfxb_forward_noalloc(C.byref(d), fake, fake, fields, None, 0, 1, None)
    assert rc == -1
    msg = lib.rfxb_last_error().decode()
    assert "count" in msg or "table" in msg, msg
