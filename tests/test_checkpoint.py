"""State files (rfx/checkpoint.py) and the resumable plan state.

CPU: without h5py the HDF5 helpers raise the reference's ImportError; with
an in-memory stand-in for h5py they write the reference's groups, datasets
and attributes and read them back.  GPU: a CPML run with a DFT plane saved
to a state file after N1 steps, restored into a fresh plan and continued for
N2 steps equals the uninterrupted N1 + N2 run bit for bit; a blob of another
shape is rejected.
"""

import numpy as np
import pytest

import rfx_b200
from rfx_b200 import checkpoint as ck


class _Attrs(dict):
    pass


class _Group:
    def __init__(self):
        self.items = {}
        self.attrs = _Attrs()

    def create_group(self, name):
        g = _Group()
        self.items[name] = g
        return g

    def create_dataset(self, name, data):
        self.items[name] = np.array(data)
        return self.items[name]

    def __getitem__(self, name):
        return self.items[name]

    def __contains__(self, name):
        return name in self.items

    def __iter__(self):
        return iter(self.items)


class _FakeH5:
    """The part of h5py's File/Group/Dataset interface rfx/checkpoint.py uses."""
    files = {}

    class File(_Group):
        def __init__(self, path, mode):
            super().__init__()
            self.path, self.mode = str(path), mode
            if mode == "r":
                self.items = _FakeH5.files[self.path].items

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            if self.mode == "w":
                _FakeH5.files[self.path] = self
            return False


def test_hdf5_helpers_raise_without_h5py(tmp_path, monkeypatch):
    monkeypatch.setattr(ck, "h5py", None)
    st = rfx_b200.FDTDState(*(np.zeros((2, 2, 2), np.float32),) * 6, step=0)
    with pytest.raises(ImportError, match="h5py is required"):
        ck.save_state(tmp_path / "s.h5", st)
    with pytest.raises(ImportError, match="h5py is required"):
        ck.load_materials(tmp_path / "m.h5")


def test_hdf5_helpers_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(ck, "h5py", _FakeH5)
    rng = np.random.default_rng(3)
    g = rfx_b200.Grid(freq_max=10e9, domain=(0.01, 0.01, 0.01), cpml_layers=2)
    f = [rng.standard_normal(g.shape).astype(np.float32) for _ in range(6)]
    st = rfx_b200.FDTDState(*f, step=17)
    ck.save_state(tmp_path / "s.h5", st, grid=g)
    raw = _FakeH5.files[str(tmp_path / "s.h5")]
    assert set(raw["state"].items) == {"ex", "ey", "ez", "hx", "hy", "hz"}
    assert raw["state"].attrs["step"] == 17
    st2, meta = ck.load_state(tmp_path / "s.h5")
    for a, b in zip(f, (st2.ex, st2.ey, st2.ez, st2.hx, st2.hy, st2.hz)):
        np.testing.assert_array_equal(a, b)
    assert st2.step == 17 and meta["shape"] == tuple(g.shape) and meta["cpml_layers"] == 2
    m = rfx_b200.MaterialArrays(f[0], f[1], f[2])
    ck.save_materials(tmp_path / "m.h5", m)
    m2 = ck.load_materials(tmp_path / "m.h5")
    np.testing.assert_array_equal(m2.sigma, f[1])
    ck.save_snapshots(tmp_path / "n.h5", {"ez": np.stack(f[:3])}, grid=g, dt=g.dt)
    snaps, meta = ck.load_snapshots(tmp_path / "n.h5")
    np.testing.assert_array_equal(snaps["ez"], np.stack(f[:3]))
    assert meta["n_steps"] == 3 and meta["dt"] == g.dt


@pytest.mark.gpu
def test_plan_state_resume_is_bit_exact(cuda, tmp_path):
    import torch
    from rfx_b200.simulation import prepare_device_run
    g = rfx_b200.Grid(freq_max=20e9, domain=(0.012, 0.014, 0.011), dx=1e-3, cpml_layers=5)
    n1, n2 = 70, 90
    n = n1 + n2
    t = np.arange(n, dtype=np.float32) * np.float32(g.dt)
    w = rfx_b200.GaussianPulse(f0=25e9, bandwidth=0.5)(t).astype(np.float32)
    c = (g.nx // 2, g.ny // 2, g.nz // 2)
    rng = np.random.default_rng(5)
    eps = (1.0 + rng.random(g.shape)).astype(np.float32)
    mats = rfx_b200.MaterialArrays(eps, np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    planes = [rfx_b200.init_dft_plane_probe(2, c[2] + 2, "ez", [22e9, 27e9], g.shape)]
    kw = dict(cpml_axes="xyz", pec_axes="", sources=[(*c, "ez", w)], probes=[(c[0] + 2, c[1], c[2], "ez")],
              dft_planes=planes, pec_mask=None, dft_time_offset=1)

    def fields(p):
        return [x.cpu().numpy() for x in p.store_fields()]

    a = prepare_device_run(g, mats, n, **kw)
    try:
        a.plan.advance(0, n, a.src_table, a.probe_out, a.dft_accs, a.dft_phases)
        ref_f, ref_acc, ref_ts = fields(a.plan), a.dft_accs[0].cpu().numpy(), a.probe_out.cpu().numpy()
    finally:
        a.plan.close()
    b = prepare_device_run(g, mats, n, **kw)
    try:
        b.plan.advance(0, n1, b.src_table, b.probe_out, b.dft_accs, b.dft_phases)
        ck.save_plan_state(tmp_path / "run.npz", b.plan, n1, grid=g)
        acc, ts = b.dft_accs[0].clone(), b.probe_out.clone()
    finally:
        b.plan.close()
    r = prepare_device_run(g, mats, n, **kw)
    try:
        step, meta = ck.load_plan_state(tmp_path / "run.npz", r.plan)
        assert step == n1 and meta["cpml_layers"] == 5
        r.dft_accs[0].copy_(acc)
        r.probe_out.copy_(ts)
        r.plan.advance(step, n - step, r.src_table, r.probe_out, r.dft_accs, r.dft_phases)
        for x, y in zip(fields(r.plan), ref_f):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(r.dft_accs[0].cpu().numpy(), ref_acc)
        np.testing.assert_array_equal(r.probe_out.cpu().numpy(), ref_ts)
    finally:
        r.plan.close()
    # a blob from another grid is rejected by the C ABI
    g2 = rfx_b200.Grid(freq_max=20e9, domain=(0.012, 0.014, 0.012), dx=1e-3, cpml_layers=5)
    m2 = rfx_b200.MaterialArrays(*(np.ones(g2.shape, np.float32),) * 3)
    o = prepare_device_run(g2, m2, 4, cpml_axes="xyz", pec_axes="", sources=[], probes=[], dft_planes=[],
                           pec_mask=None, dft_time_offset=1)
    try:
        blob = np.load(tmp_path / "run.npz")["blob"]
        with pytest.raises(RuntimeError, match="code -2"):
            o.plan.restore_state(blob)
        with pytest.raises(RuntimeError, match="code -1"):
            o.plan.restore_state(np.zeros(256, np.uint8))
    finally:
        o.plan.close()
    torch.cuda.synchronize()
