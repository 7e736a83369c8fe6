"""The reference's own acceptance gates for the graded-lane decay stop
(rfx tests/test_nonuniform_until_decay.py), restated on the oracle (CPU) and
on the CUDA path (GPU), on the reference's scene (`_build_nu_case`, :70-80:
a 16 x 16 x 24-cell graded-dz box, dz 12 x 0.4 mm then 12 x 0.6 mm, dx 0.5 mm,
CPML 4, a GaussianPulse(10 GHz, bandwidth 0.5) Ez current source at
(4, 4, 4) mm and an Ez probe at (4, 4, 8) mm).

* Gate B (:83-172): the interior-energy stop fires strictly between
  min_steps and max_steps, the last `decay_energy_consecutive` checks are
  below decay_by times the peak held at that check, the stop step is the last
  check's step, and the probe spectrum at the stop matches a 3x longer fixed
  run (peak bin within one bin, peak amplitude within 2 %, every bin carrying
  at least 5 % of the non-DC maximum within 1e-2);
* Gate C (:175-230): decay_by = 0 runs exactly N steps with a check after
  every chunk and matches the fixed run within the reference's envelope
  (5e-6 of the probe scale, 2e-6 of the E scale, 1e-4 of the H scale);
* chunking (:233-265): one chunk of N steps and four chunks of N/4 give the
  same probe series and fields bit for bit.

These gates are independent of this project's restatement of the stop rule:
they are the criteria the reference itself holds its decay loop to."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from tests.scenarios import rel_l2

DZ = np.array([0.4e-3] * 12 + [0.6e-3] * 12)
GATE_B = dict(decay_by=1e-4, check_interval=50, min_steps=100, max_steps=3000, decay_energy_consecutive=2)
N_FORCED = 200
TS_ENVELOPE, E_ENVELOPE, H_ENVELOPE = 5e-6, 2e-6, 1e-4
TOL = 1e-4   # CUDA path against the oracle (probe traces)
COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")


def _indices():
    """Source and probe cells from the graded position_to_index (host logic)."""
    import rfx_b200
    from rfx_b200.nonuniform import position_to_index
    pg = rfx_b200.make_nonuniform_grid((0.008, 0.008), DZ, 0.5e-3, cpml_layers=4)
    return pg, position_to_index(pg, (0.004, 0.004, 0.004)), position_to_index(pg, (0.004, 0.004, 0.008))


def _oracle_case(n_table):
    pg, src, prb = _indices()
    g = oracle.make_nonuniform_grid((0.008, 0.008), DZ, 0.5e-3, cpml_layers=4)
    assert g.shape == (pg.nx, pg.ny, pg.nz)
    mats = (np.ones(g.shape, np.float32), np.zeros(g.shape, np.float32), np.ones(g.shape, np.float32))
    w = oracle.current_source_waveform(g, src, "ez", mats, n_table, f0=10e9, bandwidth=0.5)
    return g, mats, [(*src, "ez", w)], [(*prb, "ez")]


def _product_case(n_table):
    import rfx_b200
    from rfx_b200.sources import GaussianPulse, make_current_source
    pg, src, prb = _indices()
    shape = (pg.nx, pg.ny, pg.nz)
    mats = rfx_b200.MaterialArrays(np.ones(shape, np.float32), np.zeros(shape, np.float32),
                                   np.ones(shape, np.float32))
    s = make_current_source(pg, src, "ez", GaussianPulse(f0=10e9, bandwidth=0.5), n_table, mats)
    return pg, mats, [s], [(*prb, "ez")]


def _spectrum_gate(ts_stop, ts_ref):
    """Gate B's spectral witness: returns (peak-bin shift, peak amplitude
    ratio, in-band per-bin error)."""
    n_ref = ts_ref.shape[0]
    padded = np.zeros(n_ref)
    padded[:ts_stop.shape[0]] = ts_stop
    spec_ref = np.abs(np.fft.rfft(ts_ref))
    spec_dec = np.abs(np.fft.rfft(padded))
    k_ref, k_dec = int(np.argmax(spec_ref)), int(np.argmax(spec_dec))
    band = spec_ref >= 0.05 * float(np.max(spec_ref[1:]))
    return abs(k_dec - k_ref), spec_dec[k_ref] / spec_ref[k_ref], float(np.max(np.abs(spec_dec[band] / spec_ref[band] - 1.0)))


def _check_gate_b(steps, checks):
    kw = GATE_B
    assert kw["min_steps"] <= steps < kw["max_steps"], f"stop after {steps} steps"
    assert len(checks) >= kw["decay_energy_consecutive"]
    assert all(u < kw["decay_by"] * p for _, u, p in checks[-kw["decay_energy_consecutive"]:])
    assert checks[-1][0] == steps


def _check_envelope(ts_fixed, ts_decay, f_fixed, f_decay):
    ts_scale = float(np.max(np.abs(ts_fixed)))
    assert float(np.max(np.abs(ts_fixed - ts_decay))) <= TS_ENVELOPE * ts_scale
    e_scale = max(float(np.max(np.abs(f_fixed[c]))) for c in range(3))
    h_scale = max(float(np.max(np.abs(f_fixed[c]))) for c in range(3, 6))
    for c in range(6):
        bound = (E_ENVELOPE * e_scale) if c < 3 else (H_ENVELOPE * h_scale)
        assert float(np.max(np.abs(np.asarray(f_fixed[c]) - np.asarray(f_decay[c])))) <= bound


# --------------------------------------------------------------------------- oracle (CPU)

def _oracle_decay(**kw):
    g, mats, srcs, probes = _oracle_case(kw["max_steps"])
    return oracle.run_until_decay_nonuniform(g, mats, sources=srcs, probes=probes, dx_arr=g.dx_arr,
                                             dy_arr=g.dy_arr, **kw)


@pytest.mark.slow
def test_oracle_gate_b_stop_fires_with_trace_and_spectral_witness():
    res, steps, checks = _oracle_decay(**GATE_B)
    _check_gate_b(steps, checks)
    g, mats, srcs, probes = _oracle_case(3 * steps)
    ref = oracle.run_nonuniform(g, mats, 3 * steps, sources=srcs, probes=probes)
    shift, ratio, inband = _spectrum_gate(res.time_series[:, 0], ref.time_series[:, 0])
    print(f"oracle: stop after {steps} steps; peak shift {shift}, ratio {ratio:.5f}, in-band error {inband:.3e}")
    assert shift <= 1 and abs(ratio - 1.0) <= 0.02 and inband <= 1e-2


def test_oracle_gate_c_forced_n_and_chunking():
    kw = dict(decay_by=0.0, check_interval=50, min_steps=1, max_steps=N_FORCED, decay_energy_consecutive=2)
    res, steps, checks = _oracle_decay(**kw)
    assert steps == N_FORCED and res.time_series.shape[0] == N_FORCED
    assert [s for s, _, _ in checks] == [50, 100, 150, 200]
    assert all(u >= 0.0 for _, u, _ in checks)
    g, mats, srcs, probes = _oracle_case(N_FORCED)
    fixed = oracle.run_nonuniform(g, mats, N_FORCED, sources=srcs, probes=probes)
    _check_envelope(fixed.time_series, res.time_series, [fixed.state[c] for c in COMPS],
                    [res.state[c] for c in COMPS])
    one, _, _ = _oracle_decay(**dict(kw, check_interval=N_FORCED))
    assert np.array_equal(one.time_series, res.time_series)
    for c in COMPS:
        assert np.array_equal(np.asarray(one.state[c]), np.asarray(res.state[c]))


# --------------------------------------------------------------------------- CUDA path (GPU)

def _product_decay(**kw):
    import rfx_b200
    pg, mats, srcs, probes = _product_case(kw["max_steps"])
    return rfx_b200.run_nonuniform_until_decay(pg, mats, sources=srcs, probes=probes, **kw)


def _fields(state):
    return [np.asarray(getattr(state, c)) for c in COMPS]


@pytest.mark.gpu
def test_gate_b_stop_fires_with_trace_and_spectral_witness(cuda):
    import rfx_b200
    out = _product_decay(**GATE_B)
    ts = np.asarray(out["time_series"])
    steps = ts.shape[0]
    _check_gate_b(steps, out["decay_checks"])
    pg, mats, srcs, probes = _product_case(3 * steps)
    ref = rfx_b200.run_nonuniform(pg, mats, 3 * steps, sources=srcs, probes=probes)
    shift, ratio, inband = _spectrum_gate(ts[:, 0], np.asarray(ref["time_series"])[:, 0])
    res, o_steps, _ = _oracle_decay(**GATE_B)
    print(f"CUDA: stop after {steps} steps (oracle {o_steps}); peak shift {shift}, ratio {ratio:.5f}, "
          f"in-band error {inband:.3e}; probe relL2 against the oracle "
          f"{rel_l2(ts[:, 0], res.time_series[:, 0]):.2e}")
    assert shift <= 1 and abs(ratio - 1.0) <= 0.02 and inband <= 1e-2
    assert steps == o_steps
    assert rel_l2(ts[:, 0], res.time_series[:, 0]) < TOL


@pytest.mark.gpu
def test_gate_c_forced_n_and_chunking(cuda):
    import rfx_b200
    kw = dict(decay_by=0.0, check_interval=50, min_steps=1, max_steps=N_FORCED, decay_energy_consecutive=2)
    out = _product_decay(**kw)
    ts = np.asarray(out["time_series"])
    assert ts.shape[0] == N_FORCED and out["state"].step == N_FORCED
    assert [s for s, _, _ in out["decay_checks"]] == [50, 100, 150, 200]
    assert all(u >= 0.0 for _, u, _ in out["decay_checks"])
    pg, mats, srcs, probes = _product_case(N_FORCED)
    fixed = rfx_b200.run_nonuniform(pg, mats, N_FORCED, sources=srcs, probes=probes)
    _check_envelope(np.asarray(fixed["time_series"]), ts, _fields(fixed["state"]), _fields(out["state"]))
    one = _product_decay(**dict(kw, check_interval=N_FORCED))
    assert np.array_equal(np.asarray(one["time_series"]), ts)
    for a, b in zip(_fields(one["state"]), _fields(out["state"])):
        assert np.array_equal(a, b)
