"""Device-side failure paths of the persistent step kernels, exercised
without faulting the GPU: a pipeline wait made to run out (one CTA does not
issue one plane's TMA boxes, every wait is limited to a few hundred polls)
and a poisoned work-queue entry (an empty x range).  In both cases the
kernels finish, the status word reports the failure to the host
(RFXB_E_TIMEOUT = -6, RFXB_E_WORK = -7), and a fresh sweep on the same
device afterwards runs clean and reproduces the undisturbed result bit for
bit."""

import numpy as np
import pytest


def _sweep():
    import torch

    from rfx_b200.batch import Sweep
    from rfx_b200.workloads import batched_sweep
    insts = batched_sweep(seed=3, n_inst=3, n_steps=60, n_lo=40, n_hi=72)
    sw = Sweep(insts, 60, device=torch.device("cuda", 0), batched=True)
    _, lim = sw.batch.launch_config()
    assert lim["fwd_persist"] >= 1 and lim["adj_persist"] == 1
    sw.batch.set_launch_config(fwd_persist=2, adj_persist=1)
    return sw


def _result(sw):
    Js, grads = sw.run()
    sw.check_device()
    return np.array([float(j) for j in Js]), [g.detach().cpu().numpy().copy() for g in grads]


def _lib():
    from rfx_b200 import _lib
    return _lib.load()


def _clean_rerun_matches(J0, g0):
    sw = _sweep()
    try:
        J, g = _result(sw)
        assert np.array_equal(J, J0)
        for a, b in zip(g, g0):
            assert np.array_equal(a, b)
    finally:
        sw.close()


@pytest.mark.gpu
def test_forward_wait_that_runs_out_is_reported(cuda):
    sw = _sweep()
    try:
        J0, g0 = _result(sw)
        assert _lib().rfxb_batch_debug_fault(sw.batch._h, 0, 256) == 0
        sw.forward()
        with pytest.raises(RuntimeError, match=r"code -6\).*ran out"):
            sw.check_device()
    finally:
        sw.close()
    _clean_rerun_matches(J0, g0)


@pytest.mark.gpu
def test_reverse_wait_that_runs_out_is_reported(cuda):
    sw = _sweep()
    try:
        J0, g0 = _result(sw)
        sw.forward()
        _, gs = sw.objectives()
        sw.check_device()
        assert _lib().rfxb_batch_debug_fault(sw.batch._h, 0, 256) == 0
        sw.backward(gs)
        with pytest.raises(RuntimeError, match=r"code -6\).*ran out"):
            sw.check_device()
    finally:
        sw.close()
    _clean_rerun_matches(J0, g0)


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1, 4])
def test_poisoned_work_item_is_rejected(cuda, which):
    """Lists 0 / 1: forward CPML / CPML-free tiles; 4: reverse CPML-free."""
    sw = _sweep()
    try:
        J0, g0 = _result(sw)
        assert _lib().rfxb_batch_debug_poison(sw.batch._h, which, 0) == 0
        if which < 2:
            sw.forward()
        else:
            sw.forward()
            _, gs = sw.objectives()
            sw.backward(gs)
        with pytest.raises(RuntimeError, match=r"code -7\).*invalid work item"):
            sw.check_device()
    finally:
        sw.close()
    _clean_rerun_matches(J0, g0)
