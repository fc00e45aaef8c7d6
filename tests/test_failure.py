"""Failure detection without faulting the GPU: bounded device waits, host-side input
checks, iteration caps."""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200._lib import ArielError, lib
from ariel_b200.flipsim import Batch

from helpers import dambreak, params


@pytest.mark.gpu
def test_grid_barrier_times_out_and_reports():
    # a barrier that nothing releases must give up after its budget and report, leaving the
    # context usable
    assert lib().ariel_selftest_barrier_timeout(50.0) == A.ARIEL_ERR_DEVICE_TIMEOUT
    b = Batch([dambreak(8)], params())
    b.init()
    b.step(1)
    b.close()


@pytest.mark.gpu
def test_nan_input_rejected():
    b = Batch([dambreak(8)], params())
    pos = np.array([[0.5, np.nan, 0.5]], np.float32)
    with pytest.raises(ArielError) as e:
        b.set_particles(pos, np.zeros((1, 3), np.float32), np.ones(1, np.float32), np.ones(1, np.int32))
    assert e.value.code == A.ARIEL_ERR_NAN
    b.close()


@pytest.mark.gpu
def test_not_converged_is_reported():
    prm = params(precision=A.PREC_FP64, stop=A.STOP_REL, tol=1e-12, max_iters=2, fail_on_not_converged=1)
    b = Batch([dambreak(16)], prm)
    b.init()
    with pytest.raises(ArielError) as e:
        b.step(1)
    assert e.value.code == A.ARIEL_ERR_NOT_CONVERGED
    st = b.stats()
    assert st.pcg_converged == 0 and st.pcg_iterations == 2
    b.close()


@pytest.mark.gpu
def test_invalid_arguments():
    with pytest.raises(ArielError) as e:
        Batch([dambreak(1)], params())
    assert e.value.code == A.ARIEL_ERR_INVALID_ARG
    b = Batch([dambreak(8)], params())
    with pytest.raises(ArielError) as e:
        b.step(1)  # before Init
    assert e.value.code == A.ARIEL_ERR_STATE
    b.close()
