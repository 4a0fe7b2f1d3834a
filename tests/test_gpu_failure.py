"""Failure detection without a GPU fault.  Every mbarrier wait in the tensor-core kernels is bounded:
when it runs out it sets bit 1 of the launch's status word and returns, and the host turns a non-zero
status into TRPDRV_ERR_DEVICE.  trpdrv_selftest_bounded_wait runs that same wait on a barrier that
nothing completes, with a short limit: the wait must give up after the limit, report it, and leave the
device usable.  Argument checks come before any device work and run on the CPU."""
import numpy as np
import pytest


@pytest.mark.parametrize("limit", [0.0, -1.0, 10.5, float("nan")])
def test_selftest_rejects_limits_outside_the_range(T, limit):
    with pytest.raises(T.TrpdrvError) as e:
        T.selftest_bounded_wait(limit)
    assert e.value.status == 1


@pytest.mark.gpu
@pytest.mark.parametrize("limit", [0.02, 0.25])
def test_bounded_wait_gives_up_and_reports(T, limit):
    status, elapsed = T.selftest_bounded_wait(limit)
    assert status == 2, f"status word {status}: the wait on a barrier nothing completes must give up"
    # the clock is read every 256 polls: the wait ends shortly after the limit, never before it
    assert limit <= elapsed < limit + 0.5, elapsed


@pytest.mark.gpu
def test_device_stays_usable_after_a_wait_runs_out(T):
    s = T.synth_system(4, 40, seed=5)
    T.clear_error()
    before = T.cbody(s, 2, 3, 1, 1)
    status, _ = T.selftest_bounded_wait(0.02)
    assert status == 2
    after = T.cbody(s, 2, 3, 1, 1)
    assert np.array_equal(np.array(before), np.array(after))
    assert T.last_error()[0] == 0  # the wait's status is returned to the caller, not recorded as a failure
