"""GPU tests of registered host arrays for the drop-in entry points (trpdrv_register_host): calls whose
pointers lie inside registered arrays read the device copies and give the same bits as calls that
copy their slices; a registered array changed on the host is seen only after trpdrv_refresh_host."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRIPLES = [(1, 1, 1, 1), (3, 2, 2, 1), (4, 4, 3, 1), (5, 1, 5, 1), (2, 3, 1, 1)]


def _calls(T, s):
    out = []
    for i, j, k, klo in TRIPLES:
        out.append(T.cbody(s, i, j, k, klo))
    return np.array(out)


def test_registered_inputs_give_the_same_bits_and_refresh(T):
    s = T.synth_system(5, 48, seed=81)
    T.finalize()
    want = _calls(T, s)
    T.register_system(s)
    try:
        assert np.array_equal(_calls(T, s), want)
        # a registered array changed on the host: stale until refreshed
        s.arrays["jvv"] *= 1.5
        assert np.array_equal(_calls(T, s), want)
        T.refresh_host(s.arrays["jvv"])
        changed = _calls(T, s)
        assert not np.array_equal(changed, want)
    finally:
        T.unregister_system(s)
    assert np.array_equal(_calls(T, s), changed)  # unregistered: read from the host again, same values


def test_registration_rejects_overlaps_and_unknown_arrays(T, monkeypatch):
    s = T.synth_system(3, 16, seed=82)
    T.register_host(s.arrays["t2"])
    try:
        with pytest.raises(T.TrpdrvError) as ei:
            T.register_host(s.arrays["t2"][8:])  # inside the registered range
        assert ei.value.status == 1
        with pytest.raises(T.TrpdrvError):
            T.refresh_host(s.arrays["jvv"])
    finally:
        T.unregister_host(s.arrays["t2"])
    with pytest.raises(T.TrpdrvError):
        T.unregister_host(s.arrays["t2"])


def test_finalize_drops_registrations(T):
    s = T.synth_system(5, 16, seed=83)  # the triples of TRIPLES need nocc >= 5
    T.register_system(s)
    T.finalize()
    with pytest.raises(T.TrpdrvError):
        T.refresh_host(s.arrays["t2"])
    want = _calls(T, s)  # still correct after finalize (per-call copies)
    T.finalize()
    assert np.array_equal(_calls(T, s), want)
