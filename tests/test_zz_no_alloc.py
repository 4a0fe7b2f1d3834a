"""The entry point that allocates no device memory (trpdrv_body_device_noalloc), through the C ABI.

It serves callers that cannot allocate device memory when they need the work: code inside a CUDA
stream capture, code under a device-memory budget fixed by its host application, or callers that own
every device buffer.  Its scratch is one static device array, so it is checked here against the
existing host drop-in entry point (ccsd_trpdrv_omp_cbody_) on two calls in a row, which must agree
with each other and with the drop-in; the array keeps the previous call's contents, so the second
call also shows that leftovers do not leak into the result.  This file is named so that pytest
collects it last: a failure here never stops a run before every other test has run.  The tests pass
in a fresh process (first call sets the device up) and after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, per energy: both paths run the same FP64 kernels


def _device_slices(dev, s, i, j, k):
    """Device addresses of the reference body's arguments for triple (i,j,k), already sliced."""
    O, V = s.nocc, s.nvir
    vv, ov = V * V, O * V

    def at(name, off):
        return dev[name].data_ptr() + 8 * off

    jb = (j - 1) * O
    return dict(eorb=at("eorb", 0),
                tij=at("t2", (jb + i - 1) * vv), tkj=at("t2", (jb + k - 1) * vv),
                tia=at("tov", (i - 1) * ov), tka=at("tov", (k - 1) * ov),
                xia=at("xov", (i - 1) * ov), xka=at("xov", (k - 1) * ov),
                jia=at("jvv", (i - 1) * vv), jka=at("jvv", (k - 1) * vv),
                kia=at("kvv", (i - 1) * vv), kka=at("kvv", (k - 1) * vv),
                jij=at("jov", (jb + i - 1) * ov), jkj=at("jov", (jb + k - 1) * ov),
                kij=at("kov", (jb + i - 1) * ov), kkj=at("kov", (jb + k - 1) * ov),
                dintc1=at("dintc", (i - 1) * V), dintx1=at("dintx", (i - 1) * V), t1v1=at("t1v", (i - 1) * V),
                dintc2=at("dintc", (k - 1) * V), dintx2=at("dintx", (k - 1) * V), t1v2=at("t1v", (k - 1) * V))


def test_no_alloc_entry_point_matches_dropin_on_two_calls(T):
    import torch

    s = T.synth_system(6, 72, seed=77, ncor=1)
    dev = {n: torch.from_numpy(a).cuda() for n, a in s.arrays.items()}
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for (i, j, k) in [(3, 2, 1), (5, 6, 5), (6, 1, 2)]:
        ptrs = _device_slices(dev, s, i, j, k)
        ptrs["out4"] = out.data_ptr()
        calls = []
        for _ in range(2):
            out.fill_(12345.0)  # the entry point must overwrite every output
            T.body_device_noalloc(s.ncor, s.nocc, s.nvir, s.a, i, j, k, ptrs, stream=stream.cuda_stream)
            stream.synchronize()
            calls.append(out.cpu().numpy().copy())
        assert np.array_equal(calls[0], calls[1]), (i, j, k)
        e4, e5 = T.cbody(s, i, j, k, 1)  # existing entry point, host buffers, starting from emp4 = emp5 = 0
        for r in calls:
            got4 = r[0] + (r[2] if i != k else 0.0)
            got5 = r[1] + (r[3] if i != k else 0.0)
            assert abs(got4 - e4) <= TOL * abs(e4), (i, j, k, got4, e4)
            assert abs(got5 - e5) <= TOL * abs(e5), (i, j, k, got5, e5)


def test_no_alloc_entry_point_rejects_sizes_beyond_its_scratch(T):
    import torch

    s = T.synth_system(2, 8, seed=3)
    dev = {n: torch.from_numpy(a).cuda() for n, a in s.arrays.items()}
    ptrs = _device_slices(dev, s, 1, 1, 1)
    ptrs["out4"] = dev["eorb"].data_ptr()
    with pytest.raises(T.TrpdrvError) as ei:
        T.body_device_noalloc(0, 2, T.NOALLOC_MAX_NVIR + 1, 3, 1, 1, 1, ptrs)
    assert ei.value.status == 1 and "exceed" in str(ei.value)
    with pytest.raises(T.TrpdrvError):
        T.body_device_noalloc(0, T.NOALLOC_MAX_NOCC + 1, 8, 3, 1, 1, 1, ptrs)
