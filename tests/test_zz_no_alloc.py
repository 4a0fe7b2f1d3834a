"""The entry point that allocates no device memory (trpdrv_body_device_noalloc), through the C ABI.

It serves callers that cannot call cudaMalloc when they need the work: an application that reserves
device memory up front in its own pool and gives libraries a fixed budget, a plug-in inside a
framework that owns every device buffer, or a loop that cannot pay for an allocation per call.  Its
scratch is one static device array, so it is checked here against the existing host drop-in entry
point (ccsd_trpdrv_omp_cbody_, on its plain per-triple path: the same kernels) on two calls in a row,
which must agree with each other and with the drop-in; the array keeps the previous call's contents, so the second call also shows that leftovers
do not leak into the result.  The cases cover the 16-byte vector copies and the scalar ones (odd nvir,
pointers off a 16-byte boundary), the size limit (nocc = 64, nvir = 256), and every triple of a golden
system made by the reference itself.  This file is named so that pytest collects it last: a failure
here never stops a run before every other test has run.  The tests pass in a fresh process (the
first call sets the device up) and after the other tests.
"""
import os

import numpy as np
import pytest

from conftest import RECORD_RTOL, TOTAL_RTOL, assert_records_close, assert_total_close, load_golden, system_from_golden

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, per energy: both paths run the same FP64 kernels


def _to_device(s, offset=0):
    """Device copies of the system's arrays; offset > 0 starts every array that many doubles into its
    buffer (8-byte but not 16-byte aligned for odd offsets)."""
    import torch
    dev = {}
    for n, a in s.arrays.items():
        buf = torch.zeros(a.size + offset, dtype=torch.float64, device="cuda")
        buf[offset:].copy_(torch.from_numpy(np.ascontiguousarray(a)))
        dev[n] = (buf, offset)
    return dev


def _device_slices(dev, s, i, j, k):
    """Device addresses of the reference body's arguments for triple (i,j,k), already sliced."""
    O, V = s.nocc, s.nvir
    vv, ov = V * V, O * V

    def at(name, off):
        buf, base = dev[name]
        return buf.data_ptr() + 8 * (base + off)

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


def _noalloc_twice(T, s, dev, i, j, k):
    """Two calls in a row for one triple; both records (emp4i, emp5i, emp4k, emp5k)."""
    import torch
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    ptrs = _device_slices(dev, s, i, j, k)
    ptrs["out4"] = out.data_ptr()
    calls = []
    for _ in range(2):
        out.fill_(12345.0)  # the entry point must overwrite every output
        T.body_device_noalloc(s.ncor, s.nocc, s.nvir, s.a, i, j, k, ptrs, stream=stream.cuda_stream)
        stream.synchronize()
        calls.append(out.cpu().numpy().copy())
    return calls


def _dropin_plain(T, s, i, j, k):
    """The existing entry point on its plain per-triple path (the kernels this entry point runs too),
    from host buffers, starting from emp4 = emp5 = 0."""
    old = os.environ.get("TRPDRV_DROPIN_PATH")
    os.environ["TRPDRV_DROPIN_PATH"] = "plain"
    try:
        return T.cbody(s, i, j, k, 1)
    finally:
        if old is None:
            del os.environ["TRPDRV_DROPIN_PATH"]
        else:
            os.environ["TRPDRV_DROPIN_PATH"] = old


def _check_against_dropin(T, s, dev, triples):
    for (i, j, k) in triples:
        calls = _noalloc_twice(T, s, dev, i, j, k)
        assert np.array_equal(calls[0], calls[1]), (i, j, k)
        e4, e5 = _dropin_plain(T, s, i, j, k)
        for r in calls:
            got4 = r[0] + (r[2] if i != k else 0.0)
            got5 = r[1] + (r[3] if i != k else 0.0)
            assert abs(got4 - e4) <= TOL * abs(e4), (i, j, k, got4, e4)
            assert abs(got5 - e5) <= TOL * abs(e5), (i, j, k, got5, e5)


def test_no_alloc_entry_point_matches_dropin_on_two_calls(T):
    s = T.synth_system(6, 72, seed=77, ncor=1)
    _check_against_dropin(T, s, _to_device(s), [(3, 2, 1), (5, 6, 5), (6, 1, 2)])


@pytest.mark.parametrize("shape,offset", [((5, 37), 0), ((6, 72), 1)])
def test_no_alloc_scalar_copy_path(T, shape, offset):
    """Odd nvir, or every pointer 8 bytes off a 16-byte boundary: the GEMM takes its scalar copies."""
    nocc, nvir = shape
    s = T.synth_system(nocc, nvir, seed=78)
    _check_against_dropin(T, s, _to_device(s, offset), [(2, 1, 1), (nocc, nocc, 3), (4, 2, 4)])


def test_no_alloc_at_its_size_limit(T):
    """nocc = TRPDRV_NOALLOC_MAX_NOCC, nvir = TRPDRV_NOALLOC_MAX_NVIR, where the static scratch is
    full.  Only the j = 1 blocks of T2, JOV and KOV are built (a triple (i, 1, k) reads no other)."""
    O, V = T.NOALLOC_MAX_NOCC, T.NOALLOC_MAX_NVIR
    rng = np.random.default_rng(2024)
    eorb = np.concatenate([np.sort(rng.uniform(-2.0, -0.5, O)), np.sort(rng.uniform(0.2, 3.0, V))])
    arrays = {"eorb": eorb,
              "t2": rng.uniform(-0.05, 0.05, O * V * V), "jvv": rng.uniform(-0.1, 0.1, O * V * V),
              "kvv": rng.uniform(-0.1, 0.1, O * V * V), "tov": rng.uniform(-0.02, 0.02, O * V * O),
              "xov": rng.uniform(-0.02, 0.02, O * V * O), "jov": rng.uniform(-0.1, 0.1, O * O * V),
              "kov": rng.uniform(-0.1, 0.1, O * O * V), "dintc": rng.uniform(-0.1, 0.1, O * V),
              "dintx": rng.uniform(-0.1, 0.1, O * V), "t1v": rng.uniform(-0.02, 0.02, O * V)}
    s = T.System(0, O, V, O + 1, arrays)
    _check_against_dropin(T, s, _to_device(s), [(O, 1, O), (O, 1, 1)])


def test_no_alloc_matches_the_reference_golden_records(T):
    """Every triple of a system the reference itself evaluated (ncor = 2, odd nvir = 33)."""
    g = load_golden("g_c2_o5_v33")
    s = system_from_golden(g)
    dev = _to_device(s)
    recs = []
    for (i, j, k) in g["triples"]:
        recs.append(_noalloc_twice(T, s, dev, i, j, k)[1])
    recs = np.array(recs)
    assert_records_close(recs, g["records"], rtol=RECORD_RTOL)
    tot4 = sum(r[0] + (r[2] if t[0] != t[2] else 0.0) for r, t in zip(recs, g["triples"]))
    tot5 = sum(r[1] + (r[3] if t[0] != t[2] else 0.0) for r, t in zip(recs, g["triples"]))
    assert_total_close(tot4, g["emp4"], rtol=TOTAL_RTOL, what="emp4")
    assert_total_close(tot5, g["emp5"], rtol=TOTAL_RTOL, what="emp5")


def test_no_alloc_entry_point_rejects_sizes_beyond_its_scratch(T):
    s = T.synth_system(2, 8, seed=3)
    dev = _to_device(s)
    ptrs = _device_slices(dev, s, 1, 1, 1)
    ptrs["out4"] = dev["eorb"][0].data_ptr()
    with pytest.raises(T.TrpdrvError) as ei:
        T.body_device_noalloc(0, 2, T.NOALLOC_MAX_NVIR + 1, 3, 1, 1, 1, ptrs)
    assert ei.value.status == 1 and "exceed" in str(ei.value)
    with pytest.raises(T.TrpdrvError):
        T.body_device_noalloc(0, T.NOALLOC_MAX_NOCC + 1, 8, 3, 1, 1, 1, ptrs)
