"""GPU tests of the reference-facing body entry point (ccsd_trpdrv_omp_cbody_) on its fused path.

With even nocc and nvir (and TRPDRV_WRITE_F unset) each call stages its triple's slices into a
one-triple layout and runs the fused TMA kernel; otherwise, or with TRPDRV_DROPIN_PATH=plain, the
plain per-triple kernels.  Both are checked here against the reference's golden records, against
each other, with registered and partly registered inputs, with k-chunked slices (klo > 1), with
shapes and virtual indices that change from call to call, and at the full nocc=40, nvir=300 size.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, system_from_golden

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _want(rec, i, k):
    return rec[0] + (rec[2] if i != k else 0.0), rec[1] + (rec[3] if i != k else 0.0)


def _close(got, want, tol=TOL, scale=None):
    s = scale if scale is not None else max(abs(want), 1e-300)
    return abs(got - want) <= tol * s


@pytest.mark.parametrize("name", ["g_o4_v24", "g_o10_v60", "g_o6_v40_nk2", "g_o3_v70"])
def test_dropin_matches_reference_golden_records(T, name):
    g = load_golden(name)
    s = system_from_golden(g)
    ijkl = T.enumerate_triples(s.nocc, g["nkpass"])
    recs = np.array(g["records"])
    scale4, scale5 = np.max(np.abs(recs[:, 0])) + np.max(np.abs(recs[:, 2])), np.max(np.abs(recs[:, 1])) + \
        np.max(np.abs(recs[:, 3]))
    for t in range(len(ijkl)):
        i, j, k, klo = (int(v) for v in ijkl[t])
        e4, e5 = T.cbody(s, i, j, k, klo)
        w4, w5 = _want(recs[t], i, k)
        assert _close(e4, w4, scale=scale4) and _close(e5, w5, scale=scale5), (name, t, e4, w4, e5, w5)


def test_fused_and_plain_dropin_paths_agree(T, monkeypatch):
    s = T.synth_system(8, 64, seed=91)
    ijkl = T.enumerate_triples(8, 3)  # k-chunked: klo > 1 for most triples
    picks = ijkl[::17]
    fused = [T.cbody(s, *(int(v) for v in r), emp4=0.5, emp5=-0.25) for r in picks]
    monkeypatch.setenv("TRPDRV_DROPIN_PATH", "plain")
    plain = [T.cbody(s, *(int(v) for v in r), emp4=0.5, emp5=-0.25) for r in picks]
    for (f4, f5), (p4, p5) in zip(fused, plain):
        assert _close(f4, p4, 1e-12, abs(p4) + 1.0) and _close(f5, p5, 1e-12, abs(p5) + 1.0)


def test_registered_and_partly_registered_inputs_give_the_same_bits(T):
    s = T.synth_system(6, 48, seed=92)
    triples = [(1, 1, 1, 1), (4, 2, 3, 1), (6, 6, 6, 1), (5, 3, 2, 1)]
    want = [T.cbody(s, *t) for t in triples]
    T.register_system(s)
    try:
        assert [T.cbody(s, *t) for t in triples] == want
    finally:
        T.unregister_system(s)
    for name in ("t2", "jvv", "xov", "kov"):  # some inputs from device copies, the rest from the host
        T.register_host(s.arrays[name])
    try:
        assert [T.cbody(s, *t) for t in triples] == want
    finally:
        for name in ("t2", "jvv", "xov", "kov"):
            T.unregister_host(s.arrays[name])


def test_shapes_and_virtual_index_change_between_calls(T, O):
    """Calls alternate between two shapes (the staging layout is rebuilt) and use several `a`: every
    call matches the oracle's body."""
    fn_port = O.port_body_fn()
    systems = [T.synth_system(4, 24, seed=93), T.synth_system(6, 40, seed=94, ncor=1)]
    for rep in range(2):
        for s in systems:
            nbf = s.ncor + s.nocc + s.nvir
            for a in (s.ncor + s.nocc + 1, s.ncor + s.nocc + 5, nbf):  # virtual a: denominators away from 0
                s2 = T.System(s.ncor, s.nocc, s.nvir, a, s.arrays)
                for (i, j, k) in ((2, 1, 2), (s.nocc, s.nocc - 1, 1)):
                    got = T.cbody(s2, i, j, k, 1, 0.125, 0.0625)
                    want = T.body_call(fn_port, s2, i, j, k, 1, 0.125, 0.0625)
                    assert _close(got[0], want[0], 1e-12, abs(want[0]) + 1.0), (rep, a, i, j, k)
                    assert _close(got[1], want[1], 1e-12, abs(want[1]) + 1.0), (rep, a, i, j, k)


def test_full_size_dropin_matches_the_reference_fixture(T):
    path = os.path.join(GOLDEN, "big_c2_o40_v300.json")
    if not os.path.exists(path):
        pytest.skip("full-size fixture not generated")
    with open(path) as f:
        g = json.load(f)["systems"][0]
    s = T.synth_system(g["nocc"], g["nvir"], seed=g["seed"], a=g["a"])
    ijkl = T.enumerate_triples(g["nocc"], 1)
    recs = np.array(g["records"])
    scale4 = np.max(np.abs(recs[:, 0])) + np.max(np.abs(recs[:, 2]))
    scale5 = np.max(np.abs(recs[:, 1])) + np.max(np.abs(recs[:, 3]))
    for q in range(0, len(g["record_index"]), 97):
        t = g["record_index"][q]
        i, j, k, klo = (int(v) for v in ijkl[t])
        e4, e5 = T.cbody(s, i, j, k, klo)
        w4, w5 = _want(recs[q], i, k)
        assert _close(e4, w4, scale=scale4) and _close(e5, w5, scale=scale5), (t, e4, w4, e5, w5)


def _call_with_buffers(T, s, bufs, i, j, k, klo):
    """ccsd_trpdrv_omp_cbody_ on caller buffers (dict of BODY_ORDER name -> array) for triple (i,j,k)."""
    import ctypes as C
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    fn = T.lib.ccsd_trpdrv_omp_cbody_
    f = np.zeros((8, s.nvir * s.nvir))
    ints = [C.c_int(v) for v in (s.ncor, s.nocc, s.nvir)]
    idx = [C.c_int(v) for v in (s.a, i, j, k, klo)]
    e4, e5 = C.c_double(0.0), C.c_double(0.0)
    fn(*[f[q].ctypes.data_as(dp) for q in range(8)], s.arrays["eorb"].ctypes.data_as(dp), *[C.byref(v) for v in ints],
       C.byref(e4), C.byref(e5), *[C.byref(v) for v in idx], *[bufs[n].ctypes.data_as(dp) for n in T.BODY_ORDER])
    return e4.value, e5.value


def test_refilled_buffers_are_seen_on_every_call(T):
    """A caller that refills the same host buffers between calls (as the NWChem driver does per (i, a)
    and (k, j) block): the staging compares contents, not pointers, so every call sees its own data,
    including calls where only the k-role or only the i-role buffers change."""
    s = T.synth_system(6, 40, seed=95)
    O, V = s.nocc, s.nvir
    sizes = {n: (V * V if n in ("tij", "tkj", "jia", "jka", "kia", "kka") else
                 O * V if n in ("tia", "tka", "xia", "xka", "jij", "jkj", "kij", "kkj") else V) for n in T.BODY_ORDER}
    bufs = {n: np.zeros(sizes[n]) for n in T.BODY_ORDER}
    ijkl = T.enumerate_triples(O, 1)
    for t in list(range(0, len(ijkl), 3)) + [5, 5, 0]:  # repeats and jumps: unchanged, k-only and full refills
        i, j, k, klo = (int(v) for v in ijkl[t])
        sl = T.triple_slices(s, i, j, k, k)  # the k-chunk base at k: the buffers hold exactly one block
        for n in T.BODY_ORDER:
            np.copyto(bufs[n], sl[n][:sizes[n]])
        got = _call_with_buffers(T, s, bufs, i, j, k, k)
        want = T.cbody(s, i, j, k, klo)
        assert _close(got[0], want[0], 1e-12, abs(want[0]) + 1e-300) and \
            _close(got[1], want[1], 1e-12, abs(want[1]) + 1e-300), (t, got, want)
