"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline leg).

ctypes access to the two CPU checkers built by oracle/Makefile:
  * liboracle.so          — the project's plain-C restatement (trpdrv_oracle.c) of
                            omp/ccsd_trpdrv_omp_cbody.c:31-145 and omp/ccsd_tengy_c99.c:5-119;
  * _ref/libtrpdrv_ref.so — the reference's own omp/ccsd_trpdrv_omp_cbody.c + omp/ccsd_tengy_c99.c,
                            compiled unmodified against OpenBLAS 0.3.30 (the "reference" CPU path).
Both are driven over the same triple loop (omp/test.c:160-195) by oracle_run_system().  Nothing in
the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libtrpdrv_ref.so")
REF_TEST = os.path.join(HERE, "_ref", "test_c99")
TEST_B200 = os.path.join(HERE, "_ref", "test_c99_b200")
TEST_F77_B200 = os.path.join(HERE, "_ref", "test_f77_b200")

_dp = C.POINTER(C.c_double)

TENSOR_NAMES = ("eorb", "t2", "jvv", "kvv", "tov", "xov", "jov", "kov", "dintc", "dintx", "t1v")


class OracleSystem(C.Structure):
    _fields_ = [("ncor", C.c_int), ("nocc", C.c_int), ("nvir", C.c_int), ("a", C.c_int)] + \
               [(n, C.c_void_p) for n in TENSOR_NAMES]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            raise FileNotFoundError(f"{ORACLE_LIB} missing: run `make -C oracle oracle`")
        _lib = C.CDLL(ORACLE_LIB)
        _lib.oracle_run_system.restype = C.c_int64
        _lib.oracle_run_system.argtypes = [C.POINTER(OracleSystem), C.c_int, C.c_int64, C.c_int64, C.c_void_p,
                                           C.c_void_p, C.c_int, _dp, _dp]
        _lib.oracle_sum_records.restype = None
        _lib.oracle_sum_records.argtypes = [_dp, C.POINTER(C.c_int32), C.c_int64, _dp]
        _lib.oracle_enumerate.restype = C.c_int64
        _lib.oracle_enumerate.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int32)]
        _lib.oracle_count_triples.restype = C.c_int64
        _lib.oracle_count_triples.argtypes = [C.c_int]
        _lib.oracle_dgemm.restype = None
        _lib.oracle_dgemm.argtypes = [C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, _dp, C.c_int,
                                      _dp, C.c_int, C.c_double, _dp, C.c_int]
        _lib.oracle_tengy.restype = None
        _lib.oracle_tengy.argtypes = [_dp] * 15 + [C.c_double] + [_dp] * 4 + [C.c_int] * 3
        _lib.oracle_tensor_elems.restype = C.c_int64
        _lib.oracle_tensor_elems.argtypes = [C.c_int] * 4
        _lib.oracle_synth_fill.restype = C.c_int64
        _lib.oracle_synth_fill.argtypes = [C.c_int] * 4 + [C.c_uint64, C.c_int, _dp, C.c_int64]
        _lib.oracle_time_body.restype = None
        _lib.oracle_time_body.argtypes = [C.POINTER(OracleSystem), C.c_int, C.c_int64, C.c_int64, C.c_void_p,
                                          _dp, _dp]
    return _lib


def have_reference() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    """The compiled reference body (OpenBLAS inside); OpenBLAS is pinned to one thread per call."""
    global _ref
    if _ref is None:
        if not have_reference():
            raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference exists")
        _ref = C.CDLL(REF_LIB)
        for so in glob.glob(os.path.join(_scipy_libs(), "libscipy_openblas-*.so")):
            ob = C.CDLL(so)
            ob.scipy_openblas_set_num_threads.argtypes = [C.c_int]
            ob.scipy_openblas_set_num_threads(1)
    return _ref


def _scipy_libs():
    import scipy
    return os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))


def _struct(s) -> OracleSystem:
    o = OracleSystem()
    o.ncor, o.nocc, o.nvir, o.a = s.ncor, s.nocc, s.nvir, s.a
    for n in TENSOR_NAMES:
        arr = s.arrays[n]
        assert arr.dtype == np.float64 and arr.flags.c_contiguous
        setattr(o, n, C.c_void_p(arr.ctypes.data))
    return o


class SynthSystem:
    """One seeded system in the slice layout of trpdrv_oracle.h (arrays: name -> float64 ndarray)."""

    def __init__(self, ncor, nocc, nvir, a):
        self.ncor, self.nocc, self.nvir, self.a = ncor, nocc, nvir, a
        self.arrays = {}

    def nbytes(self) -> int:
        return sum(int(v.nbytes) for v in self.arrays.values())


A_DEPENDENT = ("jvv", "kvv", "dintc", "dintx", "t1v")


def synth_system(nocc: int, nvir: int, seed: int = 1, ncor: int = 0, dist: int = 0, a: int | None = None,
                 a_block: int = 0) -> SynthSystem:
    """The seeded synthetic system of the product's generator, restated (oracle_synth_fill): `a`
    defaults to the first virtual orbital ncor+nocc+1; a_block = m takes virtual index a + m of the
    sweep, whose a-dependent tensors (jvv, kvv, dintc, dintx, t1v) come from seed + 7919 m."""
    if a is None:
        a = ncor + nocc + 1
    s = SynthSystem(ncor, nocc, nvir, a + a_block)
    L = lib()
    for t, name in enumerate(TENSOR_NAMES):
        n = int(L.oracle_tensor_elems(t, ncor, nocc, nvir))
        buf = np.empty(n, dtype=np.float64)
        sd = seed + 7919 * a_block if name in A_DEPENDENT else seed
        if L.oracle_synth_fill(t, ncor, nocc, nvir, sd, dist, buf.ctypes.data_as(_dp), n) != n:
            raise ValueError(f"oracle_synth_fill({name}) refused its arguments")
        s.arrays[name] = buf
    return s


def time_body(s, which: str = "reference", nkpass: int = 1, t_begin: int = 0, t_end: int | None = None,
              emp4: float = 0.0, emp5: float = 0.0):
    """Serial body calls over triples [t_begin, t_end) of the driver order, as omp/test.c:160-195 makes
    them (the body accumulates emp4/emp5 itself; nothing else runs).  Returns (emp4, emp5)."""
    L = lib()
    if t_end is None:
        t_end = count_triples(s.nocc)
    fn = C.cast(ref().ccsd_trpdrv_omp_cbody_ if which == "reference" else L.oracle_cbody, C.c_void_p)
    e4, e5 = C.c_double(emp4), C.c_double(emp5)
    st = _struct(s)
    L.oracle_time_body(C.byref(st), nkpass, t_begin, t_end, fn, C.byref(e4), C.byref(e5))
    return e4.value, e5.value


def count_triples(nocc: int) -> int:
    return int(lib().oracle_count_triples(nocc))


def enumerate_triples(nocc: int, nkpass: int = 1) -> np.ndarray:
    n = count_triples(nocc)
    out = np.zeros((n, 4), dtype=np.int32)
    lib().oracle_enumerate(nocc, nkpass, out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out


def run_system(s, which: str = "port", nkpass: int = 1, t_begin: int = 0, t_end: int | None = None,
               nthreads: int = 0):
    """Runs triples [t_begin, t_end) of the driver order through the restatement ("port") or the
    compiled reference ("reference").  Returns (records (n,4) = emp4i emp5i emp4k emp5k,
    totals (emp4, emp5) long-double compensated, mismatch count)."""
    L = lib()
    n_all = count_triples(s.nocc)
    if t_end is None or t_end > n_all:
        t_end = n_all
    n = max(0, t_end - t_begin)
    rec = np.zeros((max(n, 1), 4))
    tot = np.zeros(2)
    body = tengy = None
    if which == "reference":
        R = ref()
        body = C.cast(R.ccsd_trpdrv_omp_cbody_, C.c_void_p)
        tengy = C.cast(R.ccsd_tengy_omp, C.c_void_p)
    elif which != "port":
        raise ValueError(which)
    st = _struct(s)
    mism = L.oracle_run_system(C.byref(st), nkpass, t_begin, t_end, body, tengy, nthreads,
                               rec.ctypes.data_as(_dp), tot.ctypes.data_as(_dp))
    return rec[:n], tot, int(mism)


def sum_records(rec: np.ndarray, ijkl: np.ndarray):
    tot = np.zeros(2)
    rec = np.ascontiguousarray(rec, dtype=np.float64)
    ijkl = np.ascontiguousarray(ijkl, dtype=np.int32)
    lib().oracle_sum_records(rec.ctypes.data_as(_dp), ijkl.ctypes.data_as(C.POINTER(C.c_int32)), len(rec),
                             tot.ctypes.data_as(_dp))
    return tot


def dgemm(ta: str, tb: str, alpha, A, B, beta, Cm):
    """Column-major dgemm on Fortran-ordered numpy arrays (restatement)."""
    m, n = Cm.shape
    k = A.shape[1] if ta == "N" else A.shape[0]
    lib().oracle_dgemm(ta.encode(), tb.encode(), m, n, k, alpha, A.ctypes.data_as(_dp), A.shape[0],
                       B.ctypes.data_as(_dp), B.shape[0], beta, Cm.ctypes.data_as(_dp), Cm.shape[0])


def tengy(f8, vecs, eorb, eaijk, ncor, nocc, nvir, which="port"):
    """f8 rows in argument order f1n f1t f2n f2t f3n f3t f4n f4t; vecs dintc1 dintx1 t1v1 dintc2 dintx2 t1v2."""
    out = [C.c_double() for _ in range(4)]
    fp = [np.ascontiguousarray(f8[q]).ctypes.data_as(_dp) for q in range(8)]
    vp = [np.ascontiguousarray(v).ctypes.data_as(_dp) for v in vecs]
    if which == "reference":
        fn = ref().ccsd_tengy_omp
        fn.argtypes = [_dp] * 15 + [C.c_double] + [_dp] * 4 + [C.c_int] * 3
        fn.restype = None
    else:
        fn = lib().oracle_tengy
    fn(*fp, *vp, eorb.ctypes.data_as(_dp), eaijk, *[C.byref(o) for o in out], ncor, nocc, nvir)
    return tuple(o.value for o in out)


def ref_body_fn():
    """The compiled reference ccsd_trpdrv_omp_cbody_ as a ctypes function with its 39 arguments."""
    fn = ref().ccsd_trpdrv_omp_cbody_
    ip = C.POINTER(C.c_int)
    fn.argtypes = [_dp] * 9 + [ip] * 3 + [_dp] * 2 + [ip] * 5 + [_dp] * 20
    fn.restype = None
    return fn


def port_body_fn():
    fn = lib().oracle_cbody
    ip = C.POINTER(C.c_int)
    fn.argtypes = [_dp] * 9 + [ip] * 3 + [_dp] * 2 + [ip] * 5 + [_dp] * 20
    fn.restype = None
    return fn
