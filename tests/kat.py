"""The reference driver's own fixture and loop, restated for tests (omp/test.c:55-62, 94-195).

Every array is make_array(n)[i] = 1/(100+i); a = 1 is fixed; the triple loop runs klo / j / i / k with
the same bounds and the +-1000 wrap of emp4/emp5 after every call.  The final print of
`test_c99 10 60 100000` (full loop) is the known answer emp4=2.647247 emp5=-1.560018.
"""
import ctypes as C

import numpy as np

_dp = C.POINTER(C.c_double)


def make_array(n):
    return 1.0 / (100.0 + np.arange(n, dtype=np.float64))


def run_make_array_loop(body_fn, nocc, nvir, nkpass=1, maxiter=100000):
    """Calls body_fn (39-argument reference signature) exactly as omp/test.c:160-195 does and returns
    the driver's final "emp4=%f emp5=%f" line and the number of calls."""
    ncor = 0
    nbf = ncor + nocc + nvir
    lnvv, lnov = nvir * nvir, nocc * nvir
    kchunk = (nocc - 1) // nkpass + 1
    A = {}
    A["eorb"] = make_array(nbf)
    for n in ("f1n", "f2n", "f3n", "f4n", "f1t", "f2t", "f3t", "f4t"):
        A[n] = make_array(lnvv)
    A["Tij"] = make_array(lnvv)
    A["Tkj"] = make_array(kchunk * lnvv)
    A["Tia"] = make_array(lnov * nocc)
    A["Tka"] = make_array(kchunk * lnov)
    A["Xia"] = make_array(lnov * nocc)
    A["Xka"] = make_array(kchunk * lnov)
    A["Jia"] = make_array(lnvv)
    A["Jka"] = make_array(kchunk * lnvv)
    A["Kia"] = make_array(lnvv)
    A["Kka"] = make_array(kchunk * lnvv)
    A["Jij"] = make_array(lnov * nocc)
    A["Jkj"] = make_array(kchunk * lnov)
    A["Kij"] = make_array(lnov * nocc)
    A["Kkj"] = make_array(kchunk * lnov)
    for n in ("dintc1", "dintc2", "dintx1", "dintx2", "t1v1", "t1v2"):
        A[n] = make_array(lnvv)
    P = {n: a.ctypes.data_as(_dp) for n, a in A.items()}
    c_ncor, c_nocc, c_nvir = C.c_int(ncor), C.c_int(nocc), C.c_int(nvir)
    emp4, emp5 = C.c_double(0.0), C.c_double(0.0)
    a = C.c_int(1)
    it = 0
    for klo in range(1, nocc + 1, kchunk):
        khi = min(nocc, klo + kchunk - 1)
        for j in range(1, nocc + 1):
            for i in range(1, nocc + 1):
                for k in range(klo, min(khi, i) + 1):
                    ci, cj, ck, cklo = C.c_int(i), C.c_int(j), C.c_int(k), C.c_int(klo)
                    body_fn(P["f1n"], P["f1t"], P["f2n"], P["f2t"], P["f3n"], P["f3t"], P["f4n"], P["f4t"],
                            P["eorb"], C.byref(c_ncor), C.byref(c_nocc), C.byref(c_nvir), C.byref(emp4),
                            C.byref(emp5), C.byref(a), C.byref(ci), C.byref(cj), C.byref(ck), C.byref(cklo),
                            P["Tij"], P["Tkj"], P["Tia"], P["Tka"], P["Xia"], P["Xka"], P["Jia"], P["Jka"],
                            P["Kia"], P["Kka"], P["Jij"], P["Jkj"], P["Kij"], P["Kkj"],
                            P["dintc1"], P["dintx1"], P["t1v1"], P["dintc2"], P["dintx2"], P["t1v2"])
                    it += 1
                    if it == maxiter:
                        return "emp4=%f emp5=%f" % (emp4.value, emp5.value), it
                    if emp4.value > 1000.0:
                        emp4.value -= 1000.0
                    if emp4.value < -1000.0:
                        emp4.value += 1000.0
                    if emp5.value > 1000.0:
                        emp5.value -= 1000.0
                    if emp5.value < -1000.0:
                        emp5.value += 1000.0
    return "emp4=%f emp5=%f" % (emp4.value, emp5.value), it
