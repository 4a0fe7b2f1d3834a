"""The benchmark's roofline denominators: the issue-rate probes in lib/libtrpdrv_probe.so (a measurement
tool beside the product library).  CPU: the library exports both probes.  GPU: the FP64 DMMA probe and
the tcgen05 int8 probe (one SM, CTA pair, stage handshake) return rates inside the B200's physical
range, and the int8 rate grows with the instruction's N (the emulated form's N = 64 issues below the
N = 256 rate)."""
import ctypes as C
import os
import subprocess

import pytest

from conftest import ROOT

PROBE = os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib", "libtrpdrv_probe.so")


def _lib():
    lib = C.CDLL(PROBE)
    lib.trpdrv_probe_fp64_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.trpdrv_probe_fp64_peak.restype = C.c_int
    lib.trpdrv_probe_int8_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.trpdrv_probe_int8_peak.restype = C.c_int
    lib.trpdrv_probe_int8_rate.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.trpdrv_probe_int8_rate.restype = C.c_int
    return lib


def test_probe_library_exports_both_probes():
    out = subprocess.run(["nm", "-D", "--defined-only", PROBE], capture_output=True, text=True, check=True).stdout
    names = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert {"trpdrv_probe_fp64_peak", "trpdrv_probe_int8_peak", "trpdrv_probe_int8_rate"} <= names


def test_int8_probe_rejects_unsupported_arguments():
    v = C.c_double(0.0)
    lib = _lib()
    assert lib.trpdrv_probe_int8_peak(-1, 96, C.byref(v)) != 0  # checked before any device call
    assert lib.trpdrv_probe_int8_rate(-1, 64, 3, C.byref(v)) != 0


@pytest.mark.gpu
def test_probe_rates_are_physical():
    lib = _lib()
    v = C.c_double(0.0)
    assert lib.trpdrv_probe_fp64_peak(0, 2, C.byref(v)) == 0
    assert 15.0 < v.value < 45.0, v.value  # DMMA m16n8k8, TFLOP/s (148 SMs x 1.965 GHz x 128 = 37.2)
    rates = {}
    for n in (64, 256):
        assert lib.trpdrv_probe_int8_peak(0, n, C.byref(v)) == 0
        rates[n] = v.value
    # 148 SMs x 1.965 GHz x 8192 int8 multiply-adds x 2 = 4.77 POPS is the most the device can issue
    assert 1000.0 < rates[64] < rates[256] < 4800.0, rates
    # the CTA-pair form (M = 256) and the stage-handshake form run and stay in the same range
    for flags in (1, 2):
        assert lib.trpdrv_probe_int8_rate(0, 64, flags, C.byref(v)) == 0
        assert 1000.0 < v.value < 4800.0, (flags, v.value)
