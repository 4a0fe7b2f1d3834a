"""Python binding of libtrpdrv_b200.so (ctypes over the C ABI in include/trpdrv.h).

The library is the product: hand-written sm_100a kernels behind the reference's C entry points
(ccsd_trpdrv_omp_cbody_, ccsd_tengy_omp, ... from omp/ccsd_trpdrv_omp_cbody.c:31-44 and
omp/ccsd_tengy_c99.c:5-14) plus a batched plan interface.  This module only marshals numpy arrays
into those calls; it has no compute path of its own and raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("TRPDRV_LIB") or os.path.join(os.path.dirname(_HERE), "lib", "libtrpdrv_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include")

MODE_PLAIN = 0
MODE_FUSED = 1
MODE_EMULATED = 2
DIST_UNIFORM = 0
DIST_LOGUNIFORM = 1

# tensor ids (TRPDRV_T_*)
T_EORB, T_T2, T_JVV, T_KVV, T_TOV, T_XOV, T_JOV, T_KOV, T_DINTC, T_DINTX, T_T1V = range(11)
TENSOR_NAMES = ("eorb", "t2", "jvv", "kvv", "tov", "xov", "jov", "kov", "dintc", "dintx", "t1v")

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA runtime error", 3: "out of memory",
          4: "no usable sm_100 device", 5: "call out of order", 6: "unsupported",
          7: "device-side check failed"}


class TrpdrvError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


if not os.path.exists(LIB_PATH):
    raise ImportError(f"libtrpdrv_b200.so not built at {LIB_PATH}; run `python -c "
                      f"'import __graft_entry__ as g; g.build()'` from the repository root")
lib = C.CDLL(LIB_PATH)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class SystemStruct(C.Structure):
    _fields_ = [("ncor", C.c_int), ("nocc", C.c_int), ("nvir", C.c_int), ("a", C.c_int)] + \
               [(n, C.c_void_p) for n in TENSOR_NAMES]


class OptionsStruct(C.Structure):
    _fields_ = [("mode", C.c_int), ("nkpass", C.c_int), ("rank", C.c_int), ("world", C.c_int),
                ("device", C.c_int), ("tile", C.c_int), ("ctas_per_sm", C.c_int),
                ("use_graph", C.c_int), ("mma_k", C.c_int), ("staging", C.c_int), ("slices", C.c_int),
                ("batch", C.c_int), ("a_count", C.c_int), ("target_digits", C.c_int),
                ("reserved", C.c_int * 2)]

STAGING_AUTO, STAGING_CPASYNC, STAGING_TMA = 0, 1, 2

BODY_DEVICE_FIELDS = ("eorb", "tij", "tkj", "tia", "tka", "xia", "xka", "jia", "jka", "kia", "kka", "jij", "jkj",
                      "kij", "kkj", "dintc1", "dintx1", "t1v1", "dintc2", "dintx2", "t1v2", "out4")
NOALLOC_MAX_NVIR, NOALLOC_MAX_NOCC = 256, 64


class BodyDeviceArgs(C.Structure):
    """trpdrv_body_device_args: one triple on caller-owned device pointers (already sliced)."""
    _fields_ = [("ncor", C.c_int), ("nocc", C.c_int), ("nvir", C.c_int), ("a", C.c_int), ("i", C.c_int),
                ("j", C.c_int), ("k", C.c_int)] + [(n, C.c_void_p) for n in BODY_DEVICE_FIELDS]


def _proto(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_proto("trpdrv_last_error", C.c_int, [])
_proto("trpdrv_last_error_message", C.c_char_p, [])
_proto("trpdrv_status_string", C.c_char_p, [C.c_int])
_proto("trpdrv_clear_error", None, [])
_proto("trpdrv_version", C.c_int, [])
_proto("trpdrv_options_default", None, [C.POINTER(OptionsStruct)])
_proto("trpdrv_plan_create", C.c_int, [C.POINTER(C.c_void_p), C.POINTER(SystemStruct), C.c_int,
                                       C.POINTER(OptionsStruct)])
_proto("trpdrv_plan_upload", C.c_int, [C.c_void_p, C.POINTER(SystemStruct), C.c_void_p])
_proto("trpdrv_plan_upload_execute", C.c_int, [C.c_void_p, C.POINTER(SystemStruct), C.c_int, C.c_void_p])
_proto("trpdrv_plan_bind_device", C.c_int, [C.c_void_p, C.POINTER(SystemStruct)])
_proto("trpdrv_plan_execute", C.c_int, [C.c_void_p, C.c_void_p])
_proto("trpdrv_plan_energies", C.c_int, [C.c_void_p, _dp, _dp])
_proto("trpdrv_plan_num_triples", C.c_int64, [C.c_void_p, C.c_int])
_proto("trpdrv_plan_triples", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int32)])
_proto("trpdrv_plan_triple_energies", C.c_int, [C.c_void_p, C.c_int, _dp])
_proto("trpdrv_plan_last_launches", C.c_int64, [C.c_void_p])
_proto("trpdrv_plan_staging", C.c_int, [C.c_void_p])


class TuneCandidate(C.Structure):
    _fields_ = [("staging", C.c_int), ("mma_k", C.c_int), ("ctas_per_sm", C.c_int), ("batch", C.c_int),
                ("edge_pack", C.c_int), ("ms_estimate", C.c_double)]


class TuneResult(C.Structure):
    _fields_ = [("ncand", C.c_int), ("chosen", C.c_int), ("from_cache", C.c_int), ("cand", TuneCandidate * 8),
                ("slices", C.c_int), ("est_rel_err", C.c_double)]


_proto("trpdrv_plan_autotune", C.c_int, [C.c_void_p, C.POINTER(TuneResult)])
_proto("trpdrv_plan_last_kernel_ms", C.c_int, [C.c_void_p, _dp])
_proto("trpdrv_plan_destroy", C.c_int, [C.c_void_p])
_proto("trpdrv_run", C.c_int, [C.POINTER(SystemStruct), C.c_int, C.POINTER(OptionsStruct), _dp, _dp])
_proto("trpdrv_count_triples", C.c_int64, [C.c_int])
_proto("trpdrv_enumerate_triples", C.c_int64, [C.c_int, C.c_int, C.POINTER(C.c_int32)])
_proto("trpdrv_partition", C.c_int, [_dp, C.c_int64, C.c_int, C.POINTER(C.c_int64)])
_proto("trpdrv_shard_triples", C.c_int64, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32)])
_proto("trpdrv_tensor_a_dependent", C.c_int, [C.c_int])
_proto("trpdrv_processing_order", C.c_int, [C.POINTER(C.c_int32), C.c_int64, C.c_int, C.POINTER(C.c_int32)])
_proto("trpdrv_upload_spans", C.c_int64,
       [C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int64, C.c_int, C.POINTER(C.c_int64)])
_proto("trpdrv_triple_flops", C.c_double, [C.c_int, C.c_int])
_proto("trpdrv_tensor_elems", C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int])
_proto("trpdrv_synth_fill", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, _dp,
                                      C.c_size_t])
_proto("trpdrv_body_device_noalloc", C.c_int, [C.POINTER(BodyDeviceArgs), C.c_void_p])
_proto("trpdrv_finalize", None, [])
_proto("trpdrv_register_host", C.c_int, [C.c_void_p, C.c_size_t])
_proto("trpdrv_refresh_host", C.c_int, [C.c_void_p])
_proto("trpdrv_unregister_host", C.c_int, [C.c_void_p])
_proto("trpdrv_selftest_bounded_wait", C.c_int, [C.c_double, _ip, _dp])
_body_args = [_dp] * 9 + [_ip] * 3 + [_dp] * 2 + [_ip] * 5 + [_dp] * 20
for _n in ("ccsd_trpdrv_omp_cbody_", "ccsd_trpdrv_omp_fbody_", "ccsd_trpdrv_cbody_", "ccsd_trpdrv_opencl_"):
    _proto(_n, None, _body_args)
_tengy_args = [_dp] * 15 + [C.c_double] + [_dp] * 4 + [C.c_int] * 3
_proto("ccsd_tengy_omp", None, _tengy_args)
_proto("ccsd_tengy", None, _tengy_args)
_proto("ccsd_tengy_omp_", None, [_dp] * 15 + [_dp] + [_dp] * 4 + [_ip] * 3)


def _check(rc: int):
    if rc != 0:
        raise TrpdrvError(rc, lib.trpdrv_last_error_message().decode(errors="replace"))


def last_error() -> tuple[int, str]:
    return lib.trpdrv_last_error(), lib.trpdrv_last_error_message().decode(errors="replace")


def clear_error():
    lib.trpdrv_clear_error()


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


# --------------------------------------------------------------------------------------------
# host-side helpers
# --------------------------------------------------------------------------------------------
def count_triples(nocc: int) -> int:
    return int(lib.trpdrv_count_triples(nocc))


def enumerate_triples(nocc: int, nkpass: int = 1) -> np.ndarray:
    """(n, 4) int32 array of i, j, k, klo (1-based) in the reference driver's order."""
    n = count_triples(nocc)
    out = np.zeros((max(n, 1), 4), dtype=np.int32)
    lib.trpdrv_enumerate_triples(nocc, nkpass, out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out[:n]


def partition(costs: Optional[Sequence[float]], n: int, world: int) -> np.ndarray:
    bounds = np.zeros(world + 1, dtype=np.int64)
    if costs is None:
        cp = None
    else:
        carr = np.ascontiguousarray(costs, dtype=np.float64)
        assert carr.size == n
        cp = carr.ctypes.data_as(_dp)
    _check(lib.trpdrv_partition(cp, n, world, bounds.ctypes.data_as(C.POINTER(C.c_int64))))
    return bounds


def shard_triples(nocc: int, nkpass: int, rank: int, world: int) -> np.ndarray:
    """(n, 3) int32 i, j, k (1-based): the triples a plan with this rank/world processes."""
    n = int(lib.trpdrv_shard_triples(nocc, nkpass, rank, world, None))
    if n < 0:
        raise TrpdrvError(1, f"shard_triples({nocc}, {nkpass}, {rank}, {world})")
    out = np.zeros((max(n, 1), 3), dtype=np.int32)
    lib.trpdrv_shard_triples(nocc, nkpass, rank, world, out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out[:n]


def processing_order(ijk: np.ndarray, block: int = 0) -> np.ndarray:
    """Permutation position -> list index in which fused plans process the triples ijk ((n, 3), 1-based)."""
    a = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
    out = np.zeros(max(len(a), 1), dtype=np.int32)
    rc = lib.trpdrv_processing_order(a.ctypes.data_as(C.POINTER(C.c_int32)), len(a), block,
                                     out.ctypes.data_as(C.POINTER(C.c_int32)))
    if rc != 0:
        raise TrpdrvError(1, "processing_order: bad arguments")
    return out[:len(a)]


def upload_spans(ijk: np.ndarray, order: Optional[np.ndarray], chunks: int) -> np.ndarray:
    """Span bounds (positions of the processing order) that trpdrv_plan_upload_execute launches one by
    one: spans are [b[s], b[s+1])."""
    a = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
    o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
    out = np.zeros(max(chunks, 0) + 1, dtype=np.int64)
    ns = lib.trpdrv_upload_spans(a.ctypes.data_as(C.POINTER(C.c_int32)),
                                 None if o is None else o.ctypes.data_as(C.POINTER(C.c_int32)), len(a), chunks,
                                 out.ctypes.data_as(C.POINTER(C.c_int64)))
    if ns < 0:
        raise TrpdrvError(1, "upload_spans: bad arguments")
    return out[:ns + 1]


def triple_flops(nocc: int, nvir: int) -> float:
    return float(lib.trpdrv_triple_flops(nocc, nvir))


def tensor_elems(tensor: int, ncor: int, nocc: int, nvir: int) -> int:
    return int(lib.trpdrv_tensor_elems(tensor, ncor, nocc, nvir))


def tensor_a_dependent(tensor: int) -> bool:
    """Whether the tensor holds one block per virtual index in an a sweep (options a_count)."""
    return bool(lib.trpdrv_tensor_a_dependent(tensor))


# --------------------------------------------------------------------------------------------
# systems
# --------------------------------------------------------------------------------------------
@dataclass
class System:
    """One system in the library's slice layout (trpdrv.h): all triples of the virtual indices
    a .. a + a_count - 1; the a-dependent tensors hold a_count blocks (plans need a_count=a_count)."""
    ncor: int
    nocc: int
    nvir: int
    a: int
    arrays: dict = field(default_factory=dict)  # name -> contiguous float64 ndarray (host) or device ptr
    a_count: int = 1

    def a_view(self, ai: int) -> "System":
        """The single-`a` system of virtual index a + ai (views of the a-dependent blocks)."""
        out = System(self.ncor, self.nocc, self.nvir, self.a + ai)
        for t, name in enumerate(TENSOR_NAMES):
            arr = self.arrays[name]
            if tensor_a_dependent(t):
                n = tensor_elems(t, self.ncor, self.nocc, self.nvir)
                arr = arr[ai * n:(ai + 1) * n]
            out.arrays[name] = arr
        return out

    def struct(self, device_ptrs: Optional[dict] = None) -> SystemStruct:
        s = SystemStruct()
        s.ncor, s.nocc, s.nvir, s.a = self.ncor, self.nocc, self.nvir, self.a
        for name in TENSOR_NAMES:
            if device_ptrs is not None:
                setattr(s, name, C.c_void_p(int(device_ptrs[name])))
            else:
                arr = self.arrays[name]
                setattr(s, name, C.c_void_p(arr.ctypes.data))
        return s

    def nbytes(self) -> int:
        return sum(int(a.nbytes) for a in self.arrays.values())


def synth_system(nocc: int, nvir: int, seed: int = 1, ncor: int = 0, dist: int = DIST_UNIFORM,
                 a: Optional[int] = None, alloc=None, a_count: int = 1, a_block: int = 0) -> System:
    """Seeded synthetic system.  `a` defaults to the first virtual orbital (ncor+nocc+1), which keeps
    every denominator e_b + e_c + eaijk >= 2.1 under these distributions.  `alloc(n)` may return a
    preallocated (e.g. pinned) float64 buffer of n elements.  With a_count > 1 the a-dependent
    tensors get a_count blocks; block 0 is the a_count = 1 system's, block m is generated from seed
    + 7919 m.  a_block = m starts the sweep at its block m instead (virtual index a + m): with
    a_count = 1 that is one a of the molecule, equal to synth_system(..., a_count=m+1).a_view(m)."""
    if a is None:
        a = ncor + nocc + 1
    if a_block < 0:
        raise TrpdrvError(1, f"a_block {a_block}: must be >= 0")
    sysm = System(ncor, nocc, nvir, a + a_block, a_count=a_count)
    for t, name in enumerate(TENSOR_NAMES):
        n = tensor_elems(t, ncor, nocc, nvir)
        dep = tensor_a_dependent(t)
        blocks = a_count if dep else 1
        buf = alloc(n * blocks) if alloc is not None else np.empty(n * blocks, dtype=np.float64)
        for m in range(blocks):
            mm = m + a_block if dep else m
            _check(lib.trpdrv_synth_fill(t, ncor, nocc, nvir, seed + 7919 * mm, dist, _ptr(buf[m * n:]), n))
        sysm.arrays[name] = buf
    return sysm


def triple_slices(s: System, i: int, j: int, k: int, klo: int) -> dict:
    """The reference body's pointer arguments for triple (i,j,k) (1-based) as numpy views, with the
    k-chunk base at klo exactly as omp/test.c passes them (omp/test.c:173-176)."""
    O, V = s.nocc, s.nvir
    vv, ov = V * V, O * V
    A = s.arrays
    jb = (j - 1) * O
    return dict(
        eorb=A["eorb"],
        tij=A["t2"][(jb + i - 1) * vv:], tkj=A["t2"][(jb + klo - 1) * vv:],
        tia=A["tov"][(i - 1) * ov:], tka=A["tov"][(klo - 1) * ov:],
        xia=A["xov"][(i - 1) * ov:], xka=A["xov"][(klo - 1) * ov:],
        jia=A["jvv"][(i - 1) * vv:], jka=A["jvv"][(klo - 1) * vv:],
        kia=A["kvv"][(i - 1) * vv:], kka=A["kvv"][(klo - 1) * vv:],
        jij=A["jov"][(jb + i - 1) * ov:], jkj=A["jov"][(jb + klo - 1) * ov:],
        kij=A["kov"][(jb + i - 1) * ov:], kkj=A["kov"][(jb + klo - 1) * ov:],
        dintc1=A["dintc"][(i - 1) * V:], dintx1=A["dintx"][(i - 1) * V:], t1v1=A["t1v"][(i - 1) * V:],
        dintc2=A["dintc"][(k - 1) * V:], dintx2=A["dintx"][(k - 1) * V:], t1v2=A["t1v"][(k - 1) * V:],
    )


BODY_ORDER = ("tij", "tkj", "tia", "tka", "xia", "xka", "jia", "jka", "kia", "kka", "jij", "jkj", "kij",
              "kkj", "dintc1", "dintx1", "t1v1", "dintc2", "dintx2", "t1v2")


def body_call(fn, s: System, i: int, j: int, k: int, klo: int, emp4: float = 0.0, emp5: float = 0.0,
              f: Optional[np.ndarray] = None):
    """Calls a reference-signature body `fn` (a ctypes function) for one triple; returns the updated
    (emp4, emp5).  `f` (8, nvir*nvir) receives f1n f1t f2n f2t f3n f3t f4n f4t in argument order."""
    sl = triple_slices(s, i, j, k, klo)
    V = s.nvir
    if f is None:
        f = np.zeros((8, V * V), dtype=np.float64)
    fp = [f[q].ctypes.data_as(_dp) for q in range(8)]
    ints = [C.c_int(v) for v in (s.ncor, s.nocc, s.nvir)]
    e4, e5 = C.c_double(emp4), C.c_double(emp5)
    idx = [C.c_int(v) for v in (s.a, i, j, k, klo)]
    arrs = [np.ascontiguousarray(sl[n]).ctypes.data_as(_dp) if not sl[n].flags.c_contiguous
            else sl[n].ctypes.data_as(_dp) for n in BODY_ORDER]
    fn(*fp, sl["eorb"].ctypes.data_as(_dp), *[C.byref(v) for v in ints], C.byref(e4), C.byref(e5),
       *[C.byref(v) for v in idx], *arrs)
    return e4.value, e5.value


def cbody(s: System, i: int, j: int, k: int, klo: int, emp4=0.0, emp5=0.0, f=None, entry="ccsd_trpdrv_omp_cbody_"):
    return body_call(getattr(lib, entry), s, i, j, k, klo, emp4, emp5, f)


def register_host(arr: np.ndarray):
    """trpdrv_register_host: the drop-in entry points read pointers inside `arr` from a device copy."""
    _check(lib.trpdrv_register_host(C.c_void_p(arr.ctypes.data), arr.nbytes))


def refresh_host(arr: np.ndarray):
    _check(lib.trpdrv_refresh_host(C.c_void_p(arr.ctypes.data)))


def unregister_host(arr: np.ndarray):
    _check(lib.trpdrv_unregister_host(C.c_void_p(arr.ctypes.data)))


def selftest_bounded_wait(limit_seconds: float = 0.05) -> tuple[int, float]:
    """trpdrv_selftest_bounded_wait: runs the kernels' bounded mbarrier wait on a barrier that nothing
    completes; returns (status word, seconds waited).  A correct wait gives up: status 2."""
    st, el = C.c_int(0), C.c_double(0.0)
    _check(lib.trpdrv_selftest_bounded_wait(float(limit_seconds), C.byref(st), C.byref(el)))
    return st.value, el.value


def register_system(s: "System"):
    """Registers every array of a host system (its tensors stay unchanged while drop-in calls run)."""
    for name in TENSOR_NAMES:
        register_host(s.arrays[name])


def unregister_system(s: "System"):
    for name in TENSOR_NAMES:
        unregister_host(s.arrays[name])


def tengy(f8: np.ndarray, vecs: Sequence[np.ndarray], eorb: np.ndarray, eaijk: float, ncor: int, nocc: int,
          nvir: int, entry: str = "ccsd_tengy_omp"):
    """Calls the library's tengy drop-in.  f8 rows in argument order f1n f1t f2n f2t f3n f3t f4n f4t;
    vecs = dintc1, dintx1, t1v1, dintc2, dintx2, t1v2.  Returns (emp4i, emp5i, emp4k, emp5k)."""
    out = [C.c_double(0.0) for _ in range(4)]
    fp = [np.ascontiguousarray(f8[q]).ctypes.data_as(_dp) for q in range(8)]
    vp = [np.ascontiguousarray(v).ctypes.data_as(_dp) for v in vecs]
    if entry == "ccsd_tengy_omp_":
        order = [vp[0], vp[3], vp[1], vp[4], vp[2], vp[5]]
        e = C.c_double(eaijk)
        ints = [C.c_int(v) for v in (ncor, nocc, nvir)]
        lib.ccsd_tengy_omp_(*fp, *order, eorb.ctypes.data_as(_dp), C.byref(e), *[C.byref(o) for o in out],
                            *[C.byref(v) for v in ints])
    else:
        getattr(lib, entry)(*fp, *vp, eorb.ctypes.data_as(_dp), eaijk, *[C.byref(o) for o in out],
                            ncor, nocc, nvir)
    return tuple(o.value for o in out)


# --------------------------------------------------------------------------------------------
# plans
# --------------------------------------------------------------------------------------------
def options(mode=MODE_FUSED, nkpass=1, rank=0, world=1, device=-1, ctas_per_sm=0, use_graph=1,
            mma_k=0, staging=STAGING_AUTO, slices=0, batch=0, a_count=1, target_digits=0) -> OptionsStruct:
    o = OptionsStruct()
    lib.trpdrv_options_default(C.byref(o))
    o.mode, o.nkpass, o.rank, o.world, o.device = mode, nkpass, rank, world, device
    o.ctas_per_sm, o.use_graph, o.staging = ctas_per_sm, use_graph, staging
    if mma_k:
        o.mma_k = mma_k
    if slices:
        o.slices = slices
    if batch:
        o.batch = batch
    o.a_count = a_count
    o.target_digits = target_digits
    return o


class Plan:
    """Device storage + work queue for a batch of systems (trpdrv_plan_*)."""

    def __init__(self, systems: Sequence[System], **opt):
        self.systems = list(systems)
        self._shapes = (SystemStruct * len(self.systems))()
        for q, s in enumerate(self.systems):
            st = self._shapes[q]
            st.ncor, st.nocc, st.nvir, st.a = s.ncor, s.nocc, s.nvir, s.a
        if "a_count" not in opt:  # the systems' a sweep (all alike)
            counts = {getattr(s, "a_count", 1) for s in self.systems}
            if len(counts) != 1:
                raise TrpdrvError(1, f"systems of one plan must share a_count, got {sorted(counts)}")
            opt["a_count"] = counts.pop()
        self.opt = options(**opt)
        self.h = C.c_void_p()
        _check(lib.trpdrv_plan_create(C.byref(self.h), self._shapes, len(self.systems), C.byref(self.opt)))

    def upload(self, systems: Optional[Sequence[System]] = None, stream: int = 0):
        systems = self.systems if systems is None else systems
        arr = (SystemStruct * len(systems))(*[s.struct() for s in systems])
        _check(lib.trpdrv_plan_upload(self.h, arr, C.c_void_p(stream) if stream else None))

    def upload_execute(self, systems: Optional[Sequence[System]] = None, chunks: int = 0, stream: int = 0):
        """trpdrv_plan_upload_execute: upload and execute with the T2/JOV/KOV copies overlapped with the
        fused kernel, j range by j range."""
        systems = self.systems if systems is None else systems
        arr = (SystemStruct * len(systems))(*[s.struct() for s in systems])
        _check(lib.trpdrv_plan_upload_execute(self.h, arr, chunks, C.c_void_p(stream) if stream else None))

    def bind_device(self, ptrs: Sequence[dict]):
        arr = (SystemStruct * len(self.systems))(*[s.struct(p) for s, p in zip(self.systems, ptrs)])
        _check(lib.trpdrv_plan_bind_device(self.h, arr))

    def execute(self, stream: int = 0):
        _check(lib.trpdrv_plan_execute(self.h, C.c_void_p(stream) if stream else None))

    def energies(self):
        n = len(self.systems)
        e4 = np.zeros(n)
        e5 = np.zeros(n)
        _check(lib.trpdrv_plan_energies(self.h, e4.ctypes.data_as(_dp), e5.ctypes.data_as(_dp)))
        return e4, e5

    def num_triples(self, sys: int = 0) -> int:
        return int(lib.trpdrv_plan_num_triples(self.h, sys))

    def triples(self, sys: int = 0) -> np.ndarray:
        n = self.num_triples(sys)
        out = np.zeros((max(n, 1), 3), dtype=np.int32)
        _check(lib.trpdrv_plan_triples(self.h, sys, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out[:n]

    def triple_energies(self, sys: int = 0) -> np.ndarray:
        n = self.num_triples(sys)
        out = np.zeros((max(n, 1), 4))
        _check(lib.trpdrv_plan_triple_energies(self.h, sys, out.ctypes.data_as(_dp)))
        return out[:n]

    def autotune(self) -> dict:
        """trpdrv_plan_autotune: times the compiled variants on a sample of this plan's work and keeps the
        fastest.  Returns {"candidates": [...], "chosen": i, "from_cache": 0 timed now, 1 process cache, 2 file
        cache (TRPDRV_TUNE_CACHE)}."""
        r = TuneResult()
        _check(lib.trpdrv_plan_autotune(self.h, C.byref(r)))
        cands = [{"staging": c.staging, "mma_k": c.mma_k, "ctas_per_sm": c.ctas_per_sm, "batch": c.batch,
                  "edge_pack": c.edge_pack, "ms_estimate": c.ms_estimate} for c in r.cand[:r.ncand]]
        return {"candidates": cands, "chosen": r.chosen, "from_cache": int(r.from_cache), "slices": r.slices,
                "est_rel_err": r.est_rel_err}

    def staging(self) -> int:
        """1 = cp.async, 2 = TMA staging in the fused kernel (0 for plain plans)."""
        return int(lib.trpdrv_plan_staging(self.h))

    def last_launches(self) -> int:
        return int(lib.trpdrv_plan_last_launches(self.h))

    def last_kernel_ms(self) -> float:
        ms = C.c_double(0.0)
        _check(lib.trpdrv_plan_last_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def close(self):
        if self.h:
            lib.trpdrv_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(systems: Sequence[System], **opt):
    """One call from host arrays to per-system totals (trpdrv_run)."""
    arr = (SystemStruct * len(systems))(*[s.struct() for s in systems])
    o = options(**opt)
    e4 = np.zeros(len(systems))
    e5 = np.zeros(len(systems))
    _check(lib.trpdrv_run(arr, len(systems), C.byref(o), e4.ctypes.data_as(_dp), e5.ctypes.data_as(_dp)))
    return e4, e5


def body_device_noalloc(ncor: int, nocc: int, nvir: int, a: int, i: int, j: int, k: int, ptrs: dict,
                        stream: int = 0):
    """trpdrv_body_device_noalloc: `ptrs` maps BODY_DEVICE_FIELDS to device addresses (ints).
    Asynchronous on `stream`; raises TrpdrvError on a rejected call."""
    args = BodyDeviceArgs()
    args.ncor, args.nocc, args.nvir, args.a, args.i, args.j, args.k = ncor, nocc, nvir, a, i, j, k
    for n in BODY_DEVICE_FIELDS:
        setattr(args, n, C.c_void_p(int(ptrs[n])) if ptrs.get(n) else None)
    _check(lib.trpdrv_body_device_noalloc(C.byref(args), C.c_void_p(stream) if stream else None))


def finalize():
    lib.trpdrv_finalize()
