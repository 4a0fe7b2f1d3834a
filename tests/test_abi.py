"""The C-ABI library loads and exports exactly what include/trpdrv.h declares (CPU only; no compute)."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "trpdrv.h")
LIB = os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib", "libtrpdrv_b200.so")

REFERENCE_SYMBOLS = {
    # symbol: reference file it replaces
    "ccsd_trpdrv_omp_cbody_": "omp/ccsd_trpdrv_omp_cbody.c:31-44",
    "ccsd_trpdrv_omp_fbody_": "omp/ccsd_trpdrv_omp_f77.f:1-9",
    "ccsd_trpdrv_cbody_": "ocl/ccsd_trpdrv_cbody.c:31",
    "ccsd_trpdrv_opencl_": "ocl/ccsd_trpdrv_opencl.c:31",
    "ccsd_tengy_omp": "omp/ccsd_tengy_c99.c:5-14",
    "ccsd_tengy": "ocl/ccsd_tengy.c:3-12",
    "ccsd_tengy_omp_": "omp/ccsd_tengy_f77.f:1-5",
}


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
        name = m.group(1)
        if name in ("if", "sizeof", "defined") or name.isupper():
            continue
        # keep identifiers that start a top-level declaration (preceded by a type)
        before = text[:m.start()].rstrip()
        if before.endswith(("void", "int", "int64_t", "double", "size_t", "char *", "*")) or \
                re.search(r"(void|int|int64_t|double|size_t|char \*|\*)\s*$", before):
            names.add(name)
    return names


def exported_functions():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_loads(T):
    assert T.lib.trpdrv_version() >= 10000
    assert os.path.exists(LIB)


def test_every_declared_function_is_exported():
    decl = declared_functions()
    exp = exported_functions()
    assert set(REFERENCE_SYMBOLS) <= decl
    missing = decl - exp
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_nothing_exported_beyond_the_header():
    extra = exported_functions() - declared_functions()
    assert not extra, f"exported but not declared in trpdrv.h: {sorted(extra)}"


def test_reference_symbols_resolvable_through_ctypes(T):
    for name in REFERENCE_SYMBOLS:
        assert getattr(T.lib, name) is not None


def test_header_compiles_as_c_and_cxx(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "trpdrv.h"\nint main(void){trpdrv_options o; trpdrv_options_default(&o); return o.world - 1;}\n')
    for comp, extra in (("gcc", ["-std=c99"]), ("g++", ["-x", "c++"])):
        subprocess.run([comp, *extra, "-I", os.path.join(ROOT, "include"), "-c", str(src), "-o",
                        str(tmp_path / "t.o")], check=True)


def test_status_strings(T):
    for code in range(8):
        assert T.lib.trpdrv_status_string(code).decode()


def _build_c_caller(out_dir):
    lib_dir = os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib")
    exe = os.path.join(str(out_dir), "c_plan_caller")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_plan_caller.c"), "-o", exe, "-L", lib_dir, "-ltrpdrv_b200",
                    "-Wl,-rpath," + lib_dir], check=True)
    return exe


def test_c_caller_of_the_plan_interface_compiles_and_links(tmp_path):
    """A C99 program using the plan interface (tests/c_plan_caller.c) builds against the header and links
    against libtrpdrv_b200.so; running it needs a GPU (tests/test_gpu_parity.py)."""
    assert os.access(_build_c_caller(tmp_path), os.X_OK)


HEADER_FP32 = os.path.join(ROOT, "include", "trpdrv_fp32.h")
LIB_FP32 = os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib", "libtrpdrv_b200_fp32.so")


def test_fp32_library_exports_exactly_its_header():
    """libtrpdrv_b200_fp32.so (the FP32 parity form) exports the float entry points of
    include/trpdrv_fp32.h (gpu-omp/ccsd_trpdrv_omp_cbody.c:38-51, gpu-omp/ccsd_tengy_c99.c:5-14) and
    nothing else."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER_FP32).read(), flags=re.S)
    decl = set(re.findall(r"^\s*(?:void|int|const char \*)\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, flags=re.M))
    assert {"ccsd_trpdrv_omp_cbody_", "ccsd_trpdrv_omp_fbody_", "ccsd_tengy_omp"} <= decl
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_FP32], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert exported == decl


def test_fp32_header_compiles_as_c_and_cxx(tmp_path):
    src = tmp_path / "t32.c"
    src.write_text('#include "trpdrv_fp32.h"\nint main(void){return trpdrv_fp32_last_error();}\n')
    for comp, extra in (("gcc", ["-std=c99"]), ("g++", ["-x", "c++"])):
        subprocess.run([comp, *extra, "-I", os.path.join(ROOT, "include"), "-c", str(src), "-o",
                        str(tmp_path / "t32.o")], check=True)
