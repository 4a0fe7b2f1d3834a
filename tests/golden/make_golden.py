"""Generates the golden fixtures in tests/golden/ from the REFERENCE ITSELF.

The reference's omp/ccsd_trpdrv_omp_cbody.c and omp/ccsd_tengy_c99.c, compiled unmodified by
oracle/Makefile into oracle/_ref/libtrpdrv_ref.so (OpenBLAS 0.3.30), are run over every triple of a
few small seeded systems (inputs from the library's counter-based generator, trpdrv_synth_fill).
For each triple the fixture stores emp4i, emp5i, emp4k, emp5k (the reference body's f arrays fed to
the reference ccsd_tengy_omp), plus long-double compensated totals and per-tensor checksums of the
inputs, so a change of the generator is detected rather than silently changing the fixture.

It also records the known-answer print of the reference driver itself:
    oracle/_ref/test_c99 10 60 100000   ->   "emp4=2.647247 emp5=-1.560018"
and of the reference's single-precision variant (gpu-omp/test.c + gpu-omp/ccsd_trpdrv_omp_cbody.c,
unmodified, host build; `python tests/golden/make_golden.py fp32` writes only this file):
    oracle/_ref/test_fp32 10 60 100000  ->   kat_test_fp32_10_60.json

Run from the repository root where the reference sources exist:
    make -C oracle && python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
import trpdrv_b200 as T  # noqa: E402

# name: (ncor, nocc, nvir, seed, dist, nkpass)
CASES = {
    "g_o4_v24": (0, 4, 24, 11, T.DIST_UNIFORM, 1),
    "g_o6_v40_nk2": (0, 6, 40, 12, T.DIST_UNIFORM, 2),
    "g_c2_o5_v33": (2, 5, 33, 13, T.DIST_UNIFORM, 1),
    "g_o4_v30_log": (0, 4, 30, 14, T.DIST_LOGUNIFORM, 1),
    "g_o10_v60": (0, 10, 60, 15, T.DIST_UNIFORM, 1),
    "g_o3_v70": (0, 3, 70, 16, T.DIST_UNIFORM, 1),
}


def checksums(s):
    return {n: [float(np.sum(a)), float(np.sum(a * a))] for n, a in s.arrays.items()}


def fp32_kat(out_dir):
    runs = []
    for argv in (["10", "60", "100000"], ["10", "60", "100000", "3"], ["12", "50", "100000", "2"]):
        kat = subprocess.run([os.path.join(os.path.dirname(O.REF_TEST), "test_fp32"), *argv], capture_output=True,
                             text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1"))
        line = [ln for ln in kat.stdout.splitlines() if ln.startswith("emp4=")][0]
        runs.append({"argv": argv, "line": line})
        print("fp32", argv, line)
    with open(os.path.join(out_dir, "kat_test_fp32_10_60.json"), "w") as f:
        json.dump({"command": "test_fp32 10 60 100000", "line": runs[0]["line"], "runs": runs,
                   "source": "reference gpu-omp/test.c + gpu-omp/ccsd_trpdrv_omp_cbody.c (single precision), "
                             "unmodified, host build with OpenBLAS sgemm"}, f, indent=1)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "fp32":
        fp32_kat(os.path.dirname(os.path.abspath(__file__)))
        return
    if os.environ.get("OMP_NUM_THREADS") != "1":
        # one OpenMP thread inside the reference tengy: a fixed reduction order, reproducible fixtures
        os.execvpe(sys.executable, [sys.executable, os.path.abspath(__file__)],
                   dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1"))
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, (ncor, nocc, nvir, seed, dist, nkpass) in CASES.items():
        s = T.synth_system(nocc, nvir, seed=seed, ncor=ncor, dist=dist)
        rec, tot, mism = O.run_system(s, "reference", nkpass=nkpass, nthreads=1)
        assert mism == 0, name
        ijkl = O.enumerate_triples(nocc, nkpass)
        doc = {
            "generator": "trpdrv_synth_fill (splitmix64 counter stream)",
            "source": "oracle/_ref/libtrpdrv_ref.so = reference omp/ccsd_trpdrv_omp_cbody.c + omp/ccsd_tengy_c99.c",
            "ncor": ncor, "nocc": nocc, "nvir": nvir, "a": s.a, "seed": seed, "dist": dist, "nkpass": nkpass,
            "checksums": checksums(s),
            "triples": ijkl[:, :3].tolist(),
            "records": [[float(repr_f) for repr_f in r] for r in rec],
            "emp4": float(tot[0]), "emp5": float(tot[1]),
        }
        with open(os.path.join(out_dir, name + ".json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))
        print(name, len(rec), tot)

    runs = []
    for argv in (["10", "60", "100000"], ["10", "60", "100000", "3"], ["12", "50", "100000", "2"]):
        kat = subprocess.run([O.REF_TEST, *argv], capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1"))
        line = [ln for ln in kat.stdout.splitlines() if ln.startswith("emp4=")][0]
        runs.append({"argv": argv, "line": line})
        print(argv, line)
    with open(os.path.join(out_dir, "kat_test_c99_10_60.json"), "w") as f:
        json.dump({"command": "test_c99 10 60 100000", "line": runs[0]["line"], "runs": runs,
                   "source": "reference omp/test.c + omp/ccsd_trpdrv_omp_cbody.c + omp/ccsd_tengy_c99.c, unmodified"},
                  f, indent=1)
    fp32_kat(out_dir)


if __name__ == "__main__":
    main()
