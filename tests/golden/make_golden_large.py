"""Generates the full-size golden fixtures tests/golden/big_*.json from the REFERENCE ITSELF.

The three full-size workloads of the benchmark, each run over EVERY triple of one `a` through the
reference's omp/ccsd_trpdrv_omp_cbody.c + omp/ccsd_tengy_c99.c compiled unmodified by oracle/Makefile
(oracle/_ref/libtrpdrv_ref.so, OpenBLAS 0.3.30 on one thread per call, triples spread over the host
cores):

  big_c2_o40_v300       nocc=40, nvir=300, uniform distributions, seed 2024, a = 41 (32,800 triples)
  big_c3_o30_v400_log   nocc=30, nvir=400, log-uniform integral magnitudes in [1e-6, 1], seed 2024,
                        a = 31 (13,950 triples)
  big_c4_six            six systems (8,80) (12,150) (16,220) (24,310) (32,380) (40,450), seed 2024 + q,
                        a = nocc + 1 (60,296 triples)

Each system stores the long-double compensated totals over all of its triples, the records
(emp4i, emp5i, emp4k, emp5k) of every 13th triple of the driver order (every triple for systems of
fewer than 2,500 triples), and input checksums.  Inputs come from the oracle's restatement of the
counter-based generator (oracle.synth_system), so nothing from the product library is involved.

Run from the repository root where the reference sources exist (about 12 minutes on 8 cores):
    make -C oracle && python tests/golden/make_golden_large.py [c2|c3|c4 ...]
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

SEED = 2024
STRIDE = 13
FULL_BELOW = 2500
WORKLOADS = {
    "c2": ("big_c2_o40_v300", 0, [(40, 300, SEED)]),
    "c3": ("big_c3_o30_v400_log", 1, [(30, 400, SEED)]),
    "c4": ("big_c4_six", 0, [(o, v, SEED + q) for q, (o, v) in
                             enumerate([(8, 80), (12, 150), (16, 220), (24, 310), (32, 380), (40, 450)])]),
}


def checksums(s):
    return {n: [float(np.sum(a)), float(np.sum(a * a))] for n, a in s.arrays.items()}


def one_system(nocc, nvir, seed, dist):
    s = O.synth_system(nocc, nvir, seed=seed, dist=dist, a=nocc + 1)
    t0 = time.time()
    rec, tot, mism = O.run_system(s, "reference", nthreads=os.cpu_count() or 1)
    assert mism == 0
    n = len(rec)
    stride = 1 if n < FULL_BELOW else STRIDE
    idx = np.arange(0, n, stride)
    print(f"  ({nocc},{nvir}) seed {seed}: {n} triples in {time.time() - t0:.0f} s, emp4={tot[0]!r} emp5={tot[1]!r}",
          flush=True)
    return {"ncor": 0, "nocc": nocc, "nvir": nvir, "a": s.a, "seed": seed, "dist": dist, "nkpass": 1,
            "triples_total": n, "record_stride": stride, "checksums": checksums(s),
            "record_index": idx.tolist(), "records": rec[idx].tolist(),
            "emp4": float(tot[0]), "emp5": float(tot[1])}


def main():
    if os.environ.get("OMP_NUM_THREADS") is None:
        # the triples run in parallel; each reference call is then single-threaded inside (nested
        # OpenMP off, OpenBLAS on one thread), so every record has a fixed reduction order
        os.execvpe(sys.executable, [sys.executable, os.path.abspath(__file__), *sys.argv[1:]],
                   dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1), OPENBLAS_NUM_THREADS="1",
                        OMP_MAX_ACTIVE_LEVELS="1"))
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for key in (sys.argv[1:] or list(WORKLOADS)):
        name, dist, shapes = WORKLOADS[key]
        print(name, flush=True)
        doc = {"source": "oracle/_ref/libtrpdrv_ref.so = reference omp/ccsd_trpdrv_omp_cbody.c + "
                         "omp/ccsd_tengy_c99.c, unmodified, every triple of one a per system",
               "generator": "oracle_synth_fill (splitmix64 counter stream, the product generator's recipe)",
               "systems": [one_system(o, v, sd, dist) for o, v, sd in shapes]}
        with open(os.path.join(out_dir, name + ".json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
