"""Benchmark of the CCSD(T) triples body on B200: one JSON line on rank 0.

Default workload: the fused persistent FP64 kernel over every (i,j,k) triple of one `a` at
nocc=40, nvir=300 (32,800 triples, 16.06 TFLOP per step), seeded synthetic inputs resident in HBM
(1.52 GB > the 126 MB L2, so no L2 flush is needed between steps).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload c2|c3|c4]

--impl b200 (default): `value` = triples/s of the fused kernel on device-resident inputs (CUDA events,
  max over ranks); `e2e` = the same metric through the C ABI with host buffers (pinned host -> device
  copy of every input tensor, execute, device -> host read of the energies inside the timed region;
  one trpdrv_plan_upload_execute call, which copies T2/JOV/KOV span by span under the fused kernel,
  with the upload-then-execute figure beside it);
  `roofline` = FP64 tensor-pipe fraction of the fused kernel against the FP64 DMMA peak measured live
  by the library's probe; `plain_gpu` = the plain per-triple GPU path (16 GEMMs + tengy per triple) on a
  bounded sample; `cpu_baseline` = the reference's own CPU body (oracle/_ref, OpenBLAS) on a bounded
  sample with all host threads (rank 0, N = 1 only).
--impl reference: the reference's CPU path alone (oracle/_ref/libtrpdrv_ref.so: the reference
  omp/ccsd_trpdrv_omp_cbody.c + omp/ccsd_tengy_c99.c compiled unmodified), each step a bounded sample of
  the same workload's triples; rank 0 only.
  The default line also carries `emulated`: the emulated-FP64 form (Ozaki int8 digit slices on the
  tcgen05 tensor cores, TRPDRV_MODE_EMULATED) on the same inputs for 5..8 slices, with its speedup over
  the native FP64 fused kernel, its error against it and its int8 rate against the device's int8 peak
  (the larger of cuBLASLt's int8 GEMM and the library's tcgen05 issue probe at N = 256).
--workload c3: the emulated form at nocc=30, nvir=400 with log-uniform integral magnitudes in
  [1e-6, 1]: `value` = triples/s of the emulated form (7 slices), beside the native FP64 fused kernel
  on the same system and the slice sweep with its errors.
--workload c1: the plain per-triple FP64 path (one grouped 16-GEMM launch and one tengy launch per
  triple) at nocc=20, nvir=200, every triple per step, beside the reference's CPU body.
--workload c4: six systems of uneven size, (8,80) (12,150) (16,220) (24,310) (32,380) (40,450), in
  one fused FP64 launch: `value` = aggregate triples/s; per-system energies checked against
  single-system plans; compared with one plain FP64 launch pair per triple, serially per system.
--probe-int8: the tcgen05 int8 issue-probe table (N = 64 / 128 / 256 for one SM, a CTA pair and the
  contraction kernel's stage handshake) as one JSON line; nothing else runs.
With torchrun (N > 1) every rank runs the whole workload for its own virtual index a (weak scaling: the
a loop of the full (T) is what partitions into independent units; `value` counts the triples of all
ranks), and one NCCL all-reduce of the energies per step sums the ranks' (T) contributions.  With
--scaling strong the triples of one a are split over the ranks instead.
"""
import os

# The reference arm times the reference's CPU path (OpenMP tengy + OpenBLAS, serial body calls) with a
# passive OpenMP wait policy: libgomp reads its environment when it is first loaded, so this precedes
# every import.  The B200 arm runs its CPU baseline as a separate reference-arm process.
import sys  # noqa: E402

if "--impl" in sys.argv and sys.argv[sys.argv.index("--impl") + 1:][:1] == ["reference"]:
    os.environ.setdefault("OMP_WAIT_POLICY", "passive")

import argparse  # noqa: E402
import json  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import time  # noqa: E402

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200"))

METRIC = "(T) triples/s & FP64-equiv TFLOP/s, fused/emulated vs plain FP64 GPU"
NOCC, NVIR, SEED = 40, 300, 2024
C1 = (20, 200)
C3 = (30, 400)
C4 = [(8, 80), (12, 150), (16, 220), (24, 310), (32, 380), (40, 450)]
SLICES = (5, 6, 7, 8)
DEFAULT_SLICES = 7
TARGET_DIGITS = 11  # emp4/emp5 relative error bar of the plain FP64 form


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nocc", type=int, default=None, help="default 40 (c2) / 30 (c3)")
    ap.add_argument("--nvir", type=int, default=None, help="default 300 (c2) / 400 (c3)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--mma-k", type=int, default=8, choices=[4, 8, 16], help="FP64 MMA shape of the fused kernel (before autotuning)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="N > 1: weak = every rank runs the whole workload for its own virtual index a (the "
                         "outer loop of the full (T)); strong = the triples of one a are split over the ranks")
    ap.add_argument("--no-emulated", action="store_true", help="skip the emulated-FP64 sweep of the default line")
    ap.add_argument("--no-sub-legs", action="store_true",
                    help="skip the default line's c3 / c4 sub-legs (N = 1) and strong split (N > 1)")
    ap.add_argument("--profile", action="store_true",
                    help="the timed plan only (c2/c4: fused FP64; c3: emulated, 7 slices), no probes, e2e, plain "
                         "or CPU legs: the command profiled with ncu")
    ap.add_argument("--probe-int8", action="store_true",
                    help="print the tcgen05 int8 issue-probe table (N = 64/128/256; one SM, CTA pair, stage "
                         "handshake) as one JSON line and exit")
    args = ap.parse_args()
    if args.profile:
        args.no_cpu_baseline = args.no_plain = True
        args.no_emulated = args.workload != "c3"
    dn, dv = {"c1": C1, "c3": C3}.get(args.workload, (NOCC, NVIR))
    args.nocc = dn if args.nocc is None else args.nocc
    args.nvir = dv if args.nvir is None else args.nvir
    return args


def workload_text(name, nocc, nvir):
    n = nocc * nocc * (nocc + 1) // 2
    if name == "c1":
        return (f"plain per-triple FP64 path (one grouped 16-GEMM launch + one tengy launch per triple), "
                f"nocc={nocc} nvir={nvir}, all {n} (i,j,k) triples of one a per step")
    if name == "c3":
        return (f"emulated-FP64 triples body (Ozaki int8 digit slices on tcgen05, {DEFAULT_SLICES} slices, "
                f"FP64 energies), nocc={nocc} nvir={nvir}, log-uniform integral magnitudes in [1e-6, 1], "
                f"all {n} (i,j,k) triples of one a per step")
    return f"fused persistent FP64 triples body, nocc={nocc} nvir={nvir}, all {n} (i,j,k) triples of one a per step"


def workload(nocc, nvir, name="c2"):
    n = nocc * nocc * (nocc + 1) // 2
    return {"workload": workload_text(name, nocc, nvir), "nocc": nocc, "nvir": nvir, "triples_per_step": n,
            "flop_per_triple": 16.0 * nvir * nvir * (nvir + nocc),
            "l2": "inputs resident in HBM exceed the 126 MB L2; no flush between steps"}


# ------------------------------------------------------------------------------------------------
# CPU reference path (test infrastructure: oracle/_ref is the reference compiled unmodified)
# ------------------------------------------------------------------------------------------------
def time_reference_cpu(nocc, nvir, budget_s=12.0, seed=None, dist=0, min_triples=16):
    """Times the reference body (omp/ccsd_trpdrv_omp_cbody.c + omp/ccsd_tengy_c99.c, unmodified, OpenBLAS)
    over consecutive triples of the synthetic system, serially as omp/test.c:160-195 calls it (the body
    accumulates emp4/emp5 itself; nothing else runs), each call using every host thread (OpenMP +
    OpenBLAS).  Inputs come from the oracle's restatement of the generator, so nothing of the product
    is loaded.  Returns (triples/s, triples timed, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C
    import glob
    import oracle as O
    ncpu = os.cpu_count() or 1
    O.ref()
    for so in glob.glob(os.path.join(O._scipy_libs(), "libscipy_openblas-*.so")):
        ob = C.CDLL(so)
        ob.scipy_openblas_set_num_threads.argtypes = [C.c_int]
        ob.scipy_openblas_set_num_threads(ncpu)
    s = O.synth_system(nocc, nvir, seed=SEED if seed is None else seed, dist=dist, a=nocc + 1)
    O.time_body(s, "reference", t_begin=0, t_end=2)  # warm-up (thread pools, pages)
    n_all = nocc * nocc * (nocc + 1) // 2
    done, t0, chunk = 0, time.perf_counter(), 4
    e4 = e5 = 0.0
    while True:
        hi = min(n_all, done + chunk)
        e4, e5 = O.time_body(s, "reference", t_begin=done, t_end=hi, emp4=e4, emp5=e5)
        done = hi
        el = time.perf_counter() - t0
        if done >= n_all or (el >= budget_s and done >= min_triples):
            break
    return done / el, done, el, ncpu


def workload_shapes(name, nocc, nvir):
    """(nocc, nvir, seed, dist) of every system of a workload."""
    if name == "c4":
        return [(o, v, SEED + q, 0) for q, (o, v) in enumerate(C4)]
    return [(nocc, nvir, SEED, 1 if name == "c3" else 0)]


def parallelism_text(gpus, scaling, nsys=1):
    if scaling == "weak":
        return (f"{gpus} rank(s), each running the whole workload for its own virtual index a (weak scaling); "
                f"one all-reduce of {2 * nsys} doubles per step sums the (T) contributions")
    return f"triples sharded over {gpus} rank(s), one all-reduce of {2 * nsys} doubles per step"


def config_for(args):
    """The `config` object of the line, identical in both arms for the same arguments."""
    shapes = workload_shapes(args.workload, args.nocc, args.nvir)
    mult = args.gpus if args.scaling == "weak" else 1  # weak scaling: every rank runs the whole workload
    counts = [mult * o * o * (o + 1) // 2 for o, _, _, _ in shapes]
    l2 = "inputs resident in HBM exceed the 126 MB L2; no flush between steps"
    if args.workload == "c4":
        return {"workload": "fused persistent FP64 triples body over six systems of uneven size in one launch: "
                            + ", ".join(f"({o},{v})" for o, v, _, _ in shapes) + f"; all {sum(counts)} triples of "
                            f"one a each",
                "systems": [{"nocc": o, "nvir": v, "triples": c} for (o, v, _, _), c in zip(shapes, counts)],
                "triples_per_step": sum(counts),
                "flop_per_step": sum(c * 16.0 * v * v * (v + o) for c, (o, v, _, _) in zip(counts, shapes)),
                "l2": l2, "parallelism": parallelism_text(args.gpus, args.scaling, len(shapes))}
    cfg = workload(args.nocc, args.nvir, args.workload)
    cfg["triples_per_step"] = counts[0]
    if args.workload == "c3":
        cfg["slices"] = DEFAULT_SLICES
    if args.workload == "c1":
        cfg["l2"] = "inputs (0.17 GB) exceed the 126 MB L2; no flush between steps"
    cfg["parallelism"] = parallelism_text(args.gpus, args.scaling)
    return cfg


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    shapes = workload_shapes(args.workload, args.nocc, args.nvir)
    counts = [o * o * (o + 1) // 2 for o, _, _, _ in shapes]
    weights = [c * 16.0 * v * v * (v + o) for c, (o, v, _, _) in zip(counts, shapes)]
    n_all, flop_all = sum(counts), sum(weights)
    budget = 4.0 / len(shapes)
    vals, secs, per_step = [], [], None
    for step in range(args.warmup + args.steps):
        sec, sec_full, timed, ncpu = 0.0, 0.0, 0, os.cpu_count()
        for c, (o, v, sd, dist) in zip(counts, shapes):
            rate, n, el, ncpu = time_reference_cpu(o, v, budget_s=budget, seed=sd, dist=dist,
                                                   min_triples=4 if len(shapes) > 1 else 16)
            sec += el
            sec_full += c / rate  # the system's full triple count at its sampled rate
            timed += n
        per_step = (timed, ncpu)
        if step >= args.warmup:
            vals.append(n_all / sec_full)
            secs.append(sec)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "triples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs),
        "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded counter-based generator, reference config distributions)",
        "config": config_for(args),
        "cpu_baseline": {"value": value, "unit": "triples/s", "cores": per_step[1], "kind": "reference",
                         "sample": f"each step: {per_step[0]} consecutive triples of the driver order (every "
                                   f"system sampled, about {budget:.0f} s each), serial calls of the reference "
                                   f"body with {per_step[1]} OpenMP (passive wait) + OpenBLAS threads; "
                                   f"ms_per_step is the sampled step, value the full workload's triples over "
                                   f"the time the sampled rate(s) give it"},
        "e2e": {"value": value, "unit": "triples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "tflops_fp64_equiv": value * flop_all / n_all / 1e12,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
# B200 arm
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [[c.strip() for c in ln.split(",")] for ln in out.splitlines() if ln.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        power = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        load = [v for v in sm if v > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(power) if power else None}


def read_profile_traffic():
    """DRAM bytes per fused launch from the committed ncu summary (profiles/), or None."""
    path = os.path.join(ROOT, "profiles", "fused_tma_nocc40_nvir300.md")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        ln = ln.lstrip("*- \t")
        if ln.startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Ranks:
    """torch.distributed plumbing: one process per GPU, NCCL; everything here is a no-op at N = 1."""

    def __init__(self):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(self.local)
        self.dev = torch.device("cuda", self.local)
        if self.world > 1:
            import datetime
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=self.dev)
        # a stream of our own: the library's launches and the timing events go to the same stream (a
        # handle of 0 would make each plan fall back to its own stream, which the events would not see)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.sp = self.stream.cuda_stream
        assert self.sp != 0
        self.set_scaling("strong")

    def set_scaling(self, scaling):
        """weak: each rank's plans take the whole workload (for its own a); strong: plans split it."""
        self.weak = scaling == "weak"
        self.shard = dict(rank=0, world=1) if self.weak else dict(rank=self.rank, world=self.world)
        self.mult = self.world if self.weak else 1  # workloads per step, summed over ranks

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def sum(self, vals):
        if self.world == 1:
            return list(vals)
        t = self.torch.tensor(list(vals), dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t)
        return t.tolist()

    def max(self, v):
        if self.world == 1:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def probe_fp64_peak(kind, device):
    """TFLOP/s of the FP64 issue-rate probe (lib/libtrpdrv_probe.so, a measurement tool built beside the
    library): kind 1..3 = DMMA m16n8k4/k8/k16 with register operands, 4 = scalar DFMA."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib", "libtrpdrv_probe.so"))
    lib.trpdrv_probe_fp64_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.trpdrv_probe_fp64_peak.restype = C.c_int
    out = C.c_double()
    rc = lib.trpdrv_probe_fp64_peak(device, kind, C.byref(out))
    if rc:
        raise RuntimeError(f"FP64 probe kind {kind} failed with CUDA error {rc}")
    return out.value


def probe_int8_peak(n, device, flags=0):
    """TOPS of the int8 issue-rate probe (lib/libtrpdrv_probe.so): tcgen05.mma.kind::i8 K=32 with the given
    N, digit-like shared-memory operands in the emulated form's order; flags 0 = one issuing thread per
    SM (M=128), 1 = CTA pairs (cta_group::2, M=256), 2 = one SM behind the contraction kernel's two-stage
    stage handshake."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib", "libtrpdrv_probe.so"))
    lib.trpdrv_probe_int8_rate.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.trpdrv_probe_int8_rate.restype = C.c_int
    out = C.c_double()
    rc = lib.trpdrv_probe_int8_rate(device, n, flags, C.byref(out))
    if rc:
        raise RuntimeError(f"int8 probe N={n} flags={flags} failed with status {rc}")
    return out.value


def run_int8_probe_table():
    """--probe-int8: the issue rate of every probe form on GPU 0, with cycles per instruction per SM."""
    import torch
    props = torch.cuda.get_device_properties(0)
    clock_hz = 1.965e9
    rows = []
    for flags, form in ((0, "one SM, M=128"), (1, "CTA pair, M=256"), (2, "one SM, M=128, stage handshake")):
        for n in (64, 128, 256):
            tops = probe_int8_peak(n, 0, flags)
            # per SM and instruction: 128 rows x N x 32 multiply-adds, 2 operations each
            cyc = 2.0 * 128 * n * 32 * props.multi_processor_count / (tops * 1e12) * clock_hz
            rows.append({"form": form, "n": n, "tops": round(tops, 1), "cycles_per_instruction_at_1965mhz": round(cyc, 1)})
    print(json.dumps({"int8_issue_probe": rows, "device": props.name, "sms": props.multi_processor_count}), flush=True)


def measure_peaks(T, R, skip):
    """FP64: the library's probes (DMMA m16n8k4/k8/k16, DFMA) and cuBLAS DGEMM 8192^3.  int8: cuBLASLt int8
    GEMM 8192^3 (torch._int_mm) and the library's tcgen05 int8 issue probe at N = 64 (the emulated form's
    instruction) and N = 256; the larger of cuBLASLt and the N = 256 probe is the denominator of the
    emulated form's tensor-pipe fraction."""
    torch = R.torch
    probe, cublas_dgemm, int8, int8_mma = {1: 0.0, 2: 0.0, 3: 0.0, 4: 0.0}, 0.0, None, {}
    if skip:
        return probe, cublas_dgemm, int8, int8_mma
    probe = {k: probe_fp64_peak(k, R.local) for k in (1, 2, 3, 4)}
    int8_mma = {n: probe_int8_peak(n, R.local) for n in (64, 256)}

    def best_of(fn, flop, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return reps * flop / (e0.elapsed_time(e1) * 1e-3) / 1e12

    a = torch.randn(8192, 8192, dtype=torch.float64, device=R.dev)
    cublas_dgemm = best_of(lambda: torch.matmul(a, a), 2 * 8192 ** 3)
    del a
    try:
        ai = torch.randint(-64, 65, (8192, 8192), dtype=torch.int8, device=R.dev)
        int8 = best_of(lambda: torch._int_mm(ai, ai), 2 * 8192 ** 3, reps=10)
        del ai
    except Exception:
        int8 = None
    return probe, cublas_dgemm, int8, int8_mma


def time_plan(T, R, plan, steps, warmup):
    """Device time per step (CUDA events on the launching stream, max over ranks), the plan's kernel time
    per step (events around its launches), launches, and the all-reduced per-system energies."""
    torch = R.torch

    def step():
        plan.execute(stream=R.sp)
        e4, e5 = plan.energies()
        return R.sum(list(e4) + list(e5))

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    R.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms, launches, tot = [], 0, None
    start.record(R.stream)
    for _ in range(steps):
        tot = step()
        kernel_ms.append(plan.last_kernel_ms())
        launches += plan.last_launches()
    end.record(R.stream)
    torch.cuda.synchronize()
    R.barrier()
    torch.cuda.synchronize()
    elapsed = R.max(start.elapsed_time(end) * 1e-3)
    n = len(plan.systems)
    return elapsed / steps, statistics.mean(kernel_ms), launches, tot[:n], tot[n:]


def time_e2e(T, R, plan, steps, warmup, streamed=False):
    """Through the C ABI with host buffers: pinned host -> device copy of every input, execute, device ->
    host read of the energies; seconds per step, max over ranks.  streamed: one
    trpdrv_plan_upload_execute call (T2/JOV/KOV copied span by span under the fused kernel), else
    trpdrv_plan_upload then trpdrv_plan_execute."""
    torch = R.torch
    times = []
    for it in range(warmup + steps):
        torch.cuda.synchronize()
        R.barrier()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(R.stream)
        if streamed:
            plan.upload_execute(stream=R.sp)
        else:
            plan.upload(stream=R.sp)
            plan.execute(stream=R.sp)
        e4, e5 = plan.energies()
        t1.record(R.stream)
        torch.cuda.synchronize()
        R.sum(list(e4) + list(e5))
        el = R.max(t0.elapsed_time(t1) * 1e-3)
        if it >= warmup:
            times.append(el)
    return statistics.mean(times)


def emulated_ops_per_triple(nocc, nvir, slices):
    """Algorithmic int8 operations of one triple in the emulated form: two 2V x 2V x (V + O) products
    per digit pair, slices (slices + 1) / 2 digit pairs, 2 operations per multiply-add."""
    return 2 * (2 * nvir) ** 2 * (nvir + nocc) * 2 * slices * (slices + 1) / 2


def emulated_sweep(T, R, systems, ref_e4, ref_e5, steps, warmup, slice_list, int8_peak, fp64_peak=None,
                   int8_n64=None):
    """The emulated form on the same systems for each slice count: triples/s, FP64-equivalent TFLOP/s,
    int8 tensor-pipe rate (against the device's int8 peak, and against the issue rate of the N = 64
    instruction the form uses) and its error against the native FP64 fused result."""
    out = {}
    n_all = R.mult * sum(T.count_triples(s.nocc) for s in systems)  # every rank's triples
    flop = R.mult * sum(T.count_triples(s.nocc) * T.triple_flops(s.nocc, s.nvir) for s in systems)
    for sl in slice_list:
        with T.Plan(systems, mode=T.MODE_EMULATED, slices=sl, **R.shard, device=R.local) as p:
            p.upload(stream=R.sp)
            tune = p.autotune()
            sec, kms, launches, e4, e5 = time_plan(T, R, p, steps, warmup)
            mine = sum(p.num_triples(q) * emulated_ops_per_triple(s.nocc, s.nvir, sl) for q, s in enumerate(systems))
        ops = R.sum([mine])[0]
        r4 = max(abs(a - b) / abs(b) for a, b in zip(e4, ref_e4))
        r5 = max(abs(a - b) / abs(b) for a, b in zip(e5, ref_e5))
        int8_tops = ops / sec / 1e12
        out[str(sl)] = {"value": n_all / sec, "unit": "triples/s", "ms_per_step": 1e3 * sec,
                        "tflops_fp64_equiv": flop / sec / 1e12, "kernel_ms": kms, "gpu_launches": launches,
                        "int8_tops": int8_tops, "int8_frac": (int8_tops / int8_peak) if int8_peak else None,
                        "int8_frac_of_n64_issue": (int8_tops / int8_n64) if int8_n64 else None,
                        "emp4_rel_err_vs_fp64": r4, "emp5_rel_err_vs_fp64": r5,
                        "fp64_roofline_frac": (flop / sec / 1e12) / fp64_peak if fp64_peak else None,
                        "batch": tune["candidates"][tune["chosen"]]["batch"]}
    # the 1e-11 relative accuracy target on emp4 and emp5: the autotuner picks the slice count
    with T.Plan(systems, mode=T.MODE_EMULATED, target_digits=TARGET_DIGITS, **R.shard,
                device=R.local) as p:
        p.upload(stream=R.sp)
        tune = p.autotune()
        sec, kms, launches, e4, e5 = time_plan(T, R, p, steps, warmup)
    r4 = max(abs(a - b) / abs(b) for a, b in zip(e4, ref_e4))
    r5 = max(abs(a - b) / abs(b) for a, b in zip(e5, ref_e5))
    out["target"] = {"target_digits": TARGET_DIGITS, "slices": tune["slices"], "est_rel_err": tune["est_rel_err"],
                     "value": n_all / sec, "unit": "triples/s", "ms_per_step": 1e3 * sec,
                     "tflops_fp64_equiv": flop / sec / 1e12,
                     "fp64_roofline_frac": (flop / sec / 1e12) / fp64_peak if fp64_peak else None,
                     "emp4_rel_err_vs_fp64": r4, "emp5_rel_err_vs_fp64": r5, "gpu_launches": launches,
                     "batch": tune["candidates"][tune["chosen"]]["batch"] if tune["candidates"] else None}
    return out


def plain_sample(T, R, s, flop_triple, frac=16):
    """The plain per-triple path (BASELINE config 1's method) on 1/frac of one system's triples."""
    torch = R.torch
    with T.Plan([s], mode=T.MODE_PLAIN, rank=0, world=frac, device=R.local) as pp:
        pp.upload(stream=R.sp)
        pp.execute(stream=R.sp)
        pp.energies()
        pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        pe0.record(R.stream)
        pp.execute(stream=R.sp)
        pe1.record(R.stream)
        pp.energies()
        pms = pe0.elapsed_time(pe1)
        nplain = pp.num_triples(0)
    return {"value": nplain / (pms * 1e-3), "unit": "triples/s",
            "sample": f"{nplain} triples (1/{frac} of nocc={s.nocc} nvir={s.nvir}, driver order), one grouped "
                      f"16-GEMM launch + one tengy launch per triple",
            "tflops_fp64_equiv": nplain * flop_triple / (pms * 1e-3) / 1e12}


def dropin_leg(T, s, ntrip=512):
    """The reference-facing entry point ccsd_trpdrv_omp_cbody_ called once per triple from host buffers,
    as omp/test.c:160-195 calls it (wall clock: every call returns its energies to the host).  The
    39 arguments of every call are prepared before the timed loop (raw addresses), so the loop is one
    foreign call per triple.  Timed with per-call copies of the slices (the default) and with the
    system's arrays registered as unchanging (trpdrv_register_host: no per-call transfer)."""
    import ctypes as C
    ijkl = T.enumerate_triples(s.nocc, 1)[:ntrip]
    # pageable host memory, like the reference driver's own arrays (omp/test.c:112-146)
    s = T.System(s.ncor, s.nocc, s.nvir, s.a, {k: np.array(v, copy=True) for k, v in s.arrays.items()})
    fn = C.CFUNCTYPE(None, *([C.c_void_p] * 39))(C.cast(T.lib.ccsd_trpdrv_omp_cbody_, C.c_void_p).value)
    f = np.zeros((8, s.nvir * s.nvir))
    emp = np.zeros(2)
    fp = [f[q].ctypes.data for q in (0, 1, 2, 3, 4, 5, 6, 7)]  # f1n f1t f2n f2t f3n f3t f4n f4t
    keep, calls = [], []
    for i, j, k, klo in ijkl:
        ints = np.array([s.ncor, s.nocc, s.nvir, s.a, i, j, k, klo], dtype=np.int32)
        keep.append(ints)
        sl = T.triple_slices(s, int(i), int(j), int(k), int(klo))
        calls.append(tuple(fp + [sl["eorb"].ctypes.data] + [ints.ctypes.data + 4 * q for q in range(3)] +
                           [emp.ctypes.data, emp.ctypes.data + 8] + [ints.ctypes.data + 4 * q for q in range(3, 8)] +
                           [sl[n].ctypes.data for n in T.BODY_ORDER]))
    out = {}
    for label in ("per_call_copies", "registered_inputs"):
        if label == "registered_inputs":
            T.register_system(s)
        for args in calls[:8]:  # warm-up
            fn(*args)
        emp[:] = 0.0
        t0 = time.perf_counter()
        for args in calls:
            fn(*args)
        el = time.perf_counter() - t0
        if label == "registered_inputs":
            T.unregister_system(s)
        out[label] = {"value": len(calls) / el, "unit": "triples/s", "emp4": float(emp[0]), "emp5": float(emp[1])}
    out["sample"] = (f"the first {len(calls)} triples of the driver order at nocc={s.nocc} nvir={s.nvir}, one "
                     f"ccsd_trpdrv_omp_cbody_ call each from pageable host buffers (wall clock; arguments prepared "
                     f"before the timed loop)")
    return out


def cpu_leg(args, R, workload_name=None):
    """The reference's CPU body on this host's cores: the reference arm of this script run as its own
    process (only the oracle's libraries loaded, passive OpenMP wait), three steps of about 4 s."""
    if R.rank != 0 or R.world != 1 or args.no_cpu_baseline:
        return None
    wl = workload_name or args.workload
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", "3", "--warmup", "1",
           "--workload", wl]
    if wl in ("c1", "c2", "c3"):
        cmd += ["--nocc", str(args.nocc), "--nvir", str(args.nvir)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env, check=True).stdout
        line = json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])
        cb = dict(line["cpu_baseline"])
        cb["sample"] = "a reference-arm process of this script (" + " ".join(cmd[2:]) + "): " + cb["sample"]
        return cb
    except Exception as ex:  # the reference build is missing
        return {"value": None, "unit": "triples/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"unavailable: {ex}"}


def base_line(args, R, value, sec, config):
    return {"metric": METRIC, "value": value, "unit": "triples/s", "n_gpus": R.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
            "scaling": "weak" if R.weak else "strong",
            "vs_baseline": None, "data": "synthetic (seeded counter-based generator, reference config distributions)",
            "config": config}


def fp64_roofline(achieved, peak, traffic, kms):
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": traffic,
            "peak_source": "measured live on this device: max of the FP64 probes (lib/libtrpdrv_probe.so) (DMMA m16n8k4/k8/k16 "
                           "and DFMA, register operands, 50 ms bursts) and cuBLAS DGEMM 8192^3; "
                           "MEASURED_PEAKS.json has no FP64 entry",
            "kernel_ms": kms}


def reference_fixture(name):
    """Totals the reference itself computed for a full-size workload (tests/golden/make_golden_large.py):
    a list of {"nocc", "nvir", "emp4", "emp5"} per system, or None when the fixture is absent."""
    path = os.path.join(ROOT, "tests", "golden", name + ".json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return [{k: g[k] for k in ("nocc", "nvir", "emp4", "emp5")} for g in json.load(f)["systems"]]


def rel_errors(e4, e5, ref):
    if not ref:
        return None
    return [{"nocc": g["nocc"], "nvir": g["nvir"], "emp4": abs(a - g["emp4"]) / abs(g["emp4"]),
             "emp5": abs(b - g["emp5"]) / abs(g["emp5"])} for a, b, g in zip(e4, e5, ref)]


def sub_leg_c3(T, R, steps, warmup):
    """The precision workload at reduced length: nocc=30, nvir=400, log-uniform integral magnitudes,
    the emulated form at its default 7 slices and the FP64 fused kernel, both against the reference's
    totals for this system (tests/golden/big_c3_o30_v400_log.json)."""
    o, v = C3
    s = T.synth_system(o, v, seed=SEED, a=o + 1, dist=T.DIST_LOGUNIFORM)
    n = T.count_triples(o)
    out = {"workload": f"nocc={o} nvir={v}, log-uniform integral magnitudes in [1e-6, 1], all {n} triples of one a",
           "steps": steps, "warmup": warmup}
    ref = reference_fixture("big_c3_o30_v400_log")
    for label, opt in (("emulated_7", dict(mode=T.MODE_EMULATED, slices=DEFAULT_SLICES)),
                       ("fused_fp64", dict(mode=T.MODE_FUSED))):
        with T.Plan([s], **opt, device=R.local) as p:
            p.upload(stream=R.sp)
            p.autotune()
            sec, kms, launches, e4, e5 = time_plan(T, R, p, steps, warmup)
        out[label] = {"value": n / sec, "unit": "triples/s", "ms_per_step": 1e3 * sec,
                      "tflops_fp64_equiv": n * T.triple_flops(o, v) / sec / 1e12, "gpu_launches": launches,
                      "rel_err_vs_reference": rel_errors(e4, e5, ref)}
    out["speedup_emulated_vs_fp64"] = out["emulated_7"]["value"] / out["fused_fp64"]["value"]
    return out


def sub_leg_c4(T, R, steps, warmup, peak):
    """Six systems of uneven size in one fused FP64 launch, aggregate triples/s, each system's totals
    against the reference's (tests/golden/big_c4_six.json)."""
    systems = [T.synth_system(o, v, seed=SEED + q, a=o + 1) for q, (o, v) in enumerate(C4)]
    n = sum(T.count_triples(x.nocc) for x in systems)
    flop = sum(T.count_triples(x.nocc) * T.triple_flops(x.nocc, x.nvir) for x in systems)
    with T.Plan(systems, mode=T.MODE_FUSED, device=R.local) as p:
        p.upload(stream=R.sp)
        p.autotune()
        sec, kms, launches, e4, e5 = time_plan(T, R, p, steps, warmup)
    return {"workload": "six systems " + ", ".join(f"({o},{v})" for o, v in C4) + f" in one fused launch, {n} "
                        f"triples", "steps": steps, "warmup": warmup,
            "value": n / sec, "unit": "triples/s", "ms_per_step": 1e3 * sec, "tflops_fp64_equiv": flop / sec / 1e12,
            "roofline_frac": (flop / (kms * 1e-3) / 1e12) / peak, "gpu_launches": launches,
            "rel_err_vs_reference": rel_errors(e4, e5, reference_fixture("big_c4_six"))}


def strong_split(T, R, args, steps, warmup):
    """N > 1: the triples of the c2 system's first a split over the ranks (strong scaling), beside the
    default split over a; every rank takes part (the same collective steps on all ranks)."""
    s = T.synth_system(args.nocc, args.nvir, seed=SEED, a=args.nocc + 1)
    with T.Plan([s], mode=T.MODE_FUSED, rank=R.rank, world=R.world, device=R.local) as p:
        p.upload(stream=R.sp)
        sec, kms, launches, e4, e5 = time_plan(T, R, p, steps, warmup)
    n = T.count_triples(args.nocc)
    return {"value": n / sec, "unit": "triples/s", "ms_per_step": 1e3 * sec, "n_gpus": R.world,
            "workload": f"the {n} triples of one a at nocc={args.nocc} nvir={args.nvir}, split over the ranks",
            "emp4": e4[0], "emp5": e5[0]}


def run_c1(args, T, R, systems, in_bytes, n_all, flop_all, probe, cublas_dgemm, fp64_probe, peak):
    """the plain per-triple path on every triple of (20, 200), checked against the fused
    FP64 kernel on the same inputs (both are checked against the reference by the tests)."""
    with T.Plan(systems, mode=T.MODE_PLAIN, **R.shard, device=R.local) as p:
        p.upload(stream=R.sp)
        clocks = ClockSampler(R.local)
        clocks.start()
        time.sleep(0.3)
        sec, kms, launches, e4, e5 = time_plan(T, R, p, args.steps, args.warmup)
        ck = clocks.stop()
        rec = p.triple_energies(0)
        my_flop = p.num_triples(0) * T.triple_flops(args.nocc, args.nvir)
        e2e_sec = None if args.profile else time_e2e(T, R, p, args.steps, args.warmup)
    with T.Plan(systems, mode=T.MODE_FUSED, **R.shard, device=R.local) as f:
        f.upload(stream=R.sp)
        fsec, _, _, f4, f5 = time_plan(T, R, f, 1, 1)
        frec = f.triple_energies(0)
    dev = float(np.max(np.abs(rec - frec) / np.maximum(np.max(np.abs(frec), axis=0), 1e-300)))
    if R.rank != 0:
        R.close()
        return
    cfg = config_for(args)
    achieved = my_flop / (kms * 1e-3) / 1e12
    line = base_line(args, R, n_all / sec, sec, cfg)
    line.update({
        "dtype": "f64", "tflops_fp64_equiv": flop_all / sec / 1e12,
        "roofline": fp64_roofline(achieved, peak, None, kms), "fp64_probe_tflops": fp64_probe,
        "e2e": {"value": (n_all / e2e_sec) if e2e_sec else None, "unit": "triples/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": 16,
                "path": "trpdrv_plan_upload (pinned host) + trpdrv_plan_execute + trpdrv_plan_energies"},
        "gpu_launches": launches, "clocks": ck, "emp4": e4[0], "emp5": e5[0],
        "fused_fp64": {"value": n_all / fsec, "unit": "triples/s", "records_max_rel_dev_vs_plain": dev},
        "cpu_baseline": cpu_leg(args, R),
    })
    print(json.dumps(line), flush=True)
    R.close()


def run_b200_arm(args):
    import trpdrv_b200 as T
    R = Ranks()
    R.set_scaling(args.scaling)
    # weak scaling: rank r runs the workload for its own virtual index a = first virtual + r of the same
    # molecule (block r of the a sweep: its own J, K, dintc, dintx, t1v; T2, TOV, XOV, JOV, KOV and the
    # orbital energies shared); rank 0 is the N = 1 workload
    off = R.rank if R.weak else 0

    # inputs in pinned host memory (the e2e leg copies them every step)
    pinned = []

    def alloc(n):
        t = R.torch.empty(n, dtype=R.torch.float64).pin_memory()
        pinned.append(t)
        return t.numpy()

    if args.workload == "c4":
        systems = [T.synth_system(o, v, seed=SEED + q, a=o + 1, alloc=alloc, a_block=off)
                   for q, (o, v) in enumerate(C4)]
    else:
        dist = T.DIST_LOGUNIFORM if args.workload == "c3" else T.DIST_UNIFORM
        systems = [T.synth_system(args.nocc, args.nvir, seed=SEED, a=args.nocc + 1, dist=dist, alloc=alloc,
                                  a_block=off)]
    in_bytes = sum(s.nbytes() for s in systems)
    # triples and FLOPs of one step over all ranks
    n_all = R.mult * sum(T.count_triples(s.nocc) for s in systems)
    flop_all = R.mult * sum(T.count_triples(s.nocc) * T.triple_flops(s.nocc, s.nvir) for s in systems)

    probe, cublas_dgemm, int8_cublaslt, int8_mma = measure_peaks(T, R, args.profile)
    int8_peak = max([v for v in (int8_cublaslt, int8_mma.get(256)) if v] or [0.0]) or None
    int8_peaks = {"cublaslt_8192": int8_cublaslt, "mma_probe_m128n64": int8_mma.get(64),
                  "mma_probe_m128n256": int8_mma.get(256)}
    peak = max(max(probe.values()), cublas_dgemm) or 1.0
    fp64_probe = {"dmma_m16n8k4": probe[1], "dmma_m16n8k8": probe[2], "dmma_m16n8k16": probe[3],
                  "dfma": probe[4], "cublas_dgemm_8192": cublas_dgemm}

    if args.workload == "c1":
        run_c1(args, T, R, systems, in_bytes, n_all, flop_all, probe, cublas_dgemm, fp64_probe, peak)
        return

    if args.profile and args.workload == "c3":
        with T.Plan(systems, mode=T.MODE_EMULATED, slices=DEFAULT_SLICES, **R.shard,
                    device=R.local) as p:
            p.upload(stream=R.sp)
            sec, kms, launches, e4, e5 = time_plan(T, R, p, args.steps, args.warmup)
        if R.rank == 0:
            print(json.dumps({"profile": "emulated", "slices": DEFAULT_SLICES, "nocc": args.nocc, "nvir": args.nvir,
                              "ms_per_step": 1e3 * sec, "kernel_ms": kms, "gpu_launches": launches}), flush=True)
        R.close()
        return

    # the native FP64 fused kernel (the headline of c2 and c4, the comparison of c3)
    plan = T.Plan(systems, mode=T.MODE_FUSED, **R.shard, device=R.local, mma_k=args.mma_k)
    plan.upload(stream=R.sp)
    tune = None if args.profile else plan.autotune()  # outside the timed region
    my_flop = sum(plan.num_triples(q) * T.triple_flops(s.nocc, s.nvir) for q, s in enumerate(systems))
    clocks = None
    if args.workload != "c3":
        clocks = ClockSampler(R.local)
        clocks.start()
        time.sleep(0.3)
    sec, kms, launches, e4, e5 = time_plan(T, R, plan, args.steps, args.warmup)
    ck = clocks.stop() if clocks else None
    e2e_sec = e2e_serial_sec = None
    if not args.profile and args.workload != "c3":
        e2e_sec = time_e2e(T, R, plan, args.steps, args.warmup, streamed=True)
        e2e_serial_sec = time_e2e(T, R, plan, args.steps, args.warmup)
    # per-system energies of the batch against single-system plans (c4)
    singles = None
    if args.workload == "c4":
        singles = []
        for q, s in enumerate(systems):
            with T.Plan([s], mode=T.MODE_FUSED, **R.shard, device=R.local) as p1:
                p1.upload(stream=R.sp)
                _, _, _, a4, a5 = time_plan(T, R, p1, 1, 0)
            singles.append(bool(a4[0] == e4[q] and a5[0] == e5[q]))
    plan.close()
    achieved = my_flop / (kms * 1e-3) / 1e12

    # emulated-FP64 form on the same systems
    emulated = None
    if not args.no_emulated and args.workload in ("c2", "c3"):
        if args.workload == "c3":
            clocks = ClockSampler(R.local)
            clocks.start()
            time.sleep(0.3)
        emulated = emulated_sweep(T, R, systems, e4, e5, args.steps, args.warmup, SLICES, int8_peak, peak,
                                  int8_mma.get(64))
        if args.workload == "c3":
            ck = clocks.stop()
    emu_e2e_sec = None
    if args.workload == "c3" and not args.no_emulated:
        with T.Plan(systems, mode=T.MODE_EMULATED, slices=DEFAULT_SLICES, **R.shard,
                    device=R.local) as p:
            p.upload(stream=R.sp)
            emu_e2e_sec = time_e2e(T, R, p, args.steps, args.warmup)

    # plain per-triple GPU path: a bounded sample of each system, serially
    plain = None
    if not args.no_plain and R.rank == 0:
        if args.workload == "c4":
            per = [plain_sample(T, R, s, T.triple_flops(s.nocc, s.nvir), frac=32) for s in systems]
            serial_sec = sum(T.count_triples(s.nocc) / pl["value"] for s, pl in zip(systems, per))
            plain = {"value": (n_all / R.mult) / serial_sec, "unit": "triples/s",  # one GPU
                     "sample": "1/32 of each system's triples, one grouped 16-GEMM launch + one tengy launch per "
                               "triple, systems one after another; serial time extrapolated by triple counts",
                     "tflops_fp64_equiv": (flop_all / R.mult) / serial_sec / 1e12, "per_system": per}
        else:
            s = systems[0]
            plain = plain_sample(T, R, s, T.triple_flops(s.nocc, s.nvir))

    # default line: the precision and uneven-batch workloads at reduced length, and at N > 1 the strong
    # split of one a beside the split over a
    sub = None
    if args.workload == "c2" and not args.profile and not args.no_sub_legs:
        sub = {}
        if R.world == 1:
            sub["c3"] = sub_leg_c3(T, R, 3, 1)
            sub["c4"] = sub_leg_c4(T, R, 2, 1, peak)
        elif R.weak:
            sub["strong_split"] = strong_split(T, R, args, 3, 1)
    if R.rank != 0:
        R.close()
        return
    traffic = read_profile_traffic() if args.workload == "c2" else None
    if args.workload == "c3":
        emu = emulated[str(DEFAULT_SLICES)] if emulated else None
        value = emu["value"] if emu else n_all / sec
        wsec = (emu["ms_per_step"] * 1e-3) if emu else sec
        cfg = config_for(args)
        line = base_line(args, R, value, wsec, cfg)
        line.update({
            "dtype": "int8 (emulated f64)",
            "tflops_fp64_equiv": flop_all / wsec / 1e12,
            "roofline": {"bound": "tensor", "achieved": emu["int8_tops"] if emu else None, "peak": int8_peak,
                         "unit": "TOPS (int8)", "frac": emu["int8_frac"] if emu else None, "traffic": None,
                         "peak_source": "measured live on this device: max of cuBLASLt int8 GEMM 8192^3 "
                                        "(torch._int_mm) and the tcgen05 int8 issue probe at M=128 N=256 "
                                        "(lib/libtrpdrv_probe.so); achieved = algorithmic int8 operations of the "
                                        "digit-pair products over the whole step (slicing, products and FP64 "
                                        "energies)",
                         "kernel_ms": emu["kernel_ms"] if emu else None},
            "fp64_fused": {"value": n_all / sec, "unit": "triples/s", "ms_per_step": 1e3 * sec,
                           "tflops_fp64_equiv": flop_all / sec / 1e12, "roofline_frac": achieved / peak,
                           "emp4": e4[0], "emp5": e5[0]},
            "speedup_vs_fp64_fused": (value / (n_all / sec)),
            "emulated_slices": emulated,
            "int8_peak_tops": int8_peak, "int8_peaks_tops": int8_peaks, "fp64_probe_tflops": fp64_probe,
            "e2e": {"value": (n_all / emu_e2e_sec) if emu_e2e_sec else None, "unit": "triples/s",
                    "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": 16,
                    "path": "trpdrv_plan_upload (pinned host) + trpdrv_plan_execute + trpdrv_plan_energies"},
            "gpu_launches": emu["gpu_launches"] if emu else launches,
            "clocks": ck, "plain_gpu": plain,
            "speedup_vs_plain": (value / R.world / plain["value"]) if plain else None,  # per GPU
            "cpu_baseline": cpu_leg(args, R),
        })
    else:
        value = n_all / sec
        line = base_line(args, R, value, sec, config_for(args))
        line.update({
            "dtype": "f64",
            "fused_mma": (f"m16n8k{tune['candidates'][tune['chosen']]['mma_k']} f64 (autotuned)"
                          if tune and tune.get("candidates") else f"m16n8k{args.mma_k} f64"),
            "tflops_fp64_equiv": flop_all / sec / 1e12,
            "roofline": fp64_roofline(achieved, peak, traffic, kms),
            "fp64_probe_tflops": fp64_probe,
            "e2e": {"value": (n_all / e2e_sec) if e2e_sec else None, "unit": "triples/s",
                    "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": 16 * len(systems),
                    "path": "trpdrv_plan_upload_execute (pinned host; T2/JOV/KOV copied span by span under "
                            "the fused kernel) + trpdrv_plan_energies",
                    "upload_then_execute": (n_all / e2e_serial_sec) if e2e_serial_sec else None},
            "gpu_launches": launches,
            "clocks": ck,
            "plain_gpu": plain,
            "speedup_vs_plain": (value / R.world / plain["value"]) if plain else None,  # per GPU
            "autotune": tune,
        })
        if args.workload == "c4":
            line["emp4"], line["emp5"] = e4, e5
            line["per_system_equals_single_runs"] = singles
            line["cpu_baseline"] = cpu_leg(args, R)
        else:
            line["emp4"], line["emp5"] = e4[0], e5[0]
            # the all-reduced totals are one a's (T) contribution unless N > 1 ranks each ran their own a
            one_a = (args.nocc, args.nvir) == (NOCC, NVIR) and not (R.weak and R.world > 1)
            line["rel_err_vs_reference"] = rel_errors(e4, e5, reference_fixture("big_c2_o40_v300")) if one_a else None
            line["cpu_baseline"] = cpu_leg(args, R)
            if not args.profile and not args.no_plain:
                line["dropin"] = dropin_leg(T, systems[0])
            if sub is not None:
                line.update(sub)
            if emulated:
                emu = emulated[str(DEFAULT_SLICES)]
                tgt = emulated["target"]
                line["emulated"] = {"default_slices": DEFAULT_SLICES, "value": emu["value"], "unit": "triples/s",
                                    "speedup_vs_fp64_fused": emu["value"] / value,
                                    "speedup_vs_plain": (emu["value"] / R.world / plain["value"]) if plain else None,
                                    "at_target_1e-11": {"slices": tgt["slices"], "value": tgt["value"],
                                                        "speedup_vs_fp64_fused": tgt["value"] / value,
                                                        "speedup_vs_plain": (tgt["value"] / R.world / plain["value"])
                                                        if plain else None},
                                    "int8_peak_tops": int8_peak, "int8_peaks_tops": int8_peaks,
                                    "slices": emulated}
    print(json.dumps(line), flush=True)
    R.close()


def main():
    args = parse()
    if args.probe_int8:
        run_int8_probe_table()
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_b200_arm(args)


if __name__ == "__main__":
    main()
