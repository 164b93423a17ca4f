#!/usr/bin/env python
"""Benchmark: plain single-vector HMVM y = H x on one B200 (per rank).

Workload (the GPU configuration of the reference's HMVM path): a synthetic
H-matrix built with HACApK's rules -- N=262,144 points uniform on the unit
sphere (seeded), kernel 1/(4*pi*|x-y|) with self-term 1.0, bisection cluster
tree with leaf size 32, admissibility eta=2.0, ACA eps=1e-4 -- and x uniform in
[-1,1] from the seed.  A step is one HMVM over the whole matrix (5 GB in FP64,
far larger than the 126 MB L2, so no L2 flush is needed between steps).

Arms
  (default)          the B200 library: device-resident x/y (value) and, through
                     the C ABI with pinned host buffers, H2D x + HMVM + D2H y
                     per step (e2e).
  --impl reference   the reference's own CPU HMVM (hmvm_omp_2<double,0>,
                     compiled from its sources into oracle/_ref; falls back to
                     the C restatement in oracle/) on all host cores.

Multi-GPU: the HMVM does not shard in the reference (one process, one
device); N ranks run N independent replicas ("replicas only"), value is the
total HMVM/s of all ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libhmvm_ref.so")
REF_CUDA_SO = os.path.join(ROOT, "oracle", "_ref", "libhmvm_ref_cuda.so")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "mixed"])
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--geometry", default="sphere")
    ap.add_argument("--eps", type=float, default=1e-4)
    ap.add_argument("--eta", type=float, default=2.0)
    ap.add_argument("--leaf", type=int, default=32)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bound on the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stage1-cfg", type=int, default=-1)
    ap.add_argument("--stage2-cfg", type=int, default=-1)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--kernel", type=int, default=-1, help="0: register-streaming, 1: TMA-ring (default)")
    ap.add_argument("--nrhs", type=int, default=1, help="right-hand sides per step (multi-RHS HMVM when > 1)")
    ap.add_argument("--x-dist", default="uniform", choices=["uniform", "normal"], help="entries of x / X")
    ap.add_argument("--lr-format", default="fp16", choices=["fp16", "bf16"], help="mixed plans: 16-bit factor format")
    ap.add_argument("--mesh", default=None,
                    help="single workload: the ppohBEM collocation matrix of this .pbf mesh instead of a generated one")
    ap.add_argument("--mesh-eps", type=float, default=1e-6, help="--mesh: ACA tolerance (the reference driver's 1e-6)")
    ap.add_argument("--graph", action="store_true",
                    help="nrhs 1: time CUDA-graph replays of one captured apply (stage times from a profiled pass after)")
    ap.add_argument("--workload", default="single", choices=["single", "batch"],
                    help="batch: many independent H-matrices of uneven N in one CUDA-graph replay")
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--batch-nmin", type=int, default=4096)
    ap.add_argument("--batch-nmax", type=int, default=131072)
    ap.add_argument("--batch-rhs-max", type=int, default=16)
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary workloads (FP32, mixed, multi-RHS) timed after the headline")
    ap.add_argument("--secondary-steps", type=int, default=40, help="timed steps of each single-vector secondary leg")
    ap.add_argument("--no-batch-leg", action="store_true",
                    help="default run: skip the batch workload (config C4) among the secondary legs")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own hybrid2 CUDA kernels on this GPU")
    ap.add_argument("--reference-gpu-runs", type=int, default=20, help="timed runs of the reference's GPU kernel")
    ap.add_argument("--no-cpu-variants", action="store_true",
                    help="skip the reference's full OpenMP variant sweep and its one-core hmvm_seq_2")
    return ap.parse_args()


# ---- the reference's CPU HMVM (CPU baseline / reference arm) ---------------
class CpuReference:
    """hmvm_omp_2<double,0> from the reference build (kind "reference"), else
    the oracle's restatement of it (kind "port")."""

    def __init__(self, hm):
        P = C.c_void_p
        self.nd = hm.nd
        self._i32 = [np.ascontiguousarray(getattr(hm, n), dtype=np.int32)
                     for n in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2")]
        self._rm = hm.rowmat
        # the reference's matrix2 holds int offsets (hacapk.h:28,31): beyond 2^31 elements only the port runs
        if os.path.exists(REF_SO) and hm.len <= np.iinfo(np.int32).max:
            self.kind = "reference"
            lib = C.CDLL(REF_SO)
            lib.ref_wrap2.restype = C.c_void_p
            lib.ref_wrap2.argtypes = [C.c_int] * 4 + [P] * 9
            lib.ref_omp2_d.argtypes = [C.c_void_p, P, P, C.c_int]
            lib.ref_seq2_d.argtypes = [C.c_void_p, P, P, C.c_int]
            lib.ref_omp_bench_d.argtypes = [C.c_void_p, P, C.c_char_p, C.c_int]
            lib.ref_omp_bench_d.restype = C.c_int
            lib.ref_max_threads.restype = C.c_int
            self.lib = lib
            self.h = lib.ref_wrap2(hm.nd, hm.nlf, hm.ktmax, hm.len,
                                   *[a.ctypes.data_as(P) for a in self._i32], hm.rowmat.ctypes.data_as(P))
            self.threads = int(lib.ref_max_threads())
        else:
            self.kind = "port"
            lib = C.CDLL(ORACLE_SO)
            lib.orc_omp2_d.argtypes = [C.c_int32, C.c_int32, C.c_int32] + [P] * 11 + [C.c_int]
            lib.orc_max_threads.restype = C.c_int
            self.lib = lib
            self._i64 = [self._i32[k] for k in range(6)] + [np.ascontiguousarray(hm.a1, np.int64),
                                                             np.ascontiguousarray(hm.a2, np.int64)]
            self.hm = hm
            self.threads = int(lib.orc_max_threads())

    def run(self, x, y):
        P = C.c_void_p
        if self.kind == "reference":
            self.lib.ref_omp2_d(self.h, x.ctypes.data_as(P), y.ctypes.data_as(P), 0)
        else:
            hm = self.hm
            self.lib.orc_omp2_d(hm.nd, hm.nlf, hm.ktmax, *[a.ctypes.data_as(P) for a in self._i64],
                                hm.rowmat.ctypes.data_as(P), x.ctypes.data_as(P), y.ctypes.data_as(P), 0)

    def time_sample(self, x, max_seconds):
        """The reference's own loop shape (hmvm_omp.cpp:992-1021): L runs, the
        first 5 discarded; L bounded so the sample stays near max_seconds."""
        y = np.empty(self.nd)
        t0 = time.perf_counter()
        self.run(x, y)
        one = max(time.perf_counter() - t0, 1e-6)
        L = int(min(10, max(6, max_seconds / one)))
        ts = []
        for _ in range(L):
            t0 = time.perf_counter()
            self.run(x, y)
            ts.append(time.perf_counter() - t0)
        kept = ts[5:]
        return y, dict(runs=L, kept=len(kept), min=min(kept), avg=sum(kept) / len(kept), max=max(kept))


# ---- clocks -----------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = []
        maxes = []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                maxes.append(float(r[1]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 4 + k and r[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value: float, dist, device) -> float:
    """The largest `value` over all ranks (timings are reported as the slowest rank)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


DTYPES = {"fp64": "f64", "fp32": "f32",
          "mixed": "mixed: f32/f16/e4m3 low-rank, f32/f64 dense storage; f32 segment sums, f64 rows and x, y"}

# ncu summaries that carry traffic_per_algorithmic_byte lines, by the kernel they
# captured: FP64 stream kernel, mixed kernel (FP16 factors), wide tensor-core
# kernel (mixed, FP16 factors, 128 right-hand sides)
TRAFFIC_PROFILES = {"fp64": os.path.join(ROOT, "profiles", "stream_kernel_fp64_sphere65536.md"),
                    "mixed": os.path.join(ROOT, "profiles", "mixed_kernel_fp16_sphere65536.md"),
                    "tcw": os.path.join(ROOT, "profiles", "tcw_kernel_mixed_sphere65536_nrhs128.md")}


def traffic_ratio(stage: int, precision: str = "fp64"):
    """DRAM bytes per algorithmic byte of a stage kernel, from the committed ncu
    summary (a capture of a smaller case of the same kernel), or None."""
    path = TRAFFIC_PROFILES.get(precision)
    if path is None:
        return None
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) == 3 and parts[0] == "traffic_per_algorithmic_byte" and parts[1] == f"stage{stage}":
                return float(parts[2])
    except OSError:
        pass
    return None


def measured_peak_gbs():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def build_matrix(a):
    from hacapk_hmvm_b200 import HMatrix

    if a.mesh:
        return HMatrix.from_mesh(a.mesh, eps=a.mesh_eps)
    return HMatrix.generate(a.n, a.geometry, eta=a.eta, eps=a.eps, leaf_size=a.leaf, seed=a.seed)


# The reference's published best CUDA times (hybrid2, src_hmvm/src_cpp/result/time_<matrix>_<d|f>.csv,
# hardware not stated) for the matrices whose meshes it ships: (faces, seconds per HMVM).
PUBLISHED = {"216h": (21600, {"fp64": 1.002e-3, "fp32": 6.638e-4}),
             "sample": (600, {"fp64": 1.920e-5, "fp32": 1.674e-5})}


def published_hmvm_per_s(a, hm):
    if not a.mesh or a.nrhs != 1:
        return None
    for key, (faces, t) in PUBLISHED.items():
        if key in os.path.basename(a.mesh) and hm.nd == faces and a.precision in t:
            return 1.0 / t[a.precision]
    return None


def workload_config(a, hm):
    if a.mesh:
        mb = hm.stored_elements() * (4 if a.precision == "fp32" else 8) / 1e6
        return {
            "workload": f"ppohBEM collocation matrix of {os.path.basename(a.mesh)} (N={hm.nd}, HACApK leaf 15, "
                        f"eta 2, ACA eps {a.mesh_eps:g}), single-vector HMVM, {a.precision.upper()}",
            "nrhs": a.nrhs, "n": hm.nd, "mesh": os.path.basename(a.mesh), "aca_eps": a.mesh_eps,
            "nlf": hm.nlf, "n_lowrank": int((hm.ltmtx == 1).sum()), "n_dense": int((hm.ltmtx == 2).sum()),
            "stored_elements": hm.stored_elements(), "precision": a.precision,
            "l2": (f"matrix {mb:.0f} MB, above the 126 MB L2" if mb > 126 else
                   f"matrix {mb:.1f} MB fits the 126 MB L2 (not an HBM figure)"),
            "parallelism": f"replicas x{a.gpus}",
        }
    return {
        "workload": f"{a.geometry} N={a.n} leaf={a.leaf} eta={a.eta} ACA eps={a.eps:g}, "
                    + ("single-vector HMVM, " if a.nrhs == 1 else f"multi-RHS HMVM nrhs={a.nrhs}, ")
                    + f"{a.precision.upper()}" + (f" ({a.lr_format} factors)" if a.precision == "mixed" else ""),
        "nrhs": a.nrhs,
        "n": a.n, "geometry": a.geometry, "leaf_size": a.leaf, "eta": a.eta, "aca_eps": a.eps,
        "nlf": hm.nlf, "n_lowrank": int((hm.ltmtx == 1).sum()), "n_dense": int((hm.ltmtx == 2).sum()),
        "stored_elements": hm.stored_elements(), "precision": a.precision,
        "l2": "inputs larger than L2 (the matrix streamed each step is far above 126 MB)",
        "parallelism": f"replicas x{a.gpus}",
    }


def run_reference(a, rank):
    if rank != 0:
        return
    hm = build_matrix(a)
    rng = np.random.default_rng(a.seed)
    x = rng.uniform(-1.0, 1.0, hm.nd) if a.x_dist == "uniform" else rng.standard_normal(hm.nd)
    cpu = CpuReference(hm)
    y = np.empty(hm.nd)
    for _ in range(max(a.warmup, 1)):
        cpu.run(x, y)
    # Each step is one full HMVM; cap the number of steps so the arm stays within a few minutes.
    t0 = time.perf_counter()
    cpu.run(x, y)
    one = time.perf_counter() - t0
    steps = int(max(1, min(a.steps, 120.0 / max(one, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(steps):
        cpu.run(x, y)
    dt = time.perf_counter() - t0
    value = steps / dt
    sample = f"{steps} full HMVMs (hmvm_omp_2<double,0>) over the whole matrix"
    line = {
        "impl": "reference", "metric": "HMVM/s", "value": value, "unit": "HMVM/s", "n_gpus": a.gpus,
        "steps": steps, "warmup": a.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": (f"the ppohBEM mesh {os.path.basename(a.mesh)}" if a.mesh else "synthetic (seeded HACApK-rule H-matrix")
                + f"; x {'uniform[-1,1]' if a.x_dist == 'uniform' else 'standard normal'}" + ("" if a.mesh else ")"),
        "config": workload_config(a, hm),
        "gbytes_per_s": hm.algorithmic_bytes(8) / (dt / steps) / 1e9,
        "cpu_baseline": {"value": value, "unit": "HMVM/s", "cores": cpu.threads, "kind": cpu.kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "HMVM/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# Right-hand sides from which FP32 and mixed workloads run on the wide tensor-core form.
TC_WIDE_MIN = 32  # from here the wide tensor-core form (128 right-hand sides per pass)
TC16_MIN = 16     # mixed plans from here: the 16-wide tensor-core pass


def plan_width(precision, nrhs):
    """nrhs_max of the plan a workload of nrhs right-hand sides runs on."""
    if precision in ("fp32", "mixed") and nrhs >= TC_WIDE_MIN:
        return 128
    if precision == "mixed" and nrhs >= TC16_MIN:
        return 16
    return min(nrhs, 8)


def make_plan(hm, precision, nrhs, lr_format, device, a=None):
    """The plan a workload runs on: single-vector plans for nrhs 1, multi-RHS
    plans sized for the pass width otherwise: the wide tensor-core form (128
    right-hand sides per pass) from 32 right-hand sides, the 16-wide
    tensor-core pass for mixed plans from 16."""
    from hacapk_hmvm_b200 import Plan

    kw = {}
    if a is not None:
        kw = dict(stage1_cfg=a.stage1_cfg, stage2_cfg=a.stage2_cfg, ctas_per_sm=a.ctas_per_sm, kernel=a.kernel)
    return Plan(hm, precision, device=device, nrhs_max=plan_width(precision, nrhs),
                mixed_lr_format=lr_format if precision == "mixed" else None, **kw)


def kernel_name(plan, info, nrhs):
    if info["kernel"] == 4:
        return "hmvm_tcw_kernel"
    if nrhs > 1:
        return "hmvm_tc_kernel" if (plan.precision == "mixed" and info["nrhs_max"] >= 16) else "hmvm_multi_kernel"
    return {0: "hmvm_tile_kernel", 1: "hmvm_stream_kernel", 2: "hmvm_mixed_kernel"}[info["kernel"]]


def passes_of(plan, nrhs):
    """Matrix streams per multi-RHS apply (one per pass)."""
    if nrhs <= 1:
        return 1
    per_pass = max(plan.multi_kernel_count(min(nrhs, 2)), 1)
    return max(1, plan.multi_kernel_count(nrhs) // per_pass)


def roofline_of(plan, info, nrhs, stage_ms, napplies, ms_step, precision, lr_format="fp16"):
    """Dominant kernel's achieved bandwidth (its algorithmic bytes per launch /
    its average CUDA-event duration) and the whole step's, against the
    measured HBM peak."""
    peak, peak_kind = measured_peak_gbs()
    stage_bytes = [info["stage1_bytes"], 0, info["stage2_bytes"], 0]
    dom = int(np.argmax(stage_ms))
    dom_avg_s = stage_ms[dom] / max(napplies, 1) * 1e-3
    achieved = stage_bytes[dom] / dom_avg_s / 1e9 if dom_avg_s > 0 else 0.0
    passes = passes_of(plan, nrhs)
    elem_xy = 4 if precision == "fp32" else 8
    # a multi-RHS step streams the matrix once per pass and reads/writes every column once
    alg_bytes = info["algorithmic_bytes"] * passes + 2 * plan.nd * elem_xy * (nrhs - passes)
    kname = kernel_name(plan, info, nrhs)
    ratio, tkey = None, None
    if dom in (0, 2) and nrhs == 1 and lr_format == "fp16" and (
            (info["kernel"] == 1 and precision == "fp64") or precision == "mixed"):
        tkey = precision
    elif dom in (0, 2) and info["kernel"] == 4 and precision == "mixed" and lr_format == "fp16":
        tkey = "tcw"
    if tkey:
        ratio = traffic_ratio(1 if dom == 0 else 2, tkey)
    roof = {
        "bound": "hbm",
        "kernel": [f"{kname} (V stage)", "hmvm_reduce_kernel (V stage)", f"{kname} (row stage)",
                   "hmvm_reduce_kernel (row stage)"][dom],
        "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
        "traffic": stage_bytes[dom] * ratio if ratio else None,
        "traffic_source": None,
        "whole_step_gbs": alg_bytes / (ms_step * 1e-3) / 1e9,
        "whole_step_frac": alg_bytes / (ms_step * 1e-3) / 1e9 / peak,
        "stage_ms_avg": [s / max(napplies, 1) for s in stage_ms],
        "stage_bytes": stage_bytes,
        "passes_per_step": passes,
    }
    if ratio:
        roof["traffic_source"] = ("ncu capture of the same kernel at N=65536, scaled by algorithmic bytes ("
                                  + os.path.relpath(TRAFFIC_PROFILES[tkey], ROOT) + ")")
    return roof, alg_bytes


def time_steps(step, steps, warmup, stream, dev, dist=None):
    """ms per step over `steps` timed steps after `warmup` untimed ones (CUDA
    events on the launching stream, max over ranks)."""
    import torch

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    return max_over_ranks(e0.elapsed_time(e1), dist, dev) / steps


class CpuColumns:
    """The reference CPU HMVM (hmvm_omp_2<double,0>) of columns of X, each
    computed once."""

    def __init__(self, cpu, X):
        self.cpu, self.X, self.y = cpu, X, {}

    def __call__(self, c):
        if c not in self.y:
            yc = np.empty(self.cpu.nd)
            self.cpu.run(self.X[c], yc)
            self.y[c] = yc
        return self.y[c]


def checked_columns(nrhs):
    """Every column up to 16 right-hand sides, else a fixed sample of 8."""
    if nrhs <= 16:
        return list(range(nrhs))
    return sorted(set(int(round(v)) for v in np.linspace(0, nrhs - 1, 8)))


def cpu_bench_variants(cpu, x, seq_seconds):
    """The reference's own timed sweep of its SoA OpenMP variants
    (hmvm_omp_bench, L=10 with the first 5 discarded) and hmvm_seq_2 on one
    core (the reference proxy's loop shape, bounded to about seq_seconds)."""
    out = {}
    if cpu.kind != "reference":
        return out
    import tempfile

    with tempfile.NamedTemporaryFile("r", suffix=".txt") as f:
        rc = cpu.lib.ref_omp_bench_d(cpu.h, x.ctypes.data_as(C.c_void_p), f.name.encode(), 0)
        if rc == 0:
            rows = {}
            for line in open(f.name):
                p = line.split()
                if len(p) == 9 and p[0] == "TIME":
                    rows[p[2]] = {"min_s": float(p[4]), "max_s": float(p[6]), "avg_s": float(p[8])}
            if rows:
                best = min(rows, key=lambda k: rows[k]["min_s"])
                out["omp_variants"] = rows
                out["best_omp_variant"] = {"name": best, "value": 1.0 / rows[best]["min_s"], "unit": "HMVM/s",
                                           "cores": cpu.threads}
    y = np.empty(cpu.nd)
    t0 = time.perf_counter()
    cpu.lib.ref_seq2_d(cpu.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0)
    one = max(time.perf_counter() - t0, 1e-6)
    runs = int(min(10, max(6, seq_seconds / one)))
    ts = []
    for _ in range(runs):
        t0 = time.perf_counter()
        cpu.lib.ref_seq2_d(cpu.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0)
        ts.append(time.perf_counter() - t0)
    kept = ts[5:]
    out["seq_2_one_core"] = {"value": 1.0 / min(kept), "unit": "HMVM/s", "cores": 1,
                             "sample": f"hmvm_seq_2<double,0>, {runs} runs, first 5 discarded, min of {len(kept)}"}
    return out


# The reference's fastest published GPU variants (hybrid2; src_hmvm/src_cpp/result/
# time_216h_d.csv:469 and time_216h_f.csv:379) as (kernel index, div, mul, a2t, a2i,
# aa, da); the index encodes the knobs as hmvm_cuda2.cu:395-404 decodes them.
REF_GPU_VARIANTS = {"fp64": (356, 4, 12, 1, 1, 0, 0), "fp32": (266, 4, 13, 0, 1, 0, 0)}


def reference_gpu(cpu, x, ours, nbench):
    """The reference's own hybrid2 CUDA kernels (hmvm_cuda2.cu, built unchanged
    for sm_100a into oracle/_ref) on this GPU: their TIME line from the
    reference's own wrapper, and the relative error of one launch's y against
    the reference CPU HMVM in FP64.  ours: {"fp64": HMVM/s, "fp32": HMVM/s}."""
    import tempfile

    if cpu.kind != "reference" or not os.path.exists(REF_CUDA_SO):
        return None
    P = C.c_void_p
    lib = C.CDLL(REF_CUDA_SO)
    lib.refgpu_cuda2_bench.argtypes = [P, C.c_int, P, C.c_int, C.c_int, C.c_char_p]
    lib.refgpu_hybrid2_y.argtypes = [P, C.c_int, P] + [C.c_int] * 6 + [P]
    cpu.lib.ref_matrix2_d.restype = P
    cpu.lib.ref_matrix2_f.restype = P
    cpu.lib.ref_make_float.argtypes = [P]
    y_ref = np.empty(cpu.nd)
    cpu.run(x, y_ref)
    out = {}
    for prec in ("fp64", "fp32"):
        kidx, div, mul, a2t, a2i, aa, da = REF_GPU_VARIANTS[prec]
        f32 = prec == "fp32"
        if f32 and cpu.lib.ref_make_float(cpu.h) != 0:
            continue
        m2 = cpu.lib.ref_matrix2_f(cpu.h) if f32 else cpu.lib.ref_matrix2_d(cpu.h)
        xv = np.ascontiguousarray(x, dtype=np.float32 if f32 else np.float64)
        with tempfile.NamedTemporaryFile("r", suffix=".txt") as f:
            if lib.refgpu_cuda2_bench(m2, int(f32), xv.ctypes.data_as(P), kidx, nbench, f.name.encode()) != 0:
                continue
            line = [ln.split() for ln in open(f.name) if ln.startswith("TIME")]
        if not line or len(line[0]) != 9:
            continue
        t = line[0]
        y = np.empty(cpu.nd, dtype=xv.dtype)
        rc = lib.refgpu_hybrid2_y(m2, int(f32), xv.ctypes.data_as(P), div, mul, a2t, a2i, aa, da, y.ctypes.data_as(P))
        rate = 1.0 / float(t[4])
        out[prec] = {
            "kernel": t[2] + " (src_hmvm/src_cpp/hmvm_cuda2.cu, built unchanged for sm_100a)",
            "value": rate, "unit": "HMVM/s", "time_s": {"min": float(t[4]), "max": float(t[6]), "avg": float(t[8])},
            "timing": f"the reference's own TIME line: kernel launch + cudaDeviceSynchronize timed with omp_get_wtime, "
                      f"{5 + nbench} runs with the first 5 discarded, min (hmvm_cuda2.cu:236-302)",
            "relerr_vs_fp64_cpu_reference": (float(np.linalg.norm(y.astype(np.float64) - y_ref) /
                                                   np.linalg.norm(y_ref)) if rc == 0 else None),
            "ratio_vs_reference_gpu": (ours.get(prec) / rate) if ours.get(prec) else None,
        }
    return out or None


# Secondary workloads timed after the headline on the same matrix: (label,
# precision, right-hand sides, 16-bit factor format).  Plans are built once per
# (precision, factor format, pass kind) and reused by the legs that share them.
SECONDARY = [
    ("fp32 single-vector", "fp32", 1, None),
    ("mixed single-vector, FP16 factors", "mixed", 1, "fp16"),
    ("mixed single-vector, BF16 factors", "mixed", 1, "bf16"),
    ("mixed multi-RHS nrhs=16, FP16 factors", "mixed", 16, "fp16"),
    ("mixed multi-RHS nrhs=128, FP16 factors", "mixed", 128, "fp16"),
    ("mixed multi-RHS nrhs=16, BF16 factors", "mixed", 16, "bf16"),
    ("mixed multi-RHS nrhs=128, BF16 factors", "mixed", 128, "bf16"),
    ("fp32 multi-RHS nrhs=8", "fp32", 8, None),
    ("fp32 multi-RHS nrhs=128", "fp32", 128, None),
]


def run_secondary(a, hm, X, cpucols, fp64_rate, local_rank, stream, dev):
    import torch

    legs = []
    key_of = lambda prec, nrhs, fmt: (prec, fmt, plan_width(prec, nrhs))
    plans = {}
    for i, (label, prec, nrhs, fmt) in enumerate(SECONDARY):
        key = key_of(prec, nrhs, fmt)
        try:
            legs.append(secondary_leg(a, hm, X, cpucols, fp64_rate, local_rank, stream, dev, plans, key,
                                      label, prec, nrhs, fmt))
        except Exception as e:  # one leg's failure is reported in its place; the others still run
            legs.append({"workload": label, "precision": prec, "lr_format": fmt, "nrhs": nrhs,
                         "error": f"{type(e).__name__}: {e}"})
        # close a plan after the last leg that uses it
        if key in plans and all(key_of(p2, n2, f2) != key for (_, p2, n2, f2) in SECONDARY[i + 1:]):
            plans[key][0].close()
            del plans[key]
            torch.cuda.empty_cache()
    return legs


def secondary_leg(a, hm, X, cpucols, fp64_rate, local_rank, stream, dev, plans, key, label, prec, nrhs, fmt):
    import torch

    if key not in plans:
        t0 = time.perf_counter()
        plans[key] = (make_plan(hm, prec, nrhs, fmt, local_rank), time.perf_counter() - t0)
    plan, setup_s = plans[key]
    info = plan.info()
    ndt = np.float32 if prec == "fp32" else np.float64
    tdt = torch.float32 if prec == "fp32" else torch.float64
    xd = torch.from_numpy(X[:nrhs].astype(ndt)).to(dev)
    yd = torch.full((nrhs, hm.nd), float("nan"), dtype=tdt, device=dev)
    if nrhs == 1:
        step = lambda: plan.apply(xd[0], yd[0], stream)
    else:
        step = lambda: plan.apply_multi(xd, yd, stream)
    for _ in range(2):
        step()
    torch.cuda.synchronize(dev)
    plan.profile(True)
    steps = max(3, a.secondary_steps if nrhs == 1 else a.secondary_steps // 4)
    ms = time_steps(step, steps, a.warmup, stream, dev)
    stage_ms, napplies = plan.profile_read()
    plan.profile(False)
    plan.status()
    roof, alg = roofline_of(plan, info, nrhs, stage_ms, napplies, ms, prec, fmt or "fp16")
    Y = yd.cpu().numpy().astype(np.float64)
    errs = {}
    for c in checked_columns(nrhs):
        yc = cpucols(c)
        errs[c] = float(np.linalg.norm(Y[c] - yc) / np.linalg.norm(yc))
    rate = 1e3 / ms * nrhs
    leg = {
        "workload": label, "precision": prec, "lr_format": fmt, "nrhs": nrhs,
        "unit": "HMVM/s" if nrhs == 1 else "vectors/s", "value": rate, "ms_per_step": ms, "steps": steps,
        "ratio_vs_fp64_vectors": rate / fp64_rate,
        "relerr_vs_fp64_cpu_reference": max(errs.values()),
        "relerr_columns_checked": len(errs), "aca_eps": a.eps,
        "roofline": roof, "algorithmic_bytes_per_step": alg,
        "kernel": kernel_name(plan, info, nrhs), "plan_setup_s": setup_s,
        "device_bytes": info["device_bytes"],
        "gpu_launches": steps * (plan.kernel_count() if nrhs == 1 else plan.multi_kernel_count(nrhs)),
    }
    del xd, yd
    return leg


def run_b200(a, rank, world, local_rank):
    import torch

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist = dist_mod
    hm = build_matrix(a)
    secondary = (not a.no_secondary and a.nrhs == 1 and a.precision == "fp64" and not a.mesh and rank == 0
                 and world == 1 and not a.graph)
    rng = np.random.default_rng(a.seed)
    ncols = max(a.nrhs, 128 if secondary else 1)
    X = rng.uniform(-1.0, 1.0, (ncols, hm.nd)) if a.x_dist == "uniform" else rng.standard_normal((ncols, hm.nd))
    x = X[0]
    t0 = time.perf_counter()
    plan = make_plan(hm, a.precision, a.nrhs, a.lr_format, local_rank, a)
    setup_s = time.perf_counter() - t0
    info = plan.info()
    # x and y: FP64 for FP64 and mixed plans, FP32 for FP32 plans
    tdt = torch.float32 if a.precision == "fp32" else torch.float64
    ndt = np.float32 if a.precision == "fp32" else np.float64
    elem = 4 if a.precision == "fp32" else 8
    xd = torch.from_numpy(X[:a.nrhs].astype(ndt)).to(dev)
    yd = torch.empty((a.nrhs, hm.nd), dtype=tdt, device=dev)
    stream = torch.cuda.current_stream(dev)
    if a.nrhs == 1:
        def step():
            plan.apply(xd[0], yd[0], stream)
    else:
        def step():
            plan.apply_multi(xd, yd, stream)
    use_graph = a.graph and a.nrhs == 1
    direct_step = step
    if use_graph:
        plan.capture(xd[0], yd[0])

        def step():
            plan.replay(stream)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize(dev)

    # ---- timed region: K device-resident HMVMs ----
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(vis.split(",")[local_rank].strip() if vis else str(local_rank))
    clocks.start()
    time.sleep(0.3)
    if not use_graph:
        plan.profile(True)
    ms_step = time_steps(step, a.steps, 0, stream, dev, dist)
    if use_graph:  # stage times: a profiled pass of direct applies (a replayed graph records no events)
        plan.profile(True)
        for _ in range(min(a.steps, 200)):
            direct_step()
        torch.cuda.synchronize(dev)
    stage_ms, napplies = plan.profile_read()
    plan.profile(False)
    clk = clocks.stop()
    Y_gpu = yd.cpu().numpy().astype(np.float64)
    y_gpu = Y_gpu[0]

    # ---- e2e: the C-ABI host-buffer call, pinned buffers, copies inside ----
    xh = torch.from_numpy(X[:a.nrhs].astype(ndt)).pin_memory()
    yh = torch.empty((a.nrhs, hm.nd), dtype=tdt).pin_memory()
    xh_np, yh_np = xh.numpy(), yh.numpy()
    if a.nrhs == 1:
        def host_step():
            plan.apply_host(xh_np[0], yh_np[0], stream)
    else:
        def host_step():
            plan.apply_multi_host(xh_np, yh_np, stream)
    e2e_step = time_steps(host_step, a.e2e_steps, 3, stream, dev, dist)

    unit = "HMVM/s" if a.nrhs == 1 else "vectors/s"
    roof, alg_bytes = roofline_of(plan, info, a.nrhs, stage_ms, napplies, ms_step, a.precision, a.lr_format)
    kname = kernel_name(plan, info, a.nrhs)
    plan_keys = {"kernel": kname, "stage1_cfg": info["stage1_cfg"], "stage2_cfg": info["stage2_cfg"],
                 "ctas_per_sm": [info["ctas_per_sm"], info["stage2_ctas_per_sm"]],
                 "device_bytes": info["device_bytes"], "plan_setup_s": setup_s}
    launches = a.steps * (plan.kernel_count() if a.nrhs == 1 else plan.multi_kernel_count(a.nrhs))
    plan.close()
    del xd, yd
    torch.cuda.empty_cache()

    # ---- CPU baseline (rank 0, N=1 only) and parity of this run ----
    cpu_line = None
    rel = None
    legs = None
    ref_gpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = CpuReference(hm)
        cpucols = CpuColumns(cpu, X)
        y_cpu, st = cpu.time_sample(x, a.cpu_seconds)
        cpucols.y[0] = y_cpu
        rel = float(np.linalg.norm(y_gpu - y_cpu) / np.linalg.norm(y_cpu))
        for r in checked_columns(a.nrhs)[1:]:
            rel = max(rel, float(np.linalg.norm(Y_gpu[r] - cpucols(r)) / np.linalg.norm(cpucols(r))))
        cpu_line = {"value": 1.0 / st["min"], "unit": "HMVM/s", "cores": cpu.threads, "kind": cpu.kind,
                    "sample": f"hmvm_omp_2<double,0> on the full matrix (one vector per call), {st['runs']} runs, "
                              f"first 5 discarded, min of {st['kept']} (avg {st['avg'] * 1e3:.2f} ms)",
                    "relerr_gpu_vs_cpu": rel}
        if not a.no_cpu_variants:
            cpu_line.update(cpu_bench_variants(cpu, x, a.cpu_seconds))
        if secondary:
            legs = run_secondary(a, hm, X, cpucols, 1e3 / ms_step, local_rank, stream, dev)
            if not a.no_batch_leg:
                try:
                    legs.append(batch_leg(a, local_rank))
                except Exception as e:  # reported in its place
                    legs.append({"workload": batch_workload_text(a), "error": f"{type(e).__name__}: {e}"})
        if secondary and not a.no_reference_gpu:
            ours = {"fp64": 1e3 / ms_step}
            for leg in legs or []:
                if leg.get("workload") == "fp32 single-vector" and "value" in leg:
                    ours["fp32"] = leg["value"]
            try:
                ref_gpu = reference_gpu(cpu, x, ours, a.reference_gpu_runs)
            except Exception as e:
                ref_gpu = {"error": f"{type(e).__name__}: {e}"}
    if dist:
        dist.barrier()

    if rank == 0:
        value = world * 1e3 / ms_step * a.nrhs
        cfg = workload_config(a, hm)
        line = {
            "metric": unit, "value": value, "unit": unit, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": (value / published_hmvm_per_s(a, hm)) if published_hmvm_per_s(a, hm) else None,
            "dtype": DTYPES[a.precision],
            "data": (f"the ppohBEM mesh {os.path.basename(a.mesh)}" if a.mesh else
                     "synthetic (seeded HACApK-rule H-matrix") +
                    f"; x {'uniform[-1,1]' if a.x_dist == 'uniform' else 'standard normal'}" + ("" if a.mesh else ")"),
            "config": cfg,
            "plan": plan_keys,
            "gbytes_per_s": alg_bytes / (ms_step * 1e-3) / 1e9,
            "algorithmic_bytes_per_step": alg_bytes,
            "relerr_vs_fp64_cpu_reference": rel, "aca_eps": a.eps,
            "roofline": roof,
            "cpu_baseline": cpu_line,
            "e2e": {"value": world * 1e3 / e2e_step * a.nrhs, "unit": unit,
                    "h2d_bytes_per_step": hm.nd * elem * a.nrhs, "d2h_bytes_per_step": hm.nd * elem * a.nrhs,
                    "ms_per_step": e2e_step},
            "clocks": clk,
            "gpu_launches": launches,
        }
        if use_graph:
            line["timing"] = ("CUDA-graph replays of one captured apply (hmvm_b200_plan_replay); stage times "
                              "from a profiled pass of direct applies after the timed region")
        if legs is not None:
            line["secondary"] = legs
        if ref_gpu is not None:
            line["reference_gpu"] = ref_gpu
        print(json.dumps(line), flush=True)


def batch_specs(a):
    """The batch workload: N log-uniform in [nmin, nmax]; geometry, eta, ACA
    eps drawn per instance; 1..rhs_max right-hand sides each (seeded)."""
    rng = np.random.default_rng(a.seed + 77)
    specs = []
    for i in range(a.batch_count):
        n = int(round(np.exp(rng.uniform(np.log(a.batch_nmin), np.log(a.batch_nmax)))))
        geo = ["sphere", "cube", "plate"][int(rng.integers(3))]
        eta = [1.0, 2.0][int(rng.integers(2))]
        eps = [1e-3, 1e-4, 1e-6][int(rng.integers(3))]
        nrhs = int(rng.integers(1, a.batch_rhs_max + 1))
        specs.append((n, geo, eta, eps, nrhs, a.seed + 1000 + i))
    return specs


def measure_batch(a, local_rank, oracle=True):
    """Many independent FP32 H-matrices: the batch (every class and pass in one
    launch per stage) replayed as a CUDA graph, against a loop of per-matrix
    applies.  With oracle, the graph's first column of every instance is checked
    against the reference CPU HMVM in FP64 on the stored elements."""
    import torch

    from hacapk_hmvm_b200 import Batch, HMatrix, Plan

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    specs = batch_specs(a)
    mats = []
    t0 = time.perf_counter()
    for n, geo, eta, eps, _, seed in specs:
        mats.append(HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=a.leaf, seed=seed).to_float())
    gen_s = time.perf_counter() - t0
    nrhs = [sp[4] for sp in specs]
    rng = np.random.default_rng(a.seed)
    Xs = [torch.from_numpy(rng.uniform(-1, 1, (k, m.nd)).astype(np.float32)).to(dev) for m, k in zip(mats, nrhs)]
    Yb = [torch.empty_like(x) for x in Xs]
    Ys = [torch.empty_like(x) for x in Xs]
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    batch = Batch(mats, "fp32", device=local_rank, nrhs=nrhs)
    setup_s = time.perf_counter() - t0
    batch.capture(Xs, Yb)
    kc = batch.kernel_count()
    plans = [Plan(m, "fp32", device=local_rank, nrhs_max=min(k, 8)) for m, k in zip(mats, nrhs)]

    def seq_step():
        for pl, x, y in zip(plans, Xs, Ys):
            if x.shape[0] == 1:
                pl.apply(x[0], y[0], stream)
            else:
                pl.apply_multi(x, y, stream)

    def timed(fn, steps):
        for _ in range(max(a.warmup, 3)):
            fn()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    steps = min(a.steps, 50)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(vis.split(",")[local_rank].strip() if vis else str(local_rank))
    clocks.start()
    time.sleep(0.3)
    ms_graph = timed(lambda: batch.launch(stream), steps)
    clk = clocks.stop()
    ms_seq = timed(seq_step, max(3, steps // 4))
    batch.status()
    rel_seq = max(float(torch.linalg.norm((yb - ys).double()) / torch.linalg.norm(ys.double())) for yb, ys in zip(Yb, Ys))
    rel_inst = None
    kind = None
    if oracle:
        # every instance: its first column against the CPU HMVM (reference build, else the
        # port) in FP64 on the FP32-stored elements, one instance converted at a time
        rel_inst = []
        for i, m in enumerate(mats):
            m64 = HMatrix.from_arrays(m.nd, m.ktmax, m.ltmtx, m.kt, m.ndl, m.ndt, m.nstrtl, m.nstrtt, m.a1, m.a2,
                                      m.rowmat.astype(np.float64))
            x0 = Xs[i][0].cpu().numpy().astype(np.float64)
            yo = np.empty(m.nd)
            cpu = CpuReference(m64)
            kind = cpu.kind
            cpu.run(x0, yo)
            rel_inst.append(float(np.linalg.norm(Yb[i][0].cpu().numpy() - yo) / np.linalg.norm(yo)))
            del m64, cpu
    vecs = sum(nrhs)
    info = batch.info()
    peak, peak_kind = measured_peak_gbs()
    # each class streams its matrices once per pass (2, 4 or 8 columns per pass)
    alg = 0
    for m, k in zip(mats, nrhs):
        w = 2 if k <= 2 else 4 if k <= 4 else 8
        alg += m.stored_elements() * 4 * -(-k // w) + 8 * m.nd * k
    alg = int(alg)
    out = {
        "value": vecs / (ms_graph * 1e-3), "unit": "vectors/s", "ms_per_step": ms_graph, "steps": steps,
        "specs": specs, "total_rows": int(sum(m.nd for m in mats)), "total_vectors": vecs,
        "classes": batch.class_count(), "device_bytes": info["device_bytes"], "batch_setup_s": setup_s,
        "generate_s": gen_s, "kernels_per_replay": kc,
        "sequential_baseline": {"value": vecs / (ms_seq * 1e-3), "unit": "vectors/s", "ms_per_step": ms_seq,
                                "what": "per-matrix plans, one apply/apply_multi per matrix in a loop"},
        "speedup_vs_sequential": ms_seq / ms_graph,
        "relerr_graph_vs_sequential": rel_seq,
        "relerr_vs_fp64_cpu_reference": max(rel_inst) if rel_inst else None,
        "relerr_instances_checked": len(rel_inst) if rel_inst else 0,
        "relerr_per_instance": rel_inst,
        "relerr_kind": kind,
        "roofline": {"bound": "hbm", "achieved": alg / (ms_graph * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms_graph * 1e-3) / 1e9 / peak, "peak_source": peak_kind,
                     "traffic": None, "scope": "whole graph replay (all kernels), algorithmic bytes"},
        "clocks": clk,
    }
    for pl in plans:
        pl.close()
    batch.close()
    return out


def batch_workload_text(a):
    return (f"batch of {a.batch_count} H-matrices, N log-uniform in [{a.batch_nmin}, {a.batch_nmax}], "
            f"sphere/cube/plate, eta 1|2, ACA eps 1e-3|1e-4|1e-6, 1..{a.batch_rhs_max} RHS each, FP32 storage, "
            f"one CUDA-graph replay")


def run_batch(a, rank, world, local_rank):
    """The batch workload's own JSON line."""
    r = measure_batch(a, local_rank, oracle=rank == 0 and not a.no_cpu_baseline)
    if rank == 0:
        line = {
            "metric": "vectors/s", "value": r["value"], "unit": "vectors/s", "n_gpus": world,
            "steps": r["steps"], "warmup": a.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded HACApK-rule H-matrices; X uniform[-1,1])",
            "config": {"workload": batch_workload_text(a),
                       "instances": [{"n": sp[0], "geometry": sp[1], "eta": sp[2], "eps": sp[3], "nrhs": sp[4]}
                                     for sp in r["specs"]],
                       "total_rows": r["total_rows"], "total_vectors": r["total_vectors"],
                       "classes": r["classes"], "device_bytes": r["device_bytes"],
                       "batch_setup_s": r["batch_setup_s"], "generate_s": r["generate_s"],
                       "l2": "inputs larger than L2 (the batch's matrix bytes far exceed 126 MB)"},
            "sequential_baseline": r["sequential_baseline"],
            "speedup_vs_sequential": r["speedup_vs_sequential"],
            "relerr_graph_vs_sequential": r["relerr_graph_vs_sequential"],
            "relerr_vs_fp64_cpu_reference": r["relerr_vs_fp64_cpu_reference"],
            "relerr_instances_checked": r["relerr_instances_checked"],
            "roofline": r["roofline"],
            "clocks": r["clocks"], "gpu_launches": r["steps"] * r["kernels_per_replay"],
            "kernels_per_replay": r["kernels_per_replay"],
        }
        print(json.dumps(line), flush=True)


def batch_leg(a, local_rank):
    """The batch workload as a secondary leg of the default run."""
    r = measure_batch(a, local_rank, oracle=True)
    return {"workload": batch_workload_text(a), "precision": "fp32", "unit": r["unit"], "value": r["value"],
            "ms_per_step": r["ms_per_step"], "steps": r["steps"], "classes": r["classes"],
            "kernels_per_replay": r["kernels_per_replay"], "total_vectors": r["total_vectors"],
            "sequential_baseline": r["sequential_baseline"], "speedup_vs_sequential": r["speedup_vs_sequential"],
            "relerr_vs_fp64_cpu_reference": r["relerr_vs_fp64_cpu_reference"],
            "relerr_instances_checked": r["relerr_instances_checked"], "relerr_kind": r["relerr_kind"],
            "relerr_graph_vs_sequential": r["relerr_graph_vs_sequential"], "roofline": r["roofline"],
            "gpu_launches": r["steps"] * r["kernels_per_replay"]}


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if a.workload == "batch":
            run_batch(a, rank, world, local_rank)
        else:
            run_b200(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
