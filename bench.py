"""PairHMM throughput benchmark (GCUPS) on B200, batched vs per-call, with accuracy vs the FP64 oracle.

Workload (one step = one pass of the hot path over the batch): 4096 uneven regions of 8-256 reads
(75% of length 151, else 50-250) against 2-32 haplotypes whose reference window is the region's
longest read plus 50-400 bases, FP32 with FP64 recomputation of lost pairs, prefix and suffix
sharing. GCUPS counts nominal cells (Σ read lengths x Σ haplotype lengths per region), as fgkl's
pairhmm-bench does (crates/pairhmm/src/bin/bench.rs:59, :102).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun with N ranks, every rank draws the same batch of N x 4096 regions and partitions it
by the planner's computed cells (fgkl_b200.shard); each rank runs its part, about 4096 regions, on
its own GPU. Regions are independent, so there is no data-path collective (weak scaling: the work
per GPU stays fixed as N grows); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PairHMM GCUPS, batched vs per-call on one B200, at max |dlog10L| vs FP64 oracle"
WORKLOAD = ("batched uneven PairHMM: 4096 regions, 8-256 reads (75% of length 151, else 50-250) x 2-32 "
            "haplotypes (longest read + 50-400 bases), FP32 + FP64 recomputation, prefix+suffix sharing")
FLOP_FORWARD = 12  # 4 FMUL + 4 FFMA per forward cell (fgkl kernel.rs:1011-1013)
FLOP_BACKWARD = 11  # 3 FMUL + 4 FFMA per backward cell (kernel.rs:1080-1088)
FLOP_ADJOINT = 40   # adjoint cell: backward 11 + forward 11 + gradient terms 18
# Smith-Waterman cell (GATK's recurrences, reference.rs:69-110), integer operations: the diagonal's
# score (compare, add), each gap (two adds, the compare that picks open or extend), the three-way
# choice of H (two compares), the -1e8 floor, and the traceback byte (direction and two gap bits).
SW_OPS_PER_CELL = 13
L2_BYTES = 126 * 1024 * 1024


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--regions", type=int, default=4096)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--per-call-regions", type=int, default=128)
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target work of the timed CPU reference sample")
    p.add_argument("--accuracy-seconds", type=float, default=8.0, help="target work of the FP64 oracle accuracy sample")
    p.add_argument("--reference-step-seconds", type=float, default=4.0,
                   help="target work of one step of the reference arm")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extra-configs", action="store_true", help="skip the c2/c3/c4 lines")
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch configuration")
    p.add_argument("--sw-pairs", type=int, default=16384, help="pairs of the Smith-Waterman line")
    p.add_argument("--config", default="c1", choices=["c1", "c2", "c3", "c4", "sw"],
                   help="c2/c3/c4: time only that configuration (with --regions to shrink it), for profiling")
    return p.parse_args()


# ---------------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------------

def dist_init(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def barrier(pg, device):
    if pg is not None:
        import torch

        t = torch.zeros(1, device=f"cuda:{device}")
        pg.all_reduce(t)
        torch.cuda.synchronize(device)


def max_over_ranks(pg, value, device):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{device}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", f"--id={self.device}", "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags) if f.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------------------------
# CPU baseline: fgkl's batched CPU algorithm (oracle/fgkl_cpu.c) on a bounded sample of the same
# workload, all host threads; the FP64 scalar oracle only measures accuracy
# ---------------------------------------------------------------------------------------------

def cpu_sample_regions(w, target_cells):
    cells = w.region_nominal_cells()
    picked, acc = [], 0
    for g in range(w.num_regions):
        if acc >= target_cells and picked:
            break
        picked.append(g)
        acc += int(cells[g])
    return picked, acc


def run_oracle(w, regions, threads):
    from oracle import oracle

    t0 = time.perf_counter()
    res = oracle.workload_matrix(w, regions, threads)
    return res, time.perf_counter() - t0


def run_fgkl_cpu(w, regions, threads):
    """fgkl's CPU algorithm restated (FP32 first, FP64 recomputation, prefix + suffix sharing)."""
    from oracle import oracle

    t0 = time.perf_counter()
    res, lost = oracle.fgkl_cpu_workload(w, regions, threads)
    return res, lost, time.perf_counter() - t0


def fgkl_cpu_sample(threads, regions, cells, lost):
    from oracle import oracle

    return (f"{len(regions)} regions ({cells:.3g} nominal cells) of the workload; fgkl's batched CPU algorithm "
            f"restated in C (oracle/fgkl_cpu.c: reads on SIMD lanes, FP32 first with FP64 recomputation of "
            f"{lost} lost pairs, prefix and suffix sharing, {oracle.ISA_NAMES[oracle.cpu_isa()]}), one region per "
            f"thread on {threads} threads; the Rust crate itself cannot be built here (no cargo)")


# ---------------------------------------------------------------------------------------------
# the reference arm
# ---------------------------------------------------------------------------------------------

def reference_arm(args, rank, world, pg):
    if rank != 0:
        return
    from oracle import oracle

    threads = os.cpu_count() or 1
    # The workload generators built into the oracle library: this arm never loads the CUDA library.
    w = oracle.synth_workload(1, seed=args.seed, regions=args.regions, threads=threads)
    # Calibrate the per-step sample to a few seconds of work on this host.
    regions, cells = cpu_sample_regions(w, 2e10)
    _, _, secs = run_fgkl_cpu(w, regions, threads)
    per_step_cells = cells / secs * args.reference_step_seconds
    regions, cells = cpu_sample_regions(w, per_step_cells)
    for _ in range(args.warmup):
        run_fgkl_cpu(w, regions[:8], threads)
    times, lost = [], 0
    for _ in range(args.steps):
        _, lost, s = run_fgkl_cpu(w, regions, threads)
        times.append(s)
    total = sum(times)
    value = cells * args.steps / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "regions": args.regions, "seed": args.seed, "sample_regions": len(regions),
                   "sample_nominal_cells": cells},
        "cpu_baseline": {"value": value, "unit": "GCUPS", "cores": threads, "kind": "port",
                         "sample": fgkl_cpu_sample(threads, regions, cells, lost) + " (per step)"},
        "e2e": {"value": value, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# peaks
# ---------------------------------------------------------------------------------------------

def hbm_peak_gbs():
    """HBM bandwidth for a roofline: MEASURED_PEAKS.json's copy bandwidth when the file exists,
    else 6,650 GB/s, an earlier copy measurement on these B200s."""
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            d = json.loads(path.read_text())
            for k in ("hbm_gbs", "hbm_GBps", "hbm"):
                if isinstance(d.get(k), (int, float)):
                    return float(d[k]), f"MEASURED_PEAKS.json {k} (measured)"
        except (ValueError, OSError):
            pass
    return 6650.0, "fallback 6,650 GB/s copy bandwidth (MEASURED_PEAKS.json absent)"


# ---------------------------------------------------------------------------------------------
# the other configurations: device-timed, with an oracle accuracy sample
# ---------------------------------------------------------------------------------------------

def time_device(stream, flush, fn, steps):
    import torch

    times = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    return statistics.mean(times)


def extra_configs(args, device, stream, flush, threads, which=("c2", "c3", "c4", "sw"), regions=0):
    """c2 (shared SNP haplotypes), c3 (PD-HMM) and c4 (adjoint), one device-timed line each
    (`regions` > 0 shrinks them, for profiling)."""
    from fgkl_b200 import BatchContext, Config, Precision, _lib, synthetic
    from fgkl_b200.adjoint import AdjointContext, params_from_quals
    from oracle import oracle

    steps = max(2, min(args.steps, 3))
    res = {}
    for cfg_id, name, note in ((2, "c2", "512 regions x 200 reads (151) x 128 SNP haplotypes (400), FP32 + FP64 recomputation, "
                                         "prefix+suffix sharing"),
                               (3, "c3", "PD-HMM: 1024 regions x 64 reads (151) x 16 PD haplotypes (350), 5% SNP flags, 2% "
                                         "deletions, FP32 + FP64 recomputation, prefix sharing")):
        if name not in which:
            continue
        w = synthetic.workload(cfg_id, seed=args.seed, regions=regions, threads=threads)
        ctx = BatchContext(device=device, stream=stream.cuda_stream)
        tuning = None
        if not args.no_autotune:
            # The autotuner, untimed, on 512 regions of the same generator with another seed; its
            # choice applies to the timed batch.
            tctx = BatchContext(device=device, stream=stream.cuda_stream)
            tw = synthetic.workload(cfg_id, seed=args.seed + 7919, regions=min(512, w.num_regions), threads=threads)
            chosen, _ = tctx.autotune(tw, Config(precision=Precision.FLOAT), repeats=3)
            tctx.close()
            tuning = {k: chosen[k] for k in ("streams", "grid_percent", "reads_per_warp", "rows_extra", "warps_per_block")}
            ctx.set_tuning(**tuning)
        ctx.prepare(w, Config(precision=Precision.FLOAT))
        for _ in range(2):
            ctx.run()
        t = time_device(stream, flush, ctx.run, steps)
        out, st = ctx.fetch()
        # Where the step goes: one serialised run with every launch timed by CUDA events.
        ctx.set_profiling(True)
        ctx.run()
        prof = ctx.launch_profile()
        ctx.set_profiling(False)
        nominal = w.nominal_cells()
        sample = [0]
        ref = oracle.workload_matrix(w, sample, threads)
        offs = w.output_offsets()
        # FP32 roofline of the dominant first-pass launch and of the whole step (12 FLOP a forward or
        # PD cell, 11 a backward cell), against the FP32 FMA peak measured live on this GPU.
        s_tf, p_tf, clk = C.c_double(), C.c_double(), C.c_double()
        _lib.lib().fgkl_probe_fp32_tflops(device, C.byref(s_tf), C.byref(p_tf), C.byref(clk))
        peak = max(s_tf.value, p_tf.value)
        first = [x for x in prof if not x["recomputation"]]
        dom = max(first, key=lambda x: x["ms"])
        dom_tf = (FLOP_FORWARD * dom["forward_cells"] + FLOP_BACKWARD * dom["backward_cells"]) / (dom["ms"] / 1e3) / 1e12
        step_tf = (FLOP_FORWARD * st.forward_cells + FLOP_BACKWARD * st.backward_cells) / t / 1e12
        kinds = {0: "PackedF32", 1: "OneF32", 2: "OneF64", 3: "OneF32Pd", 4: "OneF64Pd", 5: "PackedF32Pd"}
        kname = "pd_kernel" if dom["kind"] in (3, 4, 5) else "pairhmm_kernel"
        roof = {"bound": "fp32", "unit": "TFLOP/s", "peak": peak, "achieved": dom_tf, "frac": dom_tf / peak,
                "dominant_launch": {"kernel": f"{kname}<{kinds.get(dom['kind'], dom['kind'])}, {dom['rows']}>",
                                    "ms": dom["ms"], "forward_cells": dom["forward_cells"],
                                    "backward_cells": dom["backward_cells"],
                                    "share_of_serialised_time": dom["ms"] / max(1e-9, sum(x["ms"] for x in prof))},
                "whole_step": {"achieved": step_tf, "frac": step_tf / peak}}
        res[name] = {"workload": note, "regions": w.num_regions, "nominal_gcups": nominal / t / 1e9,
                     "computed_gcups": st.computed_cells / t / 1e9, "ms_per_step": 1e3 * t, "steps": steps,
                     "nominal_cells": nominal, "computed_cells": int(st.computed_cells),
                     "prefix_only_cells": int(st.prefix_only_cells), "forward_cells": int(st.forward_cells),
                     "backward_cells": int(st.backward_cells), "fallback_pairs": int(st.fallback_pairs),
                     "serialised_ms": {"first_pass": sum(x["ms"] for x in prof if not x["recomputation"]),
                                       "fp64_recomputation": sum(x["ms"] for x in prof if x["recomputation"])},
                     "max_abs_dlog10_sample": float(np.max(np.abs(out[offs[0]:offs[1]] - ref))),
                     "accuracy_sample": "region 0 against the FP64 oracle",
                     "roofline": roof,
                     "launch_tuning": tuning}
        if not args.no_cpu_baseline:
            # fgkl's CPU algorithm for this configuration (oracle/fgkl_cpu.c: the plain kernel for
            # c2, the PD kernel for c3) on a bounded sample of the same workload, all host threads.
            regs, cells = cpu_sample_regions(w, 5e9)
            _, _, secs = run_fgkl_cpu(w, regs, threads)
            target = 4.0 * cells / secs
            if target > cells * 1.5:
                regs, cells = cpu_sample_regions(w, target)
                _, lost, secs = run_fgkl_cpu(w, regs, threads)
            else:
                lost = 0
            cpu = cells / secs / 1e9
            res[name]["cpu_baseline"] = {"value": cpu, "unit": "GCUPS", "cores": threads, "kind": "port",
                                         "sample": f"{len(regs)} regions ({cells:.3g} nominal cells) of the workload; "
                                                   f"fgkl's batched {'PD' if cfg_id == 3 else 'plain'} CPU kernel "
                                                   "restated in C (oracle/fgkl_cpu.c), FP32 with FP64 recomputation"}
            res[name]["device_over_cpu"] = (nominal / t / 1e9) / cpu
        ctx.close()
    if "c4" in which:
        res["c4"] = adjoint_line(args, device, stream, flush, regions, threads)
    if "sw" in which:
        res["sw"] = smith_waterman_line(args, device, threads)
    return res


def adjoint_line(args, device, stream, flush, regions, threads):
    """c4: the adjoint, device-timed, with an accuracy sample against the FP64 scalar adjoint."""
    from fgkl_b200 import _lib, synthetic
    from fgkl_b200.adjoint import AdjointContext, params_from_quals
    from oracle import oracle

    steps = max(2, min(args.steps, 3))
    # c4: the adjoint.
    w = synthetic.workload(4, seed=args.seed, regions=regions, threads=threads)
    p = params_from_quals(w)
    actx = AdjointContext(device=device, stream=stream.cuda_stream)
    actx.prepare(w, p, False)
    actx.run()
    t = time_device(stream, flush, actx.run, steps)
    r = actx.fetch()
    nominal = w.nominal_cells()
    # Accuracy sample: region 0's reads against the FP64 scalar adjoint, summed global gradients.
    n0, h0 = int(w.region_reads[0]), int(w.region_haps[0])
    lo, hi = int(w.read_offsets[0]), int(w.read_offsets[n0])
    g_ref = np.zeros((4, hi - lo))
    for rr in range(n0):
        a, b = int(w.read_offsets[rr]), int(w.read_offsets[rr + 1])
        args_ = [x[a:b] for x in (p.gap_open_ins, p.gap_open_del, p.gap_continuation, p.base_error)]
        for h in range(h0):
            hap = w.hap_bases[int(w.hap_offsets[h]):int(w.hap_offsets[h + 1])].tobytes()
            _, *gr = oracle.adj_gradient(hap, w.bases[a:b].tobytes(), *args_)
            for k in range(4):
                g_ref[k, a - lo:b - lo] += gr[k]
    ours_g = [r.gap_open_ins, r.gap_open_del, r.gap_continuation, r.base_error]
    # FP32 roofline: per cell the backward recurrence (11 FLOP), the forward recurrence (11) and the
    # gradient terms (18: four products against the backward values, each an FMA into a per-row sum,
    # plus the prior and sign products). The backward values are recomputed once from checkpoints
    # (another 11 FLOP a cell, not counted: it is the price of keeping them on chip).
    s_tf, p_tf, clk = C.c_double(), C.c_double(), C.c_double()
    _lib.lib().fgkl_probe_fp32_tflops(device, C.byref(s_tf), C.byref(p_tf), C.byref(clk))
    fp32_peak = max(s_tf.value, p_tf.value)
    adj_tf = FLOP_ADJOINT * nominal / t / 1e12
    rel = [abs(ours_g[k][lo:hi].sum() - g_ref[k].sum()) / abs(g_ref[k].sum()) for k in range(4)]
    line = {"workload": "adjoint: 256 regions x 64 reads (151) x 8 haplotypes (350); gradients of the summed log10 "
                             "likelihood w.r.t. gap-open (ins, del), gap continuation, base error per read position",
                 "regions": w.num_regions, "nominal_gcups": nominal / t / 1e9, "ms_per_step": 1e3 * t, "steps": steps,
                 "nominal_cells": nominal, "cells_per_pair_visited": "backward sweep twice (checkpoints, then blocks), forward once",
                 "fp64_reads": r.fp64_reads,
                 "max_rel_err_global_gradients_sample": max(rel),
                 "roofline": {"bound": "fp32", "unit": "TFLOP/s", "achieved": adj_tf, "peak": fp32_peak,
                              "frac": adj_tf / fp32_peak, "flop_per_cell": FLOP_ADJOINT,
                              "peak_source": "measured FP32 FMA probe on this GPU"},
                 "accuracy_sample": "region 0 against the FP64 scalar adjoint (summed gradients)"}
    actx.close()
    return line


def sw_pairs(n_pairs, ref_len=500, alt_len=500, seed=5):
    """fgkl's sw-bench pairs (crates/smithwaterman/src/bin/bench.rs:42-53): a uniform ACGT reference,
    the alternate its first alt_len bases with 3 substitutions and 1 deletion (drawn with numpy)."""
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    pairs = []
    for _ in range(n_pairs):
        r = acgt[rng.integers(0, 4, ref_len)]
        a = r[:min(alt_len, ref_len)].copy()
        for _ in range(3):
            a[rng.integers(0, a.size)] = acgt[rng.integers(0, 4)]
        a = np.delete(a, rng.integers(0, a.size))
        pairs.append((r.tobytes(), a.tobytes()))
    return pairs


def _cigar_ops(cigar):
    """The elements of a CIGAR string."""
    import re

    return re.findall(r"\d+[MIDS]", cigar)


def smith_waterman_line(args, device, threads):
    """GATK's Smith-Waterman (fgkl crates/smithwaterman) on fgkl's sw-bench shape, one batch call."""
    from concurrent.futures import ThreadPoolExecutor

    from fgkl_b200 import BatchContext
    from fgkl_b200.sw import HAPLOTYPE_TO_REFERENCE as P, OverhangStrategy, align_batch
    from oracle import oracle

    import ctypes as C

    import numpy as np

    from fgkl_b200 import _lib
    from fgkl_b200.pairhmm import _check

    pairs = sw_pairs(args.sw_pairs)
    cells = sum(len(r) * len(a) for r, a in pairs)
    ctx = BatchContext(device=device)
    got = align_batch(pairs, P, OverhangStrategy.INDEL, ctx)  # untimed: the engine's buffers, and the results checked below
    # The timed call is the C ABI's, as a JNI caller makes it, from host arrays built once.
    refs = np.frombuffer(b"".join(r for r, _ in pairs), np.uint8)
    alts = np.frombuffer(b"".join(a for _, a in pairs), np.uint8)
    roff = np.concatenate([[0], np.cumsum([len(r) for r, _ in pairs])]).astype(np.int64)
    aoff = np.concatenate([[0], np.cumsum([len(a) for _, a in pairs])]).astype(np.int64)
    b = _lib.SwBatch(len(pairs), refs.ctypes.data_as(_lib.u8p), roff.ctypes.data_as(_lib.i64p), alts.ctypes.data_as(_lib.u8p),
                     aoff.ctypes.data_as(_lib.i64p))
    cap = int(_lib.lib().fgkl_sw_cigar_capacity(C.byref(b)))
    cigar = np.zeros(cap, np.uint32)
    counts = np.zeros(len(pairs), np.int32)
    offsets = np.zeros(len(pairs), np.int32)
    prm = P._c()
    times, kernel = [], []
    kms = C.c_float()
    for _ in range(max(3, min(args.steps, 5))):
        t0 = time.perf_counter()
        _check(_lib.lib().fgkl_sw_align_batch(ctx._ctx, C.byref(b), C.byref(prm), int(OverhangStrategy.INDEL),
                                              cigar.ctypes.data_as(C.POINTER(C.c_uint32)), cap,
                                              counts.ctypes.data_as(_lib.i32p), offsets.ctypes.data_as(_lib.i32p)))
        times.append(time.perf_counter() - t0)
        _check(_lib.lib().fgkl_sw_last_kernel_ms(ctx._ctx, C.byref(kms)))
        kernel.append(kms.value / 1e3)
    ctx.close()
    t = statistics.median(times)
    tk = statistics.median(kernel)
    alu = C.c_double()
    _check(_lib.lib().fgkl_probe_int32_alu_gops(device, C.byref(alu)))
    sw_gops = SW_OPS_PER_CELL * cells / tk / 1e9
    same = all(int(offsets[k]) == got[k].offset and counts[k] == len(_cigar_ops(got[k].cigar)) for k in range(0, len(pairs), 97))
    params = (P.match_value, P.mismatch_penalty, P.gap_open_penalty, P.gap_extend_penalty)
    sample = list(range(0, len(pairs), max(1, len(pairs) // 512)))

    def one(k):
        return oracle.sw_align(pairs[k][0], pairs[k][1], params, int(OverhangStrategy.INDEL))

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        ref = list(ex.map(one, sample))
    cpu_secs = time.perf_counter() - t0
    cpu_cells = sum(len(pairs[k][0]) * len(pairs[k][1]) for k in sample)
    differ = sum((g.cigar, g.offset) != r for g, r in zip((got[k] for k in sample), ref))
    return {"workload": f"Smith-Waterman: {len(pairs)} pairs, reference 500, alternate its first 500 bases with 3 substitutions "
                        "and 1 deletion (fgkl's sw-bench shape), haplotype-to-reference scores, Indel strategy",
            "gcups": cells / t / 1e9, "ms_per_step": 1e3 * t, "cells": cells,
            "kernel": {"ms": 1e3 * tk, "gcups": cells / tk / 1e9,
                       "timing": "CUDA events around the fill-and-traceback launch of each timed call, median"},
            "roofline": {"bound": "int32 alu", "unit": "Gop/s", "achieved": sw_gops, "peak": alu.value,
                         "frac": sw_gops / alu.value, "ops_per_cell": SW_OPS_PER_CELL,
                         "peak_source": "measured XOR and signed-max chains on this GPU (fgkl_probe_int32_alu_gops)"},
            "timing": "one fgkl_sw_align_batch call (C ABI) from host arrays built once: uploads, kernel, CIGAR packing, "
                      "downloads, wall clock",
            "timed_calls_match_the_python_call": same,
            "alignments_differing_from_oracle": differ, "oracle_sample_pairs": len(sample),
            "cpu_baseline": {"value": cpu_cells / cpu_secs / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
                             "sample": f"{len(sample)} pairs through the scalar restatement of GATK's aligner "
                                       "(oracle/sw_oracle.c), one pair per thread"}}


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------

def ours(args, rank, world, local, pg):
    import torch

    from fgkl_b200 import BatchContext, Config, PairHmm, Precision, _lib, synthetic

    device = local
    torch.cuda.set_device(device)
    threads = os.cpu_count() or 1
    if world == 1:
        w = synthetic.workload(1, seed=args.seed, regions=args.regions, threads=threads)
    else:
        # One batch of world x regions, partitioned by planned cells; this rank runs its part.
        from fgkl_b200.shard import partition_regions, region_costs

        whole = synthetic.workload(1, seed=args.seed, regions=args.regions * world, threads=threads)
        part = partition_regions(region_costs(whole), world)[rank]
        w = whole.subset(part)
        del whole
    nominal = w.nominal_cells()
    stream = torch.cuda.Stream(device=device)
    cfg = Config(precision=Precision.FLOAT)
    # Launch configuration (streams per pass, persistent grid size) from the autotuner, run untimed on
    # a batch of the same generator with another seed, then fixed for every context below.
    tuning = None
    if not args.no_autotune:
        tw = synthetic.workload(1, seed=args.seed + 7919 + rank, regions=min(args.regions, 1024), threads=threads)
        tctx = BatchContext(device=device, stream=stream.cuda_stream)
        chosen, tried = tctx.autotune(tw, cfg, repeats=3)
        tctx.close()
        tuning = {"chosen": {k: chosen[k] for k in ("streams", "grid_percent", "reads_per_warp", "rows_extra", "warps_per_block")},
                  "candidates_ms": {f"s{t['streams']}/g{t['grid_percent']}/r{t['reads_per_warp']}/x{t['rows_extra']}"
                                    f"/w{t['warps_per_block']}": round(t["ms"], 2) for t in tried},
                  "key": "streams/grid %/reads per warp/rows-per-lane step up/warps per block",
                  "tuned_on": f"{tw.num_regions} regions of the same generator, another seed (untimed)"}

    def tuned(c):
        if tuning:
            c.set_tuning(**tuning["chosen"])
        return c

    ctx = tuned(BatchContext(device=device, stream=stream.cuda_stream))
    n_out = ctx.prepare(w, cfg)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")

    # Warm-up (first run also captures the CUDA graph).
    for _ in range(args.warmup):
        ctx.run()
    torch.cuda.synchronize(device)
    out, stats = ctx.fetch()
    planned_launches = int(stats.kernel_launches)

    # Timed steps: device-resident inputs, L2 flushed between steps (untimed), events on our stream.
    times = []
    barrier(pg, device)
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                ctx.run()
                ev1.record(stream)
            ev1.synchronize()
            times.append(ev0.elapsed_time(ev1) / 1e3)
    torch.cuda.synchronize(device)
    barrier(pg, device)
    step = statistics.mean(times)
    step_max = max_over_ranks(pg, step, device)
    out, stats = ctx.fetch()
    value = nominal * world / step_max / 1e9

    # Roofline of the dominant kernel: one extra run with the launches serialised on our stream and
    # CUDA events around each (direct launches, no graph); the launch with the longest duration is the
    # dominant one; its algorithmic FP32 FLOPs (12 per forward cell, 11 per backward cell) over its
    # duration, against the FP32 FMA peak measured live on this GPU.
    with torch.cuda.stream(stream):
        flush.zero_()
    ctx.set_profiling(True)
    ctx.run()
    launches = ctx.launch_profile()
    ctx.set_profiling(False)
    dom = max(launches, key=lambda x: x["ms"])
    dom_flops = FLOP_FORWARD * dom["forward_cells"] + FLOP_BACKWARD * dom["backward_cells"]
    flops = FLOP_FORWARD * stats.forward_cells + FLOP_BACKWARD * stats.backward_cells
    s_tf, p_tf, clk = C.c_double(), C.c_double(), C.c_double()
    _lib.lib().fgkl_probe_fp32_tflops(device, C.byref(s_tf), C.byref(p_tf), C.byref(clk))
    peak = max(s_tf.value, p_tf.value)
    achieved = dom_flops / (dom["ms"] / 1e3) / 1e12
    step_achieved = flops / step / 1e12
    kind_names = {0: "PackedF32", 1: "OneF32", 2: "OneF64", 3: "OneF32Pd", 4: "OneF64Pd", 5: "PackedF32Pd"}
    dominant = {"kernel": f"pairhmm_kernel<{kind_names.get(dom['kind'], dom['kind'])}, {dom['rows']}>",
                "ms": dom["ms"], "tasks": dom["tasks"], "blocks": dom["blocks"],
                "forward_cells": dom["forward_cells"], "backward_cells": dom["backward_cells"],
                "share_of_serialised_time": dom["ms"] / max(1e-9, sum(x["ms"] for x in launches)),
                "serialised_total_ms": sum(x["ms"] for x in launches)}

    # End to end through the C ABI from host buffers: every step plans, stages and uploads its batch,
    # runs it and downloads its results (fgkl_batch_prepare / fgkl_batch_run / fgkl_batch_fetch).
    # Streamed: two contexts on one compute stream alternate, so the host planning and upload of
    # step k+1 overlap the kernels of step k, as a caller feeding batches back to back runs them.
    # Single: one context, one fgkl_batch_compute call after another, nothing overlapped (one batch's
    # latency).
    h2d = int(w.bases.size * 5 + w.read_offsets.nbytes)
    d2h = int(n_out * 8)
    from fgkl_b200.pairhmm import _check, _ptr
    L = _lib.lib()
    # The step's inputs and results live in page-locked host memory, which the copies upload from
    # and download into directly (allocated and filled untimed).
    import dataclasses

    pinned_keep = []

    def pinned_copy(a):
        t = torch.empty(a.size, dtype=torch.uint8 if a.dtype == np.uint8 else torch.float64, pin_memory=True)
        pinned_keep.append(t)
        p = t.numpy()
        p[...] = a
        return p

    w_pinned = dataclasses.replace(w, **{f: pinned_copy(getattr(w, f)) for f in ("bases", "quals", "ins_gop", "del_gop", "gcp")})
    b_in, c_in = w_pinned.as_batch(), cfg._c()
    shared = torch.cuda.Stream(device=device)
    ctxs = [tuned(BatchContext(device=device, stream=shared.cuda_stream)),
            tuned(BatchContext(device=device, stream=shared.cuda_stream))]
    outs = [pinned_copy(np.zeros(n_out, np.float64)) for _ in ctxs]
    st = _lib.Stats()
    for ctx, o in zip(ctxs, outs):  # sizes each context's device and pinned buffers, untimed
        _check(L.fgkl_batch_compute(ctx._ctx, C.byref(b_in), C.byref(c_in), _ptr(o, _lib.f64p), n_out, C.byref(st)))
    n_e2e = max(3, args.steps)

    def fetch(k):
        _check(L.fgkl_batch_fetch(ctxs[k % 2]._ctx, _ptr(outs[k % 2], _lib.f64p), n_out, C.byref(st)))

    barrier(pg, device)
    t0 = time.perf_counter()
    for k in range(n_e2e):
        ctx = ctxs[k % 2]._ctx
        _check(L.fgkl_batch_prepare(ctx, C.byref(b_in), C.byref(c_in)))
        _check(L.fgkl_batch_run(ctx))
        if k > 0:
            fetch(k - 1)
    fetch(n_e2e - 1)
    e2e_step = max_over_ranks(pg, (time.perf_counter() - t0) / n_e2e, device)
    e2e_value = nominal * world / e2e_step / 1e9
    single_times = []
    for _ in range(max(1, min(3, args.steps))):
        barrier(pg, device)
        t0 = time.perf_counter()
        _check(L.fgkl_batch_compute(ctxs[0]._ctx, C.byref(b_in), C.byref(c_in), _ptr(outs[0], _lib.f64p), n_out,
                                    C.byref(st)))
        single_times.append(time.perf_counter() - t0)
    e2e_phases = {"plan_ms": st.host_plan_ms, "pack_ms": st.host_pack_ms, "upload_ms": st.host_upload_ms,
                  "fetch_ms": st.host_fetch_ms}
    single_step = max_over_ranks(pg, statistics.mean(single_times), device)
    e2e_single = nominal * world / single_step / 1e9
    identical = all(o.tobytes() == out.tobytes() for o in outs)

    if rank != 0:
        barrier(pg, device)
        return

    # Per-call form: one fgkl_pairhmm_compute_config call per region from host buffers already in the
    # JNI layout (as the JNI shim holds them), first on one thread, then from several threads at once
    # (each calling thread gets its own engine and stream, as GATK's native threads would).
    import threading

    from fgkl_b200.pairhmm import _Flat

    pc_regions = [w.region(g) for g in range(min(args.per_call_regions, w.num_regions))]
    flats = [_Flat(reads, haps, None) for reads, haps in pc_regions]
    calls = []
    for (reads, haps), f in zip(pc_regions, flats):
        rd, hp = f.structs()
        n = len(reads) * len(haps)
        calls.append((rd, hp, np.empty(n, np.float64), n))
    c_cfg = cfg._c()
    L_pc = _lib.lib()

    def call(c):
        rd, hp, o, n = c
        _check(L_pc.fgkl_pairhmm_compute_config(C.byref(rd), C.byref(hp), C.byref(c_cfg), _ptr(o, _lib.f64p), n, None))

    for c in calls:  # untimed: the engine that serves these calls at full size
        call(c)
    pc_cells = sum(sum(len(r.bases) for r in reads) * sum(len(h) for h in haps) for reads, haps in pc_regions)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for c in calls:
        call(c)
    pc_secs = time.perf_counter() - t0
    per_call = pc_cells / pc_secs / 1e9 if pc_cells else float("nan")
    pc_threads = 8

    def per_call_threads(max_batches):
        # The same calls from pc_threads threads at once: combined into batches when they meet
        # (max_batches > 0, the library's default), or each run alone on its thread's engine.
        prev = L_pc.fgkl_set_call_combining(max_batches)
        gate = threading.Barrier(pc_threads + 1)

        def worker(k):
            for _ in range(2):  # untimed: this thread's engine (and the combining engines) at full size
                for c in calls:
                    call(c)
            gate.wait()
            for c in calls[k::pc_threads]:
                call(c)
            gate.wait()

        pool = [threading.Thread(target=worker, args=(k,)) for k in range(pc_threads)]
        for th in pool:
            th.start()
        gate.wait()
        b0, r0 = C.c_uint64(), C.c_uint64()
        L_pc.fgkl_call_combining_stats(C.byref(b0), C.byref(r0))
        t0 = time.perf_counter()
        gate.wait()
        secs = time.perf_counter() - t0
        b1, r1 = C.c_uint64(), C.c_uint64()
        L_pc.fgkl_call_combining_stats(C.byref(b1), C.byref(r1))
        for th in pool:
            th.join()
        L_pc.fgkl_set_call_combining(prev)
        return pc_cells / secs / 1e9 if pc_cells else float("nan"), b1.value - b0.value, r1.value - r0.value

    per_call_mt, mt_batches, mt_requests = per_call_threads(2)
    per_call_alone, _, _ = per_call_threads(0)

    line = {
        "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * step_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "regions": args.regions, "seed": args.seed, "pairs": n_out,
                   "nominal_cells": nominal, "computed_cells": int(stats.computed_cells),
                   "forward_cells": int(stats.forward_cells), "backward_cells": int(stats.backward_cells),
                   "prefix_only_cells": int(stats.prefix_only_cells),
                   "l2": f"inputs {w.bases.size * 5 / 2**20:.0f} MiB > L2 126 MiB; L2 also flushed (untimed) between steps",
                   "parallelism": f"one batch of {world} x {args.regions} regions partitioned by planned cells over {world} GPU(s), no collective",
                   "launch_tuning": tuning},
        "computed_gcups": stats.computed_cells / step / 1e9,
        "fallback_pairs": int(stats.fallback_pairs), "rescue_reads": int(stats.rescue_reads),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     # DRAM bytes come from an ncu capture (one pass per launch), which a timed run cannot
                     # make; they are kept with the profile summaries.
                     "traffic": None,
                     "peak_source": f"measured FP32 FMA probe on this GPU (scalar {s_tf.value:.1f}, packed {p_tf.value:.1f} "
                                    "TFLOP/s); MEASURED_PEAKS.json has no FP32 figure (it holds HBM and bf16 ones when "
                                    "present)",
                     "flop_per_cell": {"forward": FLOP_FORWARD, "backward": FLOP_BACKWARD},
                     "dominant_launch": dominant,
                     "whole_step": {"achieved": step_achieved, "frac": step_achieved / peak,
                                    "note": "all first-pass FLOPs over the whole step (concurrent bins, recomputation)"}},
        "e2e": {"value": e2e_value, "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "includes": "host planning + packing + H2D from page-locked inputs + kernels + D2H into page-locked outputs, every step",
                "form": f"{n_e2e} batches streamed through two contexts on one stream (prepare/run of batch k+1 "
                        "before fetching batch k), page-locked host buffers in and out",
                "ms_per_step": 1e3 * e2e_step,
                "single": {"value": e2e_single, "ms_per_step": 1e3 * single_step,
                           "form": "one fgkl_batch_compute call at a time, nothing overlapped",
                           "host_phases_last_call": e2e_phases},
                "bit_identical_to_device_run": identical},
        "gpu_launches": planned_launches * args.steps,
        "clocks": clocks.summary(),
    }

    if not args.no_extra_configs:
        line["configs"] = extra_configs(args, device, stream, flush, os.cpu_count() or 1)

    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        offs = w.output_offsets()
        # Accuracy against the FP64 scalar oracle on a sample of about args.accuracy_seconds.
        regions, cells = cpu_sample_regions(w, 1e9)
        ref, secs = run_oracle(w, regions, threads)
        target = args.accuracy_seconds * cells / secs
        if target > cells * 1.5:
            regions, cells = cpu_sample_regions(w, target)
            ref, secs = run_oracle(w, regions, threads)
        got = np.concatenate([out[offs[g]:offs[g + 1]] for g in regions])
        line["max_abs_dlog10"] = float(np.max(np.abs(got - ref)))
        line["accuracy_sample"] = {"regions": len(regions), "pairs": int(got.size), "oracle": "scalar FP64"}
        # The timed CPU reference: fgkl's batched algorithm on about args.cpu_seconds of work.
        regions, cells = cpu_sample_regions(w, 2e10)
        cpu, lost, secs = run_fgkl_cpu(w, regions, threads)
        target = args.cpu_seconds * cells / secs
        if target > cells * 1.5:
            regions, cells = cpu_sample_regions(w, target)
            cpu, lost, secs = run_fgkl_cpu(w, regions, threads)
        mine = np.concatenate([out[offs[g]:offs[g + 1]] for g in regions])
        line["cpu_baseline"] = {"value": cells / secs / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
                                "sample": fgkl_cpu_sample(threads, regions, cells, lost),
                                "max_abs_dlog10_vs_gpu": float(np.max(np.abs(mine - cpu)))}
    # Last in the line, so that a reader keeping only the end of a long line keeps them.
    line["per_call"] = {"value": per_call, "unit": "GCUPS", "regions": len(pc_regions),
                        "form": "one fgkl_pairhmm_compute_config call per region, JNI layout, one thread",
                        "threads": {"value": per_call_mt, "threads": pc_threads, "combined_batches": mt_batches,
                                    "combined_requests": mt_requests, "form": "8 threads, concurrent calls combined",
                                    "alone": {"value": per_call_alone, "form": "8 threads, combining off"}}}
    line["batched_over_per_call"] = value / world / per_call
    print(json.dumps(line), flush=True)
    barrier(pg, device)


def single_config(args, device):
    """One of the other configurations alone (for profiling); prints its line."""
    import torch

    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")
    regions = args.regions if args.regions != 4096 else 0
    res = extra_configs(args, device, stream, flush, os.cpu_count() or 1, (args.config,), regions)
    print(json.dumps({"config": args.config, **res[args.config]}), flush=True)


def main():
    # A fault anywhere prints the Python stack of every thread to stderr.
    faulthandler.enable()
    args = parse()
    if args.impl == "reference":
        # The reference arm is host-only: rank 0 times it, other ranks exit without work.
        reference_arm(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), None)
        return
    rank, world, local, pg = dist_init(args.gpus)
    if args.config != "c1":
        single_config(args, local)
    else:
        ours(args, rank, world, local, pg)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
