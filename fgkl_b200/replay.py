"""Replays a GATK PairHMM results dump through the batched B200 path.

GATK's HaplotypeCaller writes every read x haplotype pair it scores to a text file when run with
`--pair-hmm-results-file` (plain PairHMM) or `--pdhmm-results-file` (the partially determined HMM
of `--dragen-378-concordance-mode`). This tool rebuilds the per-region batches from such a dump,
computes them on the GPU, and reports the worst deviation from GATK's recorded likelihoods,
throughput, fallback counts, how much work haplotype sharing removes, and FNV-1a checksums of the
result bits, as fgkl's replay tools do (crates/pairhmm/src/bin/replay.rs, pdreplay.rs).

    python -m fgkl_b200.replay pairs.txt [--iters N] [--max-regions N] [--only-region N]
        [--dump-region N FILE] [--write-results DIR] [--no-suffix-sharing]
        [--modes float-nofb,float,double]
    python -m fgkl_b200.replay --pd pdpairs.txt [--iters N] [--max-regions N]

Dump formats (one line per pair, reads outer, haplotypes inner, region after region; `#` lines are
comments). Qualities are FASTQ text (Phred + 33); the likelihood is GATK's `%e` rendering:
  plain: space-separated  hap-bases read-bases read-qual ins-qual del-qual gcp log10-likelihood
  PD:    tab-separated    hap-bases hap-flags read-bases read-qual ins-qual del-qual gcp log10-likelihood
where hap-flags is Java's `Arrays.toString(byte[])` rendering ("[0, 1, 0, ...]").

`FGKL_REPLAY_DEBUG[=threshold]` prints every pair further than `threshold` (default 0.5 log10) from
GATK's value, or not finite, with the inputs that reproduce it.

The dump records no region boundaries: a read boundary shows as the haplotype list starting over,
so a region whose list repeats its first haplotype cannot be told apart and is split or dropped, as
in fgkl's tools. GATK's haplotypes within a region are distinct, so its dumps do not hit this.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .pairhmm import DEL_END, DEL_START, BatchContext, Config, PdHaplotype, Precision, Read

FNV_OFFSET = 0xCBF29CE484222325
FNV_PRIME = 0x100000001B3
MASK64 = (1 << 64) - 1
# GKL recomputes in FP64 the pairs whose 2^120-scaled FP32 result falls below 1e-28, i.e. log10
# likelihoods below about -64 (replay.rs:271-313).
BELOW_F32 = -64.0


@dataclass
class Region:
    reads: list = field(default_factory=list)
    haps: list = field(default_factory=list)  # bytes (plain) or PdHaplotype (PD)
    expected: list = field(default_factory=list)  # expected[read * len(haps) + hap]


def phred(s: str) -> bytes:
    return bytes(ord(c) - 33 for c in s)


def fastq(q: bytes) -> str:
    return "".join(chr(b + 33) for b in q)


def java_flags(s: str) -> bytes:
    """Java's Arrays.toString(byte[]) rendering back to bytes (signed values wrap, pdreplay.rs:32-39)."""
    return bytes((int(t) & 0xFF) for t in s.strip().strip("[]").split(",") if t.strip())


def _reconstruct(records, same, max_regions: int) -> list[Region]:
    """Regions from (hap, read, likelihood) records in dump order. A region's haplotype list is learnt
    from its first read (complete once the list starts over) and must repeat for every later read; a
    read boundary is recognised by the list starting over (duplicate reads are dumped back to back),
    a new region by a read boundary whose first haplotype differs, and a record that breaks the list
    mid-read discards the region so far and starts over from it (replay.rs:83-159). Regions whose
    pair count is not reads x haplotypes are dropped."""
    regions: list[Region] = []
    cur = Region()
    list_known = False
    next_hap = 0
    for hap, make_read, lk in records:
        starts_over = bool(cur.haps) and same(cur.haps[0], hap)
        if not cur.reads:
            cur.reads.append(make_read())
            cur.haps.append(hap)
            next_hap = 1
        elif not list_known:
            if starts_over:
                list_known = True
                cur.reads.append(make_read())
                next_hap = 1
            else:
                cur.haps.append(hap)
                next_hap += 1
        elif next_hap == len(cur.haps):
            if starts_over:
                cur.reads.append(make_read())
                next_hap = 1
            else:
                regions.append(cur)
                cur = Region()
                if len(regions) >= max_regions:
                    break
                cur.reads.append(make_read())
                cur.haps.append(hap)
                list_known = False
                next_hap = 1
        elif same(cur.haps[next_hap], hap):
            next_hap += 1
        else:
            cur = Region(reads=[make_read()], haps=[hap])
            list_known = False
            next_hap = 1
        cur.expected.append(lk)
    if cur.reads and len(regions) < max_regions:
        regions.append(cur)
    return [r for r in regions if len(r.expected) == len(r.reads) * len(r.haps)]


def parse_plain(path, max_regions: int = sys.maxsize) -> list[Region]:
    def records():
        with open(path) as fh:
            for line in fh:
                line = line.rstrip("\n")
                if not line or line.startswith("#"):
                    continue
                f = line.split(" ")
                if len(f) < 7:
                    continue
                yield (f[0].encode(), lambda f=f: Read(f[1].encode(), phred(f[2]), phred(f[3]), phred(f[4]), phred(f[5])),
                       float(f[6]))

    return _reconstruct(records(), lambda a, b: a == b, max_regions)


def parse_pd(path, max_regions: int = sys.maxsize) -> list[Region]:
    def records():
        with open(path) as fh:
            for line in fh:
                line = line.rstrip("\n")
                if not line or line.startswith("#"):
                    continue
                f = line.split("\t")
                if len(f) < 8:
                    continue
                yield (PdHaplotype(f[0].encode(), java_flags(f[1])),
                       lambda f=f: Read(f[2].encode(), phred(f[3]), phred(f[4]), phred(f[5]), phred(f[6])), float(f[7]))

    return _reconstruct(records(), lambda a, b: a.bases == b.bases and a.flags == b.flags, max_regions)


def write_plain_dump(regions, path) -> None:
    """Regions back in the plain dump format (GATK's `%e` likelihoods), e.g. one region to replay alone."""
    with open(path, "w") as out:
        out.write("# hap-bases read-bases read-qual read-ins-qual read-del-qual gcp expected-result\n")
        for r in regions:
            for ri, read in enumerate(r.reads):
                for hi, hap in enumerate(r.haps):
                    out.write(f"{hap.decode()} {read.bases.decode()} {fastq(read.quals)} {fastq(read.ins_gop)} "
                              f"{fastq(read.del_gop)} {fastq(read.gcp)} {r.expected[ri * len(r.haps) + hi]:e}\n")


def write_pd_dump(regions, path) -> None:
    """Regions in the PD dump format (flags as Java's Arrays.toString of signed bytes)."""
    with open(path, "w") as out:
        for r in regions:
            for ri, read in enumerate(r.reads):
                for hi, hap in enumerate(r.haps):
                    flags = "[" + ", ".join(str(b - 256 if b > 127 else b) for b in hap.flags) + "]"
                    out.write("\t".join([hap.bases.decode(), flags, read.bases.decode(), fastq(read.quals), fastq(read.ins_gop),
                                         fastq(read.del_gop), fastq(read.gcp), f"{r.expected[ri * len(r.haps) + hi]:e}"]) + "\n")


def fnv1a64(words) -> int:
    """FNV-1a over 64-bit words (each word xored in whole, then one multiply), as fgkl's replay
    checksums hash result bit patterns (replay.rs:271-313)."""
    h = FNV_OFFSET
    for w in words:
        h = ((h ^ (int(w) & MASK64)) * FNV_PRIME) & MASK64
    return h


def checksums(results: np.ndarray, expected: np.ndarray) -> tuple[int, int, int]:
    """(all result bits, bits of pairs GATK kept in FP32, those rounded to 1e-6 log10): the last one
    drops last-bit differences between platforms' log10 and keeps real kernel differences."""
    bits = results.astype(np.float64).view(np.uint64)
    kept = expected >= BELOW_F32
    return fnv1a64(bits), fnv1a64(bits[kept]), fnv1a64(round_words(results[kept] * 1e6))


def round_words(x: np.ndarray) -> np.ndarray:
    """Each value rounded half away from zero to a signed 64-bit integer, NaN to 0 and out-of-range
    values saturated, as a float-to-integer conversion after rounding does in fgkl's replay; the
    two's-complement bits as unsigned words."""
    x = np.asarray(x, np.float64)
    out = np.zeros(x.shape, np.int64)
    finite = np.isfinite(x)
    t = np.trunc(x[finite])
    frac = x[finite] - t
    r = t + np.where(np.abs(frac) >= 0.5, np.sign(x[finite]), 0.0)
    lim = 2.0 ** 63
    big, small = r >= lim, r < -lim
    vals = np.where(big | small, 0.0, r).astype(np.int64)
    vals[big] = np.iinfo(np.int64).max
    vals[small] = np.iinfo(np.int64).min
    out[finite] = vals
    out[np.isposinf(x)] = np.iinfo(np.int64).max
    out[np.isneginf(x)] = np.iinfo(np.int64).min
    return out.view(np.uint64)


def workload_of(regions):
    from .synthetic import from_regions

    return from_regions([(r.reads, r.haps) for r in regions])


def nominal_cells(regions) -> int:
    total = 0
    for r in regions:
        rb = sum(len(x.bases) for x in r.reads)
        hb = sum(len(h.bases) if isinstance(h, PdHaplotype) else len(h) for h in r.haps)
        total += rb * hb
    return total


def report_bad_pairs(regions, results: np.ndarray, threshold: float) -> None:
    k = 0
    for gi, r in enumerate(regions):
        n = len(r.haps)
        for i, e in enumerate(r.expected):
            a = results[k + i]
            if math.isfinite(a) and abs(a - e) <= threshold:
                continue
            read, hap = r.reads[i // n], r.haps[i % n]
            hb = hap.bases if isinstance(hap, PdHaplotype) else hap
            print(f"BAD region={gi} read={i // n} hap={i % n} got={a} expected={e} nreads={len(r.reads)} nhaps={n}\n"
                  f"HAP {hb.decode()}\nBASES {read.bases.decode()}\nQUALS {fastq(read.quals)}\nINS {fastq(read.ins_gop)}\n"
                  f"DEL {fastq(read.del_gop)}\nGCP {fastq(read.gcp)}", file=sys.stderr)
        k += len(r.expected)


MODES = {"float-nofb": Config(Precision.FLOAT, double_fallback=False), "float": Config(Precision.FLOAT),
         "double": Config(Precision.DOUBLE)}


def replay(regions, modes=("float-nofb", "float", "double"), iters: int = 2, share_suffixes: bool = True,
           write_results: str | None = None, stem: str = "dump", device: int = 0, pd: bool = False,
           debug_threshold: float | None = None) -> dict:
    """Computes every region in each mode through one batched context; returns the report as a dict
    (one entry per mode) and prints it."""
    w = workload_of(regions)
    expected = np.array([e for r in regions for e in r.expected], np.float64)
    cells = nominal_cells(regions)
    ctx = BatchContext(device=device)
    report = {"regions": len(regions), "pairs": int(expected.size), "cells": cells}
    # Shared work, from the planner's own counts (prefix sharing alone, and with suffix sharing).
    _, st = ctx.compute(w, Config(Precision.FLOAT, share_suffixes=share_suffixes))
    report["computed_prefix_pct"] = 100.0 * st.prefix_only_cells / max(cells, 1)
    report["computed_forward_pct"] = 100.0 * st.forward_cells / max(cells, 1)
    report["computed_backward_pct"] = 100.0 * st.backward_cells / max(cells, 1)
    print(f"regions={len(regions)} pairs={expected.size} cells={cells} computed: prefix sharing "
          f"{report['computed_prefix_pct']:.1f}%, with suffix sharing "
          f"{report['computed_forward_pct'] + report['computed_backward_pct']:.1f}% (forward "
          f"{report['computed_forward_pct']:.1f}% + backward {report['computed_backward_pct']:.1f}%); mean haps/region="
          f"{np.mean([len(r.haps) for r in regions]):.1f} mean reads/region={np.mean([len(r.reads) for r in regions]):.1f}")
    low = int(np.sum(expected < BELOW_F32))
    for label in modes:
        cfg = MODES[label]
        cfg = Config(cfg.precision, cfg.double_fallback, share_suffixes)
        best, out, stats = math.inf, None, None
        for _ in range(max(1, iters)):
            t0 = time.perf_counter()
            out, stats = ctx.compute(w, cfg)
            best = min(best, time.perf_counter() - t0)
        finite = np.isfinite(out) & np.isfinite(expected)
        worst = float(np.max(np.abs(out[finite] - expected[finite]))) if finite.any() else float("nan")
        c_all, c_kept, c_round = checksums(out, expected)
        if debug_threshold is not None:
            report_bad_pairs(regions, out, debug_threshold)
        if write_results:
            Path(write_results).mkdir(parents=True, exist_ok=True)
            out.astype("<f8").tofile(os.path.join(write_results, f"{stem}.{label}.f64"))
            expected.astype("<f8").tofile(os.path.join(write_results, f"{stem}.expected.f64"))
        fb = int(stats.fallback_pairs)
        report[label] = {"ms": 1e3 * best, "mcells_per_s": cells / best / 1e6, "max_abs_err": worst, "fallback_pairs": fb,
                         "gatk_below_f32": low, "checksum": f"{c_all:016x}", "checksum_above_threshold": f"{c_kept:016x}",
                         "checksum_rounded_1e6": f"{c_round:016x}", "results": out}
        print(f"b200   {label:<10} {1e3 * best:8.1f} ms {cells / best / 1e6:10.1f} Mcells/s  max|err| vs GATK {worst:.2e}  "
              f"kernel fallback pairs {fb} ({100.0 * fb / max(expected.size, 1):.2f}%)  GATK results below f32 threshold "
              f"{low} ({100.0 * low / max(expected.size, 1):.2f}%)  checksum {c_all:016x} (above threshold {c_kept:016x}, "
              f"rounded 1e-6 {c_round:016x})")
    ctx.close()
    return report


def pd_row_end_state(flags: bytes) -> int:
    """The deletion state a PD haplotype's rows end in: 0 normal, 1 inside, 2 after (pdreplay.rs:119-132)."""
    state = 0
    for f in flags:
        if state == 2:
            state = 0
        if f & DEL_START:
            state = 1
        if f & DEL_END:
            state = 2
    return state


def pd_summary(regions) -> dict:
    """Cells, the cells that sharing between PD haplotypes with equal bases, flags and row-end state
    could save, and flag densities (pdreplay.rs:158-196)."""
    cells = shareable = flagged_haps = flagged_cols = total_cols = 0
    for r in regions:
        rb = sum(len(x.bases) for x in r.reads)
        cells += rb * sum(len(h.bases) for h in r.haps)
        for h in r.haps:
            total_cols += len(h.flags)
            n = sum(1 for f in h.flags if f)
            flagged_cols += n
            flagged_haps += n > 0
        keys = sorted((pd_row_end_state(h.flags), list(zip(h.bases, h.flags))) for h in r.haps)
        lcp = 0
        for a, b in zip(keys, keys[1:]):
            if a[0] != b[0]:
                continue
            n = 0
            while n < min(len(a[1]), len(b[1])) and a[1][n] == b[1][n]:
                n += 1
            lcp += n
        shareable += rb * lcp
    n_haps = sum(len(r.haps) for r in regions)
    return {"cells": cells, "shareable_cells": shareable, "flagged_haps_pct": 100.0 * flagged_haps / max(n_haps, 1),
            "flagged_cols_pct": 100.0 * flagged_cols / max(total_cols, 1)}


def pd_replay(regions, iters: int = 2, device: int = 0) -> dict:
    """The PD dump through the batched context in FP32 and FP64 (pdreplay.rs:198-252). GATK writes
    -Infinity for pairs it discards after the kernel; those are left out of max|err|."""
    w = workload_of(regions)
    expected = np.array([e for r in regions for e in r.expected], np.float64)
    s = pd_summary(regions)
    print(f"regions={len(regions)} pairs={expected.size} cells={s['cells']} shareable cells={s['shareable_cells']} "
          f"({100.0 * s['shareable_cells'] / max(s['cells'], 1):.1f}%) mean haps/region={np.mean([len(r.haps) for r in regions]):.1f} "
          f"mean reads/region={np.mean([len(r.reads) for r in regions]):.1f} flagged haps={s['flagged_haps_pct']:.1f}% "
          f"flagged columns={s['flagged_cols_pct']:.2f}%")
    print(f"{'backend':<8} {'prec':<7} {'ms':>10} {'Mcells/s':>12} {'max|err|':>12} {'fallbacks':>10} {'checksum':>18}")
    ctx = BatchContext(device=device)
    report = {"regions": len(regions), "pairs": int(expected.size), **s}
    for label, prec in (("float", Precision.FLOAT), ("double", Precision.DOUBLE)):
        best, out, stats = math.inf, None, None
        for _ in range(max(1, iters)):
            t0 = time.perf_counter()
            out, stats = ctx.compute(w, Config(prec))
            best = min(best, time.perf_counter() - t0)
        keep = np.isfinite(expected)
        worst = float(np.max(np.abs(out[keep] - expected[keep]))) if keep.any() else float("nan")
        c = fnv1a64(out.astype(np.float64).view(np.uint64))
        report[label] = {"ms": 1e3 * best, "mcells_per_s": s["cells"] / best / 1e6, "max_abs_err": worst,
                         "fallback_pairs": int(stats.fallback_pairs), "checksum": f"{c:016x}", "results": out}
        print(f"{'b200':<8} {label:<7} {1e3 * best:>10.1f} {s['cells'] / best / 1e6:>12.1f} {worst:>12.2e} "
              f"{int(stats.fallback_pairs):>10} {c:>18x}")
    ctx.close()
    return report


def main(argv=None) -> int:
    p = argparse.ArgumentParser(prog="python -m fgkl_b200.replay", description=__doc__.split("\n\n")[0])
    p.add_argument("dump")
    p.add_argument("--pd", action="store_true", help="the dump is a --pdhmm-results-file (PD-HMM)")
    p.add_argument("--iters", type=int, default=2)
    p.add_argument("--max-regions", type=int, default=sys.maxsize)
    p.add_argument("--only-region", type=int)
    p.add_argument("--dump-region", nargs=2, metavar=("N", "FILE"))
    p.add_argument("--write-results")
    p.add_argument("--no-suffix-sharing", action="store_true")
    p.add_argument("--modes", default="float-nofb,float,double")
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)
    regions = (parse_pd if a.pd else parse_plain)(a.dump, a.max_regions)
    if a.dump_region:
        n = int(a.dump_region[0])
        (write_pd_dump if a.pd else write_plain_dump)([regions[n]], a.dump_region[1])
        print(f"wrote region {n} to {a.dump_region[1]}", file=sys.stderr)
    if a.only_region is not None:
        regions = [regions[a.only_region]]
    if not regions:
        print(f"no complete regions found in {a.dump}", file=sys.stderr)
        return 1
    if a.pd:
        pd_replay(regions, a.iters, a.device)
        return 0
    modes = [m for m in a.modes.split(",") if m]
    for m in modes:
        if m not in MODES:
            p.error(f"unknown mode {m}")
    dbg = os.environ.get("FGKL_REPLAY_DEBUG")
    threshold = None if dbg is None else (float(dbg) if dbg.strip() else 0.5)
    replay(regions, modes, a.iters, not a.no_suffix_sharing, a.write_results, Path(a.dump).stem, a.device,
           debug_threshold=threshold)
    return 0


if __name__ == "__main__":
    sys.exit(main())
