"""Writes tests/golden/*.json: FP64 oracle outputs on fixed seeded inputs.

fgkl keeps no numeric golden files and cannot be built here, so these fixtures come from the FP64
oracle (oracle/pairhmm_oracle.c, pinned to fgkl's known-answer tests) on inputs rebuilt draw for
draw from fgkl's own generators: they pin the oracle, the synthetic generators and the GPU path
against silent change. Regenerate with `python tests/golden/make_golden.py`.
"""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import numpy as np  # noqa: E402

from fgkl_b200 import synthetic  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    # config 0 of the benchmark: 32 reads of 151 vs 4 haplotypes of ~300, seed 0.
    "config0_seed0": ("workload", 0, 0),
    # fgkl's own test regions (crates/pairhmm/src/lib.rs tests, pd.rs tests).
    "region_11_70x120_24x300": ("region", (11, 70, 120, 24, 300)),
    "pd_region_31_70x120_24x300": ("pd_region", (31, 70, 120, 24, 300)),
}


def build(name):
    kind = CASES[name][0]
    if kind == "workload":
        return synthetic.workload(CASES[name][1], seed=CASES[name][2], regions=0, threads=8)
    if kind == "region":
        return synthetic.reference_region(*CASES[name][1])
    return synthetic.reference_pd_region(*CASES[name][1])


def adjoint_case():
    from fgkl_b200.adjoint import params_from_quals

    w = synthetic.reference_region(7, 6, 60, 3, 120)
    p = params_from_quals(w)
    reads, haps = w.region(0)
    ll, g = [], np.zeros((4, w.bases.size))
    for r, read in enumerate(reads):
        lo, hi = int(w.read_offsets[r]), int(w.read_offsets[r + 1])
        args = [a[lo:hi] for a in (p.gap_open_ins, p.gap_open_del, p.gap_continuation, p.base_error)]
        for hap in haps:
            v, *gr = O.adj_gradient(hap, read.bases, *args)
            ll.append(v)
            for k in range(4):
                g[k, lo:hi] += gr[k]
    return {"inputs": "synthetic.reference_region(7, 6, 60, 3, 120), params_from_quals", "log10": [repr(x) for x in ll],
            "gradient_sums": [repr(float(x)) for x in g.sum(axis=1)]}


def main():
    for name in CASES:
        w = build(name)
        out = O.workload_matrix(w, list(range(w.num_regions)), 8)
        (HERE / f"{name}.json").write_text(json.dumps({"case": name, "spec": str(CASES[name]),
                                                       "pairs": int(out.size), "log10": [repr(float(x)) for x in out]}) + "\n")
    (HERE / "adjoint_7_6x60_3x120.json").write_text(json.dumps(adjoint_case()) + "\n")


if __name__ == "__main__":
    main()
