"""The committed golden fixtures (tests/golden/, written by tests/golden/make_golden.py from the FP64
oracle on inputs rebuilt from fgkl's own generators): the oracle and the generators reproduce them
bit for bit on the CPU, and the GPU path matches them within the reference's tolerances."""
import json
from pathlib import Path

import numpy as np
import pytest

from fgkl_b200 import Config, Precision, synthetic
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    d = json.loads((GOLDEN / f"{name}.json").read_text())
    return np.array([float(x) for x in d["log10"]])


def workloads():
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("name", ["config0_seed0", "region_11_70x120_24x300", "pd_region_31_70x120_24x300"])
def test_oracle_reproduces_the_golden_fixture_bit_for_bit(name):
    mod = workloads()
    w = mod.build(name)
    out = O.workload_matrix(w, list(range(w.num_regions)), 8)
    assert out.tobytes() == load(name).tobytes()


def test_scalar_adjoint_reproduces_its_golden_fixture():
    mod = workloads()
    d = json.loads((GOLDEN / "adjoint_7_6x60_3x120.json").read_text())
    fresh = mod.adjoint_case()
    assert fresh["log10"] == d["log10"]
    assert fresh["gradient_sums"] == d["gradient_sums"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config0_seed0", "region_11_70x120_24x300", "pd_region_31_70x120_24x300"])
def test_gpu_path_matches_the_golden_fixture(gpu, name):
    from fgkl_b200 import BatchContext

    mod = workloads()
    w = mod.build(name)
    expected = load(name)
    for precision, tol in ((Precision.DOUBLE, 1e-9), (Precision.FLOAT, 1e-4)):
        out, _ = BatchContext().compute(w, Config(precision=precision))
        d = np.abs(out - expected)
        assert np.all(d <= tol), (name, precision, float(d.max()))
