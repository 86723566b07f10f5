"""One batch over several batch contexts (fgkl_b200.shard.MultiDeviceContext) on the GPU.

With one device here, the contexts share it: the path is the multi-device one (partition by
planned cells, one context and graph per part, reassembly in the caller's order), and the results
must carry the bits of one context running the whole batch, since a region's arithmetic does not
depend on the batch around it.
"""
import numpy as np
import pytest

from fgkl_b200 import BatchContext, Config, Precision, synthetic
from fgkl_b200.shard import MultiDeviceContext

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which, precision", [(1, Precision.FLOAT), (3, Precision.FLOAT), (1, Precision.DOUBLE)])
def test_sharded_batch_has_the_single_context_bits(gpu, which, precision):
    cfg = Config(precision=precision)
    w = synthetic.workload(which, seed=17, regions=40, threads=8)
    whole = BatchContext()
    expected, _ = whole.compute(w, cfg)
    whole.close()
    multi = MultiDeviceContext([0, 0, 0])
    got = multi.compute(w, cfg)
    assert sorted(g for p in multi.partition for g in p) == list(range(w.num_regions))
    assert got.tobytes() == expected.tobytes()
    multi.close()
