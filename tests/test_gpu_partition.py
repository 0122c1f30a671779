"""The multi-GPU split of a batch, run on one GPU: a fixed batch partitioned by fiber count
(strut_b200.distributed.partition_by_weight, as bench.py --scaling strong splits it across
ranks) and each share run in its own handle, one after another, reproduces the one-handle
histories bit for bit, record by record.  A record's result does not depend on which other
records share its handle (fixed reduction orders, per-instance masks)."""
import numpy as np
import pytest

from strut_b200 import distributed as D
from strut_b200 import model as M
from strut_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_partitioned_handles_reproduce_the_batch(gpu_lib):
    steps = 150
    params = W.batched_frame_params(10, base_seed=3000)
    cases = [W.rc_frame_case(stories=min(p["stories"], 6), bays=p["bays"], wg=p["wg"], pga_g=p["pga_g"],
                             seed=p["seed"], steps=steps) for p in params]
    models = [M.Model(c) for c in cases]
    with gpu_lib.Analysis(models) as an:
        an.run(steps, check=False)
        whole = [an.history(i) for i in range(len(models))]
        whole_status = an.instance_status()
    shares = D.partition_by_weight([m.num_fibers_total for m in models], 3)
    assert sorted(i for s in shares for i in s) == list(range(len(models)))
    for share in shares:
        sub = [models[i] for i in share]
        with gpu_lib.Analysis(sub) as an:
            an.run(steps, check=False)
            status = an.instance_status()
            for k, i in enumerate(share):
                d, e, it = an.history(k)
                assert status[k] == whole_status[i]
                assert np.array_equal(it, whole[i][2])
                assert np.array_equal(d, whole[i][0])
                assert np.array_equal(e, whole[i][1])
