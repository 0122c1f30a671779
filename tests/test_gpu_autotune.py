"""The autotuner on the GPU: every candidate launch shape of a small batch gives the first
trial's histories bit for bit (the tuner raises otherwise), the winner is one of the candidates,
and the table it writes is what lookup returns."""
import pytest

from strut_b200 import autotune as T
from strut_b200 import model as M
from strut_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_autotune_small_batch(gpu_lib, tmp_path):
    params = W.batched_frame_params(6, base_seed=1000)
    models = [M.Model(W.rc_frame_case(stories=min(p["stories"], 5), bays=p["bays"], wg=p["wg"],
                                      pga_g=p["pga_g"], seed=p["seed"], steps=120)) for p in params]
    table = tmp_path / "shapes.json"
    key, best, times = T.tune(models, 120, table=table)
    cands = T.candidates(models, False, 5)
    assert all(best[k] in cands[k] for k in T.KNOBS)
    assert len(times) >= 4
    assert T.lookup(models, False, table) == best
    assert key == T.workload_class(models, False)
