"""Oracle histories of the 20-story 6x6-bay rigid-diaphragm frame (workloads.tall_frame3d_case,
its 4000-step record) over the first STEPS steps, in both of the oracle's rounding orders (plain
and contracted multiply-adds): Newton iterations per step, the recorded displacements and
element forces, the status and the failing step.  The frame gives out a little after step 200
(an element state determination fails), which is why the record is cut there.

Writes tests/golden/tall_frame3d_4000_first215.json for tests/test_gpu_tall_frame.py.  Each
order takes about a quarter of an hour on one core (the oracle factors the 3000-dof band
densely every iteration, as Strut does on this frame); the two run in parallel processes.

    python tests/golden/make_tall_frame_golden.py
"""
import json
import multiprocessing as mp
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

STEPS = 215
OUT = Path(__file__).resolve().parent / "tall_frame3d_4000_first215.json"


def run(order: str):
    from oracle import binding
    from strut_b200 import model as M
    from strut_b200 import workloads as W

    fma = order == "contracted"
    binding.build(fma=fma)
    binding.use_fma(fma)
    m = M.Model(W.tall_frame3d_case(steps=4000))
    d, e, it, rc, failed = binding.run_transient(m, STEPS)
    return order, {"status": int(rc), "failed_step": int(failed), "iters": [int(v) for v in it],
                   "disp": d.tolist(), "eforce": e.reshape(e.shape[0], -1).tolist()}


def main():
    with mp.get_context("spawn").Pool(2) as pool:
        res = dict(pool.map(run, ["plain", "contracted"]))
    OUT.write_text(json.dumps({"record_steps": 4000, "steps": STEPS, "orders": res}) + "\n")
    print(OUT, {k: (v["status"], v["failed_step"]) for k, v in res.items()})


if __name__ == "__main__":
    main()
