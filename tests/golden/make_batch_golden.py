#!/usr/bin/env python3
"""Writes batch256_outcomes.json: the CPU oracle's outcome of every record of the 256-frame
batch (seeds 1000..1255, 2000 steps, dt 0.01 s, NormDispIncr 1e-8) at two summation orders of
the reference's algorithm, SIMD widths 8 and 1 (solver/simd_contiguous.mojo:6): per record its
status, failing step (-1: none) and Newton iterations.  The GPU batch test compares the GPU's
per-record outcome with these on every record where the two orders agree.  About 25 minutes on 8
host threads.

    python tests/golden/make_batch_golden.py [threads]
"""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import binding  # noqa: E402
from strut_b200 import model as M  # noqa: E402
from strut_b200 import workloads as W  # noqa: E402

FRAMES, STEPS, DT, SEED = 256, 2000, 0.01, 1000


def main():
    nthreads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    binding.build()
    models = [M.Model(c) for c in W.batched_frames(FRAMES, steps=STEPS, dt=DT, base_seed=SEED)]
    out = {"frames": FRAMES, "steps": STEPS, "dt": DT, "base_seed": SEED, "orders": {}}
    try:
        for w in (8, 1):
            binding.set_simd_width(w)
            t0 = time.time()
            _rc, _tot, st, fs, it = binding.run_batch(models, STEPS, nthreads, detail=True)
            out["orders"][f"simd{w}"] = {"status": st.tolist(), "failed_step": fs.tolist(),
                                          "newton_iterations": it.tolist()}
            print(f"width {w}: {int((st != 0).sum())} failed, {time.time() - t0:.0f} s", flush=True)
    finally:
        binding.set_simd_width(8)
    (HERE / "batch256_outcomes.json").write_text(json.dumps(out) + "\n")


if __name__ == "__main__":
    main()
