#!/usr/bin/env python3
"""Writes batch256_outcomes.json: the CPU oracle's outcome of every record of the 256-frame
batch (seeds 1000..1255, 2000 steps, dt 0.01 s, NormDispIncr 1e-8) under four roundings of the
reference's algorithm: SIMD widths 8 and 1 of its lane-chunked sums (solver/simd_contiguous.mojo:6),
each with separately rounded multiplies and adds (liboracle.so) and with contracted multiply-adds
(liboracle_fma.so): per record its status, failing step (-1: none) and Newton iterations.  The GPU
batch test compares the GPU's per-record outcome with these on every record where all orders
agree.  About 12 minutes per order on 8 host threads; orders already in the file are kept unless
--force is given.

    python tests/golden/make_batch_golden.py [threads] [--force]
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


ORDERS = (("simd8", 8, False), ("simd1", 1, False), ("simd8_fma", 8, True), ("simd1_fma", 1, True))


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    nthreads = int(args[0]) if args else (os.cpu_count() or 1)
    path = HERE / "batch256_outcomes.json"
    out = {"frames": FRAMES, "steps": STEPS, "dt": DT, "base_seed": SEED, "orders": {}}
    if path.exists() and "--force" not in sys.argv:
        old = json.loads(path.read_text())
        if all(old.get(k) == out[k] for k in ("frames", "steps", "dt", "base_seed")):
            out["orders"] = old["orders"]
    models = [M.Model(c) for c in W.batched_frames(FRAMES, steps=STEPS, dt=DT, base_seed=SEED)]
    try:
        for name, w, fma in ORDERS:
            if name in out["orders"]:
                continue
            binding.build(fma=fma)
            binding.use_fma(fma)
            binding.set_simd_width(w)
            t0 = time.time()
            _rc, _tot, st, fs, it = binding.run_batch(models, STEPS, nthreads, detail=True)
            out["orders"][name] = {"status": st.tolist(), "failed_step": fs.tolist(),
                                   "newton_iterations": it.tolist()}
            print(f"{name}: {int((st != 0).sum())} failed, {time.time() - t0:.0f} s", flush=True)
            path.write_text(json.dumps(out) + "\n")
    finally:
        binding.set_simd_width(8)
        binding.use_fma(False)
    path.write_text(json.dumps(out) + "\n")


if __name__ == "__main__":
    main()
