"""Autotuner of the launch shapes of a handle (strut_gpu_set_tuning).

The kernels' results do not depend on their launch shapes (fixed reduction orders, and an attempt
fan-out that keeps the sequential order's outcome), so the tuner is free to pick, per workload
class, whatever runs fastest:

  fan_out          forceBeamColumn2d attempts of an element that needed a subdivision: twelve CTAs
                   at once (1) or one after another (0)
  element_threads  640 threads per element CTA (one CTA per SM, the shortest per-element
                   iteration), 320, 224 or 160 (2D): more CTAs per SM, more elements in flight
  commit_team      64 or 128 threads per integration point in the commit kernel
  factor_ctas      CTAs of the cooperative wide-band factorisation (wide bands only)

The search is a coordinate descent from the defaults: each knob in turn takes each of its values
with the others at their best so far, every trial a fresh handle running the caller's own models
for the same steps, timed with CUDA events on the handle's stream.  Every trial's histories must
equal the first trial's bit for bit (the tuner raises otherwise).  Winners are kept in a table
keyed by workload class (ndf, fibers per section, instances, band kind), tuned_shapes.json beside
this file, which the bench and callers reuse without searching again.  Strut has no counterpart
(it runs one CPU thread).
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

from . import _abi as A
from . import runtime

TABLE = Path(__file__).resolve().parent / "tuned_shapes.json"
KNOBS = ("fan_out", "element_threads", "commit_team", "factor_ctas")
DEFAULTS = {"fan_out": 1, "element_threads": 640, "commit_team": 0, "factor_ctas": 0}


def _bucket(x: int) -> int:
    """Power-of-two bucket of a count (1, 2, 4, 8, ...)."""
    b = 1
    while b < x:
        b *= 2
    return b


def workload_class(models, wide_band: bool) -> str:
    """Key of a batch in the table: ndf, the largest section's fiber count and the instance count
    (power-of-two buckets), and whether a band lives in global memory."""
    ndf = models[0].ndf
    fibers = max((s.fiber_count for m in models for s in m.sections), default=0)
    return f"ndf{ndf}-fib{_bucket(fibers)}-inst{_bucket(len(models))}-{'wide' if wide_band else 'smem'}"


def candidates(models, wide_band: bool, max_nip: int, n_sm: int = 148):
    """Values each knob may take for this batch."""
    has_fbc2d = any(int(e.type) == A.ELEM_FORCE_BEAM_COLUMN_2D for m in models for e in m.elements)
    c = {"fan_out": [1, 0] if has_fbc2d else [1],
         "element_threads": [640, 320, 224] + ([160] if models[0].ndf == 3 else []),
         "commit_team": [0] + ([64, 128] if max_nip <= 5 else [64]),
         "factor_ctas": [0, n_sm // 4, n_sm // 2, n_sm] if wide_band else [0]}
    return c


def coordinate_search(trial, cands: dict, start: dict | None = None):
    """trial(tuning dict) -> (ms, fingerprint).  Returns (best tuning, {key: ms}) after one pass
    of coordinate descent; raises if two trials' fingerprints differ."""
    best = dict(DEFAULTS if start is None else start)
    times = {}
    ref = None

    def run(t):
        nonlocal ref
        key = json.dumps(t, sort_keys=True)
        if key not in times:
            ms, fp = trial(dict(t))
            if ref is None:
                ref = fp
            elif fp != ref:
                raise RuntimeError(f"tuning {t} changed the results")
            times[key] = ms
        return times[key]

    best_ms = run(best)
    for knob in KNOBS:
        for v in cands.get(knob, [best[knob]]):
            t = dict(best)
            t[knob] = v
            ms = run(t)
            if ms < best_ms:
                best, best_ms = t, ms
    return best, times


def _fingerprint(an) -> str:
    d, e, it = an.history_all()
    st = an.instance_status()
    h = hashlib.sha256()
    for a in (d, e, it, st):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def tune(models, steps: int, device: int = -1, save: bool = True, table: Path = TABLE):
    """Searches the launch shapes for this batch on `steps` steps of its own records; returns
    (class key, best tuning, {tuning: ms}) and, with save, records the winner in the table."""
    import torch

    with runtime.Analysis(models, device=device, tuned=False) as an:
        wide = any(an.band_info(i)[1] * 8 * models[i].num_free > 220 * 1024 for i in range(len(models)))
        max_nip = max((int(m.integrations[e.integration].num_int_pts) for m in models for e in m.elements),
                      default=1)
    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    key = workload_class(models, wide)

    def trial(t):
        with runtime.Analysis(models, device=device, tuned=False) as an:
            an.set_tuning(**t)
            stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            an.run(steps, check=False)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1), _fingerprint(an)

    best, times = coordinate_search(trial, candidates(models, wide, max_nip, n_sm))
    if save:
        tab = load_table(table)
        tab[key] = {"tuning": best, "steps": steps, "ms": times}
        table.write_text(json.dumps(tab, indent=1, sort_keys=True) + "\n")
    return key, best, times


def load_table(table: Path = TABLE) -> dict:
    return json.loads(table.read_text()) if table.exists() else {}


def lookup(models, wide_band: bool, table: Path = TABLE):
    """The table's tuning for this batch's class, or None."""
    ent = load_table(table).get(workload_class(models, wide_band))
    return dict(ent["tuning"]) if ent else None


def apply(an, table: Path = TABLE):
    """Sets the table's tuning for the analysis's batch, if its class has one; returns it."""
    wide = any(an.band_info(i)[1] * 8 * an.models[i].num_free > 220 * 1024 for i in range(len(an.models)))
    t = lookup(an.models, wide, table)
    if t:
        an.set_tuning(**t)
    return t
