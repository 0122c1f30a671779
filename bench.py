#!/usr/bin/env python3
"""Benchmark: batched plain nonlinear transient analysis of uneven 2D RC frames.

Workload (one bench step): 256 independent 2D RC moment frames (stories U{3..12}, bays
U{2..5}, forceBeamColumn2d with 5 Lobatto points and 148-fiber sections), each with its own
seeded Kanai-Tajimi record (wg U(8, 25) rad/s, PGA U(0.2, 0.6) g), Newmark (0.5, 0.25),
dt 0.01 s, 2000 steps, Newton with NormDispIncr 1e-8, BandGeneral -- the whole record, run in
one handle with per-instance convergence masks.  Inputs are synthetic (seeded generator).

Metric: records/hour (whole job).  Also reported: Newton iterations per step, fiber-state
updates/s, simulated seconds per wall second.

  value   device time of the analysis (CUDA events on the library's launching stream), model
          already resident in HBM
  e2e     the public API call a user makes: create (host -> device copy of all model data and
          records) + run + read back the recorded histories, timed on the host with device
          synchronisation, per bench step (min(K, 3) repetitions)
  roofline          the element kernel (most of the device time): fiber-state update bytes of
                    its section evaluations (80 B per Concrete02 fiber, 168 B per Steel02 fiber)
                    over its event-timed launches
  fiber_kernel      the streaming fiber-state update kernel alone (strut_gpu_section_eval_batch)
                    over as many RC column sections as the batch has fibers
  commit_kernel     the commit kernel's history reads and writes over its launches
  tall_frame3d      the 20-story 6x6-bay 3D frame (one instance, band in global memory), the
                    whole 4000-step record
Multi-GPU (one process per GPU, no collective on the data path, timing = max over ranks):
--scaling weak (default) gives every rank its own 256 frames (records seeded per rank);
--scaling strong partitions one fixed 256-frame batch across the ranks by fiber count.

Learned arm (``learned`` in the line, off with --no-learned): a per-node network trained on the
tensor cores on plain histories of 64 other frames proposes each step's first Newton guess; the
first iteration keeps it only where its residual beats the Newmark predictor's.

``--impl reference`` times the reference algorithm's CPU implementation (the CPU oracle, a
plain C restatement of Strut's path; Strut itself is Mojo and cannot be built here) on all host
cores over the same batch: every record of it, all 2000 steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_FRAMES = 256
STEPS = 2000
DT = 0.01
METRIC = "records/hour (batched plain GPU, 256 uneven 2D RC frames x 2000 steps, NormDispIncr 1e-8)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=N_FRAMES)
    ap.add_argument("--record-steps", type=int, default=STEPS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-predictor arm")
    ap.add_argument("--train-frames", type=int, default=64)
    ap.add_argument("--train-epochs", type=int, default=60)
    ap.add_argument("--learned3d-steps", type=int, default=4000,
                    help="record steps of the 3D learned-predictor arm (config 3)")
    ap.add_argument("--no-learned3d", action="store_true", help="skip the 3D learned-predictor arm")
    ap.add_argument("--no-slab", action="store_true", help="skip the batched slab-frame window (config 4)")
    ap.add_argument("--slab-frames", type=int, default=8)
    ap.add_argument("--slab-steps", type=int, default=10)
    ap.add_argument("--slab-train-frames", type=int, default=8)
    ap.add_argument("--slab-train-steps", type=int, default=40)
    ap.add_argument("--no-tall", action="store_true",
                    help="skip the large single-instance 3D frame (20 stories, 6x6 bays)")
    ap.add_argument("--tall-steps", type=int, default=4000,
                    help="timed steps of the 4000-step large 3D frame record (default: all)")
    ap.add_argument("--no-fiber", action="store_true", help="skip the streaming fiber-kernel measurement")
    ap.add_argument("--autotune", action="store_true",
                    help="search the launch shapes on the whole batch, record them in "
                         "strut_b200/tuned_shapes.json, print the result and exit")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="N > 1: every rank its own 256 frames (weak) or one batch partitioned (strong)")
    ap.add_argument("--profile-only", action="store_true",
                    help="one short analysis (for a profiler launch list); prints no bench line")
    ap.add_argument("--profile-tall", action="store_true",
                    help="with --profile-only: --tall-steps steps of the 20-story 3D frame instead")
    ap.add_argument("--element-threads", type=int, default=0,
                    help="with --profile-only: element CTA size (0: the library default)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def build_models(n_frames, steps, base_seed):
    from strut_b200 import model, workloads

    cases = workloads.batched_frames(n_frames, steps=steps, dt=DT, base_seed=base_seed)
    return [model.Model(c) for c in cases], cases


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(models, nthreads=None):
    """The CPU oracle (a C restatement of Strut's single-threaded path) over all host threads,
    on a bounded sample of the same workload: the first `nthreads` frames of the batch, each
    one whole 2000-step record on its own thread (as Strut runs a record).  Returns
    (records/hour, cores, sample text)."""
    from oracle import binding

    binding.build()
    nthreads = nthreads or os.cpu_count() or 1
    sub = models[:min(len(models), nthreads)]
    t0 = time.perf_counter()
    _rc, tot_iters, st = binding.run_batch(sub, STEPS, nthreads)
    el = time.perf_counter() - t0
    n_ok = int((st == 0).sum())
    rph = n_ok / el * 3600.0
    sample = (f"frames 0-{len(sub) - 1} of the batch, whole {STEPS}-step records, one per thread on "
              f"{nthreads} threads: {n_ok} completed in {el:.1f} s, {tot_iters / (len(sub) * STEPS):.2f} "
              f"Newton its/step")
    return rph, nthreads, sample


def tall_arm(args, device, runtime, A, torch):
    """The large single instance: the 20-story 6x6-bay 3D RC frame with rigid diaphragms
    (1029 nodes, 2660 elements, 2.77 M fibers, 3000 free dofs, band in global memory), two
    horizontal records, dt 0.005 s: device time of --tall-steps steps (default the whole
    4000-step record) after 3 warm-up steps of a separate handle (its fiber history, 2.77 M
    fibers x ~10 doubles, exceeds L2).  Beside it, the CPU oracle's time per Newton iteration on
    the first steps, scaled to the GPU run's iterations per step (the oracle refactors the band
    densely every iteration, so its step time is its iteration time x the iteration count)."""
    from strut_b200 import model as M
    from strut_b200 import workloads as W

    steps = min(args.tall_steps, 4000)
    case = W.tall_frame3d_case(steps=max(steps, 3))
    m = M.Model(case)
    with runtime.Analysis([m], device=device) as an:
        an.run(3, check=False)
    an = runtime.Analysis([m], device=device)
    stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    an.run(steps, check=False)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    _d, _e, it = an.history(0)
    status = int(an.instance_status()[0])
    done = an.steps_done
    an.close()
    ms_step = ms / max(done, 1)
    its = float(np.mean(it)) if len(it) else None
    out = {"workload": "tall_3d_rc_frame_20s_6x6b_diaphragm", "nodes": m.num_nodes,
           "elements": len(m.elements), "free_dofs": m.num_free, "fibers": m.num_fibers_total,
           "record_steps": 4000, "dt": 0.005, "steps_timed": done, "warmup_steps": 3,
           "ms_per_step": ms_step, "records_per_hour": 3600.0 / (ms_step * 4000 / 1000.0),
           "newton_its_per_step": its, "status": status}
    if not args.no_cpu_baseline and its:
        from oracle import binding as O

        O.build()
        k = 3
        t0 = time.perf_counter()
        _d, _e, cit, rc, _f = O.run_transient(m, k)
        t = time.perf_counter() - t0
        per_it = t / max(int(cit.sum()), 1)
        step_s = per_it * its
        out["cpu_baseline"] = {"value": 3600.0 / (step_s * 4000), "unit": "records/hour", "cores": 1,
                               "kind": "port", "status": int(rc),
                               "sample": f"first {k} of 4000 steps on 1 thread: {per_it:.2f} s per Newton "
                                         f"iteration, x {its:.2f} iterations per step (the GPU run's mean)"}
    return out


def fiber_arm(n_fibers, runtime, torch, peak, steps=20, warmup=3):
    """The streaming fiber-state update kernel alone: one RC column section (140 Concrete02
    and 8 Steel02 fibers) in as many instances as the batch has fibers, each with its own
    committed history; every call reads and rewrites every fiber's history once (80 B per
    Concrete02 fiber, 168 B per Steel02 fiber) at strains that cycle with a growing amplitude,
    so fibers load, unload and reverse.  Device time of `steps` calls after `warmup` calls; the
    histories (~1 GB) exceed L2."""
    from strut_b200 import model as Mo
    from strut_b200 import workloads as W

    case = {"materials": [{"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
                          {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
                          {"id": 3, "type": "Steel02", "params": dict(W.STEEL)}],
            "section": W.rc_section(1, 0.5, 0.5)}
    mats, nm, fibs, nf = Mo.section_fibers(case["section"], case["materials"])
    n = (n_fibers + nf - 1) // nf
    b = runtime.SectionBatch(mats, nm, fibs, nf, n)
    tot = steps + warmup
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    ph = torch.rand((1, n), generator=gen, device="cuda", dtype=torch.float64) * 6.283185307179586
    t = torch.arange(tot, device="cuda", dtype=torch.float64)[:, None]
    amp = (t + 1.0) / tot
    ek = torch.empty((tot, n, 2), dtype=torch.float64, device="cuda")
    ek[:, :, 0] = -3.0e-4 + 2.0e-4 * torch.sin(0.7 * t + ph)
    ek[:, :, 1] = 8.0e-3 * amp * torch.sin(0.9 * t + 2.0 * ph)
    resp = torch.empty((n, 5), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    for k in range(warmup):
        b.eval(ek[k].data_ptr(), resp.data_ptr(), commit=True, stream=s.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for k in range(warmup, tot):
        b.eval(ek[k].data_ptr(), resp.data_ptr(), commit=True, stream=s.cuda_stream)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ok = bool(torch.isfinite(resp).all().item())
    b.close()
    n_c2 = sum(1 for f in range(nf) if mats[fibs[f].material].type == 4)
    n_s2 = sum(1 for f in range(nf) if mats[fibs[f].material].type == 3)
    per_section = 80 * n_c2 + 168 * n_s2
    achieved = n * per_section / (ms / 1000.0) / 1e9
    return {"kernel": "fiber_stream_kernel", "bound": "hbm", "sections": n, "fibers": n * nf,
            "bytes_per_section": per_section, "launches": steps, "avg_launch_ms": ms,
            "fiber_state_updates_per_s": n * nf / (ms / 1000.0),
            "achieved": achieved, "peak": peak[0], "unit": "GB/s", "frac": achieved / peak[0],
            "peak_kind": peak[1], "finite": ok}


def train_predictor(models, steps, device, runtime, every, epochs, seed=7):
    """Runs `models` (recording every dof) with the plain method, builds the learned predictor's
    features and targets from the converged histories (every `every`-th step of each completed
    record) and trains the network on the tensor cores.  Returns (predictor, info)."""
    from strut_b200 import predictor as PR

    t0 = time.perf_counter()
    rec = [PR.record_all_dofs(m) for m in models]
    with runtime.Analysis(rec, device=device) as an:
        an.run(steps, check=False)
        status = an.instance_status()
        Xs, Ts = [], []
        for i, m in enumerate(rec):
            if status[i] != 0:
                continue
            X, T = PR.raw_features(m, PR.free_history(an, i))
            nn = X.shape[0] // steps
            keep = (np.arange(X.shape[0]) // nn) % every == 0
            Xs.append(X[keep])
            Ts.append(T[keep])
    X, T = np.concatenate(Xs), np.concatenate(Ts)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    pred = PR.LearnedPredictor(models[0].ndf, seed=seed)
    loss = pred.fit(X, T, epochs=epochs, batch=8192, lr=1e-3, seed=11)
    info = {"records": len(models), "samples": int(X.shape[0]), "epochs": epochs,
            "final_mse_normalised": loss, "data_s": round(t_data, 1),
            "train_s": round(time.perf_counter() - t0, 1),
            "network": f"{PR.n_features(models[0].ndf)}-128-128-{models[0].ndf} bf16 tcgen05, GELU"}
    return pred, info


def timed_run(models, steps, device, runtime, torch, pred=None):
    """One analysis of `models`, device time; returns (ms, stats, completed, histories, pred
    stats)."""
    from strut_b200 import predictor as PR

    an = runtime.Analysis(models, device=device)
    if pred is not None:
        pred.attach(an)
    stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    st = an.run(steps, check=False)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    status = an.instance_status()
    hist = an.history_all()
    ps = PR.stats(an) if pred is not None else (0, 0)
    an.close()
    return ms, st, int((status == 0).sum()), (hist, status), ps


def learned_arm(args, models, device, runtime, A, torch, world):
    """The learned+batched arm on the plain arm's batch: the per-node network (tensor-core
    kernels) is trained on histories the plain method computes for 64 other frames and records
    (seeds 5000+), then the same batch runs with the network proposing each step's first guess.
    Untimed: data generation and training; timed (device events): the analysis."""
    from strut_b200 import model as Mo, workloads as W

    tmodels = [Mo.Model(c) for c in W.batched_frames(args.train_frames, steps=args.record_steps, dt=DT,
                                                      base_seed=5000)]
    pred, info = train_predictor(tmodels, args.record_steps, device, runtime, 4, args.train_epochs)
    if world > 1:
        torch.distributed.barrier()
    ms, st, completed, _h, (offered, chosen) = timed_run(models, args.record_steps, device, runtime, torch, pred)
    if world > 1:
        t = torch.tensor([ms, completed], dtype=torch.float64, device="cuda")
        mx = t.clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t)
        ms, completed = float(mx[0].item()), int(t[1].item())
    return {
        "value": completed / (ms / 1000.0) * 3600.0, "unit": "records/hour", "ms": ms,
        "newton_its_per_step": st.global_newton_iterations / float(len(models) * args.record_steps),
        "records_completed": completed,
        "learned_guess_kept_frac": chosen / max(offered, 1),
        "train": info,
    }


def learned3d_arm(args, device, runtime, torch):
    """Config 3's learned predictor on 3D RC frames with rigid diaphragms (4 stories, 3x3 bays of
    6 m, forceBeamColumn3d columns, dispBeamColumn3d beams, 148-fiber sections, a diaphragm per
    floor) under two horizontal seeded Kanai-Tajimi records at PGA 0.4 g, dt 0.005 s: the
    41-feature network (6 dof x 4 increments, the 8 latest samples of each ground component, the
    height) is trained on the plain histories of 64 records (seeds 0-63) and evaluated on 32
    unseen records (seeds 64-95), plain and learned batches of those 32 timed on the device.  The
    frame is the largest of this family whose band fits the instance kernel's shared memory."""
    from strut_b200 import model as Mo, workloads as W

    steps = args.learned3d_steps

    def case(seed):
        return W.rc_frame3d_case(stories=4, bays_x=3, bays_y=3, steps=steps, dt=0.005, seed=seed,
                                 element="forceBeamColumn3d", beam_element="dispBeamColumn3d",
                                 diaphragm=True, bidirectional=True, pga_g=0.4)

    train = [Mo.Model(case(s)) for s in range(64)]
    pred, info = train_predictor(train, steps, device, runtime, 8, args.train_epochs)
    evals = [Mo.Model(case(s)) for s in range(64, 96)]
    ms0, st0, c0, (h0, s0), _ = timed_run(evals, steps, device, runtime, torch)
    ms1, st1, c1, (h1, s1), (offered, chosen) = timed_run(evals, steps, device, runtime, torch, pred)
    d0, d1 = h0[0], h1[0]
    ok = (s0 == 0) & (s1 == 0)
    worst = float(np.max(np.abs(d1 - d0)) / max(np.max(np.abs(d0)), 1e-300)) if ok.all() else None
    n = len(evals) * steps
    plain_rph = c0 / (ms0 / 1000.0) * 3600.0
    learned_rph = c1 / (ms1 / 1000.0) * 3600.0
    return {"workload": "diaphragm_3d_rc_frames_4s_3x3b_bidirectional", "train_records": 64,
            "eval_records": len(evals), "steps": steps, "dt": 0.005,
            "plain": {"records_per_hour": plain_rph, "ms": ms0, "newton_its_per_step": st0.global_newton_iterations / n,
                      "records_completed": c0},
            "learned": {"records_per_hour": learned_rph, "ms": ms1, "newton_its_per_step": st1.global_newton_iterations / n,
                        "records_completed": c1, "learned_guess_kept_frac": chosen / max(offered, 1)},
            "vs_plain": learned_rph / plain_rph if plain_rph else None,
            "max_disp_diff_of_peak_vs_plain": worst, "train": info}


def slab_arm(args, device, runtime, torch):
    """Config 4 on a window: a batch of `args.slab_frames` frames of the batched slab-frame set
    (stories U{10..30}, bays U{4..6} of 7 m, 2 x 2 ShellMITC4 slabs per bay, rigid diaphragms,
    two horizontal Kanai-Tajimi records at PGA U(0.3, 0.6) g, dt 0.005 s) in one handle, uneven
    sizes together; the device time of `args.slab_steps` steps after 3 warm-up steps, plain and
    with the learned predictor, whose network is retrained on the plain histories of other frames
    of the set (seeds 9000+) over the first `args.slab_train_steps` steps.  The whole set (256
    frames x 4000 steps) is out of reach of one timed run; records/hour is the batch at this
    window's rate over a 4000-step record."""
    from strut_b200 import model as Mo, workloads as W

    steps = 3 + args.slab_steps

    def build(n, seed0, st):
        return [Mo.Model(W.slab_frame3d_case(p["stories"], p["bays"], steps=st, seed=p["seed"], pga_g=p["pga_g"],
                                             wg=p["wg"]))
                for p in W.slab_frame_params(n, base_seed=seed0)]

    train = build(args.slab_train_frames, 9000, args.slab_train_steps)
    pred, info = train_predictor(train, args.slab_train_steps, device, runtime, 1, args.train_epochs)
    models = build(args.slab_frames, 8000, steps)
    out = {"workload": "slab_3d_rc_frames_10to30s_4to6b_bidirectional", "frames": len(models),
           "fibers": int(sum(m.num_fibers_total for m in models)), "free_dofs": int(sum(m.num_free for m in models)),
           "steps_timed": args.slab_steps, "warmup_steps": 3, "record_steps": 4000, "dt": 0.005, "train": info}
    for arm, p in (("plain", None), ("learned", pred)):
        an = runtime.Analysis(models, device=device)
        if p is not None:
            p.attach(an)
        an.run(3, check=False)
        stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = an.run(args.slab_steps, check=False)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        ok = int((an.instance_status() == 0).sum())
        from strut_b200 import predictor as PR

        offered, chosen = PR.stats(an) if p is not None else (0, 0)
        an.close()
        ms_step = ms / args.slab_steps
        out[arm] = {"ms_per_step": ms_step, "records_per_hour": ok * 3600.0 / (ms_step * 4000 / 1000.0),
                    "records_running": ok,
                    "newton_its_per_step": st.global_newton_iterations / float(len(models) * args.slab_steps)}
        if p is not None:
            out[arm]["learned_guess_kept_frac"] = chosen / max(offered, 1)
    out["vs_plain"] = (out["learned"]["records_per_hour"] / out["plain"]["records_per_hour"]
                       if out["plain"]["records_per_hour"] else None)
    return out


def run_reference(args):
    """The reference algorithm's CPU implementation (the oracle) on all host threads over the
    whole batch: every record, all of its steps, one record per thread at a time as Strut runs
    it.  The K bench steps are K shares of the batch run together in one pool of threads (so
    that the run's length does not depend on K); records/hour = completed records / wall time."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import binding

    binding.build()
    models, cases = build_models(args.frames, args.record_steps, 1000)
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    _rc, tot_iters, st = binding.run_batch(models, args.record_steps, nthreads)
    el = time.perf_counter() - t0
    n_ok = int((st == 0).sum())
    v = n_ok / el * 3600.0
    sample = (f"all {len(models)} frames of the batch, whole {args.record_steps}-step records on {nthreads} "
              f"threads: {n_ok} completed in {el:.1f} s, {tot_iters / (len(models) * args.record_steps):.2f} "
              f"Newton its/step")
    line = {
        "impl": "reference",
        "metric": METRIC, "value": v, "unit": "records/hour", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic (seeded Kanai-Tajimi records, generated RC frames)",
        "config": {"workload": "batched_plain_2d_rc_frames", "frames": args.frames,
                   "steps_per_record": args.record_steps, "dt": DT},
        "records_completed": n_ok,
        "cpu_baseline": {"value": v, "unit": "records/hour", "cores": nthreads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "records/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "vs_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    device = torch.cuda.current_device()
    from strut_b200 import _abi as A
    from strut_b200 import build as B
    from strut_b200 import runtime

    if rank == 0:
        B.build()
    if world > 1:
        torch.distributed.barrier()

    if args.profile_only and args.profile_tall:
        from strut_b200 import model as Mo
        from strut_b200 import workloads as W

        m = Mo.Model(W.tall_frame3d_case(steps=args.tall_steps))
        with runtime.Analysis([m], device=device) as an:
            runtime.lib().strut_gpu_set_profiling(an.h, 1)
            an.run(args.tall_steps, check=False)
            P = A.StrutKernelProfile()
            runtime.lib().strut_gpu_get_profile(an.h, __import__("ctypes").byref(P))
        if rank == 0:
            names = ("element", "instance", "commit", "predictor", "post")
            print(json.dumps({"profile": {n: {"launches": int(P.launches[i]), "ms": P.ms[i]}
                                          for i, n in enumerate(names)},
                              "workload": "tall_3d_rc_frame_20s_6x6b_diaphragm", "steps": args.tall_steps}))
        return 0

    if args.scaling == "strong" and world > 1:
        from strut_b200 import distributed as D

        all_models, all_cases = build_models(args.frames, args.record_steps, 1000)
        share = D.rank_share([m.num_fibers_total for m in all_models], world, rank)
        models = [all_models[i] for i in share]
        total_frames = args.frames
    else:
        models, _cases = build_models(args.frames, args.record_steps, 1000 + rank * args.frames)
        total_frames = args.frames * world
    n_fibers = sum(m.num_fibers_total for m in models)

    if args.profile_only:
        # host-driven loop (profiling mode): plain launches a profiler can attribute (kernel
        # nodes of a graph with conditional nodes cannot be profiled one by one)
        with runtime.Analysis(models, device=device) as an:
            if args.element_threads:
                an.set_tuning(element_threads=args.element_threads)
            runtime.lib().strut_gpu_set_profiling(an.h, 1)
            an.run(min(50, args.record_steps), check=False)
            P = A.StrutKernelProfile()
            runtime.lib().strut_gpu_get_profile(an.h, __import__("ctypes").byref(P))
        if rank == 0:
            names = ("element", "instance", "commit", "predictor", "post")
            print(json.dumps({"profile": {n: {"launches": int(P.launches[i]), "ms": P.ms[i],
                                              "algorithmic_bytes": P.bytes[i]}
                                          for i, n in enumerate(names)},
                              "frames": len(models), "steps": min(50, args.record_steps)}))
        return 0

    from strut_b200 import autotune

    if args.autotune:
        key, best, times = autotune.tune(models, args.record_steps, device=device, save=rank == 0)
        if rank == 0:
            print(json.dumps({"autotune": {"class": key, "best": best, "ms": times}}), flush=True)
        return 0

    def one_analysis(prof=False):
        an = runtime.Analysis(models, device=device)
        autotune.apply(an)
        if prof:
            runtime.lib().strut_gpu_set_profiling(an.h, 1)
        stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = an.run(args.record_steps, check=False)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        status = an.instance_status()
        if st.status not in (A.STRUT_OK, A.STRUT_NONCONVERGED):
            raise RuntimeError(f"analysis failed: status {st.status}")
        st.completed = int((status == 0).sum())
        prof_out = None
        if prof:
            P = A.StrutKernelProfile()
            runtime.lib().strut_gpu_get_profile(an.h, __import__("ctypes").byref(P))
            prof_out = P
        tuned = an.tuning()
        an.close()
        return ms, st, prof_out, tuned

    # warm-up (untimed)
    for _ in range(args.warmup):
        one_analysis()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # timed: K full batched analyses, device time
    with ClockSampler(device) as clk:
        times, stats = [], []
        for _ in range(args.steps):
            ms, st, _p, tuned = one_analysis()
            times.append(ms)
            stats.append(st)
    torch.cuda.synchronize()
    tot_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([tot_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        tot_ms = float(t.item())
    ms_per_step = tot_ms / args.steps
    st = stats[-1]
    # records that ran all steps (a record whose Newton iteration fails is masked out of the
    # batch at its failing step, as Strut would abort it; it is not counted)
    completed = st.completed
    if world > 1:
        t = torch.tensor([completed], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t)
        completed = int(t.item())
    value = completed / (ms_per_step / 1000.0) * 3600.0
    newton_per_step = st.global_newton_iterations / float(len(models) * args.record_steps)
    fiber_updates_per_s = sum(x.fiber_updates for x in stats) / (sum(times) / 1000.0)

    # end to end through the public API with host buffers (min(K, 3) repetitions)
    e2e_times = []
    h2d = d2h = 0
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with runtime.Analysis(models, device=device) as an:
            an.run(args.record_steps, check=False)
            disp, ef, it = an.history_all()
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        d2h = disp.nbytes + ef.nbytes + it.nbytes
    if world > 1:
        t = torch.tensor([max(e2e_times)], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    else:
        e2e_s = float(np.mean(e2e_times))
    # host bytes sent at create: model arrays + records
    for m in models:
        h2d += (len(m.fibers) * 32 + len(m.materials) * 96 + len(m.elements) * 48 +
                m.num_dofs * (8 * 4 + 4) + sum(len(x["values"]) * 8 for x in m.excitations))
    e2e_value = completed / e2e_s * 3600.0

    # rooflines, from one profiled analysis (host-driven loop, events around every launch)
    _ms, _st, P, _t = one_analysis(prof=True)
    peak = measured_peaks()

    def roof(k, name):
        launches = max(int(P.launches[k]), 1)
        ms_k = P.ms[k]
        achieved = (P.bytes[k] / launches) / ((ms_k / launches) / 1000.0) / 1e9 if ms_k > 0 else 0.0
        return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak[0], "unit": "GB/s",
                "frac": achieved / peak[0], "peak_kind": peak[1], "launches": int(P.launches[k]),
                "avg_launch_ms": ms_k / launches, "bytes_per_launch": P.bytes[k] / launches}

    roofline = roof(A.PROF_ELEMENT, "element_state_kernel")
    # measured DRAM traffic per launch: DRAM bytes per algorithmic byte of this kernel from one
    # ncu capture of a smaller batch of the same frames, times this run's algorithmic bytes
    roofline["traffic"] = None
    tp = ROOT / "profiles" / "element_state_kernel_dram_traffic_rc_frames96.md"
    if tp.exists():
        for line in tp.read_text().splitlines():
            if line.startswith("traffic_per_update_byte:"):
                roofline["traffic"] = float(line.split(":", 1)[1]) * roofline["bytes_per_launch"]
    commit_roof = roof(A.PROF_COMMIT, "commit_kernel")
    kernel_share = {k: P.ms[i] for k, i in (("element", 0), ("instance", 1), ("commit", 2),
                                              ("predictor", 3), ("post", 4))}

    fiber = None
    if not args.no_fiber:
        fiber = fiber_arm(n_fibers, runtime, torch, peak)

    learned = None
    if not args.no_learned:
        learned = learned_arm(args, models, device, runtime, A, torch, world)

    learned3d = None
    if rank == 0 and world == 1 and not args.no_learned3d:
        learned3d = learned3d_arm(args, device, runtime, torch)

    slab = None
    if rank == 0 and world == 1 and not args.no_slab:
        slab = slab_arm(args, device, runtime, torch)

    tall = None
    if rank == 0 and world == 1 and not args.no_tall:
        tall = tall_arm(args, device, runtime, A, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rph, cores, sample = cpu_baseline(models)
        cpu = {"value": rph, "unit": "records/hour", "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "records/hour",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "strong" if (args.scaling == "strong" and world > 1) else "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded Kanai-Tajimi records, generated RC frames)",
            "config": {"workload": "batched_plain_2d_rc_frames", "frames_total": total_frames,
                       "frames_per_gpu": len(models),
                       "steps_per_record": args.record_steps, "dt": DT,
                       "fibers_per_gpu": n_fibers,
                       "parallelism": (f"partition{world}" if args.scaling == "strong" and world > 1
                                       else f"replicas{world}"),
                       "tuned": {"fan_out": int(tuned.fan_out), "commit_team": int(tuned.commit_team),
                                 "element_threads": int(tuned.element_threads),
                                 "source": ("strut_b200/tuned_shapes.json" if autotune.lookup(models, False)
                                            else "defaults")},
                       "l2": "fiber history of the batch exceeds L2 (no flush needed)"},
            "newton_its_per_step": newton_per_step,
            "records_completed": completed,
            "records_failed_nonconvergence": total_frames - completed,
            "fiber_state_updates_per_s": fiber_updates_per_s,
            "simulated_s_per_wall_s": total_frames * args.record_steps * DT / (ms_per_step / 1000.0),
            "fanned_out_determinations": int(st.fanned_out),
            "e2e": {"value": e2e_value, "unit": "records/hour", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "repetitions": len(e2e_times)},
            "roofline": roofline,
            "commit_kernel": commit_roof,
            "kernel_ms": kernel_share,
            # launches of one analysis (profiled run, same workload) x timed analyses; the
            # displacement-record kernel runs once per step
            "gpu_launches": int(args.steps * (sum(P.launches[i] for i in range(5)) + st.steps_done)),
            "clocks": clk.summary(),
        }
        if fiber:
            line["fiber_kernel"] = fiber
        if learned:
            learned["vs_plain"] = learned["value"] / value if value else None
            line["learned"] = learned
        if learned3d:
            line["learned_3d"] = learned3d
        if slab:
            line["slab_frames_window"] = slab
        if cpu:
            line["cpu_baseline"] = cpu
        if tall:
            line["tall_frame3d"] = tall
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
