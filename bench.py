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
          synchronisation, per bench step
Multi-GPU: one process per GPU, each with its own 256 frames (records seeded per rank): weak
scaling, no collective on the data path; the timing is the max over ranks.

Learned arm (``learned`` in the line, off with --no-learned): a per-node network trained on the
tensor cores on plain histories of 64 other frames proposes each step's first Newton guess; the
first iteration keeps it only where its residual beats the Newmark predictor's.

``--impl reference`` times the reference algorithm's CPU implementation (the CPU oracle, a
plain C restatement of Strut's path; Strut itself is Mojo and cannot be built here) on all host
cores over a bounded sample of the same workload.
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
    ap.add_argument("--train-epochs", type=int, default=8)
    ap.add_argument("--no-tall", action="store_true",
                    help="skip the large single-instance 3D frame (20 stories, 6x6 bays)")
    ap.add_argument("--tall-steps", type=int, default=60,
                    help="timed steps of the 4000-step large 3D frame record")
    ap.add_argument("--profile-only", action="store_true",
                    help="one short analysis (for a profiler launch list); prints no bench line")
    ap.add_argument("--profile-tall", action="store_true",
                    help="with --profile-only: --tall-steps steps of the 20-story 3D frame instead")
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


def cpu_baseline(models, cases, nthreads=None, target_s=15.0):
    """The CPU oracle (a C restatement of Strut's single-threaded path) over all host threads,
    on a bounded sample of the same workload: the first frames of the batch for a number of
    steps sized to ~target_s of wall time.  Returns (records/hour, cores, sample text)."""
    from oracle import binding

    binding.build()
    nthreads = nthreads or os.cpu_count() or 1
    nfr = min(len(models), max(nthreads, 1) * 2)
    sub = models[:nfr]
    # probe: 20 steps on the sample
    t0 = time.perf_counter()
    binding.run_batch(sub, 20, nthreads)
    probe = time.perf_counter() - t0
    steps = int(min(STEPS, max(20, 20 * target_s / max(probe, 1e-3))))
    t0 = time.perf_counter()
    _rc, tot_iters, st = binding.run_batch(sub, steps, nthreads)
    el = time.perf_counter() - t0
    # like the GPU arm, only records that ran every step count; failed ones still cost time
    n_ok = int((st == 0).sum())
    records = n_ok * steps / float(STEPS)
    rph = records / el * 3600.0
    sample = (f"{nfr} frames of the batch x {steps} of {STEPS} steps on {nthreads} threads, "
              f"{n_ok} completed, {el:.1f} s, {tot_iters / (nfr * steps):.2f} Newton its/step")
    return rph, nthreads, sample


def tall_arm(args, device, runtime, A, torch):
    """The large single instance: the 20-story 6x6-bay 3D RC frame with rigid diaphragms
    (1029 nodes, 2660 elements, 2.77 M fibers, 3000 free dofs, band in global memory), two
    horizontal records, dt 0.005 s.  Device time of --tall-steps steps after 3 warm-up steps
    (its fiber history, 2.77 M fibers x ~10 doubles, exceeds L2); records/hour is one 4000-step
    record at that rate.  Beside it, the CPU oracle on 2 steps of the same record."""
    from strut_b200 import model as M
    from strut_b200 import workloads as W

    case = W.tall_frame3d_case(steps=args.tall_steps + 3)
    m = M.Model(case)
    an = runtime.Analysis([m], device=device)
    an.run(3, check=False)
    stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    an.run(args.tall_steps, check=False)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    _d, _e, it = an.history(0)
    status = int(an.instance_status()[0])
    an.close()
    ms_step = ms / args.tall_steps
    out = {"workload": "tall_3d_rc_frame_20s_6x6b_diaphragm", "nodes": m.num_nodes,
           "elements": len(m.elements), "free_dofs": m.num_free, "fibers": m.num_fibers_total,
           "record_steps": 4000, "dt": 0.005, "steps_timed": args.tall_steps, "warmup_steps": 3,
           "ms_per_step": ms_step, "records_per_hour": 3600.0 / (ms_step * 4000 / 1000.0),
           "newton_its_per_step": float(np.mean(it[3:])) if len(it) > 3 else None,
           "status": status}
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT))
        from oracle import binding as O

        O.build()
        t0 = time.perf_counter()
        rc = O.run_transient(m, 2)[3]
        t = (time.perf_counter() - t0) / 2.0
        out["cpu_baseline"] = {"value": 3600.0 / (t * 4000), "unit": "records/hour", "cores": 1,
                               "kind": "port", "status": int(rc),
                               "sample": f"first 2 of 4000 steps on 1 thread, {t:.2f} s/step"}
    return out


def learned_arm(args, models, device, runtime, A, torch, world):
    """The learned+batched arm: train the per-node network (tensor-core kernels) on histories the
    plain method computes for separate training frames and records (seeds 5000+), then run the
    same batch as the plain arm with the network proposing each step's first guess.  Untimed:
    data generation and training; timed (device events): the analysis."""
    from strut_b200 import model as Mo, predictor as PR, workloads as W

    t0 = time.perf_counter()
    tcases = W.batched_frames(args.train_frames, steps=args.record_steps, dt=DT, base_seed=5000)
    tmodels = [PR.record_all_dofs(Mo.Model(c)) for c in tcases]
    with runtime.Analysis(tmodels, device=device) as an:
        an.run(args.record_steps, check=False)
        status = an.instance_status()
        Xs, Ts = [], []
        for i, m in enumerate(tmodels):
            if status[i] != 0:
                continue
            X, T = PR.raw_features(m, PR.free_history(an, i))
            nn = X.shape[0] // args.record_steps
            keep = (np.arange(X.shape[0]) // nn) % 4 == 0  # every 4th step
            Xs.append(X[keep])
            Ts.append(T[keep])
    X, T = np.concatenate(Xs), np.concatenate(Ts)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    pred = PR.LearnedPredictor(tmodels[0].ndf, seed=7)
    loss = pred.fit(X, T, epochs=args.train_epochs, batch=8192, lr=1e-3, seed=11)
    t_train = time.perf_counter() - t0

    an = runtime.Analysis(models, device=device)
    pred.attach(an)
    stream = torch.cuda.ExternalStream(runtime.lib().strut_gpu_stream(an.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    st = an.run(args.record_steps, check=False)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    completed = int((an.instance_status() == 0).sum())
    offered, chosen = PR.stats(an)
    an.close()
    if world > 1:
        t = torch.tensor([ms, completed], dtype=torch.float64, device="cuda")
        mx = t.clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t)
        ms, completed = float(mx[0].item()), int(t[1].item())
    return {
        "value": completed / (ms / 1000.0) * 3600.0, "unit": "records/hour", "ms": ms,
        "newton_its_per_step": st.global_newton_iterations / float(args.frames * args.record_steps),
        "records_completed": completed,
        "learned_guess_kept_frac": chosen / max(offered, 1),
        "train": {"frames": args.train_frames, "samples": int(X.shape[0]), "epochs": args.train_epochs,
                  "final_mse_normalised": loss, "data_s": round(t_data, 1), "train_s": round(t_train, 1),
                  "network": f"{PR.n_features(tmodels[0].ndf)}-128-128-{tmodels[0].ndf} bf16 tcgen05, GELU"},
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    models, cases = build_models(args.frames, args.record_steps, 1000)
    vals = []
    info = None
    for _ in range(args.warmup):
        pass
    for _ in range(max(args.steps, 1)):
        rph, cores, sample = cpu_baseline(models, cases)
        vals.append(rph)
        info = (cores, sample)
    v = float(np.mean(vals))
    line = {
        "impl": "reference",
        "metric": METRIC, "value": v, "unit": "records/hour", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic (seeded Kanai-Tajimi records, generated RC frames)",
        "config": {"workload": "batched_plain_2d_rc_frames", "frames": args.frames,
                   "steps_per_record": args.record_steps, "dt": DT},
        "cpu_baseline": {"value": v, "unit": "records/hour", "cores": info[0], "kind": "port",
                         "sample": info[1]},
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

    models, cases = build_models(args.frames, args.record_steps, 1000 + rank * args.frames)
    n_fibers = sum(m.num_fibers_total for m in models)

    if args.profile_only:
        # host-driven loop (profiling mode): plain launches a profiler can attribute (kernel
        # nodes of a graph with conditional nodes cannot be profiled one by one)
        with runtime.Analysis(models, device=device) as an:
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

    def one_analysis(prof=False):
        an = runtime.Analysis(models, device=device)
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
        an.close()
        return ms, st, prof_out

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
            ms, st, _p = one_analysis()
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
    records = completed
    value = records / (ms_per_step / 1000.0) * 3600.0
    newton_per_step = st.global_newton_iterations / float(args.frames * args.record_steps)
    fiber_updates_per_s = st.fiber_updates / (times[-1] / 1000.0)

    # end to end through the public API with host buffers, per bench step
    e2e_times = []
    h2d = d2h = 0
    for _ in range(max(1, args.steps)):
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
    e2e_value = records / e2e_s * 3600.0

    # roofline of the dominant kernel (element state determination), one profiled analysis
    _ms, _st, P = one_analysis(prof=True)
    peak, peak_kind = measured_peaks()
    el_ms = P.ms[A.PROF_ELEMENT]
    el_launch = max(P.launches[A.PROF_ELEMENT], 1)
    el_bytes = P.bytes[A.PROF_ELEMENT]
    achieved = (el_bytes / el_launch) / ((el_ms / el_launch) / 1000.0) / 1e9
    kernel_share = {k: P.ms[i] for k, i in (("element", 0), ("instance", 1), ("commit", 2),
                                              ("predictor", 3), ("post", 4))}
    # DRAM bytes per launch: the measured traffic / algorithmic-bytes ratio of this kernel (one
    # ncu capture of a smaller batch of the same frames, traffic growing with the elements
    # processed) times this run's algorithmic bytes per launch
    traffic = None
    tp = ROOT / "profiles" / "element_state_kernel_dram_traffic_rc_frames96.md"
    if tp.exists():
        for line in tp.read_text().splitlines():
            if line.startswith("traffic_to_algorithmic_ratio:"):
                traffic = float(line.split(":", 1)[1]) * (el_bytes / el_launch)

    learned = None
    if not args.no_learned:
        learned = learned_arm(args, models, device, runtime, A, torch, world)

    tall = None
    if rank == 0 and world == 1 and not args.no_tall:
        tall = tall_arm(args, device, runtime, A, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rph, cores, sample = cpu_baseline(models, cases)
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
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded Kanai-Tajimi records, generated RC frames)",
            "config": {"workload": "batched_plain_2d_rc_frames", "frames_per_gpu": args.frames,
                       "steps_per_record": args.record_steps, "dt": DT,
                       "fibers_per_gpu": n_fibers, "parallelism": f"replicas{world}",
                       "l2": "fiber history of the batch exceeds L2 (no flush needed)"},
            "newton_its_per_step": newton_per_step,
            "records_completed": completed,
            "records_failed_nonconvergence": args.frames * world - completed,
            "fiber_state_updates_per_s": fiber_updates_per_s,
            "simulated_s_per_wall_s": args.frames * args.record_steps * DT / (times[-1] / 1000.0),
            "e2e": {"value": e2e_value, "unit": "records/hour", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"kernel": "element_state_kernel", "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "launches": int(P.launches[A.PROF_ELEMENT]),
                         "avg_launch_ms": el_ms / el_launch},
            "kernel_ms": kernel_share,
            # launches of one analysis (profiled run, same workload) x timed analyses; the
            # displacement-record kernel runs once per step
            "gpu_launches": int(args.steps * (sum(P.launches[i] for i in range(5)) + st.steps_done)),
            "clocks": clk.summary(),
        }
        if learned:
            learned["vs_plain"] = learned["value"] / value if value else None
            line["learned"] = learned
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
