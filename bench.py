"""Throughput benchmark of the B200 RSA worldline packer.

Metric: candidates tested per second (a candidate counts once its
accept/reject is decided) on seeded synthetic candidate streams.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3]
                    [--precision mixed|fp64] [--impl ours|reference]

A step is one complete packing job of the workload (every universe run from
an empty packing to its stop rule).  Multi-GPU: one process per GPU under
torchrun; universes / replicas are independent, so ranks shard them with no
data-path collective (weak scaling) and time is the max over ranks.

CPU arms.  Both time COMPLETE jobs (empty packing to the attempt cap) of a
fixed stratified sample of the workload's universes (cpu_sample): for c3, one
universe per (dim, F tercile) stratum, the one with the largest cap whose job
on the reference's CPU path fits a few seconds.  `cpu_baseline` is the oracle
(the repository's C restatement, threaded prefilter + in-order decisions) on
those jobs with the workload's conventions; `--impl reference` is the
reference's own braid_knot code compiled from its source (oracle/_ref/knot_host)
with the reference's conventions, one sample job per step in rotation.  The
packer's own rate on exactly the sample jobs is reported beside them.
"""

from __future__ import annotations

import argparse
import dataclasses
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "universe-generator_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
MIXED_SRC = os.path.join(PKG, "csrc", "ug_mixed.cu")
# DRAM bytes (read + write) of the prefilter over one complete job of the workload,
# from a 1-pass ncu capture of that job (dram__bytes_read.sum + dram__bytes_write.sum
# summed over its launches); the line reports it per launch (÷ the timed job's launch
# count).  Keyed by the SHA-256 of the prefilter source the capture ran, so a changed
# kernel reports null instead of a stale figure.
PREFILTER_TRAFFIC: dict[tuple[str, str, str], float] = {
    ("c3", "mixed", "7dce91ac1985d3ac"): 65.933716e9 + 2.547354e9,
}
FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
# reference-path cost model for picking affordable sample jobs: seconds ~ cap d T^2 / rate
REF_COST_RATE = 1.8e8
REF_JOB_BUDGET_S = 8.0


def workloads(name: str, ug, seed0: int):
    """Universes of one job (ugb200.workloads: all inputs generated from seeds)."""
    from ugb200 import workloads as W

    try:
        return W.workload(name, seed0)
    except ValueError as e:
        raise SystemExit(str(e))


def cpu_sample(us) -> list[int]:
    """Universes whose complete jobs the CPU arms time: one per (dim, F tercile)
    stratum, the largest-cap one whose reference-path job fits REF_JOB_BUDGET_S."""
    if len(us) == 1:
        return [0]
    Fs = sorted(u.T for u in us)
    t1, t2 = Fs[len(Fs) // 3], Fs[2 * len(Fs) // 3]
    strata: dict[tuple[int, int], list[int]] = {}
    for k, u in enumerate(us):
        strata.setdefault((u.dim, 0 if u.T < t1 else (1 if u.T < t2 else 2)), []).append(k)
    pick = []
    for key in sorted(strata):
        ok = [k for k in strata[key]
              if us[k].attempts * us[k].dim * us[k].T ** 2 / REF_COST_RATE <= REF_JOB_BUDGET_S]
        if ok:
            pick.append(max(ok, key=lambda k: (us[k].attempts, -k)))
    return pick


def sample_desc(us, idx) -> str:
    tot = sum(u.attempts for u in us)
    n = sum(us[k].attempts for k in idx)
    return (f"complete jobs of universes {idx} (d/T/cap: "
            + ", ".join(f"{us[k].dim}/{us[k].T}/{us[k].attempts}" for k in idx)
            + f"), {n} candidates = {100.0 * n / tot:.1f}% of the workload's {tot}")


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            return json.load(f), "measured"
    except Exception:
        return FALLBACK, "fallback"


def src_sha() -> str:
    with open(MIXED_SRC, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()[:16]


def start_clock_sampler(out_path: str):
    try:
        return subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200",
             "-i", str(int(os.environ.get("LOCAL_RANK", "0")))],
            stdout=open(out_path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def clocks_summary(path: str):
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
            v = [x.strip() for x in line.split(",")]
            if len(v) < 9:
                continue
            try:
                sm.append(float(v[1]))
                mx.append(float(v[2]))
            except ValueError:
                continue
            for n, val in zip(names, v[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
    except FileNotFoundError:
        pass
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
            "samples": len(sm)}


def cpu_baseline(us, idx, budget_s: float = 40.0):
    """The oracle (plain-C restatement of the reference path), threaded batch prefilter
    + in-order decisions on all host cores, on complete jobs of the sample universes
    with the workload's own conventions and seeds."""
    import oracle as O

    cores = os.cpu_count() or 1
    done, secs, used = 0, 0.0, []
    for k in idx:
        u = us[k]
        m = O.Model(dim=u.dim, T=u.T, rng=u.rng, zgrid=u.zgrid, excl=u.excl, cross1d=u.cross1d,
                    pin=u.pin_sin1, seed=u.seed)
        t0 = time.perf_counter()
        r = O.pack(m, u.attempts, nthreads=cores, round_size=16384, max_n=u.max_n,
                   group_mode=u.group_mode, sub_attempts=u.sub_attempts, accept_rate=u.accept_rate)
        secs += time.perf_counter() - t0
        done += r.attempts
        used.append(k)
        if secs > budget_s:
            break
    return {"value": done / secs, "unit": "candidates/s", "cores": cores, "kind": "port",
            "sample": sample_desc(us, used) + f"; {secs:.1f} s; oracle threaded prefilter + "
                      "in-order decisions, the workload's conventions and seeds",
            "universes": used}


def matched_gpu(ugb200, us, idx, prec, local, stream):
    """The packer on exactly the CPU arms' sample jobs (same universes and seeds),
    batched, device-timed: the like-for-like GPU figure beside the CPU rates."""
    import torch

    sub = [us[k] for k in idx]
    with ugb200.Packer(sub, precision=prec, device=local, stream=stream.cuda_stream,
                       rounds_per_sync=8, use_graph=True) as p:
        p.run()
        seeds = [u.seed for u in sub]
        ms, c = 0.0, 0
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            p.reset(seeds).run()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            c += sum(p.stats(k).attempts for k in range(len(sub)))
    return {"value": c / (ms / 1000.0), "unit": "candidates/s", "universes": list(idx)}


def combine_ranks(t_ms: float, cands: int, dist, device: str):
    """Whole-job numbers of a multi-rank run: the slowest rank's device time and the
    candidates of all ranks (each rank packs its own universes; no data-path
    collective, only these two reductions)."""
    import torch

    t = torch.tensor([float(t_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([int(cands)], dtype=torch.int64, device=device)
    dist.all_reduce(c)
    return float(t.item()), int(c.item())


def frames_line(packer):
    """c4's second stage: frame_bake of the packed universe (last timed job), 256 instants
    z_obs in [0.25, 0.75] pi, one path observer, the 'fit' front, a 1024 x 1024 uint32
    density grid per frame.  Timed end to end through ugb200.frames.bake_packed: the
    paths stay on the device, the 1 GiB of densities comes back to host memory."""
    from ugb200 import frames as FR

    kw = dict(observers=[("path", 0)], from_pi=0.25, to_pi=0.75, frames=256, front="fit",
              density_bins=1024, hits=False)
    FR.bake_packed(packer, 0, **{**kw, "frames": 2})  # warm-up
    t0 = time.perf_counter()
    bk = FR.bake_packed(packer, 0, **kw)
    dt = time.perf_counter() - t0
    return {"frames_per_s": 256 / dt, "ms": dt * 1e3, "paths": int(packer.stats(0).n),
            "hits": int(bk.counts.sum()), "density_sum": int(bk.density.sum()),
            "density_bytes": int(bk.density.nbytes),
            "sample": "256 frames, z_obs 0.25..0.75 pi, 1 path observer, fit front, 1024^2 density; "
                      "device-resident paths, densities copied to host"}


def precision_report(packer, us, count: int = 2048):
    """Achieved tensor-core position error against FP64 (first `count` candidates of
    every universe, all timesteps and axes) and the share of FP64 work."""
    import ugb200

    err, band, ratio = 0.0, 0.0, 0.0
    for k, u in enumerate(us):
        try:
            e, m, q = packer.mixed_error(k, 0, min(count, u.attempts))
        except ugb200.UgError:
            continue  # universe not on the tensor-core path (knot stream)
        err, band, ratio = max(err, e), max(band, m), max(ratio, q)
    st = [packer.stats(k) for k in range(len(us))]
    att = sum(s.attempts for s in st)
    ev = sum(s.evals for s in st)
    return {"max_abs_err": err, "widest_band": band, "max_err_to_band": ratio,
            "gray_frac": sum(s.gray for s in st) / max(att, 1),
            "evals_fp64_frac": sum(s.evals_fp64 for s in st) / max(ev, 1),
            "sample": f"first {count} candidates of each universe (all timesteps and axes)"}


def reference_gpu(args):
    """Informational: the reference's own GPU engines (cuda/braid_cuda.cu and
    cuda/braid_cuda3d.cu, wide builds, compiled unmodified for sm_100a by
    oracle/Makefile) on this GPU at c1 / c2 shapes with the reference's conventions;
    attempts / s from their `done:` lines' attempts over the process wall time.  Not
    bit-comparable (atomicAdd admission order)."""
    out = {}
    runs = {"c1": ("braid_cuda_w150", 64, 1_000_000), "c2": ("braid_cuda3d_w150", 128, 1_000_000)}
    for name, (exe, T, att) in runs.items():
        path = os.path.join(ROOT, "oracle", "_ref", exe)
        if not os.path.exists(path):
            out[name] = {"unavailable": f"oracle/_ref/{exe} not built"}
            continue
        cmd = [path, "-t", str(T), "--attempts", str(att), "--terms", str(T), "--maxfreq", str(T),
               "--seed", "1"]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        dt = time.perf_counter() - t0
        m = re.search(r"done: N=(\d+) in (\d+) attempts", r.stderr)
        if r.returncode or not m:
            out[name] = {"unavailable": f"{exe} exit {r.returncode}: {r.stderr.strip()[-200:]}"}
            continue
        out[name] = {"value": int(m.group(2)) / dt, "unit": "candidates/s", "N": int(m.group(1)),
                     "attempts": int(m.group(2)), "wall_s": dt, "cmd": " ".join([exe] + cmd[1:])}
    return out


def reference_arm(args, rank, world):
    """The reference's own CPU path: reference cuda/braid_knot.cu (propose, its
    eval/collide loop, index-order admission) compiled from the reference source
    (oracle/_ref/knot_host), all host threads, complete jobs of the sample universes
    (one per step, in rotation) with the reference's conventions."""
    if rank != 0:
        return 0
    import oracle as O
    import ugb200

    us, cfg = workloads(args.workload, ugb200, 0)
    exe = os.path.join(O.REF_DIR, "knot_host")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/knot_host not built"}))
        return 0
    cores = os.cpu_count() or 1
    idx = cpu_sample(us)
    done, secs, used = 0, 0.0, []
    for step in range(args.warmup + args.steps):
        k = idx[step % len(idx)]
        u = us[k]
        r = subprocess.run([exe, "--mode", "pack", "-t", str(u.T), "--dim", str(u.dim),
                            "--seed", str(1000 * step + k), "--attempts", str(u.attempts),
                            "--threads", str(cores), "--round", "16384"],
                           capture_output=True, text=True, check=True)
        m = re.search(r"in (\d+) attempts \(([0-9.]+) s", r.stderr)
        if step >= args.warmup:
            done += int(m.group(1))
            secs += float(m.group(2))
            used.append(k)
    v = done / secs if secs > 0 else 0.0
    line = {"metric": "candidates tested/s", "value": v, "unit": "candidates/s",
            "higher_is_better": True, "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, **cfg},
            "same_config": False,
            "same_config_note": "complete jobs of a stratified sample of the workload's universes "
                                "(same dim, T, attempt cap); the reference's conventions and "
                                "candidate stream; the sample is the cheap end of each stratum, "
                                "so this rate is above the workload's mean for this path",
            "cpu_baseline": {"value": v, "unit": "candidates/s", "cores": cores,
                             "kind": "reference",
                             "sample": sample_desc(us, sorted(set(used))) +
                                       "; one job per step in rotation; reference braid_knot.cu "
                                       "propose() + its eval/collide loop, threaded prefilter + "
                                       "in-order recheck, time from its done line"},
            "e2e": {"value": v, "unit": "candidates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="fixed round parameters instead of the autotuned plan (multi-universe workloads)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the FP64 single-universe sweep, the precision report and the "
                         "reference GPU engines (timing of the workload only)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own GPU engines (informational field)")
    ap.add_argument("--clocks-dir", default="",
                    help="where the nvidia-smi samples of the timed region go (default: the temp dir)")
    ap.add_argument("--profile-case", action="store_true",
                    help="run one untimed packing job of the workload and exit (for ncu captures)")
    ap.add_argument("--stride", type=int, default=1,
                    help="--profile-case: every stride-th universe of the workload")
    ap.add_argument("--max-rounds", type=int, default=0,
                    help="--profile-case: stop after this many rounds (0: run to the stop rule)")
    ap.add_argument("--universe", type=int, default=-1,
                    help="--profile-case: only this universe of the workload")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch

    import ugb200

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    prec = ugb200.PREC_MIXED if args.precision == "mixed" else ugb200.PREC_FP64
    # weak scaling: every rank packs the full universe list with its own seeds
    us, cfg = workloads(args.workload, ugb200, 1000 * rank)
    if args.profile_case:
        sub = [us[args.universe]] if args.universe >= 0 else us[::max(1, args.stride)]
        with ugb200.Packer(sub, precision=prec, device=local, use_graph=False) as p:
            p.run(max_rounds=args.max_rounds)
            st = [p.stats(k) for k in range(len(sub))]
        print(json.dumps({"profile_case": args.workload, "universes": len(sub),
                          "candidates": sum(s.attempts for s in st),
                          "evals": sum(s.evals for s in st), "rounds": max(s.rounds for s in st)}))
        return 0
    stream = torch.cuda.Stream()
    # round parameters: the autotuned plan for multi-universe workloads (cached per GPU
    # and workload; tuning time is outside every timed region), else the defaults
    rps, tuned, tune_info = 8, us, None
    if len(us) > 1 and not args.no_autotune:
        from ugb200 import autotune as A

        plan = A.tune(us, precision=prec, device=local, stream=stream.cuda_stream,
                      log=lambda m: print(m, file=sys.stderr, flush=True))
        tuned, rps = A.apply(us, plan), int(plan["rounds_per_sync"])
        tune_info = {"classes": plan["classes"], "rounds_per_sync": rps, "trials": plan["trials"],
                     "job_ms_tuned": plan["job_s"] * 1e3, "job_ms_default": plan["default_job_s"] * 1e3,
                     "cached": plan["cached"]}
    packer = ugb200.Packer(tuned, precision=prec, device=local, stream=stream.cuda_stream,
                           rounds_per_sync=rps, use_graph=True)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    base_seeds = [u.seed for u in us]  # reset() writes the new seeds into the universes

    def seeds(step):
        return [(s0 + 7919 * (step + 1)) & (2**64 - 1) for s0 in base_seeds]

    # warm-up
    for w in range(args.warmup):
        packer.reset(seeds(w)).run()
    torch.cuda.synchronize()

    # device-timed steps (inputs resident, L2 flushed between steps)
    clk_path = os.path.join(args.clocks_dir or tempfile.gettempdir(), f"clocks_rank{rank}.csv")
    sampler = start_clock_sampler(clk_path)
    times = []
    cands = 0
    launches0 = packer.counters()[0]
    for s in range(args.steps):
        with torch.cuda.stream(stream):
            flush.random_(0, 255)
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        packer.reset(seeds(args.warmup + s)).run()
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        cands += sum(packer.stats(k).attempts for k in range(len(us)))
    launches = packer.counters()[0] - launches0
    # accepted sets of the last timed job, for the FP64 single-universe comparison
    last_seeds = seeds(args.warmup + args.steps - 1)
    acc_batched = [a for a, _ in packer.accepted_all()]
    frames = frames_line(packer) if (args.workload == "c4" and rank == 0) else None
    if sampler:
        sampler.terminate()
        sampler.wait()
    t_ms = float(sum(times))
    if dist:
        t_ms, cands = combine_ranks(t_ms, cands, dist, "cuda")
    value = cands / (t_ms / 1000.0)

    # end to end through the public API with host buffers: CUDA events on the packer's
    # stream around each job (seed upload, rounds, host status syncs, and every
    # universe's accepted indices and group ids read back), ranks started together and
    # combined like `value` (max time, summed candidates)
    e2e_ms = 0.0
    e2e_c = 0
    nrep = max(1, args.steps // 2)
    _, h2d0, d2h0 = packer.counters()
    if dist:
        dist.barrier()
    for s in range(nrep):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        packer.reset(seeds(100 + s)).run()
        acc = packer.accepted_all()
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        e2e_c += sum(packer.stats(k).attempts for k in range(len(us)))
        del acc
    _, h2d1, d2h1 = packer.counters()
    h2d_b, d2h_b = (h2d1 - h2d0) // nrep, (d2h1 - d2h0) // nrep
    if dist:
        e2e_ms, e2e_c = combine_ranks(e2e_ms, e2e_c, dist, "cuda")
        _, h2d_b = combine_ranks(0.0, h2d_b, dist, "cuda")
        _, d2h_b = combine_ranks(0.0, d2h_b, dist, "cuda")
    e2e = {"value": e2e_c / (e2e_ms / 1000.0), "unit": "candidates/s",
           "h2d_bytes_per_step": h2d_b, "d2h_bytes_per_step": d2h_b}

    precision = None
    if prec == ugb200.PREC_MIXED and not args.no_extras:
        precision = precision_report(packer, us)
    packer.close()
    # per-kernel timing pass (events around each launch on the packer's stream)
    timer = ugb200.Packer(tuned, precision=prec, device=local, stream=stream.cuda_stream,
                          rounds_per_sync=rps, use_graph=False, kernel_timing=True)
    timer.reset(seeds(args.warmup)).run()
    kt = timer.kernel_times()
    st = [timer.stats(k) for k in range(len(us))]
    timer.close()
    pk_name = "k_prefilter_mixed" if prec == ugb200.PREC_MIXED else "k_prefilter64w"
    pk_ms, pk_n = kt.get(pk_name, (0.0, 0))
    evals = sum(s.evals for s in st)
    P, src = peaks()
    pk_s = pk_ms / 1000.0
    avg_s = pk_s / max(pk_n, 1)
    job_traffic = PREFILTER_TRAFFIC.get((args.workload, args.precision, src_sha()))
    traffic = job_traffic / max(pk_n, 1) if job_traffic else None
    # algorithmic units of the prefilter (per launch = job total / launches):
    #  tensor: the contraction 2 d K T per candidate (K = (F-1) + F/2; split-BF16 counted once;
    #          the mixed path evaluates all T timesteps of every candidate)
    #  HBM:    per examined (candidate, timestep) the 3^d neighbour cell offsets (8 B each) plus
    #          (4d + 4) B per accepted point examined; a 1+1 crossing test examines one
    #          stored point per (path, timestep): 8 B
    mixed = prec == ugb200.PREC_MIXED
    flops = sum(2 * u.dim * ((u.T - 1) + u.T // 2) * (u.T * s.attempts if mixed else s.evals)
                for u, s in zip(us, st))
    hbm_bytes = sum((8 * s.evals) if (u.dim == 1 and u.cross1d)
                    else (3 ** u.dim * 8 * s.evals + (4 * u.dim + 4) * s.visits)
                    for u, s in zip(us, st))
    t_ach = flops / pk_s / 1e12 if pk_s > 0 else 0.0
    h_ach = hbm_bytes / pk_s / 1e9 if pk_s > 0 else 0.0
    t_frac, h_frac = t_ach / P["bf16_tflops"], h_ach / P["hbm_gbs"]
    tensor = {"achieved": t_ach, "peak": P["bf16_tflops"], "unit": "TFLOP/s", "frac": t_frac,
              "flops_per_launch": flops / max(pk_n, 1), "peak_source": f"{src} bf16 dense (burst)"}
    hbm = {"achieved": h_ach, "peak": P["hbm_gbs"], "unit": "GB/s", "frac": h_frac,
           "bytes_per_launch": hbm_bytes / max(pk_n, 1), "peak_source": f"{src} copy bandwidth",
           "dram_gbs": traffic / avg_s / 1e9 if traffic and avg_s > 0 else None}
    main = hbm if h_frac >= t_frac else tensor  # the bound is the larger fraction
    roofline = {"bound": "hbm" if main is hbm else "tensor", "kernel": pk_name,
                "achieved": main["achieved"], "peak": main["peak"], "unit": main["unit"],
                "frac": main["frac"], "traffic": traffic, "tensor": tensor, "hbm": hbm,
                "launches": pk_n, "avg_launch_ms": pk_ms / max(pk_n, 1),
                "evals": evals, "visits": sum(s.visits for s in st),
                "kernel_share": {k: v[0] for k, v in kt.items()}, "kernel_src_sha": src_sha()}

    # the plain FP64 single-universe form on the same B200 and the same seeds: one
    # universe per packer, thread-per-candidate FP64 prefilter (the metric's
    # denominator), every universe of the workload
    fp64_plain = None
    if not args.no_extras:
        f_ms, f_c, same = 0.0, 0, True
        for k, u in enumerate(us):
            uu = ugb200.Universe(**{**u.__dict__, "seed": last_seeds[k]})
            with ugb200.Packer([uu], precision=ugb200.PREC_FP64, device=local,
                               stream=stream.cuda_stream, rounds_per_sync=8, use_graph=True) as p1:
                p1.run()  # warm-up: builds the CUDA graph of the rounds, as the batched warm-up does
                p1.reset([last_seeds[k]])
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                p1.run()
                e1.record(stream)
                e1.synchronize()
                f_ms += e0.elapsed_time(e1)
                f_c += p1.stats(0).attempts
                same = same and np.array_equal(p1.accepted(0)[0], acc_batched[k])
        fp64_plain = {"value": f_c / (f_ms / 1000.0), "unit": "candidates/s",
                      "sample": f"all {len(us)} universes of the workload, each run alone in FP64 "
                                f"with the seeds of the last timed job, {f_c} candidates",
                      "same_accepted_set": bool(same)}
        fp64_plain["mixed_batched_speedup"] = value / fp64_plain["value"]

    if rank == 0:
        line = {"metric": "candidates tested/s", "value": value, "unit": "candidates/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None,
                "dtype": "bf16x3+f32+f64" if prec == ugb200.PREC_MIXED else "f64",
                "data": "synthetic (seeded Philox candidate streams)",
                "config": {"workload": args.workload, **cfg,
                           "precision": "mixed" if prec == ugb200.PREC_MIXED else "fp64",
                           "l2": "flushed between steps (256 MiB write)",
                           "autotune": tune_info or "off (default round parameters)",
                           "parallelism": f"replicas x{world}"},
                "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "precision": precision,
                "fp64_plain_single_universe": fp64_plain,
                "frames": frames,
                "clocks": clocks_summary(clk_path)}
        if not args.no_cpu_baseline:
            idx = cpu_sample(us)
            cb = cpu_baseline(us, idx)
            same_seeds = [dataclasses.replace(t, seed=u.seed) for t, u in zip(tuned, us)]
            cb["matched_gpu"] = matched_gpu(ugb200, same_seeds, cb["universes"], prec, local, stream)
            line["cpu_baseline"] = cb
        if not args.no_extras and not args.no_reference_gpu:
            line["reference_gpu"] = reference_gpu(args)
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
