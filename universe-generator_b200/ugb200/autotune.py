"""Autotuner of the batched packer's round parameters.

The reference steers one number, its batch size, by halving and doubling it
toward 64..512 survivors per round (cuda/braid_cuda.cu:920-924).  The packer
adapts its round size on the device the same way, but three choices are fixed
before the run and decide how much of the GPU a round keeps busy:

* per universe class (dim, F octave) the round capacity (`round_size`: the
  per-round candidate buffers and the upper end of the on-device adaptation);
* per universe class the survivor capacity of a round (`surv_scale`, a factor
  on the default 2^20 / T survivors, at most 8192; the universe's `surv_cap`):
  it sets how many survivors one round can resolve before the round is cut;
* per batch the rounds per host synchronisation (`rounds_per_sync`: the length
  of the captured CUDA graph replayed between control-block reads).

Accepted sets do not depend on any of them (counter-based candidate streams,
in-order resolution), so the tuner only times.  It measures whole jobs of the
workload by coordinate descent from the defaults -- each class's round
capacity and survivor scale in turn, then the sync period -- keeps a change
only when the job gets faster by more than `min_gain`, and caches the plan on
disk keyed by the GPU and the workload's shape.
"""

from __future__ import annotations

import ctypes as C
import hashlib
import json
import math
import os
import time
from dataclasses import replace

from . import _lib as L
from .packer import Packer, Universe

ROUND_CHOICES = (4096, 16384, 65536)
SURV_CHOICES = (0.5, 1.0, 2.0)
SYNC_CHOICES = (4, 8, 16)
DEFAULT = {"round_size": 16384, "surv_scale": 1.0, "rounds_per_sync": 8}


def device_key(device: int = -1) -> str:
    name = C.create_string_buffer(256)
    sms = C.c_int32()
    L.check(L.load().ug_device_info(device, name, 256, C.byref(sms)))
    return f"{name.value.decode()} x{sms.value}SM"


def class_of(u: Universe) -> str:
    """Universe class: dimension and the octave of F (16-31, 32-63, ...)."""
    return f"d{u.dim}/F{2 ** int(math.log2(max(u.T, 16)))}"


def workload_key(us: list[Universe], precision: int) -> str:
    shape = [(u.dim, u.T, u.attempts, u.group_mode, u.cross1d, u.zgrid, u.excl) for u in us]
    h = hashlib.sha256(json.dumps([precision, shape]).encode()).hexdigest()[:16]
    return f"{len(us)}u-{h}"


def surv_cap(u: Universe, scale: float) -> int:
    """Survivor capacity for a scale on the default (2^20 / T, 256 for 1+1D), as a
    multiple of 32 in [32, 8192]; 0 (the default itself) for scale 1."""
    if scale == 1.0:
        return 0
    base = 256 if u.dim == 1 else min(8192, max(256, (1 << 20) // u.T))
    return int(min(8192, max(32, round(base * scale / 32) * 32)))


def apply(us: list[Universe], plan: dict) -> list[Universe]:
    """The universes with the plan's per-class round capacity and survivor scale."""
    out = []
    for u in us:
        c = plan.get("classes", {}).get(class_of(u), {})
        out.append(replace(u, round_size=int(c.get("round_size", DEFAULT["round_size"])),
                           surv_cap=surv_cap(u, float(c.get("surv_scale", DEFAULT["surv_scale"])))))
    return out


def _time_job(us, plan, precision, device, stream, reps) -> float:
    """Median wall seconds of one complete job (after one warm-up job)."""
    with Packer(apply(us, plan), precision=precision, device=device, stream=stream,
                rounds_per_sync=plan.get("rounds_per_sync", DEFAULT["rounds_per_sync"]),
                use_graph=True) as p:
        seeds = [u.seed for u in us]
        p.run()
        ts = []
        for r in range(reps):
            t0 = time.perf_counter()
            p.reset([(s + 7919 * (r + 1)) & (2**64 - 1) for s in seeds]).run()
            ts.append(time.perf_counter() - t0)
    ts.sort()
    return ts[len(ts) // 2]


def tune(us: list[Universe], precision: int = L.PREC_MIXED, device: int = -1, stream: int = 0,
         cache: str | None = None, reps: int = 2, min_gain: float = 0.01, budget_s: float = 120.0,
         min_share: float = 0.04, log=None, timer=None) -> dict:
    """A plan {"classes": {class: {round_size, surv_scale}}, "rounds_per_sync": n,
    "job_s": seconds, "default_job_s": seconds, "trials": n} for the universes,
    from the cache when it holds one for this GPU and workload.  Classes holding
    less than min_share of the candidates keep the defaults; the search stops
    trying new values once budget_s seconds have passed.  The defaults are timed
    twice at the start (the first timing of a process can run slow), and a plan that
    differs from them is kept only if it also beats one more timing of them at the end.  `timer(us, plan, precision,
    device, stream, reps)` times one plan (default: whole jobs on the GPU)."""
    timer = timer or _time_job
    cache = cache or os.environ.get("UG_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "ugb200", "autotune.json")
    key = f"{device_key(device)}|{workload_key(us, precision)}"
    db = {}
    if os.path.exists(cache):
        try:
            with open(cache) as f:
                db = json.load(f)
        except (OSError, ValueError):
            db = {}
    if key in db:
        return {**db[key], "cached": True}
    classes = {}
    for u in us:
        classes.setdefault(class_of(u), 0)
        classes[class_of(u)] += u.attempts
    plan = {"classes": {c: {"round_size": DEFAULT["round_size"], "surv_scale": DEFAULT["surv_scale"]}
                        for c in classes},
            "rounds_per_sync": DEFAULT["rounds_per_sync"]}
    default_plan = json.loads(json.dumps(plan))
    t_start = time.perf_counter()
    # the defaults twice: the first timing of a process can run slow
    best = min(timer(us, plan, precision, device, stream, reps), timer(us, plan, precision, device, stream, reps))
    base = best
    trials = 2
    say = log or (lambda *_: None)
    say(f"autotune: default job {best * 1e3:.1f} ms")
    total = sum(classes.values())
    # the classes holding the most candidates first
    for c in sorted(classes, key=lambda c: -classes[c]):
        if classes[c] < min_share * total:
            continue
        for knob, choices in (("round_size", ROUND_CHOICES), ("surv_scale", SURV_CHOICES)):
            cur = plan["classes"][c][knob]
            for v in choices:
                if v == cur or time.perf_counter() - t_start > budget_s:
                    continue
                trial = json.loads(json.dumps(plan))
                trial["classes"][c][knob] = v
                t = timer(us, trial, precision, device, stream, reps)
                trials += 1
                if t < best * (1.0 - min_gain):
                    say(f"autotune: {c} {knob}={v}: {t * 1e3:.1f} ms (was {best * 1e3:.1f})")
                    best, plan = t, trial
    for v in SYNC_CHOICES:
        if v == plan["rounds_per_sync"] or time.perf_counter() - t_start > budget_s:
            continue
        trial = {**plan, "rounds_per_sync": v}
        t = timer(us, trial, precision, device, stream, reps)
        trials += 1
        if t < best * (1.0 - min_gain):
            say(f"autotune: rounds_per_sync={v}: {t * 1e3:.1f} ms (was {best * 1e3:.1f})")
            best, plan = t, trial
    if json.dumps(plan, sort_keys=True) != json.dumps(default_plan, sort_keys=True):
        t = timer(us, default_plan, precision, device, stream, reps)
        trials += 1
        base = min(base, t)
        if best >= base * (1.0 - min_gain):
            say(f"autotune: defaults re-timed at {t * 1e3:.1f} ms; keeping them")
            best, plan = base, default_plan
    plan.update(job_s=best, default_job_s=base, trials=trials, tune_s=time.perf_counter() - t_start)
    db[key] = plan
    try:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        with open(cache + ".tmp", "w") as f:
            json.dump(db, f, indent=1)
        os.replace(cache + ".tmp", cache)
    except OSError:
        pass
    return {**plan, "cached": False}
