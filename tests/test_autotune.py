"""The autotuner's plan application (CPU) and, on a GPU, that a tuned plan leaves
the accepted sets unchanged."""

import numpy as np
import pytest


def test_plan_application_and_survivor_caps():
    from ugb200 import autotune as A
    from ugb200 import workloads as W

    us, _ = W.workload("c3", 0)
    classes = {A.class_of(u) for u in us}
    assert classes == {f"d{d}/F{f}" for d in (1, 2, 3) for f in (16, 32, 64, 128)}
    plan = {"classes": {"d3/F128": {"round_size": 4096, "surv_scale": 2.0},
                        "d1/F16": {"round_size": 65536, "surv_scale": 0.5}}}
    out = A.apply(us, plan)
    for u, v in zip(us, out):
        assert v.seed == u.seed and v.attempts == u.attempts and v.T == u.T
        c = A.class_of(u)
        if c == "d3/F128":
            assert v.round_size == 4096 and v.surv_cap == min(8192, round(2 * (2**20 // u.T) / 32) * 32)
        elif c == "d1/F16":
            assert v.round_size == 65536 and v.surv_cap == 128
        else:
            assert v.round_size == 16384 and v.surv_cap == 0
        assert v.surv_cap % 32 == 0 and 0 <= v.surv_cap <= 8192


@pytest.mark.gpu
def test_tuned_plan_keeps_accepted_sets(ug, tmp_path):
    from ugb200 import autotune as A

    us = [ug.Universe(dim=d, T=T, zgrid=1, excl=1, cross1d=int(d == 1), seed=40 + k, attempts=a,
                      round_size=16384)
          for k, (d, T, a) in enumerate([(1, 24, 20000), (2, 40, 60000), (3, 20, 40000), (2, 130, 8000)])]
    plan = A.tune(us, precision=1, cache=str(tmp_path / "tune.json"), reps=1, budget_s=20.0)
    assert plan["trials"] >= 2 and not plan["cached"]
    assert A.tune(us, precision=1, cache=str(tmp_path / "tune.json"))["cached"]
    forced = {"classes": {A.class_of(u): {"round_size": 4096, "surv_scale": 0.5} for u in us},
              "rounds_per_sync": 4}
    ref = None
    for p in (plan, forced):
        with ug.Packer(A.apply(us, p), precision=1, rounds_per_sync=p["rounds_per_sync"]) as pk:
            pk.run()
            got = [a for a, _ in pk.accepted_all()]
        if ref is None:
            with ug.Packer(us, precision=1) as pk:
                pk.run()
                ref = [a for a, _ in pk.accepted_all()]
        assert all(np.array_equal(a, b) for a, b in zip(got, ref))


def test_tuned_plan_must_beat_retimed_defaults(tmp_path, monkeypatch):
    """A slow first timing of the defaults (process start) must not make an equal plan
    look better: the defaults are timed again before a changed plan is kept."""
    from ugb200 import Universe
    from ugb200 import autotune as A

    monkeypatch.setattr(A, "device_key", lambda device=-1: "fake GPU x148SM")
    us = [Universe(dim=2, T=16, seed=1, attempts=1000), Universe(dim=3, T=64, seed=2, attempts=1000)]
    calls = []

    def flat(us_, plan, *a):  # every plan takes 4.0 s except the very first timing
        calls.append(plan)
        return 9.5 if len(calls) == 1 else 4.0

    out = A.tune(us, cache=str(tmp_path / "a.json"), timer=flat, budget_s=1e9)
    assert all(c["round_size"] == A.DEFAULT["round_size"] and c["surv_scale"] == A.DEFAULT["surv_scale"]
               for c in out["classes"].values())
    assert out["rounds_per_sync"] == A.DEFAULT["rounds_per_sync"]
    assert out["job_s"] == out["default_job_s"] == 4.0

    calls.clear()

    def faster_sync(us_, plan, *a):  # a real gain survives the re-timing
        calls.append(plan)
        if len(calls) == 1:
            return 9.5
        return 3.0 if plan["rounds_per_sync"] == 16 else 4.0

    out = A.tune(us, cache=str(tmp_path / "b.json"), timer=faster_sync, budget_s=1e9)
    assert out["rounds_per_sync"] == 16 and out["job_s"] == 3.0 and out["default_job_s"] == 4.0
    assert all(c["round_size"] == A.DEFAULT["round_size"] and c["surv_scale"] == A.DEFAULT["surv_scale"]
               for c in out["classes"].values())
