"""Generate tests/golden/config_parity.json: the oracle's accepted sets of the
measured workloads at their stated sizes.

    python tests/golden/make_config_golden.py [--jobs N] [--only c0,c1,...]

The oracle (oracle/ug_oracle.c, a plain-C restatement of the reference's
sequential RSA, pinned to outputs of the reference's own braid_knot) packs
every case on the CPU; no GPU is involved.  Each case stores the accepted
count, the attempts, the SHA-256 of the accepted candidate-index list (int64
little-endian, admission order) and of the group labels (int32 little-endian),
plus the first and last indices for diagnosis.  The GPU test
(tests/test_config_parity_gpu.py) runs the packer on the same cases in both
precision modes and compares.

Cases:
  c0, c1, c2, c4     the workloads of ugb200.workloads at full size (seed0 = 0)
  c3/<k>             every one of c3's 256 universes to its attempt cap
  c1_ref, c2_ref     c1 / c2 under the reference conventions (z_i = (i+1) pi / (T+1),
                     Chebyshev |d| <= 2/T)
  c1_knot            c1's shape with the reference's per-attempt xoshiro stream
                     (braid_knot.cu:207) under the reference conventions
  c1_stop            c1's shape with --until-accept-rate 1e-5 (budget 3e7; the
                     window stop ends the run at 2.25e7 candidates)
  sub_fill, sub_acc  the two-phase subpath mode (2+1, T = 24) with
                     --sub-until-fill-rate 2e-4 / --sub-until-accept-rate 1e-5
                     (phase 2 stops at 2.1875e7 / 3.75e7 of its 6e7 candidates)
"""

from __future__ import annotations

import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (ROOT, os.path.join(ROOT, "universe-generator_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

OUT = os.path.join(HERE, "config_parity.json")


def universe_dict(u) -> dict:
    keys = ("dim", "T", "terms", "rng", "zgrid", "excl", "cross1d", "pin_sin1", "group_mode",
            "round_size", "seed", "attempts", "max_n", "sub_attempts", "accept_rate",
            "sub_accept_rate", "sub_fill_rate", "euclid")
    return {k: getattr(u, k) for k in keys}


def cases() -> list[tuple[str, dict]]:
    from ugb200 import Universe
    from ugb200 import workloads as W

    out = []
    for name in ("c0", "c1", "c2", "c4"):
        us, _ = W.workload(name, 0)
        out.append((name, universe_dict(us[0])))
    us, _ = W.workload("c3", 0)
    for k, u in enumerate(us):
        out.append((f"c3/{k}", universe_dict(u)))
    out.append(("c1_ref", universe_dict(Universe(dim=2, T=64, seed=0, attempts=1_000_000,
                                                 round_size=16384))))
    out.append(("c2_ref", universe_dict(Universe(dim=3, T=128, seed=0, attempts=5_000_000,
                                                 round_size=65536))))
    out.append(("c1_knot", universe_dict(Universe(dim=2, T=64, rng=1, seed=0, attempts=1_000_000,
                                                  round_size=16384))))
    out.append(("c1_stop", universe_dict(Universe(dim=2, T=64, zgrid=1, excl=1, seed=0,
                                                  attempts=30_000_000, accept_rate=1e-5,
                                                  round_size=16384))))
    sub = dict(dim=2, T=24, zgrid=1, excl=1, seed=3, attempts=200_000, group_mode=1,
               sub_attempts=60_000_000, round_size=16384)
    out.append(("sub_fill", universe_dict(Universe(**sub, sub_fill_rate=2e-4))))
    out.append(("sub_acc", universe_dict(Universe(**sub, sub_accept_rate=1e-5))))
    return out


def sha(a) -> str:
    return hashlib.sha256(a.tobytes()).hexdigest()


def run_case(item):
    name, u = item
    import numpy as np

    import oracle as O

    m = O.Model(dim=u["dim"], T=u["T"], terms=u["terms"], rng=u["rng"], zgrid=u["zgrid"], excl=u["excl"],
                cross1d=u["cross1d"], pin=u["pin_sin1"], seed=u["seed"], euclid=u["euclid"])
    t0 = time.time()
    nth = int(os.environ.get("ORACLE_THREADS", "1"))
    r = O.pack(m, u["attempts"], max_n=u["max_n"], group_mode=u["group_mode"],
               sub_attempts=u["sub_attempts"], accept_rate=u["accept_rate"],
               sub_accept_rate=u["sub_accept_rate"], sub_fill_rate=u["sub_fill_rate"],
               nthreads=nth, round_size=16384)
    idx = np.ascontiguousarray(r.acc_idx, dtype="<i8")
    gid = np.ascontiguousarray(r.gid, dtype="<i4")
    return name, {"universe": u, "n": int(len(idx)), "n_unique": int(r.n_unique), "n_sub": int(r.n_sub),
                  "attempts": int(r.attempts), "phase1_end": int(r.phase1_end),
                  "idx_sha256": sha(idx), "gid_sha256": sha(gid),
                  "head": [int(x) for x in idx[:4]], "tail": [int(x) for x in idx[-4:]],
                  "oracle_s": round(time.time() - t0, 1)}


def cost(item) -> float:
    u = item[1]
    return u["attempts"] * u["dim"] * u["T"] * (1 + (u["sub_attempts"] > 0))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    todo = cases()
    if args.only:
        keep = args.only.split(",")
        todo = [c for c in todo if any(c[0] == k or c[0].startswith(k + "/") for k in keep)]
    old = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            old = json.load(f)["cases"]
    todo.sort(key=cost, reverse=True)
    import oracle

    oracle.build()
    res = dict(old)
    t0 = time.time()
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        for k, (name, r) in enumerate(pool.imap_unordered(run_case, todo)):
            res[name] = r
            print(f"[{k + 1}/{len(todo)}] {name}: N={r['n']} attempts={r['attempts']} "
                  f"({r['oracle_s']} s, {time.time() - t0:.0f} s total)", flush=True)
    order = sorted(res, key=lambda n: (n.split("/")[0], int(n.split("/")[1]) if "/" in n else -1))
    doc = {"generator": "tests/golden/make_config_golden.py",
           "oracle": "oracle/ug_oracle.c (sequential RSA, candidate-aligned windowed stops)",
           "hash": "sha256 of the accepted indices (int64 LE) / group labels (int32 LE), admission order",
           "cases": {n: res[n] for n in order}}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {OUT}: {len(res)} cases")
    return 0


if __name__ == "__main__":
    sys.exit(main())
