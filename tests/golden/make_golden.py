"""Generate the golden fixtures of the packing path from the reference's own code.

Run in a container that holds the reference tree (read-only) and nvcc:

    make -C oracle ref          # builds oracle/_ref/knot_host from cuda/braid_knot.cu
    python tests/golden/make_golden.py

oracle/_ref/knot_host #includes the reference's cuda/braid_knot.cu unmodified
and calls its rng_seed/propose/torus_wrap/torus_delta on the CPU, with the
eval_cand/collides_host loops of braid_knot.cu:346-372.  The fixtures hold
(1) candidate parameter streams and (2) accepted sets (attempt index plus
parameters of every admitted path) for a spread of (dim, T, terms, pin, seed).

    python tests/golden/make_golden.py --from-dumps DIR

turns dumps of the reference's own unmodified GPU packer (oracle/_ref/braid_knot,
built by `make -C oracle ref` from cuda/braid_knot.cu and run on a B200 by
the BK_RUNS commands below, `--dump DIR/bk_T{T}_d{dim}_s{seed}_p{pin}.csv`)
into tests/golden/braid_knot_b200.json.
"""

from __future__ import annotations

import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "knot_host")

STREAMS = [
    dict(T=8, dim=2, terms=0, pin=0, seed=1),
    dict(T=16, dim=3, terms=0, pin=0, seed=7),
    dict(T=12, dim=2, terms=5, pin=0, seed=3),
    dict(T=10, dim=1, terms=0, pin=1, seed=11),
    dict(T=64, dim=2, terms=0, pin=0, seed=2),
]
PACKS = [
    dict(T=16, dim=2, terms=0, pin=0, seed=1, attempts=20000),
    dict(T=16, dim=3, terms=0, pin=0, seed=2, attempts=20000),
    dict(T=8, dim=1, terms=0, pin=0, seed=3, attempts=5000),
    dict(T=12, dim=2, terms=5, pin=0, seed=4, attempts=20000),
    dict(T=16, dim=2, terms=0, pin=1, seed=5, attempts=20000),
    dict(T=24, dim=2, terms=0, pin=0, seed=6, attempts=40000),
    dict(T=10, dim=3, terms=4, pin=0, seed=8, attempts=30000),
]


BK_RUNS = [  # (T, dim, seed, attempts, pin)
    (16, 2, 1, 20000, 0), (16, 3, 2, 20000, 0), (24, 2, 6, 40000, 0),
    (16, 2, 5, 20000, 1), (32, 2, 9, 200000, 0), (12, 3, 4, 50000, 0),
]


def bk_command(T, dim, seed, attempts, pin, outdir):
    cmd = ["./oracle/_ref/braid_knot", "-t", str(T), "--dim", str(dim), "--seed", str(seed),
           "--attempts", str(attempts)]
    if pin:
        cmd.append("--pin-sin1")
    return cmd + ["--dump", f"{outdir}/bk_T{T}_d{dim}_s{seed}_p{pin}.csv"]


def from_dumps(d: str) -> None:
    out = {"generator": "reference cuda/braid_knot.cu built unmodified for sm_100a, run on a B200",
           "runs": []}
    for T, dim, seed, attempts, pin in BK_RUNS:
        rows = [x for x in open(f"{d}/bk_T{T}_d{dim}_s{seed}_p{pin}.csv").read().splitlines()
                if x and not x.startswith("#")]
        out["runs"].append({"T": T, "dim": dim, "seed": seed, "attempts": attempts, "pin": pin,
                            "command": " ".join(bk_command(T, dim, seed, attempts, pin, d)),
                            "idx": [int(x.split(",")[1]) - 1 for x in rows],
                            "head_rows": rows[:2]})
    path = os.path.join(HERE, "braid_knot_b200.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(path)


def args_of(c: dict) -> list[str]:
    a = ["-t", str(c["T"]), "--dim", str(c["dim"]), "--seed", str(c["seed"])]
    if c["terms"]:
        a += ["--terms", str(c["terms"])]
    if c["pin"]:
        a += ["--pin-sin1"]
    return a


def main() -> None:
    out = {"generator": "oracle/_ref/knot_host (reference cuda/braid_knot.cu propose)",
           "streams": [], "packs": []}
    for c in STREAMS:
        r = subprocess.run([EXE, "--mode", "stream", "--first", "0", "--count", "3", *args_of(c)],
                           capture_output=True, text=True, check=True)
        out["streams"].append({**c, "first": 0, "rows": r.stdout.strip().splitlines()})
    for c in PACKS:
        r = subprocess.run([EXE, "--mode", "pack", "--attempts", str(c["attempts"]), *args_of(c)],
                           capture_output=True, text=True, check=True)
        rows = r.stdout.strip().splitlines()
        out["packs"].append({**c, "idx": [int(x.split(",")[1]) - 1 for x in rows],
                             "head_rows": rows[:4], "tail_rows": rows[-2:],
                             "done": r.stderr.strip().splitlines()[-1].split(" (")[0]})
    path = os.path.join(HERE, "knot_reference.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(path, sum(len(p["idx"]) for p in out["packs"]), "accepted paths")


if __name__ == "__main__":
    import sys

    if len(sys.argv) > 2 and sys.argv[1] == "--from-dumps":
        from_dumps(sys.argv[2])
    else:
        main()
