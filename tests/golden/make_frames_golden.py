"""Golden frame_bake hits from the reference's own Python baker.

Run where the reference tree is present:

    python tests/golden/make_frames_golden.py

Inputs: (1) the inline 3-path dump of the reference's tests/test_frames.py (read from
that file), (2) the 45 paths of the deterministic packing T=16, dim 2, seed 1 (the
reference braid_knot stream, parameters from the oracle, which reproduces the reference
bit for bit).  Hits come from braidlab.frames.bake_reference (frames.py:246-362) of the
reference tree, which its docstring names as the oracle of the CUDA baker.
"""

from __future__ import annotations

import io
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
from oracle import REFERENCE_DIR as REF  # noqa: E402

RUN = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from braidlab.corrdim import load_axis_terms
from braidlab.frames import bake_reference
cases = json.loads(open(sys.argv[2]).read())
out = []
for c in cases:
    axes = load_axis_terms(c["dump_path"])
    kw = dict(front=c["front"], cheb=c["cheb"], speed=c["speed"], wraps=c["wraps"])
    if c["obs"][0] == "path":
        kw["observer_path"] = c["obs"][1]
    else:
        kw["observer_point"] = (c["obs"][1], c["obs"][2])
    hits = bake_reference(axes, c["z_obs"], c["z_min"], **kw)
    out.append([[int(h[0]), float(h[1]), float(h[2]), float(h[3]), float(h[4])] for h in hits])
print(json.dumps(out))
"""


def dumps():
    text = open(os.path.join(REF, "tests", "test_frames.py")).read()
    m = re.search(r'DUMP = \(\n(.*?)\n\)', text, re.S)
    inline = "".join(eval(line.strip()) for line in m.group(1).splitlines())  # string literals
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "universe-generator_b200"))
    import numpy as np

    import oracle as O
    from ugb200.io import write_dump

    model = O.Model(dim=2, T=16, rng=O.RNG_KNOT, seed=1)
    acc = O.pack(model, 20000).acc_idx
    cs = [O.candidate(model, int(i)) for i in acc]
    a2 = np.array([c["a2"] for c in cs])
    a = np.array([c["a"] for c in cs])
    b = np.array([c["b"] for c in cs])
    f = np.array([c["f"] for c in cs])
    buf = os.path.join(HERE, "_packed_dump.csv")
    write_dump(buf, 2, a2, a, b, f)
    packed = open(buf).read()
    os.remove(buf)
    return {"inline": inline, "packed": packed}


def main() -> None:
    ds = dumps()
    cases = []
    for name, spec in [
        ("inline", dict(z_obs=0.5, z_min=0.02, obs=["path", 0], front="fit")),
        ("inline", dict(z_obs=0.5, z_min=0.02, obs=["path", 0], front="budget")),
        ("inline", dict(z_obs=0.5, z_min=0.05, obs=["point", 0.1, 0.3], front="speed", cheb=False)),
        ("inline", dict(z_obs=0.35, z_min=0.02, obs=["path", 1], front="fit", wraps=2)),
        ("packed", dict(z_obs=0.5, z_min=0.02, obs=["path", 3], front="fit")),
        ("packed", dict(z_obs=0.7, z_min=0.03, obs=["point", -0.4, 0.2], front="speed")),
        ("packed", dict(z_obs=0.6, z_min=0.02, obs=["path", 0], front="budget")),
        ("packed", dict(z_obs=0.45, z_min=0.02, obs=["point", 0.0, 0.0], front="fit", cheb=False)),
    ]:
        c = {"dump": name, "front": spec["front"], "cheb": spec.get("cheb", True),
             "speed": 0.33, "wraps": spec.get("wraps"), "obs": spec["obs"],
             "z_obs_pi": spec["z_obs"], "z_min_pi": spec["z_min"]}
        cases.append(c)
    tmp = []
    for k, c in enumerate(cases):
        p = os.path.join(HERE, f"_d{k}.csv")
        open(p, "w").write(ds[c["dump"]])
        tmp.append(p)
        c["dump_path"] = p
        import math

        c["z_obs"] = c["z_obs_pi"] * math.pi
        c["z_min"] = c["z_min_pi"] * math.pi
    spec = os.path.join(HERE, "_cases.json")
    json.dump(cases, open(spec, "w"))
    r = subprocess.run([sys.executable, "-c", RUN, REF, spec], capture_output=True, text=True,
                       check=True)
    hits = json.loads(r.stdout)
    for p in tmp + [spec]:
        os.remove(p)
    for c, h in zip(cases, hits):
        del c["dump_path"]
        c["hits"] = h
    out = {"generator": "reference braidlab.frames.bake_reference", "dumps": ds, "cases": cases}
    json.dump(out, open(os.path.join(HERE, "frames_reference.json"), "w"))
    print([len(c["hits"]) for c in cases])


if __name__ == "__main__":
    main()
