"""Golden observer-view remaps from the reference's own braidlab.frames.apparent_positions
(frames.py:147-188).

Run where the reference tree is present:

    python tests/golden/make_view_golden.py

Cases: seeded hit tables (offsets up to the front radius, a hit at the pulse centre,
hits on the axes) under boosts below, at and above the 0.995 cap, a boost under the
1e-6 static threshold, both shells and both modes.  Written to view_reference.json with
every float as its exact repr.
"""

from __future__ import annotations

import json
import os
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
from braidlab.frames import HIT_DTYPE, ObserverFrame, apparent_positions
cases = json.loads(open(sys.argv[2]).read())
out = []
for c in cases:
    h = np.zeros(len(c["dx"]), HIT_DTYPE)
    h["dx"] = c["dx"]; h["dy"] = c["dy"]; h["chi"] = c["chi"]; h["src"] = np.arange(len(h)); h["z_emit"] = 1.0
    fr = ObserverFrame(1.5, 2.0, 1, 0.0, 0.0, np.array(c["beta"]), h)
    ax, ay, ld = apparent_positions(fr, c["mode"], c["cheb"])
    out.append({"ax": [float(v) for v in ax], "ay": [float(v) for v in ay], "ln_dopp": [float(v) for v in ld]})
print(json.dumps(out))
"""


def cases():
    import numpy as np

    rng = np.random.default_rng(20240601)
    out = []
    betas = [(0.3, -0.2), (0.0, 0.9), (-0.7, 0.7), (1.4, 0.3), (2e-7, 1e-7), (0.0, 0.0), (0.05, 0.01),
             (-0.995, 0.0)]
    for i, beta in enumerate(betas):
        for mode in ("moving", "static"):
            for cheb in (True, False):
                if mode == "static" and i > 1:
                    continue
                n = 48
                chi = rng.uniform(0.05, 3.0, n).astype(np.float32)
                ang = rng.uniform(-np.pi, np.pi, n)
                r = chi * rng.uniform(0.2, 1.0, n)
                dx = (r * np.cos(ang)).astype(np.float32)
                dy = (r * np.sin(ang)).astype(np.float32)
                dx[0] = dy[0] = 0.0           # at the pulse centre
                dx[1], dy[1] = chi[1], 0.0    # on the axes
                dx[2], dy[2] = 0.0, -chi[2]
                out.append({"beta": [float(beta[0]), float(beta[1])], "mode": mode, "cheb": cheb,
                            "dx": [float(v) for v in dx], "dy": [float(v) for v in dy],
                            "chi": [float(v) for v in chi]})
    return out


def main() -> None:
    cs = cases()
    tmp = os.path.join(HERE, "_view_cases.json")
    with open(tmp, "w") as fh:
        json.dump(cs, fh)
    try:
        r = subprocess.run([sys.executable, "-c", RUN, REF, tmp], capture_output=True, text=True, check=True)
    finally:
        os.remove(tmp)
    res = json.loads(r.stdout)
    for c, o in zip(cs, res):
        c.update(o)
    with open(os.path.join(HERE, "view_reference.json"), "w") as fh:
        json.dump(cs, fh)
    print(f"{len(cs)} cases")


if __name__ == "__main__":
    main()
