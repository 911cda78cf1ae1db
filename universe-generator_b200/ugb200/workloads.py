"""The synthetic packing workloads the packer is measured and checked on.

Each workload is a list of universes (one reference engine run each) plus a
description.  Every input is derived from seeds; no dataset is involved.

  c0  1+1D, F = T = 16, the crossing rule, 20 k candidates
  c1  2+1D, F = T = 64, 1 M candidates in rounds of 16 k
  c2  3+1D, F = T = 128, 5 M candidates in rounds of 64 k
  c3  256 independent universes: dims uniform in {1, 2, 3}, F log-uniform in
      [16, 256], attempt caps log-uniform in [1e4, 1e6], one seed per universe
  c4  2+1D unique-group mode, F = T = 256, 2 M candidates

All use the midpoint z grid t_k = pi (k + 1/2) / T and the open exclusion
|d| < 1/F (UG_ZGRID_MID, UG_EXCL_OPEN).  seed0 selects the seed family
(the universes' seeds are derived from it).
"""

from __future__ import annotations

import math

import numpy as np

from .packer import Universe

NAMES = ("c0", "c1", "c2", "c3", "c4")


def c3_shapes():
    """(dim, F, cap) of the 256 universes of c3, from a fixed meta-seed."""
    rng = np.random.default_rng(12345)
    out = []
    for _ in range(256):
        dim = int(rng.integers(1, 4))
        F = int(round(math.exp(rng.uniform(math.log(16), math.log(256)))))
        F = max(16, min(256, F))
        cap = int(round(math.exp(rng.uniform(math.log(1e4), math.log(1e6)))))
        out.append((dim, F, cap))
    return out


def workload(name: str, seed0: int = 0):
    """(universes, description) of workload `name`."""
    if name == "c0":
        return [Universe(dim=1, T=16, zgrid=1, excl=1, cross1d=1, seed=seed0, attempts=20000,
                         round_size=4096)], {"dim": 1, "F": 16, "T": 16, "candidates": 20000}
    if name == "c1":
        return [Universe(dim=2, T=64, zgrid=1, excl=1, seed=seed0, attempts=1_000_000,
                         round_size=16384)], {"dim": 2, "F": 64, "T": 64, "candidates": 1_000_000,
                                              "round": 16384}
    if name == "c2":
        return [Universe(dim=3, T=128, zgrid=1, excl=1, seed=seed0, attempts=5_000_000,
                         round_size=65536)], {"dim": 3, "F": 128, "T": 128, "candidates": 5_000_000,
                                              "round": 65536}
    if name == "c3":
        us = [Universe(dim=dim, T=F, zgrid=1, excl=1, cross1d=int(dim == 1),
                       seed=(seed0 * 1000003 + k) & (2**64 - 1), attempts=cap, round_size=16384)
              for k, (dim, F, cap) in enumerate(c3_shapes())]
        return us, {"universes": 256, "dims": [1, 2, 3], "F": "log-uniform[16,256]",
                    "caps": "log-uniform[1e4,1e6]", "candidates": sum(u.attempts for u in us)}
    if name == "c4":
        return [Universe(dim=2, T=256, zgrid=1, excl=1, group_mode=2, seed=seed0, attempts=2_000_000,
                         round_size=16384)], {"dim": 2, "F": 256, "T": 256, "candidates": 2_000_000,
                                              "mode": "unique-group"}
    raise ValueError(f"unknown workload {name!r}")
