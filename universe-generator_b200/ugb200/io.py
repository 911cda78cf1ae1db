"""Curve and dump writers / readers with the reference engines' file layouts.

* curve CSV: ``attempts,n`` (``attempts,n,nsub,filled`` with subpaths), one row per
  log-spaced milestone (x1.15 from 1000, cuda/braid_cuda.cu:926-929) plus the final
  row (cuda/braid_cuda.cu:1046-1060).  Admission indices are exact here, so each
  milestone row holds the count at exactly that many attempts.
* dump CSV: the 2+1 layouts of cuda/braid_cuda.cu:1062-1104 (legacy single-term
  ``ax,ay,bx,by,ax2,ay2,fx,fy[,gid]`` or multi-term ``ax2,ay2,ax_j,bx_j,fx_j,...``),
  the 3+1 layouts of cuda/braid_cuda3d.cu:1578-1613 (w axis), a 1+1 analogue (x
  axis only), and the braid_knot dump (cuda/braid_knot.cu:386-399).  Floats use
  ``%.10g`` and frequencies ``%.0f`` exactly as the engines print them.
"""

from __future__ import annotations

import csv
from pathlib import Path

import numpy as np

AXES = ("x", "y", "w")


def milestones(total: int, start: int = 1000) -> list[int]:
    out, m = [], start
    while m <= total:
        out.append(m)
        m = int(m * 1.15) + 1
    return out


def curve_rows(acc_idx: np.ndarray, attempts: int, *, n_unique_mask=None, filled=None):
    """(attempts, n[, nsub, filled]) rows: exact counts of admissions before each
    milestone, then the final row."""
    acc_idx = np.asarray(acc_idx)
    order = np.argsort(acc_idx, kind="stable")
    sidx = acc_idx[order]
    rows = []
    for m in milestones(attempts) + [attempts]:
        k = int(np.searchsorted(sidx, m, side="left"))
        if n_unique_mask is None:
            rows.append((m, k))
        else:
            u = int(np.count_nonzero(n_unique_mask[order[:k]]))
            f = int(filled[order[k - 1]]) if (filled is not None and k) else 0
            rows.append((m, u, k - u, f))
    return rows


def write_curve(path: str | Path, rows, subpaths: bool = False) -> None:
    with open(path, "w") as f:
        f.write("attempts,n,nsub,filled\n" if subpaths else "attempts,n\n")
        for r in rows:
            f.write(",".join(str(int(v)) for v in r) + "\n")


def _g(x: float) -> str:
    return "%.10g" % x


def write_dump(path: str | Path, dim: int, a2, a, b, f, gid=None) -> None:
    """Engine --dump-params layout.  a2 [n][dim], a/b/f [n][dim][nw]."""
    a2, a, b, f = (np.asarray(x) for x in (a2, a, b, f))
    n, nw = a.shape[0], a.shape[2]
    ax = AXES[:dim]
    with open(path, "w") as fh:
        if nw == 1:
            cols = [f"a{c}" for c in ax] + [f"b{c}" for c in ax] + [f"a{c}2" for c in ax] + \
                   [f"f{c}" for c in ax]
            fh.write(",".join(cols) + (",gid" if gid is not None else "") + "\n")
            for r in range(n):
                vals = [_g(a[r, k, 0]) for k in range(dim)] + \
                       ["%.0f" % b[r, k, 0] for k in range(dim)] + \
                       [_g(a2[r, k]) for k in range(dim)] + [_g(f[r, k, 0]) for k in range(dim)]
                if gid is not None:
                    vals.append(str(int(gid[r])))
                fh.write(",".join(vals) + "\n")
            return
        head = [f"a{c}2" for c in ax]
        for j in range(1, nw + 1):
            for c in ax:
                head += [f"a{c}_{j}", f"b{c}_{j}", f"f{c}_{j}"]
        fh.write(",".join(head) + (",gid" if gid is not None else "") + "\n")
        for r in range(n):
            vals = [_g(a2[r, k]) for k in range(dim)]
            for j in range(nw):
                for k in range(dim):
                    vals += [_g(a[r, k, j]), "%.0f" % b[r, k, j], _g(f[r, k, j])]
            if gid is not None:
                vals.append(str(int(gid[r])))
            fh.write(",".join(vals) + "\n")


def write_knot_dump(path: str | Path, dim: int, T: int, idx, a2, a, b, f) -> None:
    """braid_knot --dump layout: species, attempt (index + 1), per axis a2 then
    nw x (b, a, f) at %.17g (cuda/braid_knot.cu:386-399, 449-458)."""
    a2, a, b, f = (np.asarray(x) for x in (a2, a, b, f))
    nw = a.shape[2]
    with open(path, "w") as fh:
        fh.write(f"# species,attempt, then per axis: a2, then nw x (b,a,f); dim={dim} T={T} nw={nw}\n")
        for r in range(a.shape[0]):
            parts = ["0", str(int(idx[r]) + 1)]
            for k in range(dim):
                parts.append("%.17g" % a2[r, k])
                for j in range(nw):
                    parts += [str(int(b[r, k, j])), "%.17g" % a[r, k, j], "%.17g" % f[r, k, j]]
            fh.write(",".join(parts) + "\n")


def load_dump(path: str | Path):
    """Read an engine dump (any of the layouts above) into per-axis term arrays:
    returns dim, a2 [n][dim], a/b/f [n][dim][nw], gid or None."""
    with open(path) as fh:
        rows = list(csv.DictReader(fh))
    if not rows:
        raise ValueError(f"{path}: empty dump")
    fields = set(rows[0].keys())
    dim = 3 if ("aw2" in fields) else (2 if ("ay2" in fields) else 1)
    ax = AXES[:dim]
    n = len(rows)
    if f"a{ax[0]}_1" in fields:
        nw = 1
        while f"ax_{nw + 1}" in fields:
            nw += 1
        names = lambda c, j: (f"a{c}_{j + 1}", f"b{c}_{j + 1}", f"f{c}_{j + 1}")  # noqa: E731
    else:
        nw = 1
        names = lambda c, j: (f"a{c}", f"b{c}", f"f{c}")  # noqa: E731
    a2 = np.zeros((n, dim))
    a = np.zeros((n, dim, nw))
    b = np.zeros((n, dim, nw))
    f = np.zeros((n, dim, nw))
    for r, row in enumerate(rows):
        for k, c in enumerate(ax):
            a2[r, k] = float(row[f"a{c}2"])
            for j in range(nw):
                na, nb, nf = names(c, j)
                a[r, k, j] = float(row[na])
                b[r, k, j] = float(row[nb])
                f[r, k, j] = float(row[nf]) if nf in row and row[nf] != "" else 0.0
    gid = np.array([int(row["gid"]) for row in rows]) if "gid" in fields else None
    return dim, a2, a, b, f, gid
