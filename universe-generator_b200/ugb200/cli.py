"""Engine-compatible command line: a drop-in for the reference packers.

    python -m ugb200.cli [--engine braid_cuda|braid_cuda3d|braid_knot] <engine flags>

or the executables in universe-generator_b200/bin/ named like the reference binaries
(braidlab.engine.binary_name).  Accepted flags follow the engines' parsers
(cuda/braid_cuda.cu:534-584, cuda/braid_cuda3d.cu:862-913, cuda/braid_knot.cu:258-289):
the guard no-ops ``--uniform --torus --phase`` are accepted, ``--maxfreq`` must equal T
(braid_cuda.cu:597-603), ``--smart`` and ``--angle-sample`` are refused as the engines
refuse them, ``--subpaths`` with ``--sub-until-accept-rate`` / ``--sub-until-fill-rate``,
and the braid_cuda3d flags ``--euclid-collision``, ``--diag`` and ``--probe-n`` are
supported.  The outputs are the engines': curve CSV, ``--dump-params`` / ``--dump`` CSV,
the ``--diag`` CSVs and the stderr ``done: N=.. in .. attempts`` line that
braidlab.engine.parse_done reads.

Additions: ``--rng knot|philox`` (default knot: the reference's deterministic per-attempt
stream, cuda/braid_knot.cu:207), ``--zgrid ref|mid``, ``--excl ref|open``,
``--precision mixed|fp64``, ``--dim`` (braid_knot), ``--round N``.
Every failure exits 1 with a message, like the engines.
"""

from __future__ import annotations

import os
import sys

import numpy as np

from . import _lib as L
from .io import curve_rows, write_curve, write_dump, write_knot_dump
from .packer import Packer, Universe

UNSUPPORTED = {
    "--angle-sample": ("--angle-sample was removed along with the hard-wall geometry it compensated "
                       "for; the sin1 offset is always uniform (braid_cuda3d.cu:885-889)"),
    "--nu-attempts": "the second (nu) species of braid_knot is not built",
    "--nu-div": "the second (nu) species of braid_knot is not built",
}


def _die(msg: str) -> int:
    print(f"error: {msg}", file=sys.stderr)
    return 1


def filled_cells(pos: np.ndarray, cell: float) -> np.ndarray:
    """Occupied (timestep, cell) buckets after each admission, in admission
    order (the fill measure of cuda/braid_cuda.cu:865-879)."""
    n, dim, T = pos.shape
    gw = int(round(2.0 / cell))
    c = np.clip(np.floor((pos + 1.0) / cell).astype(np.int64), 0, gw - 1)
    key = np.zeros((n, T), np.int64)
    for k in range(dim):
        key = key * gw + c[:, k, :]
    key = key * T + np.arange(T)[None, :]
    seen: set[int] = set()
    out = np.zeros(n, np.int64)
    for r in range(n):
        seen.update(key[r].tolist())
        out[r] = len(seen)
    return out


def write_diag(prefix: str, px: np.ndarray, probe, probe_n: int, nb: int = 50) -> None:
    """--diag outputs of braid_cuda3d.cu:1615-1670: occupancy of the accepted worldlines'
    x over every timestep, and the probe's proposed / accepted counts per x-centre bin."""
    b = np.clip(np.floor((px.ravel() + 1.0) * 0.5 * nb).astype(np.int64), 0, nb - 1)
    occ = np.bincount(b, minlength=nb)
    centers = [-1.0 + (k + 0.5) * 2.0 / nb for k in range(nb)]
    with open(f"{prefix}_occ.csv", "w") as f:
        f.write("x_center,count\n")
        for c, v in zip(centers, occ):
            f.write(f"{c:.4f},{int(v)}\n")
    prop, acc = probe
    with open(f"{prefix}_probe.csv", "w") as f:
        f.write("x_center,proposed,accepted\n")
        for c, p_, a_ in zip(centers, prop, acc):
            f.write(f"{c:.4f},{int(p_)},{int(a_)}\n")
    print(f"diag: wrote {prefix}_occ.csv and {prefix}_probe.csv (probeN={probe_n})", file=sys.stderr)


def main(argv: list[str] | None = None, engine: str | None = None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if engine is None:
        engine = "braid_cuda"
        if "--engine" in argv:
            i = argv.index("--engine")
            engine = argv[i + 1]
            del argv[i:i + 2]
    base = engine.removesuffix("_w150")
    if base not in ("braid_cuda", "braid_cuda3d", "braid_knot"):
        return _die(f"unknown engine {engine}")
    knot = base == "braid_knot"
    # engine defaults (braid_cuda.cu:514-528, braid_knot.cu:255-257)
    T, budget = (32, 1e10) if knot else (120, 1e8)
    seed = 1 if knot else 12345
    dim = 3 if base == "braid_cuda3d" else 2
    terms = 0 if knot else 2
    curve = dump = None
    maxfreq = 0
    accept = sub_accept = sub_fill = 0.0
    pin = subpaths = euclid = False
    diag = None
    probe_n = 5_000_000
    sub_budget = 0.0
    sub_terms = 0
    max_n = 0
    rng, zgrid, excl, prec = L.RNG_KNOT, L.ZGRID_REF, L.EXCL_REF, L.PREC_MIXED
    round_size = 65536
    i = 0
    try:
        while i < len(argv):
            a = argv[i]

            def val():
                nonlocal i
                i += 1
                if i >= len(argv):
                    raise ValueError(f"{a} needs a value")
                return argv[i]

            if a in ("-t", "--timesteps"):
                T = int(val())
            elif a == "--attempts":
                budget = float(val())
            elif a == "--seed":
                seed = int(val())
            elif a in ("--uniform", "--torus", "--phase", "--sparse"):
                pass  # accepted guards; the grid kind is chosen by size
            elif a == "--smart":
                return _die("--smart was removed (frequencies are drawn uniformly)")
            elif a == "--curve":
                curve = val()
            elif a == "--maxfreq":
                maxfreq = int(val())
            elif a == "--until-accept-rate":
                accept = float(val())
            elif a == "--terms":
                terms = int(val())
            elif a == "--pin-sin1":
                pin = True
            elif a in ("--diag", "--probe-n"):
                if base != "braid_cuda3d":
                    return _die(f"{a} is a braid_cuda3d flag")
                if a == "--diag":
                    diag = val()
                else:
                    probe_n = int(float(val()))
            elif a == "--euclid-collision":
                if base != "braid_cuda3d":
                    return _die("--euclid-collision is a braid_cuda3d flag (the L2-ball exclusion)")
                euclid = True  # braid_cuda3d.cu:890-891
            elif a == "--subpaths":
                subpaths = True
            elif a == "--sub-attempts":
                sub_budget = float(val())
            elif a == "--sub-until-accept-rate":
                sub_accept = float(val())
            elif a == "--sub-until-fill-rate":
                sub_fill = float(val())
            elif a == "--sub-terms":
                sub_terms = int(val())
            elif a == "--max-n":
                max_n = int(val())
            elif a in ("--dump-params", "--dump"):
                dump = val()
            elif a == "--dim":
                dim = int(val())
            elif a == "--rng":
                rng = {"knot": L.RNG_KNOT, "philox": L.RNG_PHILOX}[val()]
            elif a == "--zgrid":
                zgrid = {"ref": L.ZGRID_REF, "mid": L.ZGRID_MID}[val()]
            elif a == "--excl":
                excl = {"ref": L.EXCL_REF, "open": L.EXCL_OPEN}[val()]
            elif a == "--precision":
                prec = {"mixed": L.PREC_MIXED, "fp64": L.PREC_FP64}[val()]
            elif a == "--round":
                round_size = int(val())
            elif a in UNSUPPORTED:
                return _die(UNSUPPORTED[a])
            else:
                return _die(f"unknown flag {a}")
            i += 1
    except (ValueError, KeyError) as e:
        return _die(str(e))
    if maxfreq not in (0, T):
        return _die(f"--maxfreq {maxfreq}: the max frequency is T={T} (the full Nyquist band)")
    if terms == 0:
        terms = T
    if terms < 2:
        terms = 2
    if sub_terms and sub_terms != terms:
        return _die("--sub-terms different from --terms is not built")
    if subpaths and dim != 2:
        return _die("subpaths is a 2+1 engine feature")
    u = Universe(dim=dim, T=T, terms=0 if terms == T else terms, rng=rng, zgrid=zgrid,
                 excl=excl, pin_sin1=int(pin), group_mode=L.GROUP_SUBPATH if subpaths else 0,
                 round_size=round_size, seed=seed, attempts=int(budget), max_n=max_n,
                 sub_attempts=int(sub_budget), accept_rate=accept, sub_accept_rate=sub_accept,
                 sub_fill_rate=sub_fill, euclid=int(euclid))
    kind = {2: "2+1", 3: "3+1", 1: "1+1"}[dim]
    print(f"{kind} (torus, phase): T={T}  modmax={max(T - 1, 2)} (maxfreq={max(T - 1, 2) + 1})  "
          f"terms={terms}  rng={'knot' if rng == L.RNG_KNOT else 'philox'}", file=sys.stderr)
    try:
        p = Packer([u], precision=prec)
        p.run()
        st = p.stats(0)
        idx, gid = p.accepted(0)
        params = p.params(0) if dump else None
        pos = p.positions(0) if (subpaths or diag) else None
        probe = p.probe(0, probe_n, 50) if diag else None
        p.close()
    except L.UgError as e:
        return _die(str(e))
    cell = 2.0 / T if excl == L.EXCL_REF else 1.0 / T
    ncell = T * int(round(2.0 / cell)) ** dim
    filled = filled_cells(pos, cell) if subpaths else None
    if knot:
        print(f"done: N={st.n} (primary {st.n}, nu 0) in {st.attempts} attempts", file=sys.stderr)
    elif base == "braid_cuda3d":
        print(f"done: N={st.n_unique} in {st.phase1_end} attempts", file=sys.stderr)
    else:
        # braid_cuda.cu:945 -- the 2+1 engine also reports the occupied grid cells
        k1 = int(np.count_nonzero(idx < st.phase1_end))
        f1 = (int(filled[k1 - 1]) if k1 else 0) if subpaths else st.filled
        print(f"done: N={st.n_unique} in {st.phase1_end} attempts, filled {f1}/{ncell} cells "
              f"({100.0 * f1 / ncell:.3f}%)", file=sys.stderr)
    if subpaths:
        sub_att = st.attempts - st.phase1_end
        if sub_att >= (int(sub_budget) if sub_budget > 0 else int(budget)):
            why = "attempt budget"
        elif sub_fill > 0 and sub_accept <= 0:
            why = "fill-rate"
        elif sub_accept > 0 and sub_fill <= 0:
            why = "accept-rate"
        else:
            why = "accept-rate or fill-rate"
        print(f"sub done ({why}): Nsub={st.n_sub} in {sub_att} attempts, filled {st.filled}/{ncell} "
              f"cells ({100.0 * st.filled / ncell:.3f}%)", file=sys.stderr)
    if diag:
        write_diag(diag, pos[:, 0, :], probe, probe_n)
    if curve:
        if knot:
            with open(curve, "w") as f:
                f.write("attempt,n,species\n")
                for k, ix in enumerate(idx):
                    f.write(f"{int(ix) + 1},{k + 1},0\n")
        else:
            uniq = (gid == np.arange(len(gid))) if subpaths else None
            write_curve(curve, curve_rows(idx, st.attempts, n_unique_mask=uniq, filled=filled),
                        subpaths=subpaths)
    if dump:
        if knot:
            write_knot_dump(dump, dim, T, idx, params["a2"], params["a"], params["b"], params["f"])
        else:
            write_dump(dump, dim, params["a2"], params["a"], params["b"], params["f"],
                       gid=gid if subpaths else None)
        print(f"dump-params: wrote {len(idx)} worldlines to {dump}", file=sys.stderr)
    return 0


def entry() -> None:
    sys.exit(main(engine=os.path.basename(sys.argv[0]) if not sys.argv[0].endswith(".py") else None))


if __name__ == "__main__":
    sys.exit(main())
