"""Job and Campaign: the identity of a packing run (reference braidlab/config.py:15-158).

Field names, defaults, validation, ``Job.key`` and ``Job.name`` are kept identical
because stores and remote workspaces are keyed by them.
"""

from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Job:
    """One packing run: (dim, T, seed) at a stop threshold."""

    dim: int
    t: int
    seed: int
    accept_rate: float
    max_attempts: float
    band: str = "nyq"          # fixed identity column: the band is always max frequency = T
    euclid: bool = False       # L2 exclusion (--euclid-collision)
    sparse: bool = False       # sparse grid (--sparse, 3+1)
    terms: int = 2             # sinusoid terms per axis incl. sin1 (--terms)
    subpaths: bool = False     # second-phase subpath packing (2+1 only)
    sub_attempts: float = 0    # fixed phase-2 budget (0 = rate stop only)
    tag: str = ""              # variant tag, part of the name only

    def __post_init__(self) -> None:
        if self.band != "nyq":
            raise ValueError(f"band must be 'nyq' (the max frequency is T), got {self.band!r}")
        if self.subpaths and self.dim != 2:
            raise ValueError("subpaths is a 2+1 engine feature (dim must be 2)")

    @property
    def key(self) -> tuple[int, str, int, int, float, int]:
        return (self.dim, self.band, self.t, self.seed, self.accept_rate, self.terms)

    @property
    def name(self) -> str:
        parts = [f"d{self.dim}_{self.band}_T{self.t}_s{self.seed}"]
        if self.euclid:
            parts.append("eu")
        parts.append("ph")
        if self.sparse:
            parts.append("sp")
        if self.terms != 2:
            parts.append(f"tm{self.terms}")
        if self.subpaths:
            parts.append("sub")
        if self.tag:
            parts.append(self.tag)
        return "_".join(parts)

    @property
    def maxfreq(self) -> int:
        return self.t


@dataclass(frozen=True)
class Campaign:
    """A declarative experiment expanding into Jobs (T x seed x terms)."""

    name: str
    dim: int
    t_values: tuple[int, ...]
    seeds: tuple[int, ...]
    accept_rate: float
    max_attempts: float = 3e12
    dump: bool = False
    euclid: bool = False
    sparse: bool = False
    terms_values: tuple[int, ...] = (2,)
    terms_track_t: bool = False
    subpaths: bool = False
    sub_attempts: float = 0
    tag: str = ""

    def __post_init__(self) -> None:
        if self.dim not in (2, 3):
            raise ValueError(f"dim must be 2 or 3, got {self.dim}")
        if self.accept_rate <= 0:
            raise ValueError("accept_rate must be > 0")
        if any(k < 2 for k in self.terms_values):
            raise ValueError(f"terms_values must all be >= 2, got {self.terms_values}")
        if self.terms_track_t and self.terms_values != (2,):
            raise ValueError("terms_track_t and terms_values are mutually exclusive")
        if self.subpaths and self.dim != 2:
            raise ValueError("subpaths is a 2+1 engine feature (dim must be 2)")

    def jobs(self) -> list[Job]:
        out = []
        for t in self.t_values:
            for s in self.seeds:
                for k in self.terms_values:
                    out.append(Job(dim=self.dim, t=t, seed=s, accept_rate=self.accept_rate,
                                   max_attempts=self.max_attempts, euclid=self.euclid,
                                   sparse=self.sparse, terms=t if self.terms_track_t else k,
                                   subpaths=self.subpaths, sub_attempts=self.sub_attempts,
                                   tag=self.tag))
        return out
