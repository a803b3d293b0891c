"""State and frame value types, mirroring kete's ``State`` (src/kete_core/src/state.rs:76-131)
and ``Frames`` enum as seen from Python."""
from __future__ import annotations

import enum
from dataclasses import dataclass, field

import numpy as np


class Frames(enum.IntEnum):
    """Coordinate frames handled on the GPU path (values are the C-ABI frame codes)."""

    Equatorial = 1
    Ecliptic = 2


@dataclass
class State:
    """An exact state: designation, TDB JD, position (AU) and velocity (AU/day) relative
    to ``center_id`` in ``frame``.  Defaults follow kete: ecliptic, Sun-centred (10)."""

    desig: str | int | None
    jd: float
    pos: np.ndarray
    vel: np.ndarray
    frame: Frames = Frames.Ecliptic
    center_id: int = 10

    def __post_init__(self):
        self.pos = np.asarray(self.pos, dtype=np.float64).reshape(3).copy()
        self.vel = np.asarray(self.vel, dtype=np.float64).reshape(3).copy()
        self.jd = float(self.jd)
        self.frame = Frames(self.frame)

    @property
    def is_finite(self) -> bool:
        return bool(np.all(np.isfinite(self.pos)) and np.all(np.isfinite(self.vel))
                    and np.isfinite(self.jd))

    @classmethod
    def new_nan(cls, desig, jd, frame=Frames.Ecliptic, center_id=10) -> "State":
        """State::new_nan (state.rs:125-135)."""
        return cls(desig, jd, [np.nan] * 3, [np.nan] * 3, frame, center_id)


@dataclass
class SimultaneousStates:
    """Collection of states at one epoch (kete_core/simult_states.rs:14-35)."""

    states: list = field(default_factory=list)
    fov: object = None

    @property
    def jd(self) -> float:
        return self.states[0].jd if self.states else float("nan")

    def __len__(self):
        return len(self.states)


def _rot():
    c, s = np.cos(0.40909280422232897), np.sin(0.40909280422232897)
    return c, s


def ecliptic_to_equatorial(v):
    c, s = _rot()
    v = np.asarray(v, dtype=np.float64)
    return np.array([v[0], c * v[1] - s * v[2], s * v[1] + c * v[2]])


def equatorial_to_ecliptic(v):
    c, s = _rot()
    v = np.asarray(v, dtype=np.float64)
    return np.array([v[0], c * v[1] + s * v[2], -s * v[1] + c * v[2]])


def change_frame(vec, from_frame, to_frame):
    if Frames(from_frame) == Frames(to_frame):
        return np.asarray(vec, dtype=np.float64)
    if Frames(from_frame) == Frames.Ecliptic:
        return ecliptic_to_equatorial(vec)
    return equatorial_to_ecliptic(vec)


def pack(states):
    """Stack states into SoA arrays: pos (3,n), vel (3,n), jd (n,)."""
    n = len(states)
    pos = np.empty((3, n))
    vel = np.empty((3, n))
    jd = np.empty(n)
    for i, s in enumerate(states):
        pos[:, i] = s.pos
        vel[:, i] = s.vel
        jd[i] = s.jd
    return pos, vel, jd
