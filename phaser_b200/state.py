"""Reconstruction state, field-compatible with phaser/state.py.

The B200 engines read and write a `ReconsState`-shaped object: phaser's own
(if phaser is installed) or these dataclasses.  Arrays stay numpy on the host
side of the boundary; the engine uploads them once and writes the results
back, so checkpoints (phaser/utils/io.py) see the usual layout:
probe (modes, y, x) complex, object (z, y, x) complex + thicknesses,
scan (..., 2) (y, x), tilt (..., 2) mrad or None.
"""
from __future__ import annotations

import dataclasses
import typing as t

import numpy

from .sampling import Sampling, ObjectSampling


@dataclasses.dataclass
class Patterns:
    patterns: numpy.ndarray       # (..., N, N) float, zero frequency in the corner
    pattern_mask: numpy.ndarray   # (N, N)


@dataclasses.dataclass
class IterState:
    engine_num: int = 0
    engine_iter: int = 0
    total_iter: int = 0
    n_engine_iters: t.Optional[int] = None
    n_total_iters: t.Optional[int] = None


@dataclasses.dataclass
class ProbeState:
    sampling: Sampling
    data: numpy.ndarray           # (modes, y, x) complex


@dataclasses.dataclass
class ObjectState:
    sampling: ObjectSampling
    data: numpy.ndarray           # (z, y, x) complex
    thicknesses: numpy.ndarray    # (z,) or empty for a single slice


@dataclasses.dataclass
class ProgressState:
    iters: numpy.ndarray = dataclasses.field(default_factory=lambda: numpy.array([], dtype=numpy.uint64))
    detector_errors: numpy.ndarray = dataclasses.field(default_factory=lambda: numpy.array([], dtype=numpy.float64))


@dataclasses.dataclass(kw_only=True)
class ReconsState:
    iter: IterState
    wavelength: float
    probe: ProbeState
    object: ObjectState
    scan: numpy.ndarray           # (..., 2) (y, x) length units
    tilt: t.Optional[numpy.ndarray] = None
    progress: ProgressState = dataclasses.field(default_factory=ProgressState)
