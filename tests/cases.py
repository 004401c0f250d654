"""Seeded synthetic reconstruction cases shared by the parity tests.

Inputs are built with numpy from a seed: a focused (optionally Hermite-mode)
probe, a jittered raster scan, a random multislice object, and patterns from
the oracle's forward model with Poisson noise.  The estimate handed to a
solver is a perturbed copy of the true object.
"""
from __future__ import annotations

import dataclasses
import typing as t

import numpy

from oracle import phaser_np as P
from phaser_b200.sampling import ObjectSampling


@dataclasses.dataclass
class Case:
    probe: numpy.ndarray
    obj: numpy.ndarray
    true_obj: numpy.ndarray
    scan: numpy.ndarray
    patterns: numpy.ndarray
    mask: numpy.ndarray
    probe_sampling: numpy.ndarray
    osamp: ObjectSampling
    thick: numpy.ndarray
    wavelength: float
    tilt: t.Optional[numpy.ndarray]

    def geom(self) -> P.Geometry:
        N = self.probe.shape[-1]
        ky, kx = P.recip_grid((N, N), self.probe_sampling, numpy.float32)
        return P.Geometry(numpy.asarray(self.osamp.corner), numpy.asarray(self.osamp.sampling), ky, kx, self.thick)

    def props(self, bwlim=2 / 3):
        g = self.geom()
        return P.make_propagators(g.ky, g.kx, self.probe_sampling, self.wavelength, self.thick, bwlim)


def make_case(seed: int, N: int = 64, M: int = 2, S: int = 3, scan_shape=(4, 4), step_px: float = 4.0,
              samp: float = 0.2, kv: float = 300e3, tilt: bool = False, counts: float = 1e5,
              dz: float = 20.0, defocus: float = 100.0, conv: float = 25.0, pad_px: float = 5.0) -> Case:
    rng = numpy.random.default_rng(seed)
    lam = P.electron_wavelength(kv)
    ps = numpy.array([samp, samp])
    ky, kx = P.recip_grid((N, N), ps, numpy.float32)
    base = P.make_focused_probe(ky, kx, lam, conv, defocus=defocus).astype(numpy.complex64)
    if M > 1:
        probe = P.hermite_modes(base, M, 0.7, [0.5, 1 / 3, 1 / 6, 0.1, 0.1, 0.1, 0.1][:M - 1])
    else:
        probe = base[None]
    probe = probe.astype(numpy.complex64)
    scan = P.raster_scan(scan_shape, step_px * samp, numpy.float32)
    scan = (scan + rng.uniform(-0.5, 0.5, scan.shape) * samp).astype(numpy.float32)
    osamp = ObjectSampling.from_scan(scan, ps, N / 2 * ps + pad_px * ps)
    H, W = (int(v) for v in osamp.shape)
    thick = numpy.full(S, dz, dtype=numpy.float32) if S > 1 else numpy.array([], numpy.float32)
    phase = rng.normal(0, 0.3, (S, H, W))
    true_obj = (numpy.exp(1j * phase) * rng.uniform(0.85, 1.0, (S, H, W))).astype(numpy.complex64)
    est = (numpy.exp(1j * 0.6 * phase) * 0.97).astype(numpy.complex64)
    tl = rng.normal(0, 3.0, scan.shape).astype(numpy.float32) if tilt else None
    # patterns from the gradient-engine forward model
    g = P.Geometry(numpy.asarray(osamp.corner), numpy.asarray(osamp.sampling), ky, kx, thick)
    props = P.make_propagators(ky, kx, ps, lam, thick)
    flat = scan.reshape(-1, 2)
    psi0, cuts, _, _ = P.cutout_group(g, probe * numpy.float32(1.2), true_obj, flat)
    pt = P.tilt_propagators(ky, kx, thick, props, None if tl is None else tl.reshape(-1, 2))
    psi = P._forward(psi0, cuts, pt)
    wave = P.fft2c(psi[-1] * cuts[:, -1, None])
    inten = numpy.sum(P.abs2(wave), axis=1)
    pats = (rng.poisson(inten * counts) / counts).astype(numpy.float32)
    mask = numpy.ones((N, N), numpy.float32)
    return Case(probe, est, true_obj, scan, pats.reshape(*scan_shape, N, N), mask, ps, osamp, thick, lam, tl)
