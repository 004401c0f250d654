"""Host-side optics used once per engine: Fresnel propagators and probes.

The propagator table is built exactly as phaser/engines/common/simulation.py:160-190
builds it (complex64 Fresnel kernel from phaser/utils/optics.py:190-211 times the
2/3 band limit), so the device kernels multiply by the reference's own values.
The probe helpers (optics.py:30-136) generate synthetic inputs.
"""
from __future__ import annotations

import math
import typing as t

import numpy


def _cdt(dtype):
    return numpy.complex64 if numpy.dtype(dtype) == numpy.float32 else numpy.complex128


def fresnel_propagator(ky, kx, wavelength: float, delta_z: float, tilt=(0., 0.)) -> numpy.ndarray:
    tx, ty = numpy.tan(tilt[0] * 1e-3), numpy.tan(tilt[1] * 1e-3)
    k2 = ky ** 2 + kx ** 2
    return numpy.exp(-1.j * numpy.pi * delta_z * (wavelength * k2 - 2. * (kx * tx + ky * ty))).astype(_cdt(k2.dtype))


def make_propagators(ky, kx, probe_sampling, wavelength: float, thicknesses,
                     bwlim_frac: t.Optional[float] = 2 / 3) -> t.Optional[numpy.ndarray]:
    """(S-1, N, N) band-limited propagators, one per slice gap; equal gaps (to 5
    decimals) share a kernel.  None for a single slice."""
    gaps = numpy.asarray(thicknesses)[:-1]
    if len(gaps) == 0:
        return None
    if bwlim_frac is not None:
        limit = numpy.min(1 / (2 * numpy.asarray(probe_sampling, numpy.float64))) * bwlim_frac
        band = (ky ** 2 + kx ** 2) <= limit ** 2
    else:
        band = numpy.ones(ky.shape, dtype=numpy.bool_)
    kernels: t.Dict[float, numpy.ndarray] = {}
    rows = []
    for dz in gaps:
        key = round(float(dz), 5)
        if key not in kernels:
            kernels[key] = fresnel_propagator(ky, kx, wavelength, float(dz)).astype(_cdt(ky.dtype)) * band
        rows.append(kernels[key])
    return numpy.stack(rows, axis=0)


def _ifft2c(a):
    return numpy.fft.fftshift(numpy.fft.ifft2(a, norm='ortho'), axes=(-2, -1))


def make_focused_probe(ky, kx, wavelength: float, aperture: float, defocus: float = 0.) -> numpy.ndarray:
    """Circular aperture (mrad) with defocus (+ = overfocus), unit intensity."""
    th2 = (ky * wavelength) ** 2 + (kx * wavelength) ** 2
    probe = numpy.exp(-2.j * numpy.pi * (defocus / (2. * wavelength)) * th2)
    probe = probe * (th2 <= (aperture * 1e-3) ** 2)
    probe = probe / numpy.sqrt(numpy.sum(probe.real ** 2 + probe.imag ** 2))
    return _ifft2c(probe).astype(_cdt(ky.dtype))


def make_hermite_modes(base: numpy.ndarray, n_modes: int, base_mode_power: float = 0.7,
                       rel_powers=1.0) -> numpy.ndarray:
    """Orthonormal Hermite-Gauss perturbation modes of `base` with the given powers."""
    rdt = numpy.float32 if base.dtype == numpy.complex64 else numpy.float64
    rel = numpy.array(rel_powers, dtype=rdt).ravel()
    rel = numpy.pad(rel, (0, n_modes - rel.size - 1), mode='edge')[:n_modes - 1]
    powers = numpy.concatenate([[base_mode_power], (1.0 - base_mode_power) * rel])
    i = numpy.arange(n_modes)
    diag = numpy.ceil((numpy.sqrt(8 * i + 9) - 3) / 2).astype(numpy.int64)
    xo = (i - diag * (diag + 1) / 2).astype(numpy.int64)
    yo = diag - xo
    yy, xx = numpy.indices(base.shape, dtype=rdt)
    mag = base.real ** 2 + base.imag ** 2
    yy = yy - numpy.sum(yy * mag) / numpy.sum(mag)
    xx = xx - numpy.sum(xx * mag) / numpy.sum(mag)
    modes = numpy.empty((n_modes, *base.shape), dtype=base.dtype)
    for k in range(n_modes):
        mode = yy ** yo[k] * xx ** xo[k] * base
        for p in range(k):
            mode = mode - modes[p] * numpy.sum(modes[p] * numpy.conj(mode))
        modes[k] = mode / numpy.sqrt(numpy.sum(mode.real ** 2 + mode.imag ** 2))
    return modes * numpy.sqrt(powers)[:, None, None].astype(modes.dtype)


def electron_wavelength(energy_ev: float) -> float:
    """Relativistic electron wavelength [angstrom] (phaser/utils/physics.py:59-62)."""
    return 1.23984244e4 / math.sqrt(energy_ev * (2 * 5.1099906e5 + energy_ev))
