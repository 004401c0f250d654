"""Sampling grids (host geometry), field-compatible with phaser's.

`Sampling` follows phaser/utils/num.py:545-670 (probe / detector grid) and
`ObjectSampling` phaser/utils/object.py:190-331 (object grid, cutout
indices).  Index arithmetic is float64 with numpy's round-half-to-even,
identical to the reference; the GPU kernels repeat the same IEEE operations.
"""
from __future__ import annotations

import typing as t

import numpy


class Sampling:
    def __init__(self, shape, *, extent=None, sampling=None):
        self.shape = numpy.broadcast_to(numpy.asarray(shape).astype(numpy.int_), (2,))
        if extent is not None:
            self.extent = numpy.broadcast_to(numpy.asarray(extent, numpy.float64), (2,))
            self.sampling = self.extent / self.shape
        elif sampling is not None:
            self.sampling = numpy.broadcast_to(numpy.asarray(sampling, numpy.float64), (2,))
            self.extent = self.sampling * self.shape
        else:
            raise ValueError("Either 'extent' or 'sampling' must be specified")

    @property
    def k_max(self) -> numpy.ndarray:
        return (1 / (2 * self.sampling)).astype(numpy.float64)

    def recip_grid(self, *, dtype=numpy.float64, xp=None):
        """(ky, kx) fftfreq meshgrid, zero frequency in the corner (num.py:651-670)."""
        ky = numpy.fft.fftfreq(int(self.shape[0]), self.sampling[0]).astype(dtype)
        kx = numpy.fft.fftfreq(int(self.shape[1]), self.sampling[1]).astype(dtype)
        return tuple(numpy.meshgrid(ky, kx, indexing='ij'))

    def recip_axes(self, dtype=numpy.float32) -> t.Tuple[numpy.ndarray, numpy.ndarray]:
        return (numpy.fft.fftfreq(int(self.shape[0]), self.sampling[0]).astype(dtype),
                numpy.fft.fftfreq(int(self.shape[1]), self.sampling[1]).astype(dtype))


class ObjectSampling:
    def __init__(self, shape, sampling, corner=None, region_min=None, region_max=None):
        self.shape = numpy.broadcast_to(numpy.asarray(shape).astype(numpy.int_), (2,))
        self.sampling = numpy.broadcast_to(numpy.asarray(sampling, numpy.float64), (2,))
        self.region_min = None if region_min is None else numpy.broadcast_to(numpy.asarray(region_min, numpy.float64), (2,))
        self.region_max = None if region_max is None else numpy.broadcast_to(numpy.asarray(region_max, numpy.float64), (2,))
        if corner is None:
            corner = -self.extent / 2. + self.sampling / 2.
        self.corner = numpy.broadcast_to(numpy.asarray(corner, numpy.float64), (2,))

    @property
    def extent(self) -> numpy.ndarray:
        return (self.shape * self.sampling).astype(numpy.float64)

    @classmethod
    def from_scan(cls, scan, sampling, pad=0.) -> 'ObjectSampling':
        """Grid covering the scan plus `pad` (object.py:246-255)."""
        sampling = numpy.asarray(sampling, numpy.float64)
        pad = numpy.broadcast_to(pad, (2,)).astype(numpy.float64)
        smin = numpy.array([float(numpy.nanmin(scan[..., i])) for i in range(2)])
        smax = numpy.array([float(numpy.nanmax(scan[..., i])) for i in range(2)])
        n = numpy.ceil((2. * pad + smax - smin) / sampling).astype(numpy.int_) + 1
        return cls((n[0], n[1]), sampling, smin - pad, smin, smax)

    def pos_to_object_idx(self, pos, cutout_shape) -> numpy.ndarray:
        """float64 index of a cutout's top-left pixel (object.py:291-301)."""
        half = -numpy.maximum(0., numpy.array(cutout_shape[-2:], numpy.float64) - 1.) / 2.
        return ((numpy.asarray(pos) - self.corner) / self.sampling + half).astype(numpy.float64)

    def cutout_starts(self, pos, cutout_shape) -> numpy.ndarray:
        return numpy.round(self.pos_to_object_idx(pos, cutout_shape)).astype(numpy.int64)

    def get_subpx_shifts(self, pos, cutout_shape) -> numpy.ndarray:
        idx = self.pos_to_object_idx(pos, cutout_shape)
        return (idx - numpy.round(idx)).astype(numpy.float64) * self.sampling

    def check_bounds(self, pad=0.) -> t.Tuple[numpy.ndarray, numpy.ndarray]:
        """(min, max) corner of the region in which probe positions overlap the object
        (object.py:277-289)."""
        pad = numpy.broadcast_to(pad, (2,)).astype(numpy.float64)
        return self.corner - pad, self.corner + self.extent + pad
