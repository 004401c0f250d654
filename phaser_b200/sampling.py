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

    @property
    def min(self) -> numpy.ndarray:
        return self.corner

    @property
    def max(self) -> numpy.ndarray:
        """Position of the last pixel (object.py:205-208)."""
        return (self.corner + (self.shape - 1) * self.sampling).astype(numpy.float64)

    def __eq__(self, other: t.Any) -> bool:
        """Same shape, sampling and corner (object.py:222-230)."""
        if type(self) is not type(other):
            return False
        return (numpy.array_equal(self.shape, other.shape) and numpy.array_equal(self.sampling, other.sampling)
                and numpy.array_equal(self.corner, other.corner))

    __hash__ = object.__hash__

    def with_sampling(self, sampling) -> 'ObjectSampling':
        """The grid at pixel size `sampling` covering at least this one, half the growth on
        each side (object.py:469-480)."""
        sampling = numpy.broadcast_to(numpy.asarray(sampling, numpy.float64), (2,))
        new_shape = numpy.ceil(self.sampling / sampling * self.shape).astype(int)
        growth = sampling * new_shape - self.sampling * self.shape
        if not numpy.all(growth / self.sampling >= -1e-4):
            raise ValueError("resampled object grid would shrink")
        return ObjectSampling(tuple(new_shape), sampling, self.corner - growth / 2. + (sampling - self.sampling) / 2.,
                              self.region_min, self.region_max)

    def expand_to_scan(self, scan, pad=0.) -> 'ObjectSampling':
        """This grid padded (whole pixels) to cover every scan position plus `pad`
        (object.py:257-275)."""
        pad = numpy.broadcast_to(pad, (2,)).astype(numpy.float64)
        smin = numpy.array([float(numpy.nanmin(scan[..., i])) for i in range(2)])
        smax = numpy.array([float(numpy.nanmax(scan[..., i])) for i in range(2)])
        pad_min = numpy.ceil(numpy.maximum(0, self.min - smin + pad) / self.sampling).astype(numpy.int_)
        pad_max = numpy.ceil(numpy.maximum(0, smax - self.max + pad) / self.sampling).astype(numpy.int_)
        if numpy.all(pad_min == 0) and numpy.all(pad_max == 0):
            return self
        rmin = numpy.minimum(self.region_min, smin) if self.region_min is not None else None
        rmax = numpy.maximum(self.region_max, smax) if self.region_max is not None else None
        return ObjectSampling(tuple(self.shape + pad_min + pad_max), self.sampling, self.corner - pad_min * self.sampling,
                              rmin, rmax)

    def check_bounds(self, pad=0.) -> t.Tuple[numpy.ndarray, numpy.ndarray]:
        """(min, max) corner of the region in which probe positions overlap the object
        (object.py:277-289)."""
        pad = numpy.broadcast_to(pad, (2,)).astype(numpy.float64)
        return self.corner - pad, self.corner + self.extent + pad
