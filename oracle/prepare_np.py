"""numpy restatement of the state preparation in front of the engines
(phaser.execute.prepare_for_engine) -- TEST INFRASTRUCTURE ONLY: only tests/
import this module.

Each function names the reference file:line whose behaviour it restates
(paths relative to the phaser source tree).  scipy.ndimage.affine_transform
(scipy 1.18, order 1, mode 'grid-constant') is restated for the diagonal
matrices the preparation uses: every output sample is the bilinear
interpolation, at coordinate (m_y * i + o_y, m_x * j + o_x), of the input
extended by the constant `cval` beyond its edges.  Coordinates and weights are
float64; values keep the input dtype's precision only at the end (as scipy
does, which interpolates in float64 and casts the result).
"""
from __future__ import annotations

import dataclasses
import typing as t

import numpy

from .phaser_np import hermite_modes


@dataclasses.dataclass
class ObjGrid:
    """ObjectSampling's fields (phaser/utils/object.py:188-230)."""
    shape: numpy.ndarray
    sampling: numpy.ndarray
    corner: numpy.ndarray
    region_min: t.Optional[numpy.ndarray] = None
    region_max: t.Optional[numpy.ndarray] = None

    def __post_init__(self):
        self.shape = numpy.broadcast_to(numpy.asarray(self.shape).astype(numpy.int64), (2,))
        self.sampling = numpy.broadcast_to(numpy.asarray(self.sampling, numpy.float64), (2,))
        self.corner = numpy.broadcast_to(numpy.asarray(self.corner, numpy.float64), (2,))

    @property
    def max(self):
        return self.corner + (self.shape - 1) * self.sampling

    def same(self, other: 'ObjGrid') -> bool:
        """ObjectSampling.__eq__ (object.py:222-230): shape, sampling and corner."""
        return (numpy.array_equal(self.shape, other.shape) and numpy.array_equal(self.sampling, other.sampling)
                and numpy.array_equal(self.corner, other.corner))


def affine_linear(arr: numpy.ndarray, matrix, offset, out_shape, cval) -> numpy.ndarray:
    """scipy.ndimage.affine_transform(arr, diag(matrix), offset, out_shape, order=1,
    mode='grid-constant', cval) over the last two axes (phaser/utils/image.py:151-195
    calls it once per leading index)."""
    H, W = arr.shape[-2:]
    m = numpy.broadcast_to(numpy.asarray(matrix, numpy.float64), (2,))
    o = numpy.broadcast_to(numpy.asarray(offset, numpy.float64), (2,))
    cy = numpy.arange(out_shape[0], dtype=numpy.float64) * m[0] + o[0]
    cx = numpy.arange(out_shape[1], dtype=numpy.float64) * m[1] + o[1]
    y0, x0 = numpy.floor(cy).astype(numpy.int64), numpy.floor(cx).astype(numpy.int64)
    ty, tx = cy - y0, cx - x0
    a = arr.astype(numpy.complex128 if numpy.iscomplexobj(arr) else numpy.float64)
    out = numpy.zeros((*arr.shape[:-2], out_shape[0], out_shape[1]), a.dtype)
    for dy, wy in ((0, 1.0 - ty), (1, ty)):
        for dx, wx in ((0, 1.0 - tx), (1, tx)):
            yy, xx = y0 + dy, x0 + dx
            vy, vx = (yy >= 0) & (yy < H), (xx >= 0) & (xx < W)
            v = a[..., numpy.clip(yy, 0, H - 1)[:, None], numpy.clip(xx, 0, W - 1)[None, :]]
            v = numpy.where(vy[:, None] & vx[None, :], v, cval)
            out += (wy[:, None] * wx[None, :]) * v
    return out.astype(arr.dtype)


def resample(arr, old_shape, old_sampling, new_shape, new_sampling, cval=0.0):
    """Sampling.resample without rotation (phaser/utils/num.py:713-733): centres aligned."""
    old_shape, new_shape = numpy.asarray(old_shape, numpy.float64), numpy.asarray(new_shape, numpy.float64)
    matrix = numpy.asarray(new_sampling, numpy.float64) / numpy.asarray(old_sampling, numpy.float64)
    offset = ((old_shape - 1) - matrix * (new_shape - 1)) / 2.
    return affine_linear(arr, matrix, offset, tuple(int(v) for v in new_shape), cval)


def resample_recip(arr, old_shape, old_sampling, new_shape, new_sampling):
    """Sampling.resample_recip (num.py:735-750): the reciprocal grids (extent k_max)
    resampled like real space between fftshift and ifftshift."""
    old_shape, new_shape = numpy.asarray(old_shape), numpy.asarray(new_shape)
    k_old = 1. / (2. * numpy.asarray(old_sampling, numpy.float64))
    k_new = 1. / (2. * numpy.asarray(new_sampling, numpy.float64))
    a = numpy.fft.fftshift(arr, axes=(-1, -2))
    r = resample(a, old_shape, k_old / old_shape, new_shape, k_new / new_shape)
    return numpy.fft.ifftshift(r, axes=(-1, -2))


def with_sampling(g: ObjGrid, sampling) -> ObjGrid:
    """ObjectSampling.with_sampling (object.py:469-480)."""
    sampling = numpy.broadcast_to(numpy.asarray(sampling, numpy.float64), (2,))
    new_shape = numpy.ceil(g.sampling / sampling * g.shape).astype(int)
    growth = sampling * new_shape - g.sampling * g.shape
    assert numpy.all(growth / g.sampling >= -1e-4)
    return ObjGrid(new_shape, sampling, g.corner - growth / 2. + (sampling - g.sampling) / 2.,
                   g.region_min, g.region_max)


def expand_to_scan(g: ObjGrid, scan, pad) -> ObjGrid:
    """ObjectSampling.expand_to_scan (object.py:257-275)."""
    pad = numpy.broadcast_to(pad, (2,)).astype(numpy.float64)
    smin = numpy.array([float(numpy.nanmin(scan[..., i])) for i in range(2)])
    smax = numpy.array([float(numpy.nanmax(scan[..., i])) for i in range(2)])
    pad_min = numpy.ceil(numpy.maximum(0, g.corner - smin + pad) / g.sampling).astype(int)
    pad_max = numpy.ceil(numpy.maximum(0, smax - g.max + pad) / g.sampling).astype(int)
    if numpy.all(pad_min == 0) and numpy.all(pad_max == 0):
        return g
    rmin = numpy.minimum(g.region_min, smin) if g.region_min is not None else None
    rmax = numpy.maximum(g.region_max, smax) if g.region_max is not None else None
    return ObjGrid(g.shape + pad_min + pad_max, g.sampling, g.corner - pad_min * g.sampling, rmin, rmax)


def object_resample(arr, old: ObjGrid, new: ObjGrid, cval=1.0):
    """ObjectSampling.resample without rotation / affine (object.py:430-467): corners
    aligned, objects extended by transmission 1."""
    matrix = new.sampling / old.sampling
    offset = (new.corner - old.corner) / old.sampling
    return affine_linear(arr, matrix, offset, tuple(int(v) for v in new.shape), cval)


def interp1d(arr, old_zs, new_zs):
    """_interp1d (object.py:160-185): linear along axis 0, edge values outside."""
    slice_is = numpy.searchsorted(old_zs, new_zs) - 1
    delta = numpy.diff(old_zs)
    rdt = numpy.float32 if arr.dtype == numpy.complex64 else numpy.float64
    out = numpy.empty((len(new_zs), *arr.shape[1:]), arr.dtype)
    for i, z in enumerate(new_zs):
        if z <= old_zs[0]:
            out[i] = arr[0]
        elif old_zs[-1] <= z:
            out[i] = arr[-1]
        else:
            j = slice_is[i]
            tt = rdt((z - old_zs[j]) / delta[j])
            out[i] = ((1 - tt) * arr[j] + tt * arr[j + 1]).astype(arr.dtype)
    return out


def resample_slices(obj, old_t, new_t, align: str = 'middle', pad_mode: str = 'vacuum'):
    """resample_slices (object.py:56-157) without rescale_projected: interpolation of
    log(obj) / thickness along z at the new slice centres, times the new thickness."""
    old_t = numpy.asarray(old_t, numpy.float64)
    new_t = numpy.asarray(new_t, numpy.float64)
    if len(new_t) < 2:
        return obj if obj.shape[0] == 1 else numpy.prod(obj, axis=0, keepdims=True)
    if obj.shape[0] == 1:
        frac = (new_t / numpy.sum(new_t))[:, None, None]
        return numpy.exp((numpy.log(obj) * frac).astype(obj.dtype))
    old_zs = numpy.cumsum(old_t) - old_t / 2.
    new_zs = numpy.cumsum(new_t) - new_t / 2.
    if align == 'bottom':
        new_zs += numpy.sum(old_t) - numpy.sum(new_t)
    elif align == 'middle':
        new_zs += (numpy.sum(old_t) - numpy.sum(new_t)) / 2.
    lg = (numpy.log(obj) / old_t[:, None, None]).astype(obj.dtype)
    if pad_mode == 'edge':
        before, after = lg[0], lg[-1]
    elif pad_mode == 'average':
        before = after = numpy.nanmean(lg, axis=0)
    else:
        before = after = numpy.zeros_like(lg[0])
    old_zs = numpy.concatenate(([old_zs[0] - old_t[0]], old_zs, [old_zs[-1] + old_t[-1]]))
    lg = numpy.concatenate((before[None], lg, after[None]), axis=0)
    new = interp1d(lg, old_zs, new_zs)
    new *= new_t[:, None, None]
    return numpy.exp(new.astype(obj.dtype))


def prepare_for_engine(patterns, mask, probe, probe_sampling, obj, grid: ObjGrid, thicknesses, scan, *,
                       sim_shape=None, resize_method='pad_crop', probe_modes=1, base_mode_power=0.7,
                       obj_pad_px=5.0, slices=None):
    """phaser.execute.prepare_for_engine (execute.py:334-402) for one plan.  Returns
    (patterns, mask, probe, probe_sampling, obj, grid, thicknesses)."""
    N = numpy.asarray(probe.shape[-2:])
    psamp = numpy.asarray(probe_sampling, numpy.float64)
    if sim_shape is not None and tuple(sim_shape) != tuple(N):
        new_shape = numpy.asarray(sim_shape)
        new_samp = (psamp * N / new_shape) if resize_method == 'pad_crop' else psamp
        probe = resample(probe, N, psamp, new_shape, new_samp)
        patterns = resample_recip(patterns, N, psamp, new_shape, new_samp)
        mask = resample_recip(mask, N, psamp, new_shape, new_samp)
        N, psamp = new_shape, new_samp
    g = grid
    if not numpy.allclose(psamp, grid.sampling):
        g = with_sampling(g, psamp)
    g2 = expand_to_scan(g, scan, psamp * N / 2. + obj_pad_px * psamp)
    if not g2.same(g):
        g = g2
    if not g.same(grid):
        obj = object_resample(obj, grid, g)
    if probe_modes != probe.shape[0]:
        if probe_modes < probe.shape[0]:
            probe = probe[:probe_modes]
        else:
            probe = hermite_modes(numpy.sum(probe, axis=0), probe_modes, base_mode_power)
    if slices is not None and (len(slices) != len(thicknesses) or not numpy.allclose(slices, thicknesses)):
        obj = resample_slices(obj, thicknesses, slices)
        thicknesses = numpy.asarray(slices, dtype=numpy.asarray(thicknesses).dtype)
    return patterns, mask, probe, psamp, obj, g, thicknesses
