"""numpy restatement of phaser's multislice hot path -- TEST INFRASTRUCTURE ONLY.

Every function names the reference file:line whose behaviour it restates
(paths relative to the phaser source tree).  Arrays follow the reference's
layouts: probe (M, N, N) complex, object (S, H, W) complex, scan (P, 2) (y, x)
in length units, patterns (P, N, N) float with the zero frequency in the
corner.  All arithmetic is done in the dtype of the inputs, as the reference
does (complex64/float32 for the usual float32 plans, complex128 for the FP64
oracle).

FFT backend: `scipy.fft` (pocketfft, the same library numpy uses) so that the
CPU baseline can use several host threads (`set_fft_workers`).
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import math
import typing as t

import numpy
import scipy.fft

_FFT_WORKERS = 1


def set_fft_workers(n: int) -> None:
    """Number of host threads used by the FFTs (1 = numpy's behaviour)."""
    global _FFT_WORKERS
    _FFT_WORKERS = max(1, int(n))


# ---------------------------------------------------------------- numerics core

def fft2c(a: numpy.ndarray) -> numpy.ndarray:
    """Forward FFT, centred real space, orthonormal (phaser/utils/num.py:460-468)."""
    a = numpy.asarray(a)
    return scipy.fft.fft2(numpy.fft.ifftshift(a, axes=(-2, -1)), norm='ortho',
                          workers=_FFT_WORKERS)


def ifft2c(a: numpy.ndarray) -> numpy.ndarray:
    """Inverse FFT back to centred real space, orthonormal (phaser/utils/num.py:434-442)."""
    a = numpy.asarray(a)
    return numpy.fft.fftshift(scipy.fft.ifft2(a, norm='ortho', workers=_FFT_WORKERS),
                              axes=(-2, -1))


def abs2(x: numpy.ndarray) -> numpy.ndarray:
    """|x|^2 as re^2 + im^2 (phaser/utils/num.py:505-512)."""
    x = numpy.asarray(x)
    return x.real ** 2. + x.imag ** 2.


def real_dtype(dtype) -> type:
    dt = numpy.dtype(dtype)
    return {numpy.dtype(numpy.complex64): numpy.float32,
            numpy.dtype(numpy.complex128): numpy.float64}.get(dt, dt.type)


def complex_dtype(dtype) -> type:
    dt = numpy.dtype(dtype)
    return {numpy.dtype(numpy.float32): numpy.complex64,
            numpy.dtype(numpy.float64): numpy.complex128}.get(dt, dt.type)


def recip_grid(shape: t.Tuple[int, int], sampling: t.Sequence[float], dtype=numpy.float32):
    """(ky, kx) meshgrid of fftfreq values, zero frequency in the corner
    (phaser/utils/num.py:651-670)."""
    fy = numpy.fft.fftfreq(int(shape[0]), float(sampling[0])).astype(dtype)
    fx = numpy.fft.fftfreq(int(shape[1]), float(sampling[1])).astype(dtype)
    ky, kx = numpy.meshgrid(fy, fx, indexing='ij')
    return ky, kx


# ---------------------------------------------------------------- cutouts (a1-a4)

def object_index(pos: numpy.ndarray, corner, sampling, cutout_shape) -> numpy.ndarray:
    """Fractional object index of a cutout's top-left pixel, float64
    (phaser/utils/object.py:291-301)."""
    pos = numpy.asarray(pos)
    half = -numpy.maximum(0., numpy.array(cutout_shape[-2:], dtype=numpy.float64) - 1.) / 2.
    return ((pos - numpy.asarray(corner, numpy.float64)) / numpy.asarray(sampling, numpy.float64)
            + half).astype(numpy.float64)


def cutout_starts(pos, corner, sampling, cutout_shape) -> numpy.ndarray:
    """Integer cutout starts: float64 index rounded half-to-even
    (phaser/utils/object.py:493-495)."""
    return numpy.round(object_index(pos, corner, sampling, cutout_shape)).astype(numpy.int64)


def subpx_shifts(pos, corner, sampling, cutout_shape) -> numpy.ndarray:
    """Residual between the position and its rounded cutout, in length units,
    float64 (phaser/utils/object.py:324-331)."""
    idx = object_index(pos, corner, sampling, cutout_shape)
    return (idx - numpy.round(idx)).astype(numpy.float64) * numpy.asarray(sampling, numpy.float64)


def get_cutouts(obj: numpy.ndarray, starts: numpy.ndarray, shape: t.Tuple[int, int],
                fill=1) -> numpy.ndarray:
    """Gather (B, *obj.shape[:-2], ny, nx) cutouts; out-of-bounds pixels read
    `fill` (the GPU semantics of phaser/utils/_cuda_kernels.py:51-75 as called
    from phaser/utils/object.py:501-519)."""
    obj = numpy.asarray(obj)
    starts = numpy.asarray(starts).reshape(-1, 2)
    ny, nx = shape
    H, W = obj.shape[-2:]
    out = numpy.full((starts.shape[0], *obj.shape[:-2], ny, nx), fill, dtype=obj.dtype)
    for b, (y0, x0) in enumerate(starts):
        ya, yb = max(0, y0), min(H, y0 + ny)
        xa, xb = max(0, x0), min(W, x0 + nx)
        if ya >= yb or xa >= xb:
            continue
        out[b, ..., ya - y0:yb - y0, xa - x0:xb - x0] = obj[..., ya:yb, xa:xb]
    return out


def add_cutouts(obj: numpy.ndarray, starts: numpy.ndarray, views: numpy.ndarray) -> numpy.ndarray:
    """In-place scatter-add of views (B, ..., ny, nx) at `starts`; pixels
    outside the object are dropped (phaser/utils/object.py:540-557,
    phaser/utils/_cuda_kernels.py:78-107)."""
    starts = numpy.asarray(starts).reshape(-1, 2)
    ny, nx = views.shape[-2:]
    H, W = obj.shape[-2:]
    for b, (y0, x0) in enumerate(starts):
        ya, yb = max(0, y0), min(H, y0 + ny)
        xa, xb = max(0, x0), min(W, x0 + nx)
        if ya >= yb or xa >= xb:
            continue
        obj[..., ya:yb, xa:xb] += views[b, ..., ya - y0:yb - y0, xa - x0:xb - x0]
    return obj


# ---------------------------------------------------------------- optics (a2, a6, a18)

def fourier_shift_filter(ky, kx, shifts) -> numpy.ndarray:
    """exp(-2 pi i (x kx + y ky)) per shift (phaser/utils/optics.py:151-170)."""
    shifts = numpy.asarray(shifts, dtype=ky.dtype)
    y, x = shifts[..., 0], shifts[..., 1]
    phase = numpy.multiply.outer(x, kx) + numpy.multiply.outer(y, ky)
    return numpy.exp(numpy.array(-2.j * numpy.pi, dtype=complex_dtype(ky.dtype)) * phase)


def fresnel_propagator(ky, kx, wavelength: float, delta_z: float, tilt=(0., 0.)) -> numpy.ndarray:
    """Fresnel free-space kernel (phaser/utils/optics.py:190-211)."""
    tx, ty = numpy.tan(tilt[0] * 1e-3), numpy.tan(tilt[1] * 1e-3)
    k2 = ky ** 2 + kx ** 2
    return numpy.exp(-1.j * numpy.pi * delta_z * (wavelength * k2 - 2. * (kx * tx + ky * ty))) \
        .astype(complex_dtype(k2.dtype))


def make_propagators(ky, kx, probe_sampling, wavelength: float, thicknesses,
                     bwlim_frac: t.Optional[float] = 2. / 3.) -> t.Optional[numpy.ndarray]:
    """One band-limited propagator per slice gap, (S-1, N, N)
    (phaser/engines/common/simulation.py:160-190).  Equal gaps share one
    propagator, keyed by the gap rounded to 5 decimals (misc.py:211-218)."""
    dzs = numpy.asarray(thicknesses)[:-1]
    if len(dzs) == 0:
        return None
    cdt = complex_dtype(ky.dtype)
    if bwlim_frac is not None:
        k_max = numpy.min(1. / (2. * numpy.asarray(probe_sampling, numpy.float64)))
        limit = k_max * bwlim_frac
        band = (ky ** 2 + kx ** 2) <= limit ** 2
    else:
        band = numpy.ones(ky.shape, dtype=bool)
    cache: t.Dict[float, numpy.ndarray] = {}
    out = []
    for dz in dzs:
        key = round(float(dz), 5)
        if key not in cache:
            cache[key] = fresnel_propagator(ky, kx, wavelength, float(dz)).astype(cdt) * band
        out.append(cache[key])
    return numpy.stack(out, axis=0)


def tilt_propagators(ky, kx, thicknesses, props, tilts):
    """Per-position tilted propagators (S-1, B, N, N); untilted -> (S-1, 1, N, N)
    (phaser/engines/common/simulation.py:193-222)."""
    if props is None:
        return None
    if tilts is None:
        return props[:, None]
    cdt = complex_dtype(ky.dtype)
    dzs = numpy.asarray(thicknesses)[:-1]
    tilts = numpy.asarray(tilts)
    inner = (numpy.multiply.outer(numpy.tan(tilts[..., 0] * 1e-3), ky)
             + numpy.multiply.outer(numpy.tan(tilts[..., 1] * 1e-3), kx))
    ramps = numpy.exp(2.j * numpy.pi * numpy.multiply.outer(dzs, inner))
    return props[:, None] * ramps.astype(cdt)


def make_focused_probe(ky, kx, wavelength: float, aperture_mrad: float, defocus: float = 0.):
    """Aperture-limited defocused probe, unit intensity (phaser/utils/optics.py:30-51)."""
    theta2 = (ky * wavelength) ** 2 + (kx * wavelength) ** 2
    probe = numpy.exp(-2.j * numpy.pi * (defocus / (2. * wavelength)) * theta2)
    probe = probe * (theta2 <= (aperture_mrad * 1e-3) ** 2)
    probe = probe / numpy.sqrt(numpy.sum(abs2(probe)))
    return ifft2c(probe)


def hermite_modes(base: numpy.ndarray, n_modes: int, base_mode_power: float = 0.7,
                  rel_powers=1.0) -> numpy.ndarray:
    """Orthonormal Hermite-Gauss modes from a base probe, Gram-Schmidt'ed in
    anti-diagonal order and scaled to the given powers
    (phaser/utils/optics.py:54-136)."""
    rdt = real_dtype(base.dtype)
    rel = numpy.array(rel_powers, dtype=rdt).ravel()
    rel = numpy.pad(rel, (0, n_modes - rel.size - 1), mode='edge')[:n_modes - 1]
    powers = numpy.concatenate([[base_mode_power], (1.0 - base_mode_power) * rel])
    i = numpy.arange(n_modes)
    diag = numpy.ceil((numpy.sqrt(8 * i + 9) - 3) / 2).astype(numpy.int64)
    xo = (i - diag * (diag + 1) / 2).astype(numpy.int64)
    yo = diag - xo
    yy, xx = numpy.indices(base.shape, dtype=rdt)
    mag = abs2(base)
    cy = numpy.sum(yy * mag) / numpy.sum(mag)
    cx = numpy.sum(xx * mag) / numpy.sum(mag)
    yy = yy - cy
    xx = xx - cx
    modes = numpy.empty((n_modes, *base.shape), dtype=base.dtype)
    for k in range(n_modes):
        mode = yy ** yo[k] * xx ** xo[k] * base
        for p in range(k):
            mode = mode - modes[p] * numpy.sum(modes[p] * numpy.conj(mode))
        modes[k] = mode / numpy.sqrt(numpy.sum(abs2(mode)))
    return modes * numpy.sqrt(powers)[:, None, None].astype(modes.dtype)


def raster_scan(shape: t.Tuple[int, int], step, dtype=numpy.float64) -> numpy.ndarray:
    """(ny, nx, 2) raster around the origin (phaser/utils/scan.py:23-55)."""
    yy = numpy.arange(shape[0], dtype=dtype) - numpy.array(shape[0] / 2., dtype=dtype)
    xx = numpy.arange(shape[1], dtype=dtype) - numpy.array(shape[1] / 2., dtype=dtype)
    pts = numpy.stack(numpy.meshgrid(yy, xx, indexing='ij'), axis=-1)
    return pts * numpy.broadcast_to(numpy.array(step), (2,)).astype(dtype)


def electron_wavelength(energy_ev: float) -> float:
    """Relativistic electron wavelength in angstrom (phaser/utils/physics.py:59-62)."""
    rest = 5.1099906e5
    hc = 1.23984244e4
    return hc / math.sqrt(energy_ev * (2 * rest + energy_ev))


# ---------------------------------------------------------------- seeded groupings (a15)

def create_rng(seed: t.Any, entropy: t.Any = None) -> numpy.random.Generator:
    """PCG64 seeded by sha256(json(seed) || json(entropy)) (phaser/utils/misc.py:14-56)."""
    if seed is None:
        return numpy.random.Generator(numpy.random.PCG64(numpy.random.SeedSequence()))
    h = hashlib.sha256()
    h.update(json.dumps(seed).encode('utf-8'))
    if entropy is not None:
        h.update(json.dumps(entropy).encode('utf-8'))
    seq = numpy.random.SeedSequence(numpy.frombuffer(h.digest(), dtype=numpy.uint32))
    return numpy.random.Generator(numpy.random.PCG64(seq))


def sparse_groupings(scan_shape: t.Tuple[int, ...], max_grouping: int, seed: t.Any, i: int = 0):
    """Randomly shuffled index grid split into near-equal groups
    (phaser/utils/misc.py:96-115)."""
    idxs = numpy.indices(scan_shape)
    idxs = idxs.reshape(idxs.shape[0], -1).T
    rng = create_rng(seed, f'groupings_{i}' if i != 0 else 'groupings')
    rng.shuffle(idxs)
    return numpy.array_split(idxs.T, numpy.ceil(idxs.shape[0] / max_grouping).astype(numpy.int64), axis=-1)


def shuffled_order(n: int, seed: t.Any, i: int) -> numpy.ndarray:
    """Order in which existing groups are visited (phaser/utils/misc.py:84-93)."""
    order = numpy.arange(n)
    create_rng(seed, f"shuffle_{i}").shuffle(order)
    return order


def mask_fraction_of_groups(n_groups: int, fraction: float) -> numpy.ndarray:
    """Every k-th group computes the error (phaser/utils/misc.py:199-208)."""
    need = max(1, math.ceil(n_groups * fraction))
    if need >= n_groups:
        return numpy.ones(n_groups, dtype=bool)
    mask = numpy.zeros(n_groups, dtype=bool)
    mask[::n_groups // need] = True
    return mask


# ---------------------------------------------------------------- noise models (a8)

@dataclasses.dataclass
class NoiseModel:
    """'amplitude' / 'anscombe' / 'poisson' with the plan defaults
    (phaser/plan.py:86-99, phaser/engines/common/noise_models.py:13-112)."""
    kind: str = 'amplitude'
    eps: float = 1.0e-3
    offset: float = 0.0
    gaussian_variance: float = 0.1

    @classmethod
    def anscombe(cls, **kw) -> 'NoiseModel':
        kw.setdefault('offset', 0.375)
        return cls(kind='anscombe', **kw)

    def wave_update(self, wave, intensity, patterns, mask):
        """chi_F = mask * (sqrt(max(I_exp,0)+c) / (sqrt(I+c)+eps) - 1) * Psi
        (noise_models.py:47-64).  Poisson has no wave update (104-112)."""
        if self.kind == 'poisson':
            raise NotImplementedError("the Poisson noise model has no wave update")
        pat = numpy.maximum(patterns, 0.0)
        u = numpy.sqrt(pat + self.offset) / (numpy.sqrt(intensity + self.offset) + self.eps) - 1.0
        u = u * mask
        return u * wave

    def loss(self, intensity, patterns, mask):
        """Summed loss (noise_models.py:29-45 amplitude/anscombe, 86-102 Poisson)."""
        pat = numpy.maximum(patterns, 0.0)
        if self.kind == 'poisson':
            val = numpy.sum(mask * (intensity + self.eps + pat * (
                numpy.log(pat + self.eps) - numpy.log(intensity + self.eps) - 1.0)))
        else:
            var = 1. + self.gaussian_variance
            val = 2. * numpy.sum(mask * (numpy.sqrt(pat + self.offset)
                                         - numpy.sqrt(intensity + self.offset) - self.eps) ** 2) / var
        return val.astype(patterns.dtype)


# ---------------------------------------------------------------- per-group model

@dataclasses.dataclass
class Geometry:
    """What a group step needs to know about the reconstruction: object
    sampling (corner, sampling), probe recip grid, slice gaps and wavelength."""
    corner: numpy.ndarray          # (2,) float64
    obj_sampling: numpy.ndarray    # (2,) float64
    ky: numpy.ndarray              # (N, N) real
    kx: numpy.ndarray
    thicknesses: numpy.ndarray     # (S,) or empty


def cutout_group(geom: Geometry, probe, obj, group_scan):
    """Subpixel-shifted probes (B, M, N, N), object cutouts (B, S, N, N) and the
    shift filters (B, 1, N, N) (phaser/engines/common/simulation.py:241-260)."""
    shape = probe.shape[-2:]
    starts = cutout_starts(group_scan, geom.corner, geom.obj_sampling, shape)
    cuts = get_cutouts(obj, starts, shape, fill=1)
    shifts = subpx_shifts(group_scan, geom.corner, geom.obj_sampling, shape)
    filt = fourier_shift_filter(geom.ky, geom.kx, shifts)[:, None]
    psi0 = ifft2c(fft2c(probe) * filt)
    return psi0, cuts, starts, filt


def _forward(psi0, cuts, props_t, on_slice=None):
    """Run the multislice forward; returns the per-slice incident waves
    (S, B, M, N, N) (simulation.py:263-285 ordering)."""
    S = cuts.shape[1]
    psi = numpy.zeros((S, *psi0.shape), dtype=psi0.dtype)
    psi[0] = psi0
    for s in range(S):
        if on_slice is not None:
            on_slice(s, psi[s])
        if s < S - 1:
            psi[s + 1] = ifft2c(fft2c(psi[s] * cuts[:, s, None]) * props_t[s][:, None])
    return psi


def lsqml_dry_run(geom, probe, obj, group_scan, patterns, mask, props, tilts,
                  obj_mag, probe_mag):
    """Presolve pass (phaser/engines/conventional/solvers.py:132-167): returns
    updated obj_mag, probe_mag and per-position intensity rescale factors.
    Note the model intensity is taken from the LAST incident wave, before the
    last slice's transmission."""
    psi0, cuts, starts, _ = cutout_group(geom, probe, obj, group_scan)
    obj_mag = obj_mag + numpy.sum(abs2(numpy.prod(cuts, axis=1)), axis=0)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)
    probe_mag = probe_mag.copy()

    def illum(s, p):
        add_cutouts(probe_mag[s], starts, numpy.sum(abs2(p), axis=1))

    psi = _forward(psi0, cuts, props_t, illum)
    model_int = numpy.sum(abs2(fft2c(psi[-1])), axis=(1, -2, -1))
    exp_int = numpy.sum(patterns * mask, axis=(-2, -1))
    return obj_mag, probe_mag, exp_int / model_int


def epie_dry_run(geom, probe, obj, group_scan, patterns, mask, props, tilts):
    """ePIE presolve pass (phaser/engines/conventional/solvers.py:387-412)."""
    psi0, cuts, _, _ = cutout_group(geom, probe, obj, group_scan)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)
    psi = _forward(psi0, cuts, props_t)
    model_int = numpy.sum(abs2(fft2c(psi[-1])), axis=(1, -2, -1))
    exp_int = numpy.sum(patterns * mask, axis=(-2, -1))
    return exp_int / model_int


def _position_step(geom, psi0, cuts, chi):
    """Per-position (dy, dx) step from the probe-shift derivative
    (phaser/engines/conventional/solvers.py:275-288 and 489-502)."""
    pf = fft2c(psi0)
    pf = pf / numpy.sum(abs2(psi0), axis=(1, -1, -2), keepdims=True)
    out = []
    for k in (geom.ky, geom.kx):
        d = ifft2c(pf * -2.j * numpy.pi * k)
        prod = d * cuts[:, 0, None]
        out.append(numpy.sum(numpy.real(chi * numpy.conj(prod)), axis=(1, -1, -2))
                   / numpy.sum(abs2(prod)))
    return numpy.stack(out, axis=-1)


@dataclasses.dataclass
class LSQMLParams:
    """LSQ-ML step parameters (phaser/plan.py:105-114 defaults)."""
    beta_object: float = 1.0
    beta_probe: float = 1.0
    illum_reg_object: float = 1e-2
    illum_reg_probe: float = 1e-2
    gamma: float = 1e-4


def lsqml_group(geom, probe, obj, group_scan, patterns, mask, props, tilts,
                noise: NoiseModel, params: LSQMLParams, *, update_object=True,
                update_probe=True, update_position=True, calc_error=True):
    """One LSQ-ML mini-batch (phaser/engines/conventional/solvers.py:171-290).

    Returns a dict with the updated `object` and `probe` (new arrays), the
    group illumination `probe_mag` (S, H, W) and `obj_mag` (N, N) that the
    solver accumulates, per-position `errors` and `pos_update` (B, 2)."""
    obj = obj.copy()
    probe = probe.copy()
    S = obj.shape[0]
    eps = 1e-16
    psi0, cuts, starts, filt = cutout_group(geom, probe, obj, group_scan)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)

    gpm = numpy.zeros(obj.shape, dtype=real_dtype(obj.dtype))
    gom = numpy.sum(abs2(numpy.prod(cuts, axis=1)), axis=0)

    def illum(s, p):
        add_cutouts(gpm[s], starts, numpy.sum(abs2(p), axis=1))

    psi = _forward(psi0, cuts, props_t, illum)

    wave = fft2c(psi[-1] * cuts[:, -1, None])
    intensity = numpy.sum(abs2(wave), axis=1, keepdims=True)
    pats = patterns[:, None]
    errors = (numpy.sqrt(numpy.nansum((intensity - pats) ** 2, axis=(1, -1, -2)))
              if calc_error else None)
    chi = ifft2c(noise.wave_update(wave, intensity, pats, mask))

    for s in range(S - 1, -1, -1):
        o = cuts[:, s, None]
        dP = chi * numpy.conj(o)
        if update_object:
            dO = chi * numpy.conj(psi[s])
            num = numpy.sum(numpy.sum(numpy.real(chi * numpy.conj(dO * psi[s])),
                                      axis=(-1, -2), keepdims=True), axis=1)
            alpha_o = num / (numpy.sum(abs2(dO * psi[s])) + params.gamma)
            avg = numpy.zeros_like(obj[0])
            add_cutouts(avg, starts, numpy.sum(dO, axis=1))
            avg = avg / (gpm[s] + params.illum_reg_object)
            upd = params.beta_object * numpy.sum(alpha_o * avg * gpm[s], axis=0) / (gpm[s] + eps)
            obj[s] = obj[s] + upd
        if s > 0:
            chi = ifft2c(fft2c(dP) * numpy.conj(props_t[s - 1])[:, None])
        elif update_probe:
            avg_p = ifft2c(numpy.sum(fft2c(dP) * numpy.conj(filt), axis=0))
            avg_p = avg_p / (gom + params.illum_reg_probe)
            proj = dP * o
            alpha_p = (numpy.sum(numpy.real(chi * numpy.conj(proj)), axis=(-1, -2), keepdims=True)
                       / (numpy.sum(abs2(proj)) + params.gamma))
            probe = probe + params.beta_probe * numpy.sum(alpha_p * avg_p * gom, axis=0) / (gom + eps)

    pos_update = _position_step(geom, psi0, cuts, chi) if update_position else None
    return dict(object=obj, probe=probe, probe_mag=gpm, obj_mag=gom,
                errors=errors, pos_update=pos_update)


@dataclasses.dataclass
class EPIEParams:
    """ePIE step parameters (phaser/plan.py:117-119 defaults)."""
    beta_object: float = 1.0
    beta_probe: float = 1.0


def epie_group(geom, probe, obj, group_scan, patterns, mask, props, tilts,
               noise: NoiseModel, params: EPIEParams, *, update_object=True,
               update_probe=True, update_position=True, calc_error=True):
    """One ePIE / 3PIE mini-batch (phaser/engines/conventional/solvers.py:415-504)."""
    obj = obj.copy()
    probe = probe.copy()
    S = obj.shape[0]
    psi0, cuts, starts, filt = cutout_group(geom, probe, obj, group_scan)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)
    psi = _forward(psi0, cuts, props_t)

    wave = fft2c(psi[-1] * cuts[:, -1, None])
    intensity = numpy.sum(abs2(wave), axis=1, keepdims=True)
    pats = patterns[:, None]
    errors = (numpy.sqrt(numpy.nansum((intensity - pats) ** 2, axis=(1, -1, -2)))
              if calc_error else None)
    chi = ifft2c(noise.wave_update(wave, intensity, pats, mask))

    for s in range(S - 1, -1, -1):
        o = cuts[:, s, None]
        dP = numpy.conj(o) * chi / numpy.max(abs2(o), axis=(-1, -2), keepdims=True)
        if update_object:
            w = numpy.max(numpy.sum(abs2(psi[s]), axis=1), axis=(-1, -2), keepdims=True)
            view = params.beta_object / S * numpy.sum(numpy.conj(psi[s]) * chi, axis=1) / w
            add_cutouts(obj[s], starts, view)
        if s > 0:
            chi = ifft2c(fft2c(dP) * numpy.conj(props_t[s - 1])[:, None])
        elif update_probe:
            probe = probe + params.beta_probe * ifft2c(numpy.mean(fft2c(dP) * numpy.conj(filt), axis=0))

    pos_update = _position_step(geom, psi0, cuts, chi) if update_position else None
    return dict(object=obj, probe=probe, errors=errors, pos_update=pos_update)


# ---------------------------------------------------------------- gradient-engine model (a14)

def grad_model_loss(geom, probe, obj, group_scan, patterns, mask, props, tilts,
                    noise: NoiseModel) -> float:
    """Forward loss of the gradient engine (phaser/engines/gradient/run.py:357-405)
    without cost regularisers: the last slice transmits but does not propagate."""
    psi0, cuts, _, _ = cutout_group(geom, probe, obj, group_scan)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)
    psi = _forward(psi0, cuts, props_t)
    wave = fft2c(psi[-1] * cuts[:, -1, None])
    intensity = numpy.sum(abs2(wave), axis=1)
    return noise.loss(intensity, patterns, mask)


def grad_dry_run(geom, probe, obj, group_scan, patterns, props, tilts):
    """Gradient-engine rescale pass (phaser/engines/gradient/run.py:413-438):
    includes the last slice's transmission and uses unmasked pattern sums."""
    psi0, cuts, _, _ = cutout_group(geom, probe, obj, group_scan)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)
    psi = _forward(psi0, cuts, props_t)
    wave = fft2c(psi[-1] * cuts[:, -1, None])
    return numpy.sum(patterns, axis=(-2, -1)) / numpy.sum(abs2(wave), axis=(1, -2, -1))


# ---------------------------------------------------------------- position solvers

def steepest_descent_step(grad, step_size: float, max_step: t.Optional[float]):
    """(phaser/engines/common/position_correction.py:13-34; note the reference
    sets max_step_size = step_size, line 16)."""
    upd = step_size * grad
    if max_step is not None:
        mag = numpy.linalg.norm(upd, axis=-1, keepdims=True)
        upd = upd * (numpy.minimum(mag, max_step) / mag)
    return upd


def momentum_step(grad, state, step_size: float, max_step: t.Optional[float], momentum: float):
    """(phaser/engines/common/position_correction.py:37-61).  Returns (update, new_state)."""
    upd = step_size * grad + momentum * state
    if max_step is not None:
        mag = numpy.linalg.norm(upd, axis=-1, keepdims=True)
        upd = upd * (numpy.minimum(mag, max_step) / mag)
    return upd, upd


# ---------------------------------------------------------------- engine loop (a16)

@dataclasses.dataclass
class ConventionalRun:
    """Inputs and knobs of one conventional-engine run (the fields of
    ConventionalEnginePlan that the hot path reads, phaser/plan.py:43-132)."""
    solver: str = 'lsqml'                         # 'lsqml' | 'epie'
    niter: int = 2
    grouping: int = 64
    seed: t.Any = 'seed'
    lsqml: LSQMLParams = dataclasses.field(default_factory=LSQMLParams)
    epie: EPIEParams = dataclasses.field(default_factory=EPIEParams)
    noise: NoiseModel = dataclasses.field(default_factory=NoiseModel)
    update_object: bool = True
    update_probe: bool = True
    update_positions: bool = False
    position_solver: t.Optional[str] = None       # 'momentum' | 'steepest_descent'
    pos_step_size: float = 1e-2
    pos_max_step: t.Optional[float] = None
    pos_momentum: float = 0.9
    calc_error_fraction: float = 0.1
    bwlim_frac: t.Optional[float] = 2. / 3.


def run_conventional(run: ConventionalRun, *, probe, obj, scan, patterns, mask,
                     probe_sampling, corner, obj_sampling, thicknesses, wavelength,
                     tilt=None, iteration_callback=None):
    """Presolve + `niter` iterations of LSQ-ML or ePIE with sparse (shuffled)
    groupings (phaser/engines/conventional/run.py:15-123 with
    solvers.py:36-128 / 306-383).  Returns (probe, object, scan, errors)."""
    probe = probe.copy()
    obj = obj.copy()
    scan = scan.copy()
    rdt = real_dtype(probe.dtype)
    N = probe.shape[-1]
    ky, kx = recip_grid(probe.shape[-2:], probe_sampling, dtype=rdt)
    geom = Geometry(numpy.asarray(corner, numpy.float64), numpy.asarray(obj_sampling, numpy.float64),
                    ky, kx, numpy.asarray(thicknesses))
    props = make_propagators(ky, kx, probe_sampling, wavelength, thicknesses, run.bwlim_frac)
    scan_shape = scan.shape[:-1]
    flat_scan = scan.reshape(-1, 2)
    flat_pat = patterns.reshape(-1, N, N)
    flat_tilt = None if tilt is None else tilt.reshape(-1, 2)

    def groups_for(i, shuffle):
        return sparse_groupings(scan_shape, run.grouping, run.seed, i)

    def flat(g):
        return numpy.ravel_multi_index(tuple(g), scan_shape)

    # presolve: probe intensity rescale (solvers.py:36-63, 306-329)
    groups = groups_for(0, True)
    factors = []
    obj_mag = numpy.zeros(probe.shape[-2:], dtype=rdt)
    probe_mag = numpy.zeros(obj.shape, dtype=rdt)
    for g in groups:
        idx = flat(g)
        tl = None if flat_tilt is None else flat_tilt[idx]
        if run.solver == 'lsqml':
            obj_mag, probe_mag, f = lsqml_dry_run(geom, probe, obj, flat_scan[idx], flat_pat[idx], mask,
                                                  props, tl, obj_mag, probe_mag)
        else:
            f = epie_dry_run(geom, probe, obj, flat_scan[idx], flat_pat[idx], mask, props, tl)
        factors.append(f)
    rescale = numpy.mean(numpy.concatenate(factors))
    probe = probe * numpy.sqrt(rescale)

    calc_mask = mask_fraction_of_groups(len(groups), run.calc_error_fraction)
    pos_state = numpy.zeros_like(flat_scan)
    errors_out = []
    for it in range(1, run.niter + 1):
        groups = groups_for(it, True)
        pos_update = numpy.zeros_like(flat_scan)
        errs = []
        for gi, g in enumerate(groups):
            idx = flat(g)
            tl = None if flat_tilt is None else flat_tilt[idx]
            kw = dict(update_object=run.update_object, update_probe=run.update_probe,
                      update_position=run.update_positions, calc_error=bool(calc_mask[gi]))
            if run.solver == 'lsqml':
                res = lsqml_group(geom, probe, obj, flat_scan[idx], flat_pat[idx], mask, props, tl,
                                  run.noise, run.lsqml, **kw)
            else:
                res = epie_group(geom, probe, obj, flat_scan[idx], flat_pat[idx], mask, props, tl,
                                 run.noise, run.epie, **kw)
            obj, probe = res['object'], res['probe']
            if not (numpy.all(numpy.isfinite(obj)) and numpy.all(numpy.isfinite(probe))):
                raise ValueError(f"NaN or inf encountered in object or probe, group {gi}")
            if run.update_positions:
                pos_update[idx] = res['pos_update']
            if calc_mask[gi]:
                errs.append(res['errors'])
        if run.update_positions:
            pos_update = pos_update - numpy.mean(pos_update, axis=0)
            if run.position_solver == 'momentum':
                pos_update, pos_state = momentum_step(pos_update, pos_state, run.pos_step_size,
                                                      run.pos_max_step, run.pos_momentum)
            else:
                pos_update = steepest_descent_step(pos_update, run.pos_step_size, run.pos_step_size)
            # in place, as run.py:106 does: with the numpy backend the momentum
            # state IS this array, so it also loses the mean
            pos_update -= numpy.mean(pos_update, axis=0)
            flat_scan = flat_scan + pos_update
        err = float(numpy.nanmean(numpy.concatenate(errs))) if errs else float('nan')
        errors_out.append(err)
        if iteration_callback is not None:
            iteration_callback(it, probe, obj, flat_scan.reshape(scan.shape), err)
    return probe, obj, flat_scan.reshape(scan.shape), numpy.array(errors_out)


def noise_dloss_dI(noise: NoiseModel, intensity, patterns, mask):
    """dL/dI of NoiseModel.loss (noise_models.py:29-45 amplitude/anscombe, 86-102 Poisson)."""
    pat = numpy.maximum(patterns, 0.0)
    if noise.kind == 'poisson':
        return mask * (1.0 - pat / (intensity + noise.eps))
    var = 1. + noise.gaussian_variance
    sI = numpy.sqrt(intensity + noise.offset)
    return -2. * mask * (numpy.sqrt(pat + noise.offset) - sI - noise.eps) / (var * sI)


def grad_model_grads(geom, probe, obj, group_scan, patterns, mask, props, tilts, noise: NoiseModel,
                     with_tilt: bool = False):
    """Loss and gradients of the gradient-engine model (the adjoint of
    phaser/engines/gradient/run.py:357-405 that jax.value_and_grad evaluates).

    Complex gradients are returned as g = dL/dRe + i dL/dIm; phaser's update
    direction -conj(jax_grad) (run.py:325) equals -g.  Position gradients are
    dL/d(y, x) through the sub-pixel shift filter (the integer cutout start has no
    gradient).  Returns (loss, g_object (S,H,W), g_probe (M,N,N), g_pos (B,2))."""
    S = obj.shape[0]
    shape = probe.shape[-2:]
    psi0, cuts, starts, filt = cutout_group(geom, probe, obj, group_scan)
    props_t = tilt_propagators(geom.ky, geom.kx, geom.thicknesses, props, tilts)
    psi = _forward(psi0, cuts, props_t)
    wave = fft2c(psi[-1] * cuts[:, -1, None])
    intensity = numpy.sum(abs2(wave), axis=1)
    loss = noise.loss(intensity, patterns, mask)
    g_wave = 2. * noise_dloss_dI(noise, intensity, patterns, mask)[:, None] * wave
    g = ifft2c(g_wave)
    g_obj = numpy.zeros_like(obj)
    g_tilt = numpy.zeros((len(group_scan), 2))
    for s in range(S - 1, -1, -1):
        add_cutouts(g_obj[s], starts, numpy.sum(g * numpy.conj(psi[s]), axis=1))
        g = g * numpy.conj(cuts[:, s, None])
        if s > 0:
            G = fft2c(g)
            if with_tilt and tilts is not None:
                # psi_s = ifft2c(fft2c(psi_{s-1} O_{s-1}) P_{s-1} T), dT/dtheta = T 2 pi i dz k (1 + tan^2) 1e-3
                Y = fft2c(psi[s])
                dz = float(geom.thicknesses[s - 1])
                for j, k in enumerate((geom.ky, geom.kx)):
                    d = numpy.real(numpy.conj(G) * Y * (2j * numpy.pi * dz * k))
                    sec2 = 1.0 + numpy.tan(tilts[:, j] * 1e-3) ** 2
                    g_tilt[:, j] += numpy.sum(d, axis=(1, -1, -2)) * sec2 * 1e-3
            g = ifft2c(G * numpy.conj(props_t[s - 1])[:, None])
    g_probe = ifft2c(numpy.sum(fft2c(g) * numpy.conj(filt), axis=0))
    pf = fft2c(probe)[None] * filt
    g_pos = []
    for k in (geom.ky, geom.kx):
        d = ifft2c(pf * -2.j * numpy.pi * k)
        g_pos.append(numpy.sum(numpy.real(numpy.conj(g) * d), axis=(1, -1, -2)))
    if with_tilt:
        return loss, g_obj, g_probe, numpy.stack(g_pos, axis=-1), g_tilt
    return loss, g_obj, g_probe, numpy.stack(g_pos, axis=-1)


# ---------------------------------------------------------------- gradient engine (a14)

class OptaxNP:
    """The optax chains of phaser/engines/gradient/solvers.py:88-138 restated in
    numpy (optax is a third-party dependency of the reference; its published
    update rules are restated here):

    - 'sgd'        optax.trace(momentum, nesterov) then scale_by_learning_rate(lr,
                   flip_sign=False); without momentum only the learning rate;
    - 'adam'       optax.scale_by_adam(b1, b2, eps, eps_root, nesterov) (Kingma & Ba
                   2015, with optax's Nesterov variant), second moment |d|^2;
    - 'polyak_sgd' scale_by_learning_rate(scaling) then scale_by_polyak(max_lr,
                   f_min, eps): the stochastic Polyak step (Loizou et al. 2021)
                   min((loss - f_min) / (sum |u|^2 + eps), max_lr), 0 for a zero
                   gradient.

    `update(d, loss)` takes the descent directions d (a dict of arrays) and returns
    the dict of updates the reference adds to its parameters (run.py:107-124)."""

    def __init__(self, kind: str, props: t.Mapping[str, t.Any], params: t.Mapping[str, numpy.ndarray]):
        self.kind = kind
        self.p = dict(props)
        self.count = 0
        self.s1 = {k: numpy.zeros_like(v) for (k, v) in params.items()}
        self.s2 = {k: numpy.zeros(v.shape, real_dtype(v.dtype)) for (k, v) in params.items()}

    def update(self, d: t.Mapping[str, numpy.ndarray], loss: float) -> t.Dict[str, numpy.ndarray]:
        p = self.p
        out = {}
        if self.kind == 'sgd':
            lr, mom = p['learning_rate'], p.get('momentum')
            for k, g in d.items():
                if mom is None:
                    out[k] = lr * g
                    continue
                self.s1[k] = g + mom * self.s1[k]
                u = g + mom * self.s1[k] if p.get('nesterov', True) else self.s1[k]
                out[k] = lr * u
        elif self.kind == 'adam':
            b1, b2 = p.get('b1', 0.9), p.get('b2', 0.999)
            eps, eps_root = p.get('eps', 1e-8), p.get('eps_root', 0.0)
            self.count += 1
            c = self.count
            for k, g in d.items():
                self.s1[k] = b1 * self.s1[k] + (1. - b1) * g
                self.s2[k] = b2 * self.s2[k] + (1. - b2) * abs2(g)
                if p.get('nesterov', False):
                    mh = b1 * self.s1[k] / (1. - b1 ** (c + 1)) + (1. - b1) * g / (1. - b1 ** c)
                else:
                    mh = self.s1[k] / (1. - b1 ** c)
                nh = self.s2[k] / (1. - b2 ** c)
                out[k] = p['learning_rate'] * mh / (numpy.sqrt(nh + eps_root) + eps)
        elif self.kind == 'polyak_sgd':
            u = {k: p.get('scaling', 1.0) * g for (k, g) in d.items()}
            q = sum(float(numpy.sum(abs2(v), dtype=numpy.float64)) for v in u.values()) + p.get('eps', 0.0)
            step = 0.0 if q <= 2. ** -52 else min((float(loss) - p['f_min']) / q, p['max_learning_rate'])
            out = {k: (step * v).astype(v.dtype) for (k, v) in u.items()}
        else:
            raise ValueError(f"unknown gradient solver '{self.kind}'")
        return {k: v.astype(d[k].dtype) for (k, v) in out.items()}


@dataclasses.dataclass
class GradientRun:
    """Inputs and knobs of one gradient-engine run (GradientEnginePlan,
    phaser/plan.py:135-141): `solvers` maps a tuple of variables to
    (kind, props) as in the plan's `solvers` dict."""
    solvers: t.Dict[t.Tuple[str, ...], t.Tuple[str, t.Dict[str, t.Any]]]
    niter: int = 2
    grouping: int = 64
    seed: t.Any = 'seed'
    noise: NoiseModel = dataclasses.field(default_factory=NoiseModel)
    update_object: bool = True
    update_probe: bool = True
    update_positions: bool = False
    update_tilt: bool = False
    bwlim_frac: t.Optional[float] = 2. / 3.
    regularizers: t.Dict[str, float] = dataclasses.field(default_factory=dict)   # name -> cost
    tv_eps: float = 1e-8


_PER_ITER = ('positions', 'tilt')


def run_gradient(run: GradientRun, *, probe, obj, scan, patterns, mask, probe_sampling, corner,
                 obj_sampling, thicknesses, wavelength, tilt=None, return_tilt: bool = False):
    """Rescale + `niter` iterations of the gradient engine with sparse groupings
    (phaser/engines/gradient/run.py:156-349): per group the model's gradients,
    the descent directions -g / B (probe) and -g / (B sum|P|^2) (others), the
    per-group solvers applied at once; positions updated once per iteration
    from the gathered group directions, minus their mean.  Returns
    (probe, object, scan, mean loss per iteration)."""
    probe = probe.copy()
    obj = obj.copy()
    rdt = real_dtype(probe.dtype)
    N = probe.shape[-1]
    ky, kx = recip_grid(probe.shape[-2:], probe_sampling, dtype=rdt)
    geom = Geometry(numpy.asarray(corner, numpy.float64), numpy.asarray(obj_sampling, numpy.float64),
                    ky, kx, numpy.asarray(thicknesses))
    props = make_propagators(ky, kx, probe_sampling, wavelength, thicknesses, run.bwlim_frac)
    scan_shape = scan.shape[:-1]
    flat_scan = scan.reshape(-1, 2).copy()
    flat_pat = patterns.reshape(-1, N, N)
    flat_tilt = None if tilt is None else tilt.reshape(-1, 2)

    def flat(g):
        return numpy.ravel_multi_index(tuple(g), scan_shape)

    factors = []
    for g in sparse_groupings(scan_shape, run.grouping, run.seed, 0):
        idx = flat(g)
        tl = None if flat_tilt is None else flat_tilt[idx]
        factors.append(grad_dry_run(geom, probe, obj, flat_scan[idx], flat_pat[idx], props, tl))
    probe = probe * numpy.sqrt(numpy.mean(numpy.concatenate(factors)))
    probe_int = numpy.sum(abs2(probe))

    flat_tilt = (numpy.zeros_like(flat_scan) if (flat_tilt is None and any('tilt' in vs for vs in run.solvers))
                 else flat_tilt)
    params = {'object': obj, 'probe': probe, 'positions': flat_scan, 'tilt': flat_tilt}
    group_solvers, iter_solvers = [], []
    for (vs, (kind, sp)) in run.solvers.items():
        sol = (frozenset(vs), OptaxNP(kind, sp, {v: params[v] for v in vs}))
        (iter_solvers if set(vs) <= set(_PER_ITER) else group_solvers).append(sol)
    enabled = {'object': run.update_object, 'probe': run.update_probe, 'positions': run.update_positions,
               'tilt': run.update_tilt}
    iter_vars = {v for sol in group_solvers + iter_solvers for v in sol[0] if enabled.get(v, False)}

    losses_out = []
    for it in range(1, run.niter + 1):
        iter_d = {k: numpy.zeros_like(flat_scan) for k in ('positions', 'tilt') if k in iter_vars}
        losses = []
        for gi, g in enumerate(sparse_groupings(scan_shape, run.grouping, run.seed, it)):
            idx = flat(g)
            B = len(idx)
            tl = None if flat_tilt is None else flat_tilt[idx]
            L, g_obj, g_probe, g_pos, g_tilt = grad_model_grads(geom, probe, obj, flat_scan[idx], flat_pat[idx],
                                                                mask, props, tl, run.noise, with_tilt=True)
            if run.regularizers:
                # cost regularisers join the loss and the gradients (gradient/run.py:398-403)
                regs = run.regularizers
                r_cost, r_grad = obj_regularizer_costs(obj, regs, B / flat_scan.shape[0], run.tv_eps)
                L = L + r_cost
                g_obj = g_obj + r_grad
                if regs.get('obj_recip_l1'):
                    r_cost, r_grad = obj_recip_l1(obj, regs['obj_recip_l1'], B / flat_scan.shape[0])
                    L = L + r_cost
                    g_obj = g_obj + r_grad
                pr = {k: v for (k, v) in regs.items() if k.startswith('probe_')}
                if pr:
                    r_cost, r_grad = probe_regularizer_costs(probe, pr, run.tv_eps)
                    L = L + r_cost
                    g_probe = g_probe + r_grad
            d = {'object': -g_obj / (probe_int * B), 'probe': -g_probe / B,
                 'positions': -g_pos / (probe_int * B), 'tilt': -g_tilt / (probe_int * B)}
            d = {k: v.astype(params[k].dtype) for (k, v) in d.items() if k in iter_vars}
            for k in ('positions', 'tilt'):
                if k in d:
                    iter_d[k][idx] = d[k]
            for (vs, sol) in group_solvers:
                dd = {k: v for (k, v) in d.items() if k in vs}
                if not dd:
                    continue
                upd = sol.update(dd, L)
                if 'probe' in upd:
                    probe = probe + upd['probe']
                if 'object' in upd:
                    obj = obj + upd['object']
            if not (numpy.all(numpy.isfinite(obj)) and numpy.all(numpy.isfinite(probe))):
                raise ValueError(f"NaN or inf encountered in object or probe, group {gi}")
            losses.append(L)
        loss = float(numpy.mean(losses))
        for (vs, sol) in iter_solvers:
            dd = {k: v for (k, v) in iter_d.items() if k in vs}
            if not dd:
                continue
            upd = sol.update(dd, loss)
            if 'positions' in upd:
                u = upd['positions']
                flat_scan = flat_scan + (u - numpy.mean(u, axis=0))
            if 'tilt' in upd:
                flat_tilt = flat_tilt + upd['tilt']   # no mean subtraction (run.py:119-123)
        losses_out.append(loss)
    if return_tilt:
        return probe, obj, flat_scan.reshape(scan.shape), numpy.array(losses_out), flat_tilt
    return probe, obj, flat_scan.reshape(scan.shape), numpy.array(losses_out)


# ---------------------------------------------------------------- constraints (a17)

def layers_taps(thicknesses, sigma: float, dtype=numpy.float32) -> numpy.ndarray:
    """Normalised Gaussian taps along z over +-2 sigma, layers taken as equally
    spaced at the mean thickness (regularizers.py:99-108)."""
    spacing = numpy.mean(thicknesses)
    r = int(numpy.ceil(2. * sigma / spacing))
    n = 2 * r + 1
    zs = ((numpy.arange(n) - (n - 1) // 2) * spacing).astype(dtype)
    taps = numpy.exp(-(zs / sigma) ** 2 / 2.)
    return (taps / numpy.sum(taps)).astype(dtype)


def regularize_layers(obj, thicknesses, sigma: float, weight: float):
    """RegularizeLayers (regularizers.py:86-132): smooth log(O) along z with the
    Gaussian taps, edges clamped (scipy 'nearest'), blend with weight."""
    if len(thicknesses) < 2:
        return obj
    taps = layers_taps(thicknesses, sigma, real_dtype(obj.dtype))
    r = (len(taps) - 1) // 2
    lg = numpy.log(obj)
    S = obj.shape[0]
    conv = numpy.zeros_like(lg)
    for s in range(S):
        for j, w in enumerate(taps):
            conv[s] += w * lg[min(max(s + r - j, 0), S - 1)]
    return (weight * numpy.exp(conv) + (1 - weight) * obj).astype(obj.dtype)


def low_pass_filter(shape, max_freq: float) -> numpy.ndarray:
    """ObjLowPass mask (regularizers.py:140-149): |k|^2 <= max_freq^2, k in 1/px."""
    ky, kx = numpy.meshgrid(numpy.fft.fftfreq(shape[0], 1.0), numpy.fft.fftfreq(shape[1], 1.0), indexing='ij')
    return (ky ** 2 + kx ** 2 <= max_freq ** 2)


def gaussian_filter(shape, sampling, sigma: float, weight: float, dtype=numpy.float32) -> numpy.ndarray:
    """ObjGaussian filter (regularizers.py:169-180): 1 - weight (1 - exp(-2 pi^2 sigma^2 k^2))."""
    ky = numpy.fft.fftfreq(shape[0], sampling[0]).astype(dtype)
    kx = numpy.fft.fftfreq(shape[1], sampling[1]).astype(dtype)
    ky, kx = numpy.meshgrid(ky, kx, indexing='ij')
    filt = numpy.exp(-(2 * numpy.pi ** 2 * sigma ** 2) * (ky ** 2 + kx ** 2)).astype(dtype)
    return (1. - weight * (1. - filt)).astype(dtype)


def fourier_filter(obj, filt):
    """O <- ifft2(filt * fft2(O)) per slice (regularizers.py:157-161, 188-192)."""
    return ifft2c(filt * fft2c(obj)).astype(obj.dtype)


def region_crop(shape, corner, sampling, region_min, region_max):
    """Rows / columns of ObjectSampling.get_region_crop (object.py:367-378) with pad 0."""
    if region_min is None:
        lo = (0, 0)
    else:
        lo = numpy.ceil((numpy.asarray(region_min) - corner) / sampling).astype(int)
    if region_max is None:
        hi = shape
    else:
        hi = numpy.floor((numpy.asarray(region_max) - corner) / sampling).astype(int) + 1
    return (max(int(lo[0]), 0), min(int(hi[0]), shape[0])), (max(int(lo[1]), 0), min(int(hi[1]), shape[1]))


def remove_phase_ramp(obj, rows, cols):
    """RemovePhaseRamp (regularizers.py:67-83, utils/image.py:30-55): per slice,
    least-squares plane a + b x + c y of the phase over the region, subtracted."""
    ph = numpy.angle(obj)
    yy, xx = numpy.indices(obj.shape[-2:], dtype=float)
    sel = numpy.zeros(obj.shape[-2:], bool)
    sel[rows[0]:rows[1], cols[0]:cols[1]] = True
    A = numpy.stack([numpy.ones(int(sel.sum())), xx[sel], yy[sel]], axis=-1)
    out = numpy.empty_like(ph)
    for s in range(obj.shape[0]):
        p = numpy.linalg.lstsq(A, ph[s][sel].astype(numpy.float64), rcond=None)[0]
        out[s] = (ph[s] - (p[0] + p[1] * xx + p[2] * yy)).astype(ph.dtype)
    return (numpy.abs(obj) * numpy.exp(1j * out)).astype(obj.dtype)


# ------------------------------------------------------- cost regularisers (f1)

def obj_regularizer_costs(obj, costs: t.Mapping[str, float], scale: float, tv_eps: float = 1e-8):
    """Object cost regularisers of the gradient engine (regularizers.py:195-351)
    and their gradients (dL/dRe + i dL/dIm), each term weighted by its cost and
    all by `scale` = B / n_pos.  Returns (cost, grad)."""
    o = obj
    grad = numpy.zeros_like(o)
    total = 0.0
    c = costs.get
    if c('obj_l1'):
        d = o - 1.0
        m = numpy.abs(d)
        total += c('obj_l1') * numpy.sum(m)
        grad += c('obj_l1') * numpy.where(m > 0, d / numpy.where(m > 0, m, 1), 0)
    if c('obj_l2'):
        d = o - 1.0
        total += c('obj_l2') * numpy.sum(abs2(d))
        grad += 2 * c('obj_l2') * d
    if c('obj_phase_l1'):
        ph = numpy.angle(o)
        total += c('obj_phase_l1') * numpy.sum(numpy.abs(ph))
        grad += c('obj_phase_l1') * numpy.sign(ph) * 1j * o / numpy.maximum(abs2(o), 1e-30)
    if c('obj_tikh'):
        for ax in (-1, -2):
            d = numpy.diff(o, axis=ax)
            total += c('obj_tikh') * numpy.sum(abs2(d))
            g = numpy.zeros_like(o)
            sl_lo = [slice(None)] * o.ndim
            sl_hi = [slice(None)] * o.ndim
            sl_lo[ax], sl_hi[ax] = slice(None, -1), slice(1, None)
            g[tuple(sl_lo)] -= 2 * d
            g[tuple(sl_hi)] += 2 * d
            grad += c('obj_tikh') * g
    if c('obj_tv'):
        gy = numpy.diff(o, axis=-2, append=o[..., -1:, :])
        gx = numpy.diff(o, axis=-1, append=o[..., :, -1:])
        tv = numpy.sqrt(abs2(gy) + abs2(gx) + tv_eps)
        total += c('obj_tv') * numpy.sum(tv)
        uy, ux = gy / tv, gx / tv
        g = -(uy + ux)
        g[..., 1:, :] += uy[..., :-1, :]
        g[..., :, 1:] += ux[..., :, :-1]
        grad += c('obj_tv') * g
    if o.shape[0] > 1 and (c('layers_tikh') or c('layers_tv')):
        d = numpy.diff(o, axis=0)
        if c('layers_tikh'):
            total += c('layers_tikh') * numpy.sum(abs2(d))
            g = numpy.zeros_like(o)
            g[:-1] -= 2 * d
            g[1:] += 2 * d
            grad += c('layers_tikh') * g
        if c('layers_tv'):
            m = numpy.abs(d)
            total += c('layers_tv') * numpy.sum(m)
            u = numpy.where(m > 0, d / numpy.where(m > 0, m, 1), 0)
            g = numpy.zeros_like(o)
            g[:-1] -= u
            g[1:] += u
            grad += c('layers_tv') * g
    return float(total) * scale, (grad * scale).astype(obj.dtype)


def obj_recip_l1(obj, cost: float, scale: float):
    """ObjRecipL1 (regularizers.py:233-253): cost * scale * sum |fft2(prod_s O_s)|.
    The centring shift of fft2 only multiplies the spectrum by a phase ramp, so the
    magnitudes are those of the plain DFT.  Returns (value, gradient on O)."""
    S = obj.shape[0]
    P = numpy.prod(obj, axis=0)
    n = P.size
    Z = numpy.fft.fft2(P) / numpy.sqrt(n)
    m = numpy.abs(Z)
    gP = numpy.fft.ifft2(numpy.where(m > 0, Z / numpy.where(m > 0, m, 1), 0)) * numpy.sqrt(n)
    grad = numpy.empty_like(obj)
    for s in range(S):
        others = numpy.prod(numpy.delete(obj, s, axis=0), axis=0) if S > 1 else numpy.ones_like(P)
        grad[s] = gP * numpy.conj(others)
    return float(numpy.sum(m)) * cost * scale, (grad * cost * scale).astype(obj.dtype)


def _tikh(R):
    """sum |diff_x R|^2 + |diff_y R|^2 over the last two axes and its gradient (g convention)."""
    total = 0.0
    g = numpy.zeros_like(R)
    for ax in (-1, -2):
        d = numpy.diff(R, axis=ax)
        total += float(numpy.sum(numpy.abs(d) ** 2))
        lo = [slice(None)] * R.ndim
        hi = [slice(None)] * R.ndim
        lo[ax], hi[ax] = slice(None, -1), slice(1, None)
        g[tuple(lo)] -= 2 * d
        g[tuple(hi)] += 2 * d
    return total, g


def probe_regularizer_costs(probe, costs: t.Mapping[str, float], tv_eps: float = 1e-8):
    """Probe cost regularisers (regularizers.py:354-426), scale 1:
    probe_phase_tikh  sum |diff angle(fft2 P)|^2 (no unwrapping),
    probe_recip_tikh  sum |diff fftshift(fft2 P)|^2,
    probe_recip_tv    sum sqrt(|g_y|^2 + |g_x|^2 + eps) of fftshift(fft2 P) (forward
                      differences, zero at the far edge).
    fft2 is unitary, so the probe gradient is ifft2 of the spectrum gradient.
    Returns (value, gradient on P)."""
    R = fft2c(probe)
    total = 0.0
    gR = numpy.zeros_like(R)
    c = costs.get
    if c('probe_phase_tikh'):
        th = numpy.angle(R)
        v, gth = _tikh(th.astype(numpy.float64))
        total += c('probe_phase_tikh') * v
        m2 = numpy.abs(R) ** 2
        gR += c('probe_phase_tikh') * gth * 1j * R / numpy.where(m2 > 0, m2, 1)
    Rs = numpy.fft.fftshift(R, axes=(-1, -2))
    gRs = numpy.zeros_like(Rs)
    if c('probe_recip_tikh'):
        v, g = _tikh(Rs)
        total += c('probe_recip_tikh') * v
        gRs += c('probe_recip_tikh') * g
    if c('probe_recip_tv'):
        gy = numpy.diff(Rs, axis=-2, append=Rs[..., -1:, :])
        gx = numpy.diff(Rs, axis=-1, append=Rs[..., :, -1:])
        tv = numpy.sqrt(numpy.abs(gy) ** 2 + numpy.abs(gx) ** 2 + tv_eps)
        total += c('probe_recip_tv') * float(numpy.sum(tv))
        uy, ux = gy / tv, gx / tv
        g = -(uy + ux)
        g[..., 1:, :] += uy[..., :-1, :]
        g[..., :, 1:] += ux[..., :, :-1]
        gRs += c('probe_recip_tv') * g
    gR += numpy.fft.ifftshift(gRs, axes=(-1, -2))
    return total, ifft2c(gR).astype(probe.dtype)


def unstructured_gaussian(vals, scan, shape, corner, sampling, sigma: float, weight: float):
    """UnstructuredGaussian (regularizers.py:430-497) for per-position values
    (n, C): every object-grid pixel takes the value of its nearest scan position,
    the image is blurred with exp(-2 pi^2 sigma^2 k^2) (k from fftfreq of the
    object sampling), sampled back at each position's rounded pixel, and blended:
    weight * blurred + (1 - weight) * vals."""
    from scipy.spatial import cKDTree
    pts = scan.reshape(-1, 2).astype(numpy.float64)
    ys = corner[0] + numpy.arange(shape[0]) * sampling[0]
    xs = corner[1] + numpy.arange(shape[1]) * sampling[1]
    grid = numpy.stack(numpy.meshgrid(ys, xs, indexing='ij'), axis=-1)
    near = cKDTree(pts).query(grid)[1]
    v = vals.reshape(len(pts), -1)
    img = v[near]                                     # (H, W, C)
    ky, kx = numpy.meshgrid(numpy.fft.fftfreq(shape[0], sampling[0]), numpy.fft.fftfreq(shape[1], sampling[1]),
                            indexing='ij')
    filt = numpy.exp(-(2 * numpy.pi ** 2 * sigma ** 2) * (ky ** 2 + kx ** 2))
    blur = numpy.real(ifft2c(fft2c(numpy.moveaxis(img, -1, 0)) * filt))
    idx = numpy.round((pts - numpy.asarray(corner)) / numpy.asarray(sampling)).astype(int)
    out = numpy.moveaxis(blur, 0, -1)[idx[:, 0], idx[:, 1]]
    return (weight * out + (1 - weight) * v).reshape(vals.shape)
