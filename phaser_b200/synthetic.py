"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no datasets ship with this repository).

* object: per slice, a phase image made of Gaussian 'atoms' on a jittered
  hexagonal lattice (independent random shift per slice), amplitude 1;
* probe: circular aperture with defocus (phaser/utils/optics.py:30-51), split
  into Hermite-Gauss modes with the requested powers (optics.py:54-94);
* scan: raster around the origin (phaser/utils/scan.py:23-55), optional jitter;
* object grid: ObjectSampling.from_scan with pad = N/2 + 5 px (phaser/execute.py:270-273);
* patterns: the far-field intensity of the multislice forward model, computed by
  the B200 forward kernel, scaled to the requested electrons per pattern and
  Poisson-sampled from a seeded generator.
"""
from __future__ import annotations

import dataclasses
import typing as t

import numpy

from .optics import make_focused_probe, make_hermite_modes, electron_wavelength
from .sampling import ObjectSampling, Sampling


def lattice_phase(shape: t.Tuple[int, int], spacing: float, sigma: float, peak: float,
                  rng: numpy.random.Generator, jitter: float = 0.5) -> numpy.ndarray:
    """Sum of Gaussian atoms (sigma px, height `peak` rad) on a hexagonal lattice of
    `spacing` px with a random global shift and per-atom jitter (uniform +-jitter px)."""
    H, W = shape
    out = numpy.zeros(shape, numpy.float64)
    dy = spacing * numpy.sqrt(3) / 2
    off = rng.uniform(0, spacing, 2)
    r = int(numpy.ceil(4 * sigma))
    yy, xx = numpy.mgrid[-r:r + 1, -r:r + 1]
    rows = numpy.arange(-1, int(H / dy) + 2)
    for i in rows:
        y0 = i * dy + off[0]
        xs = numpy.arange(-1, int(W / spacing) + 2) * spacing + off[1] + (spacing / 2 if i % 2 else 0.)
        for x0 in xs:
            cy, cx = y0 + rng.uniform(-jitter, jitter), x0 + rng.uniform(-jitter, jitter)
            iy, ix = int(round(cy)), int(round(cx))
            fy, fx = cy - iy, cx - ix
            g = peak * numpy.exp(-((yy - fy) ** 2 + (xx - fx) ** 2) / (2 * sigma ** 2))
            ya, yb = max(0, iy - r), min(H, iy + r + 1)
            xa, xb = max(0, ix - r), min(W, ix + r + 1)
            if ya < yb and xa < xb:
                out[ya:yb, xa:xb] += g[ya - (iy - r):yb - (iy - r), xa - (ix - r):xb - (ix - r)]
    return out


@dataclasses.dataclass
class Dataset:
    probe: numpy.ndarray           # (M, N, N) complex64: true probe (also the initial estimate)
    true_object: numpy.ndarray     # (S, H, W) complex64
    init_object: numpy.ndarray     # (S, H, W) complex64 (reference 'random' init: phase sigma 1e-6)
    scan: numpy.ndarray            # (ny, nx, 2) float32
    mask: numpy.ndarray            # (N, N) float32
    probe_sampling: numpy.ndarray  # (2,)
    obj_sampling: ObjectSampling
    thicknesses: numpy.ndarray     # (S,) or empty
    wavelength: float
    counts: float
    description: str


def make_dataset(*, N: int, M: int, S: int, scan_shape: t.Tuple[int, int], step_px: float, sampling: float,
                 kv: float, conv_mrad: float, defocus: float, slice_thickness: float, spacing_px: float,
                 sigma_px: float, peak_rad: float, counts: float, mode_powers: t.Sequence[float] = (),
                 scan_jitter_px: float = 0.0, seed: int = 0, grid_probe_px: t.Optional[int] = None) -> Dataset:
    """A seeded dataset.  The object grid is the reference's for a probe of
    grid_probe_px pixels (N when None): a dataset prepared for a larger detector
    keeps its grid when the detector is binned down to N (prepare_for_engine only
    pads objects)."""
    rng = numpy.random.default_rng(seed)
    lam = electron_wavelength(kv)
    psamp = Sampling((N, N), sampling=(sampling, sampling))
    ky, kx = psamp.recip_grid(dtype=numpy.float32)
    base = make_focused_probe(ky, kx, lam, conv_mrad, defocus=defocus)
    if M > 1:
        powers = list(mode_powers) or [0.7] + [0.3 / (M - 1)] * (M - 1)
        rel = numpy.array(powers[1:]) / (1 - powers[0])
        probe = make_hermite_modes(base, M, powers[0], rel)
    else:
        probe = base[None]
    probe = probe.astype(numpy.complex64)
    yy = numpy.arange(scan_shape[0], dtype=numpy.float32) - numpy.float32(scan_shape[0] / 2.)
    xx = numpy.arange(scan_shape[1], dtype=numpy.float32) - numpy.float32(scan_shape[1] / 2.)
    scan = numpy.stack(numpy.meshgrid(yy, xx, indexing='ij'), -1) * numpy.float32(step_px * sampling)
    if scan_jitter_px:
        scan = scan + rng.uniform(-scan_jitter_px, scan_jitter_px, scan.shape) * sampling
    scan = scan.astype(numpy.float32)
    grid_extent = psamp.sampling * (grid_probe_px or N)
    osamp = ObjectSampling.from_scan(scan, psamp.sampling, grid_extent / 2. + 5 * psamp.sampling)
    H, W = (int(v) for v in osamp.shape)
    phase = numpy.stack([lattice_phase((H, W), spacing_px, sigma_px, peak_rad, rng) for _ in range(S)])
    true_obj = numpy.exp(1j * phase).astype(numpy.complex64)
    init = numpy.exp(1j * rng.normal(0., 1e-6, (S, H, W))).astype(numpy.complex64)
    thick = numpy.full(S, slice_thickness, numpy.float32) if S > 1 else numpy.array([], numpy.float32)
    desc = (f"{S} slice(s) of {H}x{W} Gaussian-atom lattices ({spacing_px} px, sigma {sigma_px} px, "
            f"{peak_rad} rad), probe {N}x{N} x {M} mode(s) {conv_mrad} mrad {kv / 1e3:.0f} kV "
            f"{defocus} A defocus, scan {scan_shape[0]}x{scan_shape[1]} @ {step_px} px, {counts:.0e} e/pattern")
    return Dataset(probe, true_obj, init, scan, numpy.ones((N, N), numpy.float32),
                   numpy.asarray(psamp.sampling), osamp, thick, lam, counts, desc)


# the multislice LSQ-ML benchmark configuration (8 x 2 nm slices, 128^2 probe, 4 modes, 64^2 scan)
def lsqml_multislice_config(seed: int = 0, scan: int = 64) -> Dataset:
    return make_dataset(N=128, M=4, S=8, scan_shape=(scan, scan), step_px=6.0, sampling=0.2, kv=300e3,
                        conv_mrad=25.0, defocus=200.0, slice_thickness=20.0, spacing_px=10.0, sigma_px=1.5,
                        peak_rad=0.2, counts=1e6, mode_powers=(0.70, 0.15, 0.10, 0.05), seed=seed)


# the large multislice configuration: 32 slices of 1032^2-class, probe and detector 256^2
# with 8 modes, 256 x 256 scan at 3 px, 5e5 e-/pattern.  binned=True keeps the object grid
# but bins the detector 2 x 2 to 128^2: the pixel size stays 0.2 A, the probe window
# halves to 25.6 A (the 25 mrad probe at 200 A defocus is ~10 A across), i.e.
# prepare_for_engine with sim_shape (128, 128), resize_method 'resample'.
def large_multislice_config(seed: int = 0, scan: int = 256, binned: bool = True) -> Dataset:
    return make_dataset(N=128 if binned else 256, M=8, S=32, scan_shape=(scan, scan), step_px=3.0, sampling=0.2,
                        kv=300e3, conv_mrad=25.0, defocus=200.0, slice_thickness=20.0, spacing_px=10.0,
                        sigma_px=1.5, peak_rad=0.2, counts=5e5, seed=seed, grid_probe_px=256)


# the single-slice ePIE configuration (256^2-class object, 64^2 probe, 32^2 scan)
def epie_single_slice_config(seed: int = 0) -> Dataset:
    return make_dataset(N=64, M=1, S=1, scan_shape=(32, 32), step_px=4.0, sampling=0.2, kv=200e3,
                        conv_mrad=20.0, defocus=100.0, slice_thickness=0.0, spacing_px=10.0, sigma_px=1.5,
                        peak_rad=0.4, counts=1e5, scan_jitter_px=0.5, seed=seed)


# the gradient-engine configuration (16 x 2 nm slices, 128^2 probe, 2 modes, 128^2 scan at 5 px)
def gradient_multislice_config(seed: int = 0, scan: int = 128) -> Dataset:
    return make_dataset(N=128, M=2, S=16, scan_shape=(scan, scan), step_px=5.0, sampling=0.2, kv=300e3,
                        conv_mrad=25.0, defocus=200.0, slice_thickness=20.0, spacing_px=10.0, sigma_px=1.5,
                        peak_rad=0.2, counts=1e6, mode_powers=(0.7, 0.3), seed=seed)


def simulate_patterns(ds: Dataset, *, seed: int = 0, group: int = 256, device='cuda', counts_u16: bool = False):
    """Noisy patterns (n_pos, N, N) on the device, from the B200 forward kernel: float32,
    or (counts_u16) uint16 detector counts, drawn group by group so that no float32 copy
    of the whole set is held."""
    if counts_u16:
        return _simulate_counts_u16(ds, seed=seed, group=group, device=device)
    import torch
    from .device import DeviceEngine
    N = ds.probe.shape[-1]
    n = int(numpy.prod(ds.scan.shape[:-1]))
    dummy = torch.zeros((n, N, N), dtype=torch.float32, device=device)
    eng = DeviceEngine(probe=ds.probe, obj=ds.true_object, scan=ds.scan, patterns=None, mask=ds.mask,
                       probe_sampling=ds.probe_sampling, obj_sampling=ds.obj_sampling,
                       thicknesses=ds.thicknesses, wavelength=ds.wavelength, group_max=group,
                       device=device, patterns_on_device=dummy)
    idx = numpy.arange(n, dtype=numpy.int64)
    chunks = [idx[i:i + group] for i in range(0, n, group)]
    gt, sizes = eng.group_tensor(chunks)
    out = torch.empty((n, N, N), dtype=torch.float32, device=device)
    for g, B in enumerate(sizes):
        eng.simulate(gt[g], B, out[g * group:g * group + B])
    total = out.sum(dim=(1, 2), keepdim=True)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    pats = torch.poisson(out * (ds.counts / total), generator=gen).to(torch.float32)
    del eng, dummy
    return pats


def _simulate_counts_u16(ds: Dataset, *, seed: int, group: int, device) -> 'torch.Tensor':
    import torch
    from .device import DeviceEngine
    N = ds.probe.shape[-1]
    n = int(numpy.prod(ds.scan.shape[:-1]))
    out = torch.empty((n, N, N), dtype=torch.uint16, device=device)
    eng = DeviceEngine(probe=ds.probe, obj=ds.true_object, scan=ds.scan, patterns=None, mask=ds.mask,
                       probe_sampling=ds.probe_sampling, obj_sampling=ds.obj_sampling,
                       thicknesses=ds.thicknesses, wavelength=ds.wavelength, group_max=group,
                       device=device, patterns_on_device=out)
    idx = numpy.arange(n, dtype=numpy.int64)
    chunks = [idx[i:i + group] for i in range(0, n, group)]
    gt, sizes = eng.group_tensor(chunks)
    buf = torch.empty((group, N, N), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    peak = torch.zeros((), dtype=torch.float32, device=device)
    for g, B in enumerate(sizes):
        inten = eng.simulate(gt[g], B, buf[:B])
        total = inten.sum(dim=(1, 2), keepdim=True)
        cnt = torch.poisson(inten * (ds.counts / total), generator=gen)
        peak = torch.maximum(peak, cnt.max())
        out[g * group:g * group + B] = cnt.to(torch.uint16)
    if float(peak) >= 65536:
        raise RuntimeError(f"{float(peak)} counts do not fit uint16")
    del eng, buf
    return out
