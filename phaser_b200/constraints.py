"""Group / iteration constraints of the conventional engine on the device.

phaser applies these between mini-batches / iterations
(phaser/engines/common/simulation.py:137-157 with the implementations in
phaser/engines/common/regularizers.py).  Implemented here:
  clamp_object_amplitude  (regularizers.py:20-42)   -> phb_clamp_amplitude_c64
  limit_probe_support     (regularizers.py:45-64)   -> phb_fourier_mask_c64
  layers                  (regularizers.py:86-132)  -> phb_regularize_layers_c64 (iteration only)
  obj_low_pass            (regularizers.py:135-161) -> phb_object_filter_c64
  obj_gaussian            (regularizers.py:164-192) -> phb_object_filter_c64
  remove_phase_ramp       (regularizers.py:67-83)   -> phb_remove_phase_ramp_c64
  tilt_gaussian           (regularizers.py:430-497) -> phb_smooth_position_values (iteration only)
Any other constraint name raises NotImplementedError (no silent skip).
"""
from __future__ import annotations

import typing as t

import numpy
import torch

from . import _lib
from . import plan as P


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class ClampObjectAmplitude:
    def __init__(self, eng, state, props):
        self.eng = eng
        self.amplitude = float(P.get(props, 'amplitude', 1.1))

    def apply_group(self) -> None:
        self.apply_iter()

    def apply_iter(self) -> None:
        _lib.call('phb_clamp_amplitude_c64', self.eng.object.data_ptr(), self.eng.object.numel(),
                  self.amplitude, _stream())


class LimitProbeSupport:
    def __init__(self, eng, state, props):
        self.eng = eng
        max_angle = float(P.get(props, 'max_angle'))
        fy, fx = eng.fy.cpu().numpy(), eng.fx.cpu().numpy()
        ky, kx = numpy.meshgrid(fy, fx, indexing='ij')
        mask = (kx ** 2 + ky ** 2 <= (max_angle * 1e-3 / float(state.wavelength)) ** 2).astype(numpy.float32)
        self.mask = torch.from_numpy(mask).to(eng.device)

    def apply_group(self) -> None:
        self.apply_iter()

    def apply_iter(self) -> None:
        _lib.call('phb_fourier_mask_c64', self.eng.probe.data_ptr(), self.eng.M, self.eng.N,
                  self.mask.data_ptr(), _stream())
        self.eng.probe_changed()


class RegularizeLayers:
    """Log-domain Gaussian smoothing of the object along z (iteration constraint only)."""
    per_group = False

    def __init__(self, eng, state, props):
        self.eng = eng
        self.weight = float(P.get(props, 'weight', 0.9))
        sigma = float(P.get(props, 'sigma', 50.0))
        thick = numpy.asarray(state.object.thicknesses, numpy.float64)
        self.taps = None
        if len(thick) >= 2:
            # normalised Gaussian over +-2 sigma at the mean layer spacing (regularizers.py:99-108)
            spacing = numpy.mean(thick)
            r = int(numpy.ceil(2. * sigma / spacing))
            zs = ((numpy.arange(2 * r + 1) - r) * spacing).astype(numpy.float32)
            taps = numpy.exp(-(zs / numpy.float32(sigma)) ** 2 / 2.)
            self.taps = torch.from_numpy((taps / numpy.sum(taps)).astype(numpy.float32)).to(eng.device)

    def apply_iter(self) -> None:
        if self.taps is None:
            return
        _lib.call('phb_regularize_layers_c64', self.eng.object.data_ptr(), self.eng.S, self.eng.H, self.eng.W,
                  self.taps.data_ptr(), self.taps.numel(), self.weight, _stream())


class _ObjectFilter:
    """O <- ifft2(filter * fft2(O)) on every slice of the object."""

    def __init__(self, eng, filt: numpy.ndarray):
        self.eng = eng
        self.filt = torch.from_numpy(numpy.ascontiguousarray(filt, numpy.float32)).to(eng.device)
        self.scratch = torch.empty((eng.S, eng.H, eng.W), dtype=torch.complex64, device=eng.device)

    def apply_group(self) -> None:
        self.apply_iter()

    def apply_iter(self) -> None:
        _lib.call('phb_object_filter_c64', self.eng.object.data_ptr(), self.eng.S, self.eng.H, self.eng.W,
                  self.filt.data_ptr(), self.scratch.data_ptr(), _stream())


class ObjLowPass(_ObjectFilter):
    def __init__(self, eng, state, props):
        max_freq = float(P.get(props, 'max_freq', 0.4))
        ky, kx = numpy.meshgrid(numpy.fft.fftfreq(eng.H, 1.0), numpy.fft.fftfreq(eng.W, 1.0), indexing='ij')
        super().__init__(eng, (ky ** 2 + kx ** 2 <= max_freq ** 2))


class ObjGaussian(_ObjectFilter):
    def __init__(self, eng, state, props):
        sigma, weight = float(P.get(props, 'sigma')), float(P.get(props, 'weight', 0.9))
        samp = numpy.asarray(eng.obj_sampling.sampling, numpy.float64)
        ky = numpy.fft.fftfreq(eng.H, samp[0]).astype(numpy.float32)
        kx = numpy.fft.fftfreq(eng.W, samp[1]).astype(numpy.float32)
        ky, kx = numpy.meshgrid(ky, kx, indexing='ij')
        filt = numpy.exp(-(2 * numpy.pi ** 2 * sigma ** 2) * (ky ** 2 + kx ** 2)).astype(numpy.float32)
        super().__init__(eng, (1. - weight * (1. - filt)).astype(numpy.float32))


class RemovePhaseRamp:
    """Least-squares phase plane over the scanned region removed from every slice."""

    def __init__(self, eng, state, props):
        self.eng = eng
        os_ = eng.obj_sampling
        corner, samp = numpy.asarray(os_.corner, numpy.float64), numpy.asarray(os_.sampling, numpy.float64)
        lo = (0, 0) if os_.region_min is None else numpy.ceil((numpy.asarray(os_.region_min) - corner) / samp)
        hi = ((eng.H, eng.W) if os_.region_max is None
              else numpy.floor((numpy.asarray(os_.region_max) - corner) / samp) + 1)
        self.rows = (max(int(lo[0]), 0), min(int(hi[0]), eng.H))
        self.cols = (max(int(lo[1]), 0), min(int(hi[1]), eng.W))
        self.sums = torch.zeros((eng.S, 3), dtype=torch.float64, device=eng.device)

    def apply_group(self) -> None:
        self.apply_iter()

    def apply_iter(self) -> None:
        _lib.call('phb_remove_phase_ramp_c64', self.eng.object.data_ptr(), self.eng.S, self.eng.H, self.eng.W,
                  self.rows[0], self.rows[1], self.cols[0], self.cols[1], self.sums.data_ptr(), _stream())


class TiltGaussian:
    """Gaussian smoothing of the per-position tilts over the scan (iteration constraint)."""

    def __init__(self, eng, state, props):
        if eng.tilt is None:
            raise ValueError("tilt_gaussian needs a tilt map (state.tilt)")
        self.eng = eng
        sigma, self.weight = float(P.get(props, 'sigma')), float(P.get(props, 'weight', 0.9))
        samp = numpy.asarray(eng.obj_sampling.sampling, numpy.float64)
        ky, kx = numpy.meshgrid(numpy.fft.fftfreq(eng.H, samp[0]), numpy.fft.fftfreq(eng.W, samp[1]), indexing='ij')
        filt = numpy.exp(-(2 * numpy.pi ** 2 * sigma ** 2) * (ky ** 2 + kx ** 2)).astype(numpy.float32)
        self.filt = torch.from_numpy(filt).to(eng.device)
        self.scratch = torch.empty((2 * eng.H * eng.W,), dtype=torch.complex64, device=eng.device)

    def apply_iter(self) -> None:
        e, os_ = self.eng, self.eng.obj_sampling
        _lib.call('phb_smooth_position_values', e.tilt.data_ptr(), e.scan.data_ptr(), e.n_pos, e.H, e.W,
                  float(os_.corner[0]), float(os_.corner[1]), float(os_.sampling[0]), float(os_.sampling[1]),
                  self.filt.data_ptr(), self.weight, self.scratch.data_ptr(), _stream())


_KNOWN = {'clamp_object_amplitude': ClampObjectAmplitude, 'tilt_gaussian': TiltGaussian, 'limit_probe_support': LimitProbeSupport,
          'layers': RegularizeLayers, 'obj_low_pass': ObjLowPass, 'obj_gaussian': ObjGaussian,
          'remove_phase_ramp': RemovePhaseRamp}
# the reference's GroupConstraintHook has no 'layers' (phaser/hooks/regularization.py:83-91)
_GROUP_ONLY_EXCLUDED = {'layers', 'tilt_gaussian'}


def build_constraints(hooks: t.Sequence[t.Any], eng, state, per_group: bool) -> t.List[t.Any]:
    out = []
    for h in hooks:
        if isinstance(h, str):
            name, props = h, {}
        elif isinstance(h, dict):
            h = dict(h)
            name, props = str(h.pop('type')), h
        else:
            name = getattr(h, 'type', None) or getattr(h, 'ref', '')
            props = getattr(h, 'props', None) or {}
            name = P._REF_CLASS_NAMES.get(str(name).rsplit(':', 1)[-1], name)
        cls = _KNOWN.get(str(name))
        if cls is None:
            raise NotImplementedError(f"constraint '{name}' is not implemented by the B200 backend")
        if per_group and str(name) in _GROUP_ONLY_EXCLUDED:
            raise ValueError(f"'{name}' is an iteration constraint, not a group constraint")
        out.append(cls(eng, state, props))
    return out
