"""Group / iteration constraints of the conventional engine on the device.

phaser applies these between mini-batches / iterations
(phaser/engines/common/simulation.py:137-157 with the implementations in
phaser/engines/common/regularizers.py).  Implemented here:
  clamp_object_amplitude  (regularizers.py:24-42)   -> phb_clamp_amplitude_c64
  limit_probe_support     (regularizers.py:45-64)   -> phb_fourier_mask_c64
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


_KNOWN = {'clamp_object_amplitude': ClampObjectAmplitude, 'limit_probe_support': LimitProbeSupport}


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
        out.append(cls(eng, state, props))
    return out
