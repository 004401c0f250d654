"""State preparation in front of the engines on the device:
phaser.execute.prepare_for_engine (phaser/execute.py:334-402).

    patterns, state = prepare_for_engine(patterns, state, engine_plan)

resizes the probe, the patterns and the pattern mask to the plan's
`sim_shape` (keeping the probe's extent for 'pad_crop', its pixel size for
'resample'), resamples the object onto the probe's pixel size and pads it to
the scan (`obj_pad_px`), truncates or creates probe modes (`probe_modes`,
`base_mode_power`), reslices the object along z (`slices`), and for a gradient
plan that solves for tilt creates a zero tilt map.  The arrays come back as
device tensors (patterns float32, probe and object complex64), which the
engines take as they are: the patterns stay resident between preparation and
reconstruction.  Resampling and reslicing run as CUDA kernels
(phb_resample_c64/f32, phb_resample_slices_c64, phb_project_slices); only the
grid arithmetic (host float64, as the reference) and the creation of new probe
modes from the summed probe (a few N^2 arrays) run on the host.
"""
from __future__ import annotations

import itertools
import logging
import typing as t

import numpy
import torch

from . import _lib
from . import plan as P
from .optics import make_hermite_modes
from .sampling import ObjectSampling, Sampling
from .state import Patterns

log = logging.getLogger(__name__)


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _dev(a, dtype: torch.dtype, device) -> torch.Tensor:
    if torch.is_tensor(a):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(numpy.ascontiguousarray(a)).to(device=device, dtype=dtype)


def _resample(x: torch.Tensor, out_shape, matrix, offset, cval=0.0, recip: bool = False) -> torch.Tensor:
    """Bilinear resampling of the last two axes of x (complex64 or float32) onto
    out_shape at (matrix * index + offset), constant `cval` beyond the edges."""
    H, W = x.shape[-2:]
    Ho, Wo = (int(v) for v in out_shape)
    batch = int(numpy.prod(x.shape[:-2], dtype=numpy.int64)) if x.dim() > 2 else 1
    out = torch.empty((*x.shape[:-2], Ho, Wo), dtype=x.dtype, device=x.device)
    args = (batch, H, W, out.data_ptr(), Ho, Wo, float(matrix[0]), float(matrix[1]), float(offset[0]),
            float(offset[1]))
    if x.dtype == torch.complex64:
        c = complex(cval)
        _lib.call('phb_resample_c64', x.data_ptr(), *args, c.real, c.imag, int(recip), _stream())
    elif x.dtype == torch.float32:
        _lib.call('phb_resample_f32', x.data_ptr(), *args, float(cval), int(recip), _stream())
    else:
        raise TypeError(f"cannot resample {x.dtype}")
    return out


def resample(x: torch.Tensor, old: Sampling, new: Sampling, cval=0.0) -> torch.Tensor:
    """Sampling.resample (phaser/utils/num.py:713-733): grid centres aligned."""
    matrix = new.sampling / old.sampling
    offset = ((old.shape - 1) - matrix * (new.shape - 1)) / 2.
    return _resample(x, new.shape, matrix, offset, cval)


def resample_recip(x: torch.Tensor, old: Sampling, new: Sampling) -> torch.Tensor:
    """Sampling.resample_recip (num.py:735-750) of arrays stored with the zero frequency
    in the corner: the reciprocal grids (extent k_max) resampled between fftshift and
    ifftshift, both folded into the kernel's indexing."""
    old_r = Sampling(old.shape, extent=old.k_max)
    new_r = Sampling(new.shape, extent=new.k_max)
    matrix = new_r.sampling / old_r.sampling
    offset = ((old_r.shape - 1) - matrix * (new_r.shape - 1)) / 2.
    return _resample(x, new.shape, matrix, offset, 0.0, recip=True)


def resample_object(x: torch.Tensor, old: ObjectSampling, new: ObjectSampling) -> torch.Tensor:
    """ObjectSampling.resample (object.py:430-467): corners aligned, transmission 1
    beyond the old grid."""
    matrix = new.sampling / old.sampling
    offset = (new.corner - old.corner) / old.sampling
    return _resample(x, new.shape, matrix, offset, 1.0)


_PAD_MODES = {'vacuum': 0, 'edge': 1, 'average': 2}


def resample_slices(obj: torch.Tensor, old_t, new_t, *, align: str = 'middle',
                    pad_mode: str = 'vacuum') -> torch.Tensor:
    """resample_slices (phaser/utils/object.py:56-157, without the experimental
    rescale_projected): the object's log divided by the slice thickness,
    interpolated linearly along z at the new slice centres (edges held), times the
    new thickness, exponentiated.  Single -> multi spreads the projected potential by
    thickness; multi -> single is the product of the slices."""
    old_t = numpy.asarray(old_t, numpy.float64).ravel()
    new_t = numpy.asarray(new_t, numpy.float64).ravel()
    S, H, W = obj.shape
    st = _stream()
    if len(new_t) < 2:
        if S == 1:
            return obj
        out = torch.empty((1, H, W), dtype=torch.complex64, device=obj.device)
        _lib.call('phb_project_slices', obj.data_ptr(), S, H * W, out.data_ptr(), st)
        return out
    Sn = len(new_t)
    if S == 1:
        # exp(log(obj) * t_i / sum(t)): slice 1 of the padded stack with weight 1, "thickness" 1
        old_tab = numpy.ones(1, numpy.float32)
        ja = numpy.ones(Sn, numpy.int32)
        jb = numpy.ones(Sn, numpy.int32)
        wa = numpy.ones(Sn, numpy.float32)
        wb = numpy.zeros(Sn, numpy.float32)
        scale = (new_t / numpy.sum(new_t)).astype(numpy.float32)
        mode = 0
    else:
        if len(old_t) != S:
            raise ValueError(f"Expected an object with {len(old_t)} slices, instead got object shape {tuple(obj.shape)}")
        if align not in ('top', 'middle', 'bottom'):
            raise ValueError(f"Unknown alignment type '{align}'. Expected 'top', 'middle', or 'bottom'.")
        if pad_mode not in _PAD_MODES:
            raise ValueError(f"Unknown padding mode '{pad_mode}'. Expected 'edge', 'vacuum', or 'average'.")
        old_zs = numpy.cumsum(old_t) - old_t / 2.
        new_zs = numpy.cumsum(new_t) - new_t / 2.
        if align == 'bottom':
            new_zs += numpy.sum(old_t) - numpy.sum(new_t)
        elif align == 'middle':
            new_zs += (numpy.sum(old_t) - numpy.sum(new_t)) / 2.
        zs = numpy.concatenate(([old_zs[0] - old_t[0]], old_zs, [old_zs[-1] + old_t[-1]]))
        # linear interpolation table over the padded stack (_interp1d, object.py:160-185)
        idx = numpy.searchsorted(zs, new_zs) - 1
        ja, jb = numpy.zeros(Sn, numpy.int32), numpy.zeros(Sn, numpy.int32)
        wa, wb = numpy.zeros(Sn, numpy.float32), numpy.zeros(Sn, numpy.float32)
        for i, z in enumerate(new_zs):
            if z <= zs[0]:
                ja[i], wa[i] = 0, 1.0
            elif zs[-1] <= z:
                ja[i], wa[i] = len(zs) - 1, 1.0
            else:
                j = int(idx[i])
                tt = numpy.float32((z - zs[j]) / (zs[j + 1] - zs[j]))
                ja[i], jb[i], wa[i], wb[i] = j, j + 1, numpy.float32(1) - tt, tt
        old_tab = old_t.astype(numpy.float32)
        scale = new_t.astype(numpy.float32)
        mode = _PAD_MODES[pad_mode]
    out = torch.empty((Sn, H, W), dtype=torch.complex64, device=obj.device)
    obj = obj.contiguous()
    _lib.call('phb_resample_slices_c64', obj.data_ptr(), S if S > 1 else 1, H * W, old_tab.ctypes.data,
              out.data_ptr(), Sn, scale.ctypes.data, ja.ctypes.data, jb.ctypes.data, wa.ctypes.data,
              wb.ctypes.data, mode, st)
    return out


def solves_for_tilt(engine: t.Any) -> bool:
    """Whether a gradient plan has a solver for the tilt variable (execute.py:396-400)."""
    if not (isinstance(engine, P.GradientEnginePlan) or hasattr(engine, 'solvers')):
        return False
    solvers = P.get(engine, 'solvers', {}) or {}
    return 'tilt' in set(itertools.chain.from_iterable(P.recons_vars(k) for k in dict(solvers)))


def _as_sampling(s) -> Sampling:
    if isinstance(s, Sampling):
        return s
    return Sampling(tuple(int(v) for v in s.shape), sampling=tuple(float(v) for v in s.sampling))


def _as_object_sampling(s) -> ObjectSampling:
    if isinstance(s, ObjectSampling):
        return s
    return ObjectSampling(tuple(int(v) for v in s.shape), s.sampling, s.corner,
                          getattr(s, 'region_min', None), getattr(s, 'region_max', None))


def prepare_for_engine(patterns: Patterns, state: t.Any, engine: t.Any, *,
                       device: t.Union[str, torch.device] = 'cuda') -> t.Tuple[Patterns, t.Any]:
    """phaser.execute.prepare_for_engine (execute.py:334-402) on the device; `state` is
    a ReconsState (numpy or device arrays).  Returns (patterns, state) with device
    tensors; `state` is updated in place and returned."""
    dev = torch.device(device)
    pats = patterns.patterns
    if torch.is_tensor(pats):
        pats = pats.to(dev)
        if pats.dtype not in (torch.float32, torch.uint16):
            pats = pats.to(torch.float32)
    else:
        arr = numpy.asarray(pats)
        pats = _dev(arr, torch.uint16 if arr.dtype == numpy.uint16 else torch.float32, dev)
    mask = _dev(patterns.pattern_mask, torch.float32, dev)
    probe = _dev(state.probe.data, torch.complex64, dev)
    obj = _dev(state.object.data, torch.complex64, dev)
    if probe.dim() == 2:
        probe = probe[None]
    if obj.dim() == 2:
        obj = obj[None]
    psamp = _as_sampling(state.probe.sampling)

    sim_shape = P.get(engine, 'sim_shape', None)
    if sim_shape is not None and tuple(int(v) for v in sim_shape) != tuple(probe.shape[-2:]):
        method = P.get(engine, 'resize_method', 'pad_crop')
        if method == 'pad_crop':
            new = Sampling(tuple(sim_shape), extent=psamp.extent)
        else:
            new = Sampling(tuple(sim_shape), sampling=psamp.sampling)
        log.info(f"Resampling probe and patterns to shape {tuple(new.shape)}...")
        probe = resample(probe, psamp, new)
        if pats.dtype != torch.float32:
            pats = pats.to(torch.float32)
        pats = resample_recip(pats, psamp, new)
        mask = resample_recip(mask, psamp, new)
        psamp = new

    old_grid = _as_object_sampling(state.object.sampling)
    grid = old_grid
    if not numpy.allclose(psamp.sampling, grid.sampling):
        log.info(f"Resampling object to pixel size {list(map(float, psamp.sampling))}...")
        grid = grid.with_sampling(psamp.sampling)
    pad = psamp.extent / 2. + float(P.get(engine, 'obj_pad_px', 5.0)) * psamp.sampling
    grid_pad = grid.expand_to_scan(numpy.asarray(state.scan), pad)
    if grid_pad != grid:
        log.info(f"Padding object to shape {tuple(grid_pad.shape)}")
        grid = grid_pad
    if grid != old_grid:
        obj = resample_object(obj, old_grid, grid)

    n_modes = int(P.get(engine, 'probe_modes', 1))
    if n_modes != probe.shape[0]:
        if n_modes < probe.shape[0]:
            probe = probe[:n_modes].contiguous()
        else:
            if probe.shape[0] != 1:
                log.info("Summing probe modes (in real-space) before recreating with different # of modes")
            base = torch.sum(probe, dim=0).cpu().numpy()
            modes = make_hermite_modes(base, n_modes, float(P.get(engine, 'base_mode_power', 0.7)))
            probe = torch.from_numpy(numpy.ascontiguousarray(modes, numpy.complex64)).to(dev)

    thick = numpy.asarray(state.object.thicknesses)
    new_t = P.slice_thicknesses(P.get(engine, 'slices', None))
    if new_t is not None and (len(new_t) != len(thick) or not numpy.allclose(new_t, thick)):
        log.info(f"Reslicing object from {max(1, len(thick))} to {max(1, len(new_t))} slice(s)...")
        obj = resample_slices(obj, thick, new_t)
        thick = numpy.array(new_t, dtype=thick.dtype if thick.size else numpy.float32)

    if solves_for_tilt(engine) and state.tilt is None:
        log.info("Creating new, zeroed tilt map...")
        state.tilt = numpy.zeros_like(numpy.asarray(state.scan))

    state.probe.data = probe
    state.probe.sampling = psamp
    state.object.data = obj
    state.object.sampling = grid
    state.object.thicknesses = thick
    return Patterns(pats, mask), state
