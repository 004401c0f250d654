"""A reconstruction resident on one B200, driven through the C ABI.

`DeviceEngine` owns the device tensors (object, probe, scan, patterns, the
workspace) and fills the `phb_engine` descriptor of include/phaser_b200.h.
All work is enqueued on the current torch stream; nothing synchronises
except the explicit `sync_*` / host-copy methods.
"""
from __future__ import annotations

import ctypes
import typing as t

import numpy
import torch

from . import _lib
from .optics import make_propagators
from .sampling import ObjectSampling

SOLVERS = {'lsqml': _lib.PHB_SOLVER_LSQML, 'epie': _lib.PHB_SOLVER_EPIE, 'grad': _lib.PHB_SOLVER_GRAD}


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _ptr(t_: t.Optional[torch.Tensor]) -> int:
    return 0 if t_ is None else t_.data_ptr()


class NoiseSpec(t.NamedTuple):
    kind: str = 'amplitude'       # 'amplitude' | 'anscombe' | 'poisson'
    eps: float = 1e-3
    offset: float = 0.0
    gaussian_variance: float = 0.1


def _is_complex64(a) -> bool:
    return a.dtype == (torch.complex64 if torch.is_tensor(a) else numpy.complex64)


class DeviceEngine:
    """Device-resident state + workspace of one reconstruction.

    probe (M, N, N) complex64, object (S, H, W) complex64, scan (P, 2) float32,
    patterns (P, N, N) float32 or uint16 counts (kept resident in that format),
    mask (N, N).  `probe_sampling` is the (dy, dx)
    pixel size of the probe grid; `obj_sampling` the object's ObjectSampling.
    """

    def __init__(self, *, probe: numpy.ndarray, obj: numpy.ndarray, scan: numpy.ndarray,
                 patterns: numpy.ndarray, mask: numpy.ndarray, probe_sampling, obj_sampling: ObjectSampling,
                 thicknesses, wavelength: float, tilt: t.Optional[numpy.ndarray] = None,
                 noise: NoiseSpec = NoiseSpec(), bwlim_frac: t.Optional[float] = 2 / 3,
                 group_max: int = 64, device: t.Union[str, torch.device] = 'cuda',
                 track_illumination: bool = False, patterns_on_device: t.Optional[torch.Tensor] = None):
        self.lib = _lib.load()
        if not torch.cuda.is_available():
            raise RuntimeError("the B200 backend needs a CUDA device")
        dev = torch.device(device)
        self.device = dev
        # probe and object: host arrays, or device tensors (e.g. from prepare_for_engine)
        probe = probe if torch.is_tensor(probe) else numpy.asarray(probe)
        if probe.ndim == 2:
            probe = probe[None]
        obj = obj if torch.is_tensor(obj) else numpy.asarray(obj)
        if obj.ndim == 2:
            obj = obj[None]
        if not (_is_complex64(probe) and _is_complex64(obj)):
            raise TypeError("the B200 backend computes in complex64 (plan dtype float32)")
        M, N, N2 = probe.shape
        if N != N2 or N not in (64, 128, 256):
            raise NotImplementedError(f"probe size {N}x{N2}: the B200 kernels support N in (64, 128, 256)")
        S, H, W = obj.shape
        self.N, self.M, self.S, self.H, self.W = N, M, S, H, W
        self.scan_shape = scan.shape[:-1]
        self.n_pos = int(numpy.prod(self.scan_shape))
        self.obj_sampling = obj_sampling
        self.probe_sampling = numpy.broadcast_to(numpy.asarray(probe_sampling, numpy.float64), (2,))
        self.wavelength = float(wavelength)
        self.group_max = int(group_max)
        self.noise = noise

        fy = numpy.fft.fftfreq(N, self.probe_sampling[0]).astype(numpy.float32)
        fx = numpy.fft.fftfreq(N, self.probe_sampling[1]).astype(numpy.float32)
        ky, kx = numpy.meshgrid(fy, fx, indexing='ij')
        thick = numpy.asarray(thicknesses, dtype=numpy.float32)
        props = make_propagators(ky, kx, self.probe_sampling, self.wavelength, thick, bwlim_frac)
        if props is not None and props.shape[0] != S - 1:
            raise ValueError(f"{len(thick)} thicknesses for an object of {S} slices")

        def up(a, dt):
            if torch.is_tensor(a):
                return a.detach().to(dev).contiguous().clone()
            return torch.from_numpy(numpy.ascontiguousarray(a, dtype=dt)).to(dev)

        self.probe = up(probe, numpy.complex64)
        self.object = up(obj, numpy.complex64)
        self.scan = up(numpy.asarray(scan).reshape(-1, 2), numpy.float32)
        self.tilt = None if tilt is None else up(numpy.asarray(tilt).reshape(-1, 2), numpy.float32)
        if patterns_on_device is not None:
            self.patterns = patterns_on_device.reshape(-1, N, N)
        else:
            pat = numpy.asarray(patterns).reshape(-1, N, N)
            self.patterns = up(pat, numpy.uint16 if pat.dtype == numpy.uint16 else numpy.float32)
        if self.patterns.dtype not in (torch.float32, torch.uint16) or not self.patterns.is_contiguous():
            raise TypeError("patterns must be contiguous float32 or uint16")
        if self.patterns.shape[0] != self.n_pos:
            raise ValueError(f"{self.n_pos} scan positions but {self.patterns.shape[0]} patterns")
        self.mask = up(mask, numpy.float32)
        self.props = None if props is None else up(props, numpy.complex64)
        self.thick = up(thick if len(thick) else numpy.zeros(1, numpy.float32), numpy.float32)
        self.fy, self.fx = up(fy, numpy.float32), up(fx, numpy.float32)
        self.new_obj_mag = torch.zeros((N, N), dtype=torch.float32, device=dev) if track_illumination else None
        self.new_probe_mag = (torch.zeros((S, H, W), dtype=torch.float32, device=dev)
                              if track_illumination else None)

        nbytes = self.lib.phb_engine_workspace_bytes(N, M, S, self.group_max, H, W)
        if nbytes == 0:
            raise ValueError("invalid engine sizes")
        # 256-byte aligned workspace owned by torch
        self._ws_raw = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
        off = (-self._ws_raw.data_ptr()) % 256
        self.workspace = self._ws_raw[off:off + nbytes]

        e = _lib.PhbEngine()
        e.N, e.M, e.S, e.B_max = N, M, S, self.group_max
        e.H, e.W, e.n_pos = H, W, self.n_pos
        e.corner_y, e.corner_x = float(obj_sampling.corner[0]), float(obj_sampling.corner[1])
        e.samp_y, e.samp_x = float(obj_sampling.sampling[0]), float(obj_sampling.sampling[1])
        e.object, e.probe, e.scan = self.object.data_ptr(), self.probe.data_ptr(), self.scan.data_ptr()
        e.tilt = _ptr(self.tilt)
        e.patterns, e.pattern_mask = self.patterns.data_ptr(), self.mask.data_ptr()
        e.pattern_u16 = int(self.patterns.dtype == torch.uint16)
        e.propagators = _ptr(self.props)
        e.thicknesses = self.thick.data_ptr() if self.tilt is not None else 0
        e.ky, e.kx = self.fy.data_ptr(), self.fx.data_ptr()
        e.noise = _lib.PHB_NOISE_POISSON if noise.kind == 'poisson' else _lib.PHB_NOISE_AMPLITUDE
        e.noise_eps, e.noise_offset, e.noise_var = noise.eps, noise.offset, 1.0 + noise.gaussian_variance
        e.workspace, e.workspace_bytes = self.workspace.data_ptr(), nbytes
        e.new_obj_mag, e.new_probe_mag = _ptr(self.new_obj_mag), _ptr(self.new_probe_mag)
        self.desc = e
        self._eref = ctypes.byref(self.desc)
        _lib.call('phb_engine_init', self._eref, _stream())

        # per-step scratch owned here
        self.status = torch.full((1,), -1, dtype=torch.int32, device=dev)
        self.pos_update = torch.zeros((self.n_pos, 2), dtype=torch.float32, device=dev)
        self.errors = torch.full((self.n_pos,), float('nan'), dtype=torch.float32, device=dev)
        self.n_outside = torch.zeros((1,), dtype=torch.int32, device=dev)
        self.report = torch.zeros((4,), dtype=torch.float64, device=dev)

    # ---------------------------------------------------------------- helpers
    def set_patterns(self, patterns: torch.Tensor) -> None:
        """Point the engine at another resident pattern array of the same shape and
        type (e.g. the other half of a double-buffered host->device stream)."""
        if patterns.shape != self.patterns.shape or patterns.dtype != self.patterns.dtype \
                or not patterns.is_contiguous() or patterns.device != self.patterns.device:
            raise ValueError("patterns must match the engine's resident pattern array")
        self.patterns = patterns
        self.desc.patterns = patterns.data_ptr()

    def probe_changed(self) -> None:
        _lib.call('phb_engine_probe_changed', self._eref, _stream())

    def take_state(self, other: 'DeviceEngine') -> None:
        """Continue from another engine's reconstruction of the same dataset (e.g. the
        gradient engine's result handed to LSQ-ML): object, probe, scan positions and
        tilts are copied on the device."""
        for name in ('object', 'probe', 'scan'):
            mine, theirs = getattr(self, name), getattr(other, name)
            if mine.shape != theirs.shape:
                raise ValueError(f"{name} shapes differ: {tuple(mine.shape)} vs {tuple(theirs.shape)}")
            mine.copy_(theirs)
        if self.tilt is not None and other.tilt is not None:
            self.tilt.copy_(other.tilt)
        self.probe_changed()

    def group_tensor(self, flat_groups: t.Sequence[numpy.ndarray]) -> t.Tuple[torch.Tensor, t.List[int]]:
        """Upload a list of flat position-index arrays as one (G, B_max) int64 tensor."""
        G = len(flat_groups)
        host = numpy.zeros((G, self.group_max), dtype=numpy.int64)
        sizes = []
        for i, g in enumerate(flat_groups):
            if len(g) > self.group_max:
                raise ValueError(f"group of {len(g)} positions exceeds the engine's group_max {self.group_max}")
            if len(g) == 0:
                raise ValueError("empty group")
            g = numpy.asarray(g)
            if g.min() < 0 or g.max() >= self.n_pos:
                raise IndexError(f"position index out of range [0, {self.n_pos})")
            host[i, :len(g)] = g
            sizes.append(len(g))
        pinned = torch.from_numpy(host).pin_memory()
        return pinned.to(self.device, non_blocking=True), sizes

    # ---------------------------------------------------------------- steps
    def presolve(self, groups: torch.Tensor, sizes: t.Sequence[int], solver: str = 'lsqml',
                 gradient_form: bool = False) -> float:
        """Mean measured/model intensity ratio over all positions (solvers.py:36-63)."""
        if solver == 'epie' and self.N == 256 and not gradient_form:
            raise NotImplementedError("ePIE at a 256 x 256 probe (use LSQ-ML or the gradient engine)")
        G = len(sizes)
        num = torch.zeros((G, self.group_max), dtype=torch.float64, device=self.device)
        den = torch.zeros((G, self.group_max), dtype=torch.float64, device=self.device)
        for g, B in enumerate(sizes):
            _lib.call('phb_presolve_group', self._eref, groups[g].data_ptr(), B, SOLVERS[solver],
                      int(gradient_form), num[g].data_ptr(), den[g].data_ptr(), _stream())
        n_h, d_h = num.cpu().numpy(), den.cpu().numpy()
        ratios = numpy.concatenate([(n_h[g, :B] / d_h[g, :B]).astype(numpy.float32) for g, B in enumerate(sizes)])
        return float(numpy.mean(ratios))

    def step(self, solver: str, group: torch.Tensor, B: int, *, flags: int, beta_object=1.0, beta_probe=1.0,
             illum_reg_object=1e-2, illum_reg_probe=1e-2, gamma=1e-4, group_index: int = 0,
             grad_object: t.Optional[torch.Tensor] = None, grad_probe: t.Optional[torch.Tensor] = None,
             grad_pos: t.Optional[torch.Tensor] = None, loss: t.Optional[torch.Tensor] = None,
             group_patterns: t.Optional[torch.Tensor] = None, events: t.Optional[t.Tuple[int, int]] = None,
             grad_pos_scale: float = 1.0, group_loss: t.Optional[torch.Tensor] = None,
             rows: t.Optional[t.Tuple[int, int]] = None, grad_tilt: t.Optional[torch.Tensor] = None,
             grad_tilt_scale: float = 1.0) -> None:
        """One mini-batch step (phb_solver_group).  With `rows` = (b0, b1) only those
        rows of the group run (PHB_FLAG_PARTIAL): sum reduce_views() over ranks, then
        call finish()."""
        if solver == 'epie' and self.N == 256:
            raise NotImplementedError("ePIE at a 256 x 256 probe: its per-slice maximum over the modes needs all "
                                      "modes in one cluster (use LSQ-ML or the gradient engine)")
        st = self._step_struct(solver, flags, beta_object, beta_probe, illum_reg_object, illum_reg_probe, gamma,
                               group_index, grad_object, grad_probe, grad_pos, loss, group_patterns, events,
                               grad_pos_scale, group_loss, rows)
        st.grad_tilt, st.grad_tilt_scale = _ptr(grad_tilt), float(grad_tilt_scale)
        self._last_step = st
        _lib.call('phb_solver_group', self._eref, ctypes.byref(st), group.data_ptr(), int(B), _stream())

    def finish(self, group: torch.Tensor, B: int) -> None:
        """Apply the mini-batch updates from the (rank-summed) accumulators of the last
        partial step (phb_solver_group_finish)."""
        st = _lib.PhbStep.from_buffer_copy(self._last_step)
        st.flags = int(st.flags) & ~_lib.PHB_FLAG_PARTIAL
        _lib.call('phb_solver_group_finish', self._eref, ctypes.byref(st), group.data_ptr(), int(B), _stream())

    def reduce_views(self) -> t.Tuple[torch.Tensor, torch.Tensor]:
        """float32 and float64 views of the workspace accumulators a partial step fills
        (phb_engine_reduce_layout): the buffers ranks sum before `finish`."""
        out = (ctypes.c_int64 * 4)()
        _lib.call('phb_engine_reduce_layout', self.N, self.M, self.S, self.group_max, self.H, self.W, out)
        f32 = self.workspace[out[0]:out[0] + out[1]].view(torch.float32)
        f64 = self.workspace[out[2]:out[2] + out[3]].view(torch.float64)
        return f32, f64

    def _step_struct(self, solver, flags, beta_object, beta_probe, illum_reg_object, illum_reg_probe, gamma,
                     group_index, grad_object, grad_probe, grad_pos, loss, group_patterns, events, grad_pos_scale,
                     group_loss, rows) -> _lib.PhbStep:
        st = _lib.PhbStep()
        st.solver, st.flags = SOLVERS[solver], int(flags)
        st.beta_object, st.beta_probe = float(beta_object), float(beta_probe)
        st.illum_reg_object, st.illum_reg_probe, st.gamma = float(illum_reg_object), float(illum_reg_probe), float(gamma)
        st.pos_update = self.pos_update.data_ptr()
        st.errors = self.errors.data_ptr()
        st.loss = _ptr(loss)
        st.grad_object, st.grad_probe, st.grad_pos = _ptr(grad_object), _ptr(grad_probe), _ptr(grad_pos)
        st.status, st.group_index = self.status.data_ptr(), int(group_index)
        st.group_patterns = _ptr(group_patterns)
        st.grad_pos_scale, st.group_loss = float(grad_pos_scale), _ptr(group_loss)
        if events is not None:
            st.event_begin, st.event_end = events
        if rows is not None:
            st.flags = int(st.flags) | _lib.PHB_FLAG_PARTIAL
            st.b_begin, st.b_end = int(rows[0]), int(rows[1])
        return st

    def simulate(self, group: torch.Tensor, B: int, out: t.Optional[torch.Tensor] = None) -> torch.Tensor:
        """Far-field intensity of the forward model for one group, (B, N, N)."""
        if out is None:
            out = torch.empty((B, self.N, self.N), dtype=torch.float32, device=self.device)
        _lib.call('phb_simulate_group', self._eref, group.data_ptr(), int(B), out.data_ptr(), _stream())
        return out

    def position_update(self, momentum_state: t.Optional[torch.Tensor], step_size: float,
                        max_step: t.Optional[float], momentum: float) -> None:
        lo, hi = self.obj_sampling.check_bounds(numpy.asarray(self.probe_extent()) / 2.)
        _lib.call('phb_position_update', self.scan.data_ptr(), self.pos_update.data_ptr(), _ptr(momentum_state),
                  self.n_pos, int(momentum_state is not None), float(step_size),
                  float(max_step) if max_step is not None else -1.0, float(momentum),
                  float(lo[0]), float(lo[1]), float(hi[0]), float(hi[1]), self.n_outside.data_ptr(), _stream())

    def count_outside(self) -> None:
        """Positions completely outside the object -> self.n_outside (device), the bounds
        of position_update."""
        lo, hi = self.obj_sampling.check_bounds(numpy.asarray(self.probe_extent()) / 2.)
        _lib.call('phb_count_outside', self.scan.data_ptr(), self.n_pos, float(lo[0]), float(lo[1]), float(hi[0]),
                  float(hi[1]), self.n_outside.data_ptr(), _stream())

    def probe_extent(self) -> numpy.ndarray:
        return self.probe_sampling * self.N

    def iteration_reset(self) -> None:
        _lib.call('phb_iteration_reset', self.status.data_ptr(), self.errors.data_ptr(), self.n_pos, _stream())

    def iteration_report(self, out: torch.Tensor) -> None:
        """out (4,) float64 on the device: status, n_outside, nanmean(errors), count."""
        _lib.call('phb_iteration_report', self.status.data_ptr(), self.n_outside.data_ptr(), self.errors.data_ptr(),
                  self.n_pos, out.data_ptr(), _stream())

    # ---------------------------------------------------------------- host copies
    def host_state(self) -> t.Tuple[numpy.ndarray, numpy.ndarray, numpy.ndarray]:
        return (self.probe.cpu().numpy(), self.object.cpu().numpy(),
                self.scan.cpu().numpy().reshape(*self.scan_shape, 2))
