"""ctypes binding of libphaser_b200.so (the C ABI in include/phaser_b200.h).

The library is built in-tree by `phaser_b200.build`.  There is no fallback:
if the shared object is missing or a call fails, an exception is raised.

With PHASER_B200_BOUNDS_CHECK=1 in the environment the bounds-checking build
(libphaser_b200_bounds.so, same entry points) is loaded instead: its kernels
report a position index outside [0, n_pos) as PHB_STATUS_BOUNDS in the step's
status, which the engines raise as IndexError.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / 'libphaser_b200.so'
BOUNDS_LIB_PATH = _PKG / 'libphaser_b200_bounds.so'

PHB_OK = 0
PHB_ERR_INVALID_ARG = 1
PHB_ERR_UNSUPPORTED = 2
PHB_ERR_CUDA = 3
PHB_ERR_NONFINITE = 4
PHB_ERR_OUTSIDE = 5
PHB_ERR_SCRATCH_LIMIT = 6

PHB_SOLVER_LSQML = 0
PHB_SOLVER_EPIE = 1
PHB_SOLVER_GRAD = 2

PHB_NOISE_AMPLITUDE = 0
PHB_NOISE_POISSON = 1

PHB_FLAG_UPDATE_OBJECT = 1
PHB_FLAG_UPDATE_PROBE = 2
PHB_FLAG_UPDATE_POSITION = 4
PHB_FLAG_CALC_ERROR = 8
PHB_FLAG_PARTIAL = 16
PHB_FLAG_UPDATE_TILT = 32
PHB_STATUS_INTERNAL = 1 << 30
PHB_STATUS_BOUNDS = 1 << 29

c_void_p = ctypes.c_void_p
c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_f32 = ctypes.c_float
c_f64 = ctypes.c_double
c_size = ctypes.c_size_t


class PhbEngine(ctypes.Structure):
    """Mirror of `phb_engine` (include/phaser_b200.h)."""
    _fields_ = [
        ('N', c_i32), ('M', c_i32), ('S', c_i32), ('B_max', c_i32),
        ('H', c_i64), ('W', c_i64), ('n_pos', c_i64),
        ('corner_y', c_f64), ('corner_x', c_f64), ('samp_y', c_f64), ('samp_x', c_f64),
        ('object', c_void_p), ('probe', c_void_p), ('scan', c_void_p), ('tilt', c_void_p),
        ('patterns', c_void_p), ('pattern_mask', c_void_p), ('propagators', c_void_p),
        ('thicknesses', c_void_p), ('ky', c_void_p), ('kx', c_void_p),
        ('noise', c_i32), ('noise_eps', c_f32), ('noise_offset', c_f32), ('noise_var', c_f32),
        ('workspace', c_void_p), ('workspace_bytes', c_size),
        ('new_obj_mag', c_void_p), ('new_probe_mag', c_void_p),
        ('pattern_u16', c_i32),
    ]


class PhbStep(ctypes.Structure):
    """Mirror of `phb_step` (include/phaser_b200.h)."""
    _fields_ = [
        ('solver', c_i32), ('flags', c_i32),
        ('beta_object', c_f32), ('beta_probe', c_f32),
        ('illum_reg_object', c_f32), ('illum_reg_probe', c_f32), ('gamma', c_f32),
        ('pos_update', c_void_p), ('errors', c_void_p), ('loss', c_void_p),
        ('grad_object', c_void_p), ('grad_probe', c_void_p), ('grad_pos', c_void_p),
        ('status', c_void_p), ('group_index', c_i32),
        ('group_patterns', c_void_p), ('event_begin', c_void_p), ('event_end', c_void_p),
        ('grad_pos_scale', c_f32), ('group_loss', c_void_p), ('b_begin', c_i32), ('b_end', c_i32),
        ('grad_tilt', c_void_p), ('grad_tilt_scale', c_f32),
    ]


PHB_OPTIM_SGD = 0
PHB_OPTIM_ADAM = 1
PHB_OPTIM_POLYAK = 2


class PhbObjReg(ctypes.Structure):
    """Mirror of `phb_obj_reg` (include/phaser_b200.h)."""
    _fields_ = [(n, c_f32) for n in ('l1', 'l2', 'phase_l1', 'tikh', 'tv', 'tv_eps', 'layers_tikh', 'layers_tv',
                                      'scale')]


class PhbProbeReg(ctypes.Structure):
    """Mirror of `phb_probe_reg` (include/phaser_b200.h)."""
    _fields_ = [(n, c_f32) for n in ('phase_tikh', 'recip_tikh', 'recip_tv', 'tv_eps')]


class PhbOptim(ctypes.Structure):
    """Mirror of `phb_optim` (include/phaser_b200.h)."""
    _fields_ = [
        ('kind', c_i32), ('nesterov', c_i32),
        ('param', c_void_p), ('grad', c_void_p), ('state1', c_void_p), ('state2', c_void_p),
        ('update_out', c_void_p), ('n', c_i64), ('complex_elems', c_i32),
        ('grad_scale', c_f32), ('lr', c_f32), ('momentum', c_f32), ('b1', c_f32), ('b2', c_f32),
        ('eps', c_f32), ('eps_root', c_f32), ('count', c_i64), ('polyak_sq_norm', c_void_p), ('polyak_loss', c_void_p),
        ('polyak_scaling', c_f32), ('polyak_max_lr', c_f32), ('polyak_f_min', c_f32), ('polyak_eps', c_f32),
        ('status', c_void_p), ('status_code', c_i32),
    ]


# name -> (restype, argtypes)
_SIGNATURES = {
    'phb_status_string': (ctypes.c_char_p, [c_i32]),
    'phb_version': (c_i32, []),
    'phb_last_cuda_error': (ctypes.c_char_p, []),
    'phb_cutout_starts': (c_i32, [c_void_p, c_void_p, c_i64, c_f64, c_f64, c_f64, c_f64, c_i64, c_i64,
                                  c_void_p, c_void_p, c_void_p]),
    'phb_cutout_get_c64': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i64, c_i64, c_i64,
                                   c_f32, c_f32, c_void_p, c_void_p]),
    'phb_cutout_get_f32': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i64, c_i64, c_i64,
                                   c_f32, c_void_p, c_void_p]),
    'phb_cutout_add_c64': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i64, c_i64, c_i64,
                                   c_void_p, c_void_p]),
    'phb_cutout_add_f32': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i64, c_i64, c_i64,
                                   c_void_p, c_void_p]),
    'phb_cutout_set_c64': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i64, c_i64, c_i64,
                                   c_void_p, c_void_p]),
    'phb_fft2_c64': (c_i32, [c_void_p, c_void_p, c_i64, c_i64, c_i32, c_void_p]),
    'phb_clamp_amplitude_c64': (c_i32, [c_void_p, c_i64, c_f32, c_void_p]),
    'phb_fourier_mask_c64': (c_i32, [c_void_p, c_i64, c_i64, c_void_p, c_void_p]),
    'phb_engine_workspace_bytes': (c_size, [c_i32, c_i32, c_i32, c_i32, c_i64, c_i64]),
    'phb_engine_init': (c_i32, [ctypes.POINTER(PhbEngine), c_void_p]),
    'phb_engine_probe_changed': (c_i32, [ctypes.POINTER(PhbEngine), c_void_p]),
    'phb_presolve_group': (c_i32, [ctypes.POINTER(PhbEngine), c_void_p, c_i32, c_i32, c_i32,
                                   c_void_p, c_void_p, c_void_p]),
    'phb_solver_group': (c_i32, [ctypes.POINTER(PhbEngine), ctypes.POINTER(PhbStep), c_void_p, c_i32,
                                 c_void_p]),
    'phb_solver_group_static': (c_i32, [ctypes.POINTER(PhbEngine), ctypes.POINTER(PhbStep), c_void_p, c_i32,
                                        c_void_p]),
    'phb_simulate_group': (c_i32, [ctypes.POINTER(PhbEngine), c_void_p, c_i32, c_void_p, c_void_p]),
    'phb_optimizer_update': (c_i32, [ctypes.POINTER(PhbOptim), c_void_p]),
    'phb_sq_norm_f32': (c_i32, [c_void_p, c_i64, c_f32, c_void_p, c_void_p]),
    'phb_add_centred': (c_i32, [c_void_p, c_void_p, c_i64, c_void_p]),
    'phb_regularize_layers_c64': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i32, c_f32, c_void_p]),
    'phb_object_filter_scratch_bytes': (ctypes.c_size_t, [c_i64, c_i64, c_i64]),
    'phb_object_filter_c64': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_void_p, c_void_p, c_void_p]),
    'phb_remove_phase_ramp_c64': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64, c_void_p,
                                          c_void_p]),
    'phb_object_regularizers': (c_i32, [c_void_p, c_i64, c_i64, c_i64, ctypes.POINTER(PhbObjReg), c_void_p,
                                        c_void_p, c_void_p]),
    'phb_wait_probe': (c_i32, [c_i32, c_i64, c_void_p, c_void_p]),
    'phb_conv3x3_fwd': (c_i32, [c_void_p, c_void_p, c_void_p, c_void_p, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32,
                                c_i32, c_void_p]),
    'phb_conv3x3_bwd_data': (c_i32, [c_void_p, c_void_p, c_void_p, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32,
                                     c_void_p]),
    'phb_conv3x3_bwd_weight': (c_i32, [c_void_p, c_void_p, c_void_p, c_void_p, c_i32, c_i32, c_i32, c_i32, c_i32,
                                       c_i32, c_void_p]),
    'phb_relu_bwd': (c_i32, [c_void_p, c_void_p, c_i64, c_void_p]),
    'phb_upsample2': (c_i32, [c_void_p, c_void_p, c_i64, c_i32, c_i32, c_void_p]),
    'phb_upsample2_bwd': (c_i32, [c_void_p, c_void_p, c_i64, c_i32, c_i32, c_void_p]),
    'phb_mse': (c_i32, [c_void_p, c_void_p, c_void_p, c_i64, c_void_p, c_void_p]),
    'phb_to_bf16': (c_i32, [c_void_p, c_void_p, c_i64, c_void_p]),
    'phb_pattern_features': (c_i32, [c_void_p, c_void_p, c_i32, c_i32, c_i32, c_i32, c_i32, c_void_p, c_void_p]),
    'phb_patch_targets': (c_i32, [c_void_p, c_i64, c_i64, c_void_p, c_void_p, c_i32, c_f64, c_f64, c_f64, c_f64,
                                  c_i32, c_i32, c_void_p, c_void_p]),
    'phb_stitch_patches': (c_i32, [c_void_p, c_void_p, c_void_p, c_i32, c_f64, c_f64, c_f64, c_f64, c_i32, c_i32,
                                   c_void_p, c_void_p, c_void_p, c_i64, c_i64, c_void_p]),
    'phb_stitch_finish': (c_i32, [c_void_p, c_void_p, c_void_p, c_i64, c_void_p]),
    'phb_project_slices': (c_i32, [c_void_p, c_i64, c_i64, c_void_p, c_void_p]),
    'phb_resample_c64': (c_i32, [c_void_p, c_i64, c_i32, c_i32, c_void_p, c_i32, c_i32, c_f64, c_f64, c_f64, c_f64,
                                 c_f32, c_f32, c_i32, c_void_p]),
    'phb_resample_f32': (c_i32, [c_void_p, c_i64, c_i32, c_i32, c_void_p, c_i32, c_i32, c_f64, c_f64, c_f64, c_f64,
                                 c_f32, c_i32, c_void_p]),
    'phb_resample_slices_c64': (c_i32, [c_void_p, c_i32, c_i64, c_void_p, c_void_p, c_i32, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_i32, c_void_p]),
    'phb_probe_regularizers_scratch_bytes': (ctypes.c_size_t, [c_i32, c_i32]),
    'phb_probe_regularizers': (c_i32, [c_void_p, c_i32, c_i32, ctypes.POINTER(PhbProbeReg), c_void_p, c_void_p,
                                       c_void_p, c_void_p]),
    'phb_object_recip_l1_scratch_bytes': (ctypes.c_size_t, [c_i64, c_i64, c_i64]),
    'phb_object_recip_l1': (c_i32, [c_void_p, c_i64, c_i64, c_i64, c_f32, c_void_p, c_void_p, c_void_p, c_void_p]),
    'phb_engine_reduce_layout': (c_i32, [c_i32, c_i32, c_i32, c_i32, c_i64, c_i64, ctypes.POINTER(c_i64)]),
    'phb_solver_group_finish': (c_i32, [ctypes.POINTER(PhbEngine), ctypes.POINTER(PhbStep), c_void_p, c_i32,
                                        c_void_p]),
    'phb_smooth_positions_scratch_bytes': (ctypes.c_size_t, [c_i64, c_i64]),
    'phb_smooth_position_values': (c_i32, [c_void_p, c_void_p, c_i64, c_i64, c_i64, c_f64, c_f64, c_f64, c_f64,
                                           c_void_p, c_f32, c_void_p, c_void_p]),
    'phb_position_update': (c_i32, [c_void_p, c_void_p, c_void_p, c_i64, c_i32, c_f32, c_f32, c_f32,
                                    c_f64, c_f64, c_f64, c_f64, c_void_p, c_void_p]),
    'phb_nanmean': (c_i32, [c_void_p, c_i64, c_void_p, c_void_p, c_void_p]),
    'phb_iteration_reset': (c_i32, [c_void_p, c_void_p, c_i64, c_void_p]),
    'phb_count_outside': (c_i32, [c_void_p, c_i64, c_f64, c_f64, c_f64, c_f64, c_void_p, c_void_p]),
    'phb_iteration_report': (c_i32, [c_void_p, c_void_p, c_void_p, c_i64, c_void_p, c_void_p]),
    'phb_kernel_launches': (c_i64, []),
    'phb_fp32_peak': (c_i32, [c_i32, ctypes.POINTER(c_f64), ctypes.POINTER(c_f32), c_void_p]),
    'phb_event_create': (c_i32, [ctypes.POINTER(c_void_p)]),
    'phb_event_destroy': (c_i32, [c_void_p]),
    'phb_event_record': (c_i32, [c_void_p, c_void_p]),
    'phb_event_elapsed_ms': (c_i32, [c_void_p, c_void_p, ctypes.POINTER(c_f32)]),
    'phb_check_finite_c64': (c_i32, [c_void_p, c_i64, c_void_p, c_i32, c_void_p]),
}

EXPORTED = tuple(_SIGNATURES)

_lib = None


class PhbError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = _lib
        msg = lib.phb_status_string(status).decode() if lib else str(status)
        if status == PHB_ERR_CUDA and lib is not None:
            msg += f" ({lib.phb_last_cuda_error().decode()})"
        super().__init__(f"{where}: {msg}")
        self.status = status


def load(path: os.PathLike | None = None) -> ctypes.CDLL:
    """Load the shared library (once).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if path is not None:
        p = Path(path)
    else:
        p = BOUNDS_LIB_PATH if os.environ.get('PHASER_B200_BOUNDS_CHECK', '0') == '1' else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m phaser_b200.build` "
                          "(the B200 backend has no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def raise_for_status(bad_group: int) -> None:
    """Raise for a step status word read back from the device (-1: fine).  The
    flag bits say what the group index beside them produced: an aborted kernel
    program, a position index outside the scan (bounds-checking build), or NaN / inf
    in the updated object or probe (run.py:281 check_finite)."""
    if bad_group >= PHB_STATUS_INTERNAL:
        raise RuntimeError(f"internal error: fused kernel aborted in group {bad_group - PHB_STATUS_INTERNAL}")
    if bad_group >= PHB_STATUS_BOUNDS:
        raise IndexError(f"position index outside [0, n_pos) in group {bad_group - PHB_STATUS_BOUNDS}")
    if bad_group >= 0:
        raise ValueError(f"NaN or inf encountered in object or probe, group {bad_group}")


def call(name: str, *args) -> None:
    """Call an entry point that returns a status; raise PhbError unless PHB_OK."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != PHB_OK:
        raise PhbError(rc, name)
