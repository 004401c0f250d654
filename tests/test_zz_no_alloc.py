"""The allocation-free entry point (phb_solver_group_static) against the regular
workspace entry point (phb_solver_group).

phb_solver_group_static serves callers that cannot allocate device memory when
they run a step (e.g. a plugin inside an instrument-control process whose GPU
memory is owned by the host application): its scratch is a fixed 64 MiB array
inside the library.  Two consecutive mini-batches through each entry point, on
identical inputs, must agree within the tolerance of the other parity tests
(1e-5 relative L2 for object and probe; fp32 atomics reorder sums)."""
import ctypes

import numpy
import pytest
import torch

from phaser_b200 import _lib
from phaser_b200.device import DeviceEngine

from .cases import make_case

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    return float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b))


def engine(c, group_max):
    return DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                        probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                        wavelength=c.wavelength, group_max=group_max)


def static_step(eng, group, B, flags, group_index, **kw):
    """One mini-batch through the C ABI of the allocation-free entry point."""
    st = _lib.PhbStep()
    st.solver, st.flags = _lib.PHB_SOLVER_LSQML, flags
    st.beta_object, st.beta_probe = kw['beta_object'], kw['beta_probe']
    st.illum_reg_object, st.illum_reg_probe, st.gamma = 1e-2, 1e-2, 1e-4
    st.pos_update, st.errors = eng.pos_update.data_ptr(), eng.errors.data_ptr()
    st.status, st.group_index = eng.status.data_ptr(), group_index
    desc = _lib.PhbEngine.from_buffer_copy(eng.desc)
    desc.workspace, desc.workspace_bytes = None, 0          # the static entry point needs none
    _lib.call('phb_solver_group_static', ctypes.byref(desc), ctypes.byref(st), group.data_ptr(), B,
              torch.cuda.current_stream().cuda_stream)


def test_static_scratch_matches_workspace_entry_point():
    c = make_case(seed=61, N=64, M=2, S=3, scan_shape=(4, 4))
    groups = [numpy.array([0, 5, 10, 15, 3, 12], numpy.int64), numpy.array([1, 2, 4, 7, 8, 11, 13], numpy.int64)]
    flags = (_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
             | _lib.PHB_FLAG_CALC_ERROR)
    kw = dict(beta_object=0.9, beta_probe=0.8)
    ref = engine(c, 8)
    got = engine(c, 8)
    gt_ref, sizes = ref.group_tensor(groups)
    gt_got, _ = got.group_tensor(groups)
    for gi, B in enumerate(sizes):           # two calls in a row
        ref.step('lsqml', gt_ref[gi], B, flags=flags, group_index=gi, **kw)
        static_step(got, gt_got[gi], B, flags, gi, **kw)
        torch.cuda.synchronize()
        p_ref, o_ref, _ = ref.host_state()
        p_got, o_got, _ = got.host_state()
        assert rel_l2(o_got, o_ref) < 1e-5
        assert rel_l2(p_got, p_ref) < 1e-5
        idx = groups[gi]
        assert numpy.allclose(got.errors.cpu().numpy()[idx], ref.errors.cpu().numpy()[idx], rtol=1e-5)
        assert rel_l2(got.pos_update.cpu().numpy()[idx], ref.pos_update.cpu().numpy()[idx]) < 1e-4
    assert int(got.status.cpu()[0]) == -1


def test_static_scratch_rejects_problems_beyond_its_limit():
    c = make_case(seed=62, N=64, M=1, S=1, scan_shape=(2, 2))
    eng = engine(c, 4)
    desc = _lib.PhbEngine.from_buffer_copy(eng.desc)
    desc.S = 64
    desc.H = desc.W = 4096                  # 64 slices of 4096^2: far beyond 64 MiB
    st = _lib.PhbStep()
    gt, sizes = eng.group_tensor([numpy.arange(4, dtype=numpy.int64)])
    rc = _lib.load().phb_solver_group_static(ctypes.byref(desc), ctypes.byref(st), gt[0].data_ptr(), 4,
                                             torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PHB_ERR_SCRATCH_LIMIT
    # a partial (data-parallel) share would be left where the caller cannot sum it: refused
    desc = _lib.PhbEngine.from_buffer_copy(eng.desc)
    st.flags = _lib.PHB_FLAG_PARTIAL | _lib.PHB_FLAG_UPDATE_OBJECT
    st.b_begin, st.b_end = 0, 2
    rc = _lib.load().phb_solver_group_static(ctypes.byref(desc), ctypes.byref(st), gt[0].data_ptr(), 4,
                                             torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PHB_ERR_UNSUPPORTED
