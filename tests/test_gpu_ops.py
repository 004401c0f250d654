"""GPU parity of the array-level kernels against the numpy oracle.

Tolerances: integer work (cutout indices, gathers) is compared bit-exactly;
FFTs within 2e-6 relative L2 (float32 transform error); scatter-adds within
float32 atomic-reordering noise (atol 1e-5 on O(1) values)."""
import numpy
import pytest
import torch
from numpy.testing import assert_array_equal, assert_allclose

from oracle import phaser_np as P
from phaser_b200 import numerics as X
from phaser_b200.sampling import ObjectSampling

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    return float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b))


@pytest.fixture(scope='module')
def dev():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device('cuda')


@pytest.mark.parametrize('N', [64, 128, 256])
def test_fft2_ifft2_match_oracle(dev, N):
    rng = numpy.random.default_rng(N)
    a = (rng.normal(size=(5, N, N)) + 1j * rng.normal(size=(5, N, N))).astype(numpy.complex64)
    t = torch.from_numpy(a).to(dev)
    f = X.fft2(t).cpu().numpy()
    assert rel_l2(f, P.fft2c(a)) < 2e-6
    g = X.ifft2(t).cpu().numpy()
    assert rel_l2(g, P.ifft2c(a)) < 2e-6
    back = X.ifft2(X.fft2(t)).cpu().numpy()
    assert rel_l2(back, a) < 2e-6


@pytest.mark.parametrize('N', [64, 128, 256])
def test_fft2_known_answers(dev, N):
    # centred delta -> constant; constant -> corner delta (reference tests/test_num.py:102-155)
    a = numpy.zeros((1, N, N), numpy.complex64)
    a[0, N // 2, N // 2] = N
    f = X.fft2(torch.from_numpy(a).to(dev)).cpu().numpy()
    assert_allclose(f, numpy.ones_like(a), atol=1e-5)
    c = numpy.full((1, N, N), 1 + 1j, numpy.complex64)
    g = X.fft2(torch.from_numpy(c).to(dev)).cpu().numpy()
    expect = numpy.zeros_like(c)
    expect[0, 0, 0] = N * (1 + 1j)
    assert_allclose(g, expect, atol=1e-4)


def test_cutout_starts_bit_exact(dev):
    rng = numpy.random.default_rng(7)
    osamp = ObjectSampling((300, 280), (0.21, 0.19), (-30.3, -25.1))
    pos = rng.uniform(-25, 25, (4000, 2)).astype(numpy.float32)
    # exact half-index positions exercise round-half-to-even
    idx = numpy.arange(-20, 20)
    half = numpy.stack([osamp.corner[0] + (idx + 63.5 + 0.5) * osamp.sampling[0],
                        osamp.corner[1] + (idx + 63.5) * osamp.sampling[1]], -1).astype(numpy.float32)
    pos = numpy.concatenate([pos, half])
    for shape in [(128, 128), (64, 64), (5, 4)]:
        starts, subpx = X.cutout_starts(osamp, torch.from_numpy(pos).to(dev), shape, with_subpx=True)
        assert_array_equal(starts.cpu().numpy(), P.cutout_starts(pos, osamp.corner, osamp.sampling, shape))
        assert_array_equal(subpx.cpu().numpy(),
                           P.subpx_shifts(pos, osamp.corner, osamp.sampling, shape).astype(numpy.float32))


def test_cutout_get_add_set(dev):
    rng = numpy.random.default_rng(11)
    obj = (rng.normal(size=(3, 90, 100)) + 1j * rng.normal(size=(3, 90, 100))).astype(numpy.complex64)
    starts = numpy.array([[0, 0], [-5, 10], [40, 60], [70, 85], [-30, -40], [10, 95]], numpy.int64)
    shape = (32, 32)
    t_obj = torch.from_numpy(obj).to(dev)
    t_st = torch.from_numpy(starts).to(dev)
    got = X.get_cutouts(t_obj, t_st, shape, fill=1.0).cpu().numpy()
    assert_array_equal(got, P.get_cutouts(obj, starts, shape, fill=1))      # OOB reads 1
    views = (rng.normal(size=(6, 3, 32, 32)) + 1j * rng.normal(size=(6, 3, 32, 32))).astype(numpy.complex64)
    added = X.add_cutouts(t_obj.clone(), t_st, torch.from_numpy(views).to(dev)).cpu().numpy()
    assert_allclose(added, P.add_cutouts(obj.copy(), starts, views), rtol=0, atol=1e-5)
    # set: non-overlapping views are deterministic
    st2 = numpy.array([[0, 0], [40, 50]], numpy.int64)
    v2 = views[:2]
    out = X.set_cutouts(t_obj.clone(), torch.from_numpy(st2).to(dev), torch.from_numpy(v2).to(dev)).cpu().numpy()
    ref = obj.copy()
    for (y, x), v in zip(st2, v2):
        ref[:, y:y + 32, x:x + 32] = v
    assert_array_equal(out, ref)
    # float32 variants
    fo = rng.normal(size=(1, 50, 60)).astype(numpy.float32)
    gf = X.get_cutouts(torch.from_numpy(fo).to(dev), t_st, (16, 16), fill=0.0).cpu().numpy()
    assert_array_equal(gf, P.get_cutouts(fo, starts, (16, 16), fill=0))
