"""The oracle's warm-start network layers against float64 central finite
differences (CPU only), and its bfloat16 rounding against torch's."""
import numpy
import pytest
import torch

from oracle import cnn_np as C


@pytest.mark.parametrize('stride', [1, 2])
def test_conv_backward_matches_finite_differences(stride):
    rng = numpy.random.default_rng(stride)
    x = rng.normal(size=(2, 3, 6, 6))
    w = rng.normal(size=(4, 3, 3, 3))
    b = rng.normal(size=4)
    dy = rng.normal(size=(2, 4, 6 // stride, 6 // stride))
    dx, dw, db = C.conv3x3_backward(x, w, dy, stride)

    def f(x_=x, w_=w, b_=b):
        return float(numpy.sum(dy * C.conv3x3(x_, w_, b_, stride)))
    h = 1e-6
    for arr, grad in ((x, dx), (w, dw), (b, db)):
        for _ in range(6):
            i = tuple(rng.integers(s) for s in arr.shape)
            p, m = arr.copy(), arr.copy()
            p[i] += h
            m[i] -= h
            args = {id(x): 'x_', id(w): 'w_', id(b): 'b_'}
            fd = (f(**{args[id(arr)]: p}) - f(**{args[id(arr)]: m})) / (2 * h)
            assert fd == pytest.approx(grad[i], rel=1e-6, abs=1e-8)


def test_network_gradients_match_finite_differences():
    rng = numpy.random.default_rng(5)
    params = [(rng.normal(0, 0.3, (co, ci, 3, 3)), rng.normal(0, 0.1, co)) for (ci, co, *_r) in C.LAYERS]
    x = rng.uniform(size=(2, 1, 16, 16))
    t = rng.normal(size=(2, 2, 8, 8))
    loss, grads = C.loss_and_grads(params, x, t, quantize=False)
    h = 1e-6
    for li in (0, 2, 4):
        w, b = params[li]
        for _ in range(4):
            i = tuple(rng.integers(s) for s in w.shape)
            wp, wm = w.copy(), w.copy()
            wp[i] += h
            wm[i] -= h
            lp = C.loss_and_grads([*params[:li], (wp, b), *params[li + 1:]], x, t, quantize=False)[0]
            lm = C.loss_and_grads([*params[:li], (wm, b), *params[li + 1:]], x, t, quantize=False)[0]
            assert (lp - lm) / (2 * h) == pytest.approx(grads[li][0][i], rel=1e-5, abs=1e-9)


def test_bf16_rounding_matches_torch():
    x = numpy.random.default_rng(0).normal(size=10000).astype(numpy.float32) * 10
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert numpy.array_equal(C.bf16(x), ref)
