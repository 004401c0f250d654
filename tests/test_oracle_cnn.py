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


def test_feature_window_is_the_centred_crop_and_flip_mirrors_k():
    rng = numpy.random.default_rng(3)
    p = rng.random((2, 16, 16)).astype(numpy.float32)
    f = C.pattern_features(p, 8, 1, False)
    sh = numpy.fft.fftshift(p, axes=(-2, -1))[:, 4:12, 4:12]
    ref = numpy.log1p(sh.astype(numpy.float64))
    assert numpy.allclose(f, ref / ref.max(axis=(1, 2), keepdims=True), atol=1e-7)
    # the mirror k -> -k of the stored pattern, read without flip, is the flipped read
    mirrored = p[:, (-numpy.arange(16)) % 16][:, :, (-numpy.arange(16)) % 16]
    assert numpy.allclose(C.pattern_features(p, 8, 1, True), C.pattern_features(mirrored, 8, 1, False))
    # 2x2 binning sums the counts before the log
    fb = C.pattern_features(p, 16, 2, False)
    sb = numpy.log1p(numpy.fft.fftshift(p, axes=(-2, -1)).astype(numpy.float64).reshape(2, 8, 2, 8, 2).sum((2, 4)))
    assert numpy.allclose(fb, sb / sb.max(axis=(1, 2), keepdims=True), atol=1e-7)


def test_stitch_averages_overlaps_and_leaves_the_rest_at_one():
    P, N = 4, 8
    pred = numpy.zeros((2, 2, P, P), numpy.float32)
    pred[0, 1] = 0.2
    pred[1, 1] = 0.4
    starts = numpy.array([[0, 0], [1, 0]])
    out = C.stitch(pred, starts, N, 12, 12)
    # patch rows 2..5 (first) and 3..6 (second), columns 2..5
    assert numpy.allclose(out[2, 2], 1 + 0.2j) and numpy.allclose(out[6, 2], 1 + 0.4j)
    assert numpy.allclose(out[3:6, 2:6], 1 + 0.3j)
    assert numpy.allclose(out[0], 1) and numpy.allclose(out[:, 8:], 1)
    w = numpy.zeros((P, P))
    w[0] = 1.0            # only each patch's first row counts
    outw = C.stitch(pred, starts, N, 12, 12, w)
    assert numpy.allclose(outw[2, 2], 1 + 0.2j) and numpy.allclose(outw[3, 2], 1 + 0.4j)
    assert numpy.allclose(outw[4, 2], 1)    # weight zero everywhere there
