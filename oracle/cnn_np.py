"""numpy restatement of the warm-start network's layers and of its training
step, which the GPU kernels are tested against.  TEST INFRASTRUCTURE:
only tests/ and the benchmark's baseline code import this module.

The warm start has no counterpart in the reference (it is this backend's
addition), so there is no reference file to cite; the layer definitions are
the standard ones: 3x3 convolution with zero padding 1 and stride s
(out[y, x] = b + sum w[ci, ky, kx] in[ci, s y + ky - 1, s x + kx - 1]), ReLU,
nearest-neighbour 2x upsampling, mean squared error."""
from __future__ import annotations

import numpy


def bf16(x: numpy.ndarray) -> numpy.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    u = numpy.ascontiguousarray(x, numpy.float32).view(numpy.uint32).astype(numpy.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(numpy.uint32).view(numpy.float32)


def _patches(x: numpy.ndarray, stride: int) -> numpy.ndarray:
    """(N, C, H, W) -> (N, C, 3, 3, H/s, W/s) input taps of every output pixel."""
    N, C, H, W = x.shape
    xp = numpy.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    Ho, Wo = H // stride, W // stride
    out = numpy.empty((N, C, 3, 3, Ho, Wo), x.dtype)
    for ky in range(3):
        for kx in range(3):
            out[:, :, ky, kx] = xp[:, :, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride]
    return out


def conv3x3(x, w, b, stride: int = 1, relu: bool = False):
    """x (N, Ci, H, W), w (Co, Ci, 3, 3), b (Co) -> (N, Co, H/s, W/s)."""
    p = _patches(x, stride)
    y = numpy.einsum('ncklhw,ockl->nohw', p, w, optimize=True) + b[None, :, None, None]
    return numpy.maximum(y, 0) if relu else y


def conv3x3_backward(x, w, dy, stride: int = 1):
    """Gradients (dx, dw, db) of sum(dy * conv3x3(x, w, b, stride))."""
    p = _patches(x, stride)
    dw = numpy.einsum('nohw,ncklhw->ockl', dy, p, optimize=True)
    db = dy.sum(axis=(0, 2, 3))
    dp = numpy.einsum('nohw,ockl->ncklhw', dy, w, optimize=True)
    N, C, H, W = x.shape
    dxp = numpy.zeros((N, C, H + 2, W + 2), x.dtype)
    Ho, Wo = H // stride, W // stride
    for ky in range(3):
        for kx in range(3):
            dxp[:, :, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride] += dp[:, :, ky, kx]
    return dxp[:, :, 1:-1, 1:-1], dw, db


def upsample2(x):
    return x.repeat(2, axis=-2).repeat(2, axis=-1)


def upsample2_backward(g):
    N, C, H, W = g.shape
    return g.reshape(N, C, H // 2, 2, W // 2, 2).sum(axis=(3, 5))


# (in, out, stride, relu, upsample after)
LAYERS = ((1, 32, 2, True, False), (32, 64, 2, True, False), (64, 64, 1, True, True),
          (64, 32, 1, True, False), (32, 2, 1, False, False))


def forward(params, x, quantize: bool = True):
    """Network output and the activations the backward pass needs (weights
    rounded to bfloat16 as the kernels use them unless quantize=False)."""
    q = bf16 if quantize else (lambda v: v)
    acts = [x]
    h = x
    for (ci, co, s, relu, up), (w, b) in zip(LAYERS, params):
        h = conv3x3(h, q(w), b, s, relu)
        acts.append(h)
        if up:
            h = upsample2(h)
            acts.append(h)
    return h, acts


def loss_and_grads(params, x, target, quantize: bool = True):
    """Mean squared error and its gradients with respect to every (w, b)
    (the bfloat16 rounding of the weights passes gradients straight through)."""
    q = bf16 if quantize else (lambda v: v)
    y, acts = forward(params, x, quantize)
    n = y.size
    loss = float(numpy.sum((y - target).astype(numpy.float64) ** 2) / n)
    g = 2.0 * (y - target) / n
    grads = []
    k = len(acts) - 1
    for (ci, co, s, relu, up), (w, b) in reversed(list(zip(LAYERS, params))):
        if up:
            g = upsample2_backward(g)
            k -= 1
        out = acts[k]
        if relu:
            g = g * (out > 0)
        inp = acts[k - 1]
        gx, gw, gb = conv3x3_backward(inp, q(w), g, s)
        grads.append((gw, gb))
        g = gx
        k -= 1
    return loss, grads[::-1]


def pattern_features(pats, crop: int, bin: int, flip: bool):
    """log(1 + I) over the crop x crop window centred on zero frequency of patterns
    (B, N, N) stored with zero frequency at [0, 0], binned bin x bin, mirrored k -> -k
    when flip, scaled to a maximum of 1 per pattern: (B, crop/bin, crop/bin)."""
    B, N = pats.shape[0], pats.shape[-1]
    k = numpy.arange(crop) - crop // 2          # frequency of each window pixel
    if flip:
        k = -k
    rows = (k + N) % N
    win = numpy.maximum(pats, 0)[:, rows][:, :, rows].astype(numpy.float64)
    F = crop // bin
    binned = win.reshape(B, F, bin, F, bin).sum(axis=(2, 4))
    v = numpy.log1p(binned)
    mx = v.max(axis=(1, 2), keepdims=True)
    return numpy.where(mx > 0, v / numpy.where(mx > 0, mx, 1), 0).astype(numpy.float32)


def stitch(pred, starts, N: int, H: int, W: int, window=None):
    """Patches pred (B, 2, P, P) = (Re - 1, Im) placed at the centred P x P of each
    N x N cutout (top-left `starts` (B, 2)), averaged with per-pixel weights `window`
    (P, P; uniform when None); 1 where no patch lands."""
    B, _, P, _ = pred.shape
    off = (N - P) // 2
    w = numpy.ones((P, P)) if window is None else numpy.asarray(window, numpy.float64)
    acc = numpy.zeros((H, W), numpy.complex128)
    wgt = numpy.zeros((H, W))
    for b in range(B):
        y0, x0 = int(starts[b, 0]) + off, int(starts[b, 1]) + off
        ys, xs = numpy.arange(y0, y0 + P), numpy.arange(x0, x0 + P)
        my, mx = (ys >= 0) & (ys < H), (xs >= 0) & (xs < W)
        v = (pred[b, 0] + 1.0) + 1j * pred[b, 1]
        sub = numpy.ix_(ys[my], xs[mx])
        acc[sub] += (w * v)[numpy.ix_(my, mx)]
        wgt[sub] += w[numpy.ix_(my, mx)]
    return numpy.where(wgt > 0, acc / numpy.where(wgt > 0, wgt, 1), 1.0).astype(numpy.complex64)
