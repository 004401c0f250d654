"""The warm-start network's CUDA kernels against the numpy oracle
(oracle/cnn_np.py, itself checked against finite differences on the CPU).

Weights are rounded to bfloat16 in both; accumulation is float32 on the GPU
and float64 in the oracle: layer outputs and gradients within 1e-5 relative
L2, the whole network's loss within 1e-5 and its gradients within 1e-4."""
import numpy
import pytest
import torch

from oracle import cnn_np as C
from phaser_b200 import _lib
from phaser_b200.warmstart import WarmStartNet

from .test_gpu_engine import rel_l2

pytestmark = pytest.mark.gpu


def st():
    return torch.cuda.current_stream().cuda_stream


def bf16_tensor(w):
    q = torch.empty(w.shape, dtype=torch.bfloat16, device='cuda')
    wt = torch.from_numpy(w.astype(numpy.float32)).cuda()
    _lib.call('phb_to_bf16', wt.data_ptr(), q.data_ptr(), wt.numel(), st())
    return q


# 32 / 64 output (forward) or input (data gradient, stride 1 and 2) channels run on the
# tensor cores (tcgen05 implicit GEMM, 128-pixel tiles, 16-channel reduction chunks), and
# so does the weight gradient with 17..64 output channels (a GEMM reducing over pixels);
# the others on the FP32 pipe.  Partial pixel tiles (B H^2 not a multiple of 128) and
# partial / several reduction chunks are included.
@pytest.mark.parametrize('ci,co,stride,H', [(1, 32, 2, 64), (32, 64, 2, 32), (64, 64, 1, 16), (64, 32, 1, 32),
                                            (32, 2, 1, 32), (3, 5, 1, 20), (5, 17, 2, 18), (6, 20, 1, 40),
                                            (7, 33, 1, 34), (7, 32, 1, 10), (40, 64, 2, 14), (32, 48, 1, 12),
                                            (64, 40, 2, 16)])
def test_conv_layer_matches_oracle(ci, co, stride, H):
    rng = numpy.random.default_rng(ci * 100 + co)
    B = 3
    x = rng.normal(size=(B, ci, H, H)).astype(numpy.float32)
    w = rng.normal(0, 0.3, (co, ci, 3, 3)).astype(numpy.float32)
    b = rng.normal(0, 0.1, co).astype(numpy.float32)
    dy = rng.normal(size=(B, co, H // stride, H // stride)).astype(numpy.float32)
    wq = C.bf16(w)
    xd, bd, dyd = (torch.from_numpy(a).cuda() for a in (x, b, dy))
    q = bf16_tensor(w)
    y = torch.empty((B, co, H // stride, H // stride), device='cuda')
    _lib.call('phb_conv3x3_fwd', xd.data_ptr(), q.data_ptr(), bd.data_ptr(), y.data_ptr(), B, ci, H, H, co, stride,
              1, st())
    ref = C.conv3x3(x.astype(numpy.float64), wq.astype(numpy.float64), b.astype(numpy.float64), stride, relu=True)
    assert rel_l2(y.cpu().numpy(), ref) < 1e-5
    dx = torch.empty_like(xd)
    dw = torch.zeros((co, ci, 3, 3), device='cuda')
    db = torch.zeros((co,), device='cuda')
    _lib.call('phb_conv3x3_bwd_data', dyd.data_ptr(), q.data_ptr(), dx.data_ptr(), B, ci, H, H, co, stride, st())
    _lib.call('phb_conv3x3_bwd_weight', xd.data_ptr(), dyd.data_ptr(), dw.data_ptr(), db.data_ptr(), B, ci, H, H, co,
              stride, st())
    rdx, rdw, rdb = C.conv3x3_backward(x.astype(numpy.float64), wq.astype(numpy.float64), dy.astype(numpy.float64),
                                       stride)
    assert rel_l2(dx.cpu().numpy(), rdx) < 1e-5
    assert rel_l2(dw.cpu().numpy(), rdw) < 1e-5
    assert rel_l2(db.cpu().numpy(), rdb) < 1e-5


# The weight gradient with Ci <= 64 and 17..64 output channels runs on the tensor cores at
# stride 1 and 2, CTAs striding over (image, 128-row tile) chunks: batches large enough that
# every CTA takes several chunks (both operand buffers reused); 2 and 9 output channels run
# the FP32 kernel.
@pytest.mark.parametrize('ci,co,H,B,stride', [(64, 32, 32, 40, 1), (32, 2, 64, 12, 1), (64, 64, 16, 64, 1),
                                              (20, 9, 24, 48, 1), (20, 17, 24, 48, 1), (3, 40, 20, 40, 1),
                                              (32, 64, 32, 64, 2), (1, 32, 64, 24, 2), (24, 20, 30, 48, 2)])
def test_weight_gradient_many_chunks(ci, co, H, B, stride):
    rng = numpy.random.default_rng(ci * 7 + co)
    x = rng.normal(size=(B, ci, H, H)).astype(numpy.float32)
    dy = rng.normal(size=(B, co, H // stride, H // stride)).astype(numpy.float32)
    w = C.bf16(rng.normal(0, 0.3, (co, ci, 3, 3)).astype(numpy.float32))
    xd, dyd = torch.from_numpy(x).cuda(), torch.from_numpy(dy).cuda()
    dw = torch.zeros((co, ci, 3, 3), device='cuda')
    db = torch.zeros((co,), device='cuda')
    _lib.call('phb_conv3x3_bwd_weight', xd.data_ptr(), dyd.data_ptr(), dw.data_ptr(), db.data_ptr(), B, ci, H, H, co,
              stride, st())
    _, rdw, rdb = C.conv3x3_backward(x.astype(numpy.float64), w.astype(numpy.float64), dy.astype(numpy.float64),
                                     stride)
    assert rel_l2(dw.cpu().numpy(), rdw) < 1e-5
    assert rel_l2(db.cpu().numpy(), rdb) < 1e-5


def test_network_loss_and_gradients_match_oracle():
    net = WarmStartNet(seed=3)
    rng = numpy.random.default_rng(4)
    for b in net.b:
        b.copy_(torch.from_numpy(rng.normal(0, 0.05, b.shape[0]).astype(numpy.float32)))
    x = rng.uniform(size=(4, 1, 64, 64)).astype(numpy.float32)
    t = rng.normal(0, 0.1, (4, 2, 32, 32)).astype(numpy.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = net.forward(xd)
    gy = torch.empty_like(y)
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    _lib.call('phb_mse', y.data_ptr(), td.data_ptr(), gy.data_ptr(), y.numel(), loss.data_ptr(), st())
    net.backward(gy)
    params = [(w.astype(numpy.float64), b.astype(numpy.float64)) for (w, b) in net.numpy_params()]
    ref_loss, ref_grads = C.loss_and_grads(params, x.astype(numpy.float64), t.astype(numpy.float64))
    assert float(loss.cpu()[0]) == pytest.approx(ref_loss, rel=1e-5)
    for (gw, gb), (rw, rb) in zip(zip(net.gw, net.gb), ref_grads):
        assert rel_l2(gw.cpu().numpy(), rw) < 1e-4
        assert rel_l2(gb.cpu().numpy(), rb) < 1e-4


def test_bounded_wait_gives_up_and_the_context_stays_usable():
    """The tensor-core kernels' mbarrier waits are bounded: on a barrier that nothing
    completes the wait gives up after its limit and reports it (no hang, no fault); the
    same wait sees a completed phase at once; a tensor-core layer runs afterwards."""
    out = torch.full((1,), -1, dtype=torch.int32, device='cuda')
    _lib.call('phb_wait_probe', 0, 4096, out.data_ptr(), st())
    assert int(out.cpu()[0]) == 0
    _lib.call('phb_wait_probe', 1, 4096, out.data_ptr(), st())
    assert int(out.cpu()[0]) == 1
    rng = numpy.random.default_rng(8)
    x = rng.normal(size=(2, 64, 16, 16)).astype(numpy.float32)
    w = rng.normal(0, 0.3, (64, 64, 3, 3)).astype(numpy.float32)
    b = numpy.zeros(64, numpy.float32)
    xd, bd = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
    y = torch.empty((2, 64, 16, 16), device='cuda')
    _lib.call('phb_conv3x3_fwd', xd.data_ptr(), bf16_tensor(w).data_ptr(), bd.data_ptr(), y.data_ptr(), 2, 64, 16, 16,
              64, 1, 1, st())
    ref = C.conv3x3(x.astype(numpy.float64), C.bf16(w).astype(numpy.float64), b.astype(numpy.float64), 1, relu=True)
    assert rel_l2(y.cpu().numpy(), ref) < 1e-5


def test_upsample_and_relu_kernels():
    rng = numpy.random.default_rng(6)
    x = torch.from_numpy(rng.normal(size=(2, 3, 5, 7)).astype(numpy.float32)).cuda()
    up = torch.empty((2, 3, 10, 14), device='cuda')
    _lib.call('phb_upsample2', x.data_ptr(), up.data_ptr(), 6, 5, 7, st())
    assert torch.equal(up.cpu(), torch.from_numpy(C.upsample2(x.cpu().numpy())))
    g = torch.from_numpy(rng.normal(size=(2, 3, 10, 14)).astype(numpy.float32)).cuda()
    gin = torch.empty_like(x)
    _lib.call('phb_upsample2_bwd', g.data_ptr(), gin.data_ptr(), 6, 5, 7, st())
    assert numpy.allclose(gin.cpu().numpy(), C.upsample2_backward(g.cpu().numpy()), rtol=1e-6, atol=1e-6)
    g2 = g.clone()
    _lib.call('phb_relu_bwd', g2.data_ptr(), up.data_ptr(), g2.numel(), st())
    assert torch.equal(g2.cpu(), (g * (up > 0)).cpu())


@pytest.mark.parametrize('N,crop,bin,flip', [(128, 64, 1, True), (128, 64, 1, False), (128, 128, 2, False),
                                             (64, 64, 1, True), (128, 96, 3, True)])
def test_pattern_features_match_oracle(N, crop, bin, flip):
    rng = numpy.random.default_rng(N + crop + bin + flip)
    B = 5
    pats = rng.poisson(50.0, (B + 2, N, N)).astype(numpy.float32)
    pats[0, :3, :3] = -1.0                          # negative counts are clamped to zero
    index = numpy.array([6, 0, 3, 3, 1], numpy.int64)
    F = crop // bin
    out = torch.empty((B, F, F), dtype=torch.float32, device='cuda')
    p = torch.from_numpy(pats).cuda()
    it = torch.from_numpy(index).cuda()
    _lib.call('phb_pattern_features', p.data_ptr(), it.data_ptr(), B, N, crop, bin, int(flip), out.data_ptr(), st())
    ref = C.pattern_features(pats[index], crop, bin, flip)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-6


def test_pattern_features_reject_bad_windows():
    p = torch.zeros((1, 64, 64), dtype=torch.float32, device='cuda')
    out = torch.empty((1, 64, 64), dtype=torch.float32, device='cuda')
    for crop, bin in ((128, 1), (63, 1), (64, 3), (0, 1)):
        with pytest.raises(_lib.PhbError):
            _lib.call('phb_pattern_features', p.data_ptr(), None, 1, 64, crop, bin, 0, out.data_ptr(), st())


@pytest.mark.parametrize('windowed', [False, True])
def test_stitch_matches_oracle(windowed):
    from oracle import phaser_np as O
    from phaser_b200.warmstart import stitch_window
    rng = numpy.random.default_rng(7 + windowed)
    N, P, H, W, B = 64, 32, 90, 100, 40
    corner, samp = numpy.array([-9.0, -10.0]), numpy.array([0.2, 0.2])
    # positions spread past every edge of the object: patches are clipped there
    scan = rng.uniform([-14.0, -15.0], [14.0, 15.0], (B, 2)).astype(numpy.float32)
    pred = rng.normal(0, 0.2, (B, 2, P, P)).astype(numpy.float32)
    win = stitch_window(4.0).numpy() if windowed else None
    acc = torch.zeros((H, W), dtype=torch.complex64, device='cuda')
    wgt = torch.zeros((H, W), dtype=torch.float32, device='cuda')
    pt, sc = torch.from_numpy(pred).cuda(), torch.from_numpy(scan).cuda()
    wt = None if win is None else torch.from_numpy(win).cuda()
    _lib.call('phb_stitch_patches', pt.data_ptr(), sc.data_ptr(), None, B, corner[0], corner[1], samp[0], samp[1],
              N, P, None if wt is None else wt.data_ptr(), acc.data_ptr(), wgt.data_ptr(), H, W, st())
    obj = torch.empty_like(acc)
    _lib.call('phb_stitch_finish', acc.data_ptr(), wgt.data_ptr(), obj.data_ptr(), H * W, st())
    starts = O.cutout_starts(scan.astype(numpy.float64), corner, samp, (N, N))
    ref = C.stitch(pred, starts, N, H, W, win)
    assert rel_l2(obj.cpu().numpy(), ref) < 1e-6
