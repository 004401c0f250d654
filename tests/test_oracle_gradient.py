"""The oracle's hand-written adjoint of the gradient-engine model against
central finite differences of the oracle's loss, in float64 (CPU only).

The loss itself is pinned to the reference's noise models by
test_oracle_golden.py; jax (the reference's gradient backend) is not installed
here, so the adjoint is pinned by finite differences (step 1e-3 relative on
random object pixels and probe pixels, and on positions)."""
import numpy
import pytest

from oracle import phaser_np as P

from .cases import make_case


def f64_case(seed, **kw):
    c = make_case(seed, **kw)
    return (c, c.probe.astype(numpy.complex128), c.obj.astype(numpy.complex128),
            c.patterns.reshape(-1, *c.probe.shape[-2:]).astype(numpy.float64))


def geom64(c):
    N = c.probe.shape[-1]
    ky, kx = P.recip_grid((N, N), c.probe_sampling, numpy.float64)
    return P.Geometry(numpy.asarray(c.osamp.corner), numpy.asarray(c.osamp.sampling), ky, kx, c.thick), ky, kx


@pytest.mark.parametrize('noise', [P.NoiseModel(eps=1e-2), P.NoiseModel(kind='poisson', eps=1e-3)], ids=['amp', 'poisson'])
def test_adjoint_matches_finite_differences(noise):
    c, probe, obj, pats = f64_case(71, N=32, M=2, S=3, scan_shape=(3, 3), samp=0.3, dz=15.0)
    g, ky, kx = geom64(c)
    props = P.make_propagators(ky, kx, c.probe_sampling, c.wavelength, c.thick)
    scan = c.scan.reshape(-1, 2).astype(numpy.float64)
    mask = c.mask.astype(numpy.float64)

    def loss(o=obj, p=probe, sc=scan):
        return float(P.grad_model_loss(g, p, o, sc, pats, mask, props, None, noise))

    L, g_obj, g_probe, g_pos = P.grad_model_grads(g, probe, obj, scan, pats, mask, props, None, noise)
    assert L == pytest.approx(loss(), rel=1e-12)
    rng = numpy.random.default_rng(5)
    h = 1e-3
    # object pixels inside the scanned region (where the gradient is non-zero)
    S, H, W = obj.shape
    checked = 0
    for _ in range(64):
        s, y, x = rng.integers(S), rng.integers(H // 4, 3 * H // 4), rng.integers(W // 4, 3 * W // 4)
        for part, unit in ((0, 1.0), (1, 1j)):
            op, om = obj.copy(), obj.copy()
            op[s, y, x] += h * unit
            om[s, y, x] -= h * unit
            fd = (loss(o=op) - loss(o=om)) / (2 * h)
            an = g_obj[s, y, x].real if part == 0 else g_obj[s, y, x].imag
            assert fd == pytest.approx(an, rel=2e-4, abs=1e-6 * max(1.0, abs(L)))
            checked += 1
    assert checked == 128
    for _ in range(16):
        m, y, x = rng.integers(probe.shape[0]), rng.integers(8, 24), rng.integers(8, 24)
        for part, unit in ((0, 1.0), (1, 1j)):
            pp, pm = probe.copy(), probe.copy()
            pp[m, y, x] += h * unit * abs(probe).max()
            pm[m, y, x] -= h * unit * abs(probe).max()
            fd = (loss(p=pp) - loss(p=pm)) / (2 * h * abs(probe).max())
            an = g_probe[m, y, x].real if part == 0 else g_probe[m, y, x].imag
            assert fd == pytest.approx(an, rel=2e-4, abs=1e-6 * max(1.0, abs(L)))
    for b in range(scan.shape[0]):
        for d in range(2):
            sp, sm = scan.copy(), scan.copy()
            sp[b, d] += 1e-4
            sm[b, d] -= 1e-4
            fd = (loss(sc=sp) - loss(sc=sm)) / 2e-4
            # skip positions whose integer cutout start changes within +-h
            if (P.cutout_starts(sp[b], g.corner, g.obj_sampling, probe.shape) ==
                    P.cutout_starts(sm[b], g.corner, g.obj_sampling, probe.shape)).all():
                assert fd == pytest.approx(g_pos[b, d], rel=1e-4, abs=1e-6 * max(1.0, abs(L)))


def test_tilt_adjoint_matches_finite_differences():
    c, probe, obj, pats = f64_case(73, N=32, M=2, S=3, scan_shape=(2, 2), samp=0.3, dz=15.0)
    g, ky, kx = geom64(c)
    props = P.make_propagators(ky, kx, c.probe_sampling, c.wavelength, c.thick)
    scan = c.scan.reshape(-1, 2).astype(numpy.float64)
    mask = c.mask.astype(numpy.float64)
    tilts = numpy.random.default_rng(4).normal(0, 3.0, (4, 2))
    noise = P.NoiseModel(kind='poisson', eps=1e-3)

    def loss(t_):
        return float(P.grad_model_loss(g, probe, obj, scan, pats, mask, props, t_, noise))

    *_, g_tilt = P.grad_model_grads(g, probe, obj, scan, pats, mask, props, tilts, noise, with_tilt=True)
    h = 1e-3
    for i in range(4):
        for j in range(2):
            tp, tm = tilts.copy(), tilts.copy()
            tp[i, j] += h
            tm[i, j] -= h
            fd = (loss(tp) - loss(tm)) / (2 * h)
            assert fd == pytest.approx(g_tilt[i, j], rel=1e-4, abs=1e-8)
