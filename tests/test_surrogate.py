"""The control-variate surrogate's BF16 kernels (csrc/jms_nn.cu): forward
values and gradients against the FP64 restatement in oracle/nn_oracle.py,
training, and the control-variate estimate itself."""
import numpy as np
import pytest

from oracle import nn_oracle as N


def test_oracle_gradients_by_finite_differences():
    """The restatement's backward passes are the derivatives of its forward passes."""
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 3, 8, 8))
    w = rng.normal(size=(4, 3, 3, 3))
    b = rng.normal(size=4)
    t = rng.normal(size=(2, 4, 4, 4))
    y = N.conv_fwd(x, w, b)
    dx, dw, db = N.conv_bwd(x, w, y, y - t)

    def loss(x, w, b):
        return 0.5 * ((N.conv_fwd(x, w, b) - t) ** 2).sum()

    eps = 1e-6
    for arr, g in ((w, dw), (x, dx), (b, db)):
        for _ in range(5):
            idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
            a0 = arr[idx]
            arr[idx] = a0 + eps
            lp = loss(x, w, b)
            arr[idx] = a0 - eps
            lm = loss(x, w, b)
            arr[idx] = a0
            assert abs((lp - lm) / (2 * eps) - g[idx]) < 1e-5 * max(1.0, abs(g[idx]))
    h = rng.normal(size=(3, 5, 4, 4))
    wl = rng.normal(size=(6, 5))
    bl = rng.normal(size=6)
    tt = rng.normal(size=(3, 6))
    _, do = N.mse(N.pool_linear_fwd(h, wl, bl), tt)
    dh, dwl, dbl = N.pool_linear_bwd(h, wl, do)
    for arr, g in ((h, dh), (wl, dwl), (bl, dbl)):
        idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
        a0 = arr[idx]
        arr[idx] = a0 + eps
        lp = N.mse(N.pool_linear_fwd(h, wl, bl), tt)[0]
        arr[idx] = a0 - eps
        lm = N.mse(N.pool_linear_fwd(h, wl, bl), tt)[0]
        arr[idx] = a0
        assert abs((lp - lm) / (2 * eps) - g[idx]) < 1e-7


def test_bf16_rounding_ties_to_even():
    v = N.bf16_round(np.array([1.0, 1.00390625, 1.005859375, -2.0 ** -130, 3.0e38]))
    assert v[0] == 1.0 and v[1] == 1.0 and v[2] == 1.0078125
    assert v[3] == -(2.0 ** -130) and np.isfinite(v[4])


def _f(t):
    return t.float().cpu().numpy().astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("relu,cin,size", [(True, 3, 64), (False, 10, 16)])
def test_kernels_match_oracle(relu, cin, size):
    """Forward activations within one BF16 rounding, every gradient within
    FP32 accumulation error, computed from the kernels' own stored activations;
    the network of the default inputs (ReLU, 3 x 64 x 64) and the linear one on
    10 depth bins x 16 x 16."""
    import torch

    from jmultislicelib_b200 import surrogate as SG

    B, nout = 4, 30
    net = SG.SurrogateNet(nout, B, seed=3, cin=cin, size=size, relu=relu)
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.normal(size=(B, cin, size, size)).astype(np.float32)).cuda().to(torch.bfloat16)
    t = torch.from_numpy(rng.normal(size=(B, nout)).astype(np.float32)).cuda()
    net.backward(x, t, B)
    torch.cuda.synchronize()
    h = _f(x)
    for k in range(len(net.conv)):
        w = _f(net.bf[k])
        b = _f(net.params[2 * k + 1])
        y_gpu = _f(net.act[k])
        y_ref = N.bf16_round(N.conv_fwd(h, w, b, relu=relu))
        # the FP32 and FP64 sums round to the same BF16 value except next to a tie
        assert np.abs(y_gpu - y_ref).max() <= 2.0 ** -7 * np.abs(y_ref).max()
        assert (y_gpu != y_ref).mean() < 1e-3
        h = y_gpu
    wl, bl = _f(net.params[-2]), _f(net.params[-1])
    out = N.pool_linear_fwd(h, wl, bl)
    np.testing.assert_allclose(_f(net.out[:B]), out, rtol=1e-5, atol=1e-6)
    loss, dout = N.mse(out, _f(t))
    assert abs(float(net.loss.item()) - loss) < 1e-5 * max(loss, 1.0)
    dh, dwl, dbl = N.pool_linear_bwd(h, wl, dout)
    np.testing.assert_allclose(_f(net.grads[-2]), dwl, rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(_f(net.grads[-1]), dbl, rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(_f(net.dact[-1][:B]), dh, rtol=1e-4, atol=1e-9)
    g = dh
    for k in reversed(range(len(net.conv))):
        xin = _f(x) if k == 0 else _f(net.act[k - 1])
        w = _f(net.bf[k])
        y = _f(net.act[k])
        g_in = _f(net.dact[k][:B])      # what the kernels propagated into this layer
        scale = np.abs(g).max()
        assert np.abs(g_in - g).max() <= 1e-4 * scale
        dx, dw, db = N.conv_bwd(xin, w, y, g_in, relu=relu)
        np.testing.assert_allclose(_f(net.grads[2 * k]), dw, rtol=1e-3, atol=1e-5 * np.abs(dw).max())
        np.testing.assert_allclose(_f(net.grads[2 * k + 1]), db, rtol=1e-3, atol=1e-5 * np.abs(db).max())
        g = dx


@pytest.mark.gpu
def test_training_fits_a_smooth_target():
    """Adam on the BF16 kernels fits outputs that depend on the patch content."""
    from jmultislicelib_b200 import surrogate as SG

    rng = np.random.default_rng(7)
    n = 1024
    X = rng.normal(size=(n, 3, 64, 64)).astype(np.float32)
    X[:, :, 24:40, 24:40] += rng.normal(size=(n, 3, 1, 1)).astype(np.float32) * 3.0
    feat = X[:, :, 24:40, 24:40].mean(axis=(2, 3))
    Y = np.stack([feat[:, 0], feat[:, 1] - feat[:, 2], np.abs(feat[:, 2])], 1)
    cv = SG.ControlVariate(3, batch=128, seed=2)
    hist = cv.fit(X[:896], Y[:896], X[896:], Y[896:], epochs=15, lr=2e-3)
    assert min(h[1] for h in hist) < 0.25 * hist[0][1]
    assert np.all(np.abs(cv.beta - 1.0) < 0.3)
    pred = cv.predict(X[:256])
    assert np.corrcoef(pred[:, 0], Y[:256, 0])[0, 1] > 0.9


def test_patches_are_c_ordered_and_centred():
    """The kernels read inputs as C-ordered [n][C][H][W]: patches() must return
    that layout (a strided view fed to them reads scrambled values)."""
    from jmultislicelib_b200 import surrogate as SG

    rng = np.random.default_rng(2)
    maps = rng.normal(size=(3, 40, 48))
    pos = np.array([[0.25, 0.5], [1.0, 1.75]], np.float32)
    for pool in (1, 4):
        p = SG.patches(maps, pos, 2.0, 2.0, window=16, pool=pool)
        assert p.flags["C_CONTIGUOUS"] and p.shape == (2, 3, 16 // pool, 16 // pool)
    p = SG.patches(maps, pos, 2.0, 2.0, window=16)
    px, py = int(round(0.25 / 2.0 * 48)), int(round(0.5 / 2.0 * 40))
    assert p[0, 1, 8, 8] == maps[1, py, px]          # window centred on the probe pixel
    q = SG.patches(maps, pos, 2.0, 2.0, window=16, pool=4)
    np.testing.assert_allclose(q[0, 2, 0, 0], p[0, 2, :4, :4].mean())


@pytest.mark.gpu
def test_device_patches_match_host_patches():
    """JMS_NnPatches against channel_maps + patches on a small specimen:
    depth bins of unequal length, windows that wrap around the cell."""
    from jmultislicelib_b200 import surrogate as SG
    from jmultislicelib_b200 import synthetic as S

    sp = S.make_specimen(96, 80, 2, 2, 2, 3, 5, 300.0, keep_potential=True)
    nobj, nbins = 11, 3
    rng = np.random.default_rng(4)
    pos = np.stack([rng.uniform(0, sp.a, 7), rng.uniform(0, sp.b, 7)], 1).astype(np.float32)
    var = rng.integers(0, 3, (5, nobj)).astype(np.int32)
    for window, pool in ((64, 4), (32, 1)):
        dev = SG.DevicePatches(sp, nobj, 2, pos, nbins, window=window, pool=pool)(var).cpu().numpy()
        host = np.stack([SG.patches(SG.channel_maps(sp, nobj, 2, v, nbins), pos, sp.a, sp.b, window=window, pool=pool)
                         for v in var])
        np.testing.assert_allclose(dev, host, rtol=2e-5, atol=2e-6 * np.abs(host).max())


def test_cv_estimate_is_the_control_variate_formula():
    from jmultislicelib_b200 import surrogate as SG

    rng = np.random.default_rng(1)
    f = rng.normal(size=(64, 5, 3))
    g = f + 0.1 * rng.normal(size=f.shape)
    est = SG.cv_estimate(f[:4], g[:4], g)
    np.testing.assert_allclose(est, g.mean(axis=0) + (f[:4] - g[:4]).mean(axis=0))
    # with a perfect surrogate the estimate is the full mean; beta = 0 is the plain mean
    np.testing.assert_allclose(SG.cv_estimate(f[:4], f[:4], f), f.mean(axis=0))
    np.testing.assert_allclose(SG.cv_estimate(f[:4], g[:4], g, 0.0), f[:4].mean(axis=0))


@pytest.mark.gpu
def test_control_variate_on_a_small_scan():
    """End to end on a 128^2 specimen: signals from the library's multislice,
    depth-binned potential patches (one bin per readout interval), training on
    the library's BF16 kernels, beta fitted on held-out configurations, and the
    variance of f - beta g on configurations the network never saw: the
    trained network must remove most of the phonon variance there."""
    import torch

    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import surrogate as SG
    from jmultislicelib_b200 import synthetic as S

    nx = ny = 128
    nobj, nvar, ncell = 24, 8, 2
    sp = S.make_specimen(nx, ny, ncell, ncell, 2, nvar, 11, 300.0, keep_potential=True)
    J = jb.JMS()
    J.cleanup()
    J.set_high_tension(300.0)
    J.set_grid(nx, ny, sp.a, sp.b, S.DZ_SLICE)
    pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, 1)
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
    probe = J.calc_probe(22.0)
    assert J.setup(2, [nvar, nvar], np.arange(nobj) % 2, [0, 0], 8, 3, 1) == [0, 0, 0, 0]
    for s_, gr in enumerate(sp.gratings):
        assert J.set_phase_grating(2, s_, gr) == 0
    assert J.set_propagator(2, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(2, i, d, m) == 0
    assert J.init_core(2) == 0
    assert J.set_incident_wave(2, probe) == 0
    planes = list(range(1, J.num_det_planes()))
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, sp.a, (96, 2)).astype(np.float32)
    d_pos = torch.from_numpy(pos).cuda()
    cfgs = rng.integers(0, nvar, (40, nobj)).astype(np.int32)
    nbins = len(planes)
    X = np.stack([SG.patches(SG.channel_maps(sp, nobj, 2, v, nbins), pos, sp.a, sp.b, pool=4)
                  for v in cfgs]).astype(np.float32)
    Y = np.stack([SG.signals(J, d_pos, len(pos), v, planes) for v in cfgs])
    X -= X.mean(axis=0, keepdims=True)
    Y -= Y.mean(axis=0, keepdims=True)
    nout = Y.shape[-1]
    F = Y[32:]                                   # evaluation configurations (deviations)
    # measured: 0.085 (linear network) and 0.24 (ReLU); a least-squares fit of
    # the same inputs reaches 0.07
    for relu, bar in ((False, 0.3), (True, 0.5)):
        cv = SG.ControlVariate(nout, batch=64, seed=1, cin=nbins, size=SG.PATCH // 4, relu=relu)
        hist = cv.fit(X[8:32].reshape(-1, *X.shape[2:]), Y[8:32].reshape(-1, nout),
                      X[:8].reshape(-1, *X.shape[2:]), Y[:8].reshape(-1, nout), epochs=20)
        assert len(hist) == 20 and np.all(np.isfinite(cv.beta))
        G = cv.predict(X[32:].reshape(-1, *X.shape[2:])).reshape(F.shape)
        ratio = (F - cv.beta * G).var(axis=0).mean() / F.var(axis=0).mean()
        print("control-variate variance ratio on the small scan (relu %s): %.3f" % (relu, ratio))
        assert ratio < bar, (relu, ratio)
