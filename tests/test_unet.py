"""The U-Net oracle (CPU) and the BF16 U-Net kernels against it (GPU).

CPU: the oracle's backward pass against central finite differences in
float64 (no bf16 rounding), and the flipped-weight identity used for the
data gradient.  GPU: every kernel of libsmili_unet.so against the oracle on
bf16-representable inputs (tolerance: a few bf16 ulps, since the GPU
accumulates in float32 and rounds its outputs to bf16); every layer of a
full forward/backward pass on the GPU's own stored inputs; and the whole
chain against the oracle's own bf16 chain (3 % on the gradient vector).
"""
import numpy as np
import pytest

from oracle import unet_oracle as U


def _ident(x):
    return np.asarray(x, np.float64)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    c = (4, 4, 8, 8)
    P = {k: (w.astype(np.float64), rng.standard_normal(w.shape[0]) * 0.1)
         for k, (w, b) in U.init_params(rng, c).items()}
    x = rng.standard_normal((1, 16, 16, 1))
    R = rng.standard_normal((1, 16, 16, 1))

    def loss(params):
        out, _ = U.unet_forward(params, x, rnd=_ident)
        return float(np.sum(out * R))

    _, A = U.unet_forward(P, x, rnd=_ident)
    G = U.unet_backward(P, A, R, rnd=_ident)
    h = 1e-6
    for name in ("e1a", "e2b", "ba", "d3a", "d1a", "head"):
        w, b = P[name]
        for _ in range(3):
            idx = tuple(rng.integers(0, s) for s in w.shape)
            wp, wm = w.copy(), w.copy()
            wp[idx] += h
            wm[idx] -= h
            fd = (loss({**P, name: (wp, b)}) - loss({**P, name: (wm, b)})) / (2 * h)
            assert abs(G[name][0][idx] - fd) <= 1e-5 * max(1.0, abs(fd)), (name, idx)
        j = int(rng.integers(0, b.size))
        bp, bm = b.copy(), b.copy()
        bp[j] += h
        bm[j] -= h
        fd = (loss({**P, name: (w, bp)}) - loss({**P, name: (w, bm)})) / (2 * h)
        assert abs(G[name][1][j] - fd) <= 1e-5 * max(1.0, abs(fd)), (name, "bias")


def test_flip_weights_gives_data_gradient():
    rng = np.random.default_rng(1)
    w = rng.standard_normal((5, 3, 3, 7))
    dy = rng.standard_normal((2, 9, 11, 5))
    np.testing.assert_allclose(U.conv3x3(dy, U.flip_weights(w)), U.conv3x3_dgrad(dy, w), rtol=1e-12, atol=1e-12)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0], np.float32)
    r = U.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie rounds to even
    assert r[2] == np.float32(1.0078125)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)


# --------------------------------------------------------------------- GPU
def _bf16_tensor(a):
    import torch
    return torch.as_tensor(np.asarray(U.bf16(a), np.float32)).to(torch.bfloat16).cuda()


def _np(t):
    return t.float().cpu().numpy()


def _close_bf16(got, want, ulps=2.0):
    """|got - want| <= ulps bf16 ulps of max(|want|, 1e-3 max|want|)."""
    want = np.asarray(want, np.float64)
    scale = np.maximum(np.abs(want), 1e-3 * np.max(np.abs(want)) + 1e-30)
    return np.max(np.abs(got - want) / scale) <= ulps * 2.0 ** -8


@pytest.mark.gpu
@pytest.mark.parametrize("N,H,W,Cin,Cout,relu", [(2, 16, 16, 1, 24, True), (1, 24, 40, 24, 24, True),
                                                 (2, 8, 16, 72, 24, False), (1, 16, 16, 288, 96, True),
                                                 (1, 8, 8, 192, 192, True), (2, 16, 32, 24, 1, False),
                                                 (1, 10, 18, 20, 12, True)])
def test_conv3x3_kernel(N, H, W, Cin, Cout, relu):
    import torch
    from smili_b200.warmstart import kernels as K
    rng = np.random.default_rng(N * 1000 + Cin)
    x = U.bf16(rng.standard_normal((N, H, W, Cin)))
    w = U.bf16(rng.standard_normal((Cout, 3, 3, Cin)) / np.sqrt(9 * Cin))
    b = rng.standard_normal(Cout).astype(np.float32)
    y = torch.zeros((N, H, W, Cout), dtype=torch.bfloat16, device="cuda")
    K.conv3x3(_bf16_tensor(x), N, H, W, Cin, Cin, _bf16_tensor(w), torch.as_tensor(b).cuda(), y, Cout, Cout, relu)
    want = U.conv3x3(x, w, b, relu)
    assert _close_bf16(_np(y), want)
    # accumulate into an existing output
    y0 = U.bf16(rng.standard_normal((N, H, W, Cout)))
    y = _bf16_tensor(y0)
    K.conv3x3(_bf16_tensor(x), N, H, W, Cin, Cin, _bf16_tensor(w), None, y, Cout, Cout, False, accumulate=True)
    assert _close_bf16(_np(y), U.conv3x3(x, w) + y0, ulps=3.0)


@pytest.mark.gpu
def test_conv3x3_channel_slices():
    """Read a channel slice of a wider buffer and write into another."""
    import torch
    from smili_b200.warmstart import kernels as K
    rng = np.random.default_rng(3)
    N, H, W = 2, 16, 16
    big = U.bf16(rng.standard_normal((N, H, W, 72)))
    w = U.bf16(rng.standard_normal((24, 3, 3, 24)) / 15)
    out = torch.zeros((N, H, W, 96), dtype=torch.bfloat16, device="cuda")
    K.conv3x3((_bf16_tensor(big), 48), N, H, W, 24, 72, _bf16_tensor(w), None, (out, 24), 96, 24, False)
    got = _np(out)
    assert _close_bf16(got[..., 24:48], U.conv3x3(big[..., 48:72], w))
    assert np.all(got[..., :24] == 0) and np.all(got[..., 48:] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("N,H,W,Cin,Cout", [(4, 128, 128, 24, 24), (4, 64, 64, 48, 48), (4, 32, 32, 96, 96),
                                            (4, 16, 16, 192, 192), (4, 32, 32, 288, 96), (2, 24, 40, 48, 300),
                                            (1, 8, 8, 16, 8)])
def test_conv3x3_tcgen05_matches_mma_sync(N, H, W, Cin, Cout):
    """The tcgen05 path (TMA-staged operands, accumulator in tensor memory)
    against the mma.sync path and the oracle on the U-Net's layer shapes,
    two output-channel tiles (Cout 300) and a ragged image (24 x 40); no
    bounded wait inside the kernel runs out."""
    import torch
    from smili_b200.warmstart import kernels as K
    rng = np.random.default_rng(H * 7 + Cin)
    x = U.bf16(rng.standard_normal((N, H, W, Cin)))
    w = U.bf16(rng.standard_normal((Cout, 3, 3, Cin)) / np.sqrt(9 * Cin))
    b = rng.standard_normal(Cout).astype(np.float32)
    xt, wt, bt = _bf16_tensor(x), _bf16_tensor(w), torch.as_tensor(b).cuda()
    outs = []
    try:
        for path in (0, 2, 1):  # tcgen05 (two 128-pixel tiles per CTA where H >= 16), tcgen05 (one), mma.sync
            K.set_conv_path(path)
            y = torch.zeros((N, H, W, Cout), dtype=torch.bfloat16, device="cuda")
            K.conv3x3(xt, N, H, W, Cin, Cin, wt, bt, y, Cout, Cout, True)
            torch.cuda.synchronize()
            outs.append(_np(y))
    finally:
        K.set_conv_path(0)
    assert K.tc_status() == 0
    want = U.conv3x3(x, w, b, True)
    # both accumulate the same products in FP32 (in another order) and round once to bf16
    for o in outs:
        assert _close_bf16(o, want)


@pytest.mark.gpu
@pytest.mark.parametrize("N,H,W,Cin,Cout", [(2, 16, 16, 1, 24), (2, 32, 32, 24, 24), (1, 16, 16, 288, 96),
                                            (2, 8, 8, 96, 192), (1, 12, 20, 20, 1), (3, 24, 40, 144, 48),
                                            (2, 16, 16, 72, 24), (1, 8, 16, 48, 96)])
def test_conv3x3_wgrad_kernel(N, H, W, Cin, Cout):
    import torch
    from smili_b200.warmstart import kernels as K
    rng = np.random.default_rng(Cin + Cout)
    x = U.bf16(rng.standard_normal((N, H, W, Cin)))
    dy = U.bf16(rng.standard_normal((N, H, W, Cout)))
    nsplit = 7
    partial = torch.zeros(nsplit * Cout * 9 * Cin, dtype=torch.float32, device="cuda")
    dw = torch.zeros(Cout * 9 * Cin, dtype=torch.float32, device="cuda")
    want = U.conv3x3_wgrad(x, dy)
    try:
        for path in (0, 1):  # tcgen05 (where the channel counts allow), then mma.sync
            K.set_conv_path(path)
            K.conv3x3_wgrad(_bf16_tensor(x), Cin, _bf16_tensor(dy), Cout, N, H, W, Cin, Cout, partial, nsplit, dw)
            got = dw.cpu().numpy().reshape(want.shape)
            assert np.max(np.abs(got - want)) <= 1e-4 * np.max(np.abs(want)), path
    finally:
        K.set_conv_path(0)
    assert K.tc_status() == 0
    db = torch.zeros(Cout, dtype=torch.float32, device="cuda")
    K.bias_grad(_bf16_tensor(dy), Cout, N * H * W, Cout, db)
    np.testing.assert_allclose(db.cpu().numpy(), dy.reshape(-1, Cout).sum(0), rtol=1e-4, atol=1e-3)


@pytest.mark.gpu
def test_elementwise_kernels():
    import torch
    from smili_b200.warmstart import kernels as K
    rng = np.random.default_rng(4)
    N, H, W, C = 2, 16, 24, 40
    x = U.bf16(rng.standard_normal((N, H, W, C)))
    y = torch.zeros((N, H // 2, W // 2, C), dtype=torch.bfloat16, device="cuda")
    K.avgpool2(_bf16_tensor(x), C, y, C, N, H, W, C)
    assert _close_bf16(_np(y), U.avgpool2(x), ulps=1.0)
    dy = U.bf16(rng.standard_normal((N, H // 2, W // 2, C)))
    dx = _bf16_tensor(x)
    K.avgpool2_bwd(_bf16_tensor(dy), C, dx, C, N, H, W, C, accumulate=True)
    assert _close_bf16(_np(dx), x + U.avgpool2_bwd(dy), ulps=1.0)
    up = torch.zeros((N, 2 * H, 2 * W, C), dtype=torch.bfloat16, device="cuda")
    K.upsample2(_bf16_tensor(x), C, up, C, N, H, W, C)
    assert np.array_equal(_np(up), U.upsample2(x))
    d2 = U.bf16(rng.standard_normal((N, 2 * H, 2 * W, C)))
    g = torch.zeros((N, H, W, C), dtype=torch.bfloat16, device="cuda")
    K.upsample2_bwd(_bf16_tensor(d2), C, g, C, N, H, W, C)
    assert _close_bf16(_np(g), U.upsample2_bwd(d2), ulps=1.0)
    m = _bf16_tensor(d2)
    K.relu_mask(_bf16_tensor(np.maximum(d2, 0)), C, m, C, N * 4 * H * W, C)
    assert np.array_equal(_np(m), np.where(d2 > 0, d2, 0))
    wt = torch.zeros(7 * 9 * 5, dtype=torch.bfloat16, device="cuda")
    w = U.bf16(rng.standard_normal((5, 3, 3, 7)))
    K.flip_weights(_bf16_tensor(w), wt, 5, 7)
    assert np.array_equal(_np(wt).reshape(7, 3, 3, 5), U.flip_weights(w))
    # mse and adam
    out = U.bf16(rng.standard_normal((N, H, W, 1)))
    t = rng.standard_normal((N, H, W)).astype(np.float32)
    dout = torch.zeros((N, H, W, 1), dtype=torch.bfloat16, device="cuda")
    part = torch.zeros(64, dtype=torch.float32, device="cuda")
    K.mse(_bf16_tensor(out), 1, torch.as_tensor(t).cuda(), N * H * W, dout, 1, part, 64)
    loss, grad = U.mse(out[..., 0], t)
    assert abs(float(part.sum()) - loss) <= 1e-5 * loss
    assert _close_bf16(_np(dout)[..., 0], grad, ulps=1.0)
    n = 1000
    w0, g0 = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m0, v0 = np.zeros(n), np.zeros(n)
    wt_, mt, vt = torch.as_tensor(w0).cuda(), torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")
    w16 = torch.zeros(n, dtype=torch.bfloat16, device="cuda")
    K.adam(wt_, w16, torch.as_tensor(g0).cuda(), mt, vt, n, 1e-2, 0.9, 0.999, 1e-8, 1e-4, 1)
    wr, _, _ = U.adam(w0.astype(np.float64), g0.astype(np.float64), m0, v0, 1, 1e-2, wd=1e-4)
    np.testing.assert_allclose(wt_.cpu().numpy(), wr, rtol=1e-5, atol=1e-6)
    assert np.array_equal(_np(w16), U.bf16(wt_.cpu().numpy()))


def _unet_run(seed=11, B=2, H=32, W=32):
    import torch
    from smili_b200.warmstart.unet import UNet
    net = UNet(seed=seed)
    rng = np.random.default_rng(seed + 1)
    x = U.bf16(rng.standard_normal((B, H, W)).astype(np.float32))
    t = rng.standard_normal((B, H, W)).astype(np.float32)
    net.forward(torch.as_tensor(x).cuda())
    net.loss(t)
    dout = _np(net.D["out"])
    net.backward()
    torch.cuda.synchronize()
    return net, x, dout


def _grads(net):
    grad = net.grad.cpu().numpy()
    out, o = {}, 0
    for L in net.layers:
        gw = grad[o:o + L.nw].reshape(L.cout, 3, 3, L.cin)
        o += L.nw
        out[L.name] = (gw, grad[o:o + L.cout])
        o += L.cout
    return out


@pytest.mark.gpu
def test_unet_layers_match_oracle():
    """Every layer of a full forward/backward pass, checked on the GPU's own
    stored inputs: outputs, weight and bias gradients, data gradients."""
    net, x, dout = _unet_run()
    P = net.params_bf16()
    A = {k: _np(v) for k, v in net.A.items()}
    D = {k: _np(v) for k, v in net.D.items()}
    G = _grads(net)
    c1, c2, c3, c4 = net.c
    # (layer, its input, its stored output)
    fwd = [("e1a", A["x"], A["e1a"]), ("e1b", A["e1a"], A["cat1"][..., c2:]),
           ("e2a", A["p1"], A["e2a"]), ("e2b", A["e2a"], A["cat2"][..., c3:]),
           ("e3a", A["p2"], A["e3a"]), ("e3b", A["e3a"], A["cat3"][..., c4:]),
           ("ba", A["p3"], A["ba"]), ("bb", A["ba"], A["bb"]),
           ("d3a", A["cat3"], A["d3a"]), ("d3b", A["d3a"], A["d3b"]),
           ("d2a", A["cat2"], A["d2a"]), ("d2b", A["d2a"], A["d2b"]),
           ("d1a", A["cat1"], A["d1a"]), ("d1b", A["d1a"], A["d1b"]), ("head", A["d1b"], A["out"])]
    relu = {L.name: L.relu for L in net.layers}
    for name, xin, yout in fwd:
        w, b = P[name]
        assert _close_bf16(yout, U.conv3x3(xin, w, b, relu[name]), ulps=2.0), name
    assert _close_bf16(A["p1"], U.avgpool2(A["cat1"][..., c2:]), ulps=1.0)
    assert np.array_equal(A["cat3"][..., :c4], U.upsample2(A["bb"]))
    # backward: (layer, input, masked output gradient as stored)
    dys = {"head": D["out"], "d1b": D["d1b"], "d1a": D["d1a"], "d2b": D["d2b"], "d2a": D["d2a"],
           "d3b": D["d3b"], "d3a": D["d3a"], "bb": D["bb"], "ba": D["ba"], "e3b": D["cat3"][..., c4:],
           "e3a": D["e3a"], "e2b": D["cat2"][..., c3:], "e2a": D["e2a"], "e1b": D["cat1"][..., c2:],
           "e1a": D["e1a"]}
    for name, xin, _ in fwd:
        dy = dys[name]
        ww = U.conv3x3_wgrad(xin, dy)
        gw, gb = G[name]
        assert np.max(np.abs(gw - ww)) <= 1e-3 * np.max(np.abs(ww)) + 1e-30, name
        wb = dy.reshape(-1, dy.shape[-1]).sum(0)
        assert np.max(np.abs(gb - wb)) <= 1e-3 * np.max(np.abs(wb)) + 1e-30, name
    # data gradients that are not modified after they are written (masked by
    # the consumer's ReLU where it has one)
    chain = [("head", "d1b"), ("d1b", "d1a"), ("d2b", "d2a"), ("d3b", "d3a"), ("bb", "ba")]
    for name, nxt in chain:
        want = U.conv3x3_dgrad(dys[name], P[name][0])
        want = np.where(A[nxt] > 0, want, 0.0)
        assert _close_bf16(D[nxt], want, ulps=3.0), name
    want = U.conv3x3_dgrad(dys["d1a"], P["d1a"][0])[..., :c2]
    assert _close_bf16(D["cat1"][..., :c2], want, ulps=3.0)
    assert _close_bf16(D["d2b"], np.where(A["d2b"] > 0, U.upsample2_bwd(D["cat1"][..., :c2]), 0), ulps=3.0)


@pytest.mark.gpu
def test_unet_gradients_match_oracle():
    """The whole chain against the oracle's own bf16 forward/backward from the
    same input and weights.  Independent rounding in two 15-layer chains
    (1-ulp flips, ReLU boundaries) compounds, so the bound is 3 % on the whole
    gradient vector and 10 % per layer."""
    net, x, dout = _unet_run()
    P = net.params_bf16()
    want_out, A = U.unet_forward(P, x[..., None])
    got_out = _np(net.A["out"])
    assert np.linalg.norm(got_out - want_out) / np.linalg.norm(want_out) < 1e-2
    G = U.unet_backward(P, A, dout)
    got = _grads(net)
    allg, allw = [], []
    for L in net.layers:
        for k in range(2):
            g, w = got[L.name][k].ravel(), G[L.name][k].ravel()
            assert np.linalg.norm(g - w) <= 0.1 * np.linalg.norm(w) + 1e-30, (L.name, k)
            allg.append(g)
            allw.append(w)
    g, w = np.concatenate(allg), np.concatenate(allw)
    assert np.linalg.norm(g - w) <= 0.03 * np.linalg.norm(w)
