"""Learned initial guess: the CPU oracle pinned by finite differences, the GPU
kernels and the whole network's gradients against the oracle, and a small
training run showing what the trained network saves over a zero guess."""
import numpy as np
import pytest

import cnn_oracle as co


def _weights(rng, scale=1.0):
    W = {}
    for name, ci, cout, relu in co.LAYERS:
        std = scale * (2.0 / (27 * ci)) ** 0.5
        W[name] = (rng.standard_normal((cout, 27, ci)) * std, rng.standard_normal(cout) * 0.1)
    return W


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    W = _weights(rng)
    net = co.Net(W, bf16=False)
    x0 = rng.standard_normal((1, 8, 8, 8, 16))
    tgt = rng.standard_normal((1, 8, 8, 8))
    A = net.forward(x0)
    G = net.backward(A, tgt)
    eps = 1e-6
    for name, idx in [("out", (0, 13, 5)), ("d0a", (3, 4, 40)), ("b2", (17, 26, 100)), ("e0a", (2, 0, 1)),
                      ("e2b", (10, 13, 7)), ("d2a", (5, 2, 150))]:
        w = net.w[name][0]
        old = w[idx]
        w[idx] = old + eps
        lp = net.loss(net.forward(x0), tgt)
        w[idx] = old - eps
        lm = net.loss(net.forward(x0), tgt)
        w[idx] = old
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - G[name][0][idx]) <= 1e-6 * max(1.0, abs(fd)), (name, fd, G[name][0][idx])
    # bias of a middle layer
    b = net.w["d1b"][1]
    old = b[3]
    b[3] = old + eps
    lp = net.loss(net.forward(x0), tgt)
    b[3] = old - eps
    lm = net.loss(net.forward(x0), tgt)
    b[3] = old
    assert abs((lp - lm) / (2 * eps) - G["d1b"][1][3]) <= 1e-6


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], np.float32)
    r = co.to_bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5


# ---------------------------------------------------------------- GPU kernels
def _bf(t):
    import torch
    return torch.from_numpy(co.to_bf16(t)).to(torch.bfloat16).cuda()


def _np(t):
    import torch
    torch.cuda.synchronize()
    return t.float().cpu().numpy().astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(2, 8, 8, 8), (1, 6, 10, 12), (1, 4, 16, 24)])
@pytest.mark.parametrize("cin,cout", [(16, 16), (48, 64), (32, 48), (16, 128)])
@pytest.mark.parametrize("kernel", ["box", "tile", "tcgen05"])
def test_conv3d_matches_oracle(gpu, dims, cin, cout, kernel):
    import torch
    import learned
    L = learned.klib()
    old = L.xcnn_set_box_conv(int(kernel == "box"))
    old_tc = L.xcnn_set_tc_conv(int(kernel == "tcgen05"))
    rng = np.random.default_rng(cin * 7 + cout)
    nb, d, h, w = dims
    # input window: channels [16, 16 + cin) of a buffer with cin + 32 channels
    cs = cin + 32
    xin = co.to_bf16(rng.standard_normal((nb, d, h, w, cs)))
    wt = co.to_bf16(rng.standard_normal((cout, 27, cin)) * 0.2)
    bias = rng.standard_normal(cout).astype(np.float32)
    ref = co.conv3d(xin[..., 16:16 + cin], wt, bias)
    X, Wd, Bd = _bf(xin), _bf(wt), torch.from_numpy(bias).cuda()
    ocs = cout + 16
    for flags in (0, 1, 2):
        prev = co.to_bf16(rng.standard_normal((nb, d, h, w, ocs)))
        O = _bf(prev)
        rc = L.xcnn_conv3d(learned._p(X), cs, 16, cin, learned._p(Wd), learned._p(Bd), learned._p(O), ocs, 16,
                           cout, nb, d, h, w, flags, None)
        assert rc == 0
        got = _np(O)
        exp = ref.copy()
        if flags & 1:
            exp = np.maximum(exp, 0)
        if flags & 2:
            exp = exp + prev[..., 16:16 + cout]
        exp = co.to_bf16(exp)
        # FP32 accumulation order and one-ulp BF16 rounding differences only
        tol = 2 ** -7 * np.maximum(np.abs(exp), 1e-3) + 1e-4 * np.abs(ref).max()
        assert np.all(np.abs(got[..., 16:16 + cout] - exp) <= tol), flags
        assert np.array_equal(got[..., :16], prev[..., :16])  # outside the window untouched
    # FP32 output (the prediction layer)
    O = torch.zeros((nb, d, h, w, ocs), dtype=torch.float32, device="cuda")
    assert L.xcnn_conv3d(learned._p(X), cs, 16, cin, learned._p(Wd), learned._p(Bd), learned._p(O), ocs, 16, cout,
                         nb, d, h, w, 4, None) == 0
    got = _np(O)[..., 16:16 + cout]
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    assert L.xcnn_tc_error() == 0
    L.xcnn_set_box_conv(old)
    L.xcnn_set_tc_conv(old_tc)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout", [(16, 16), (48, 32), (192, 64), (64, 128)])
def test_conv3d_wgrad_matches_oracle(gpu, cin, cout):
    import torch
    import learned
    L = learned.klib()
    rng = np.random.default_rng(cin + cout)
    nb, d, h, w = 2, 8, 6, 10
    x = co.to_bf16(rng.standard_normal((nb, d, h, w, cin)))
    g = co.to_bf16(rng.standard_normal((nb, d, h, w, cout)))
    ref = co.conv3d_wgrad(x, g)
    dw = torch.zeros((cout, 27, cin), device="cuda")
    assert L.xcnn_conv3d_wgrad(learned._p(_bf(x)), cin, 0, cin, learned._p(_bf(g)), cout, 0, cout,
                               learned._p(dw), nb, d, h, w, None) == 0
    got = _np(dw)
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.gpu
def test_network_gradients_match_oracle(gpu):
    """Full forward + backward of the GPU network against the BF16-emulating
    oracle on a 16^3 batch of four."""
    import torch
    import learned
    torch.manual_seed(0)
    net = learned.Net(seed=5)
    rng = np.random.default_rng(9)
    nb, n = 4, 16
    a = rng.standard_normal((nb, n, n, n)).astype(np.float32)
    b = rng.standard_normal((nb, n, n, n)).astype(np.float32)
    tgt = rng.standard_normal((nb, n, n, n)).astype(np.float32)
    ta, tb, tt = (torch.from_numpy(v).cuda() for v in (a, b, tgt))
    B = net._bufs(nb, n)
    net.pack(B, ta, tb)
    net.forward(B)
    loss = net.loss_and_grad(B, tt)
    net.zero_grad()
    net.backward(B)
    torch.cuda.synchronize()
    W = {name: (net.wbf[name].float().cpu().numpy(), net.b32[name].cpu().numpy()) for name, *_ in learned.LAYERS}
    onet = co.Net(W, bf16=True)
    x0 = np.zeros((nb, n, n, n, 16), np.float32)
    x0[..., 0], x0[..., 1] = a, b
    A = onet.forward(x0)
    out = _np(B["out"])
    assert np.abs(out - A["out"]).max() <= 0.02 * np.abs(A["out"]).max()
    assert abs(float(loss.item()) - onet.loss(A, tgt)) <= 1e-3 * onet.loss(A, tgt)
    G = onet.backward(A, tgt)
    # BF16 rounding of the activation gradients differs by an ulp here and
    # there (FP32 sums in another order) and the differences grow towards the
    # bottom of the network; a wrong index or a missing path gives O(1) errors
    errs = {}
    for name, *_ in learned.LAYERS:
        gw = net.gw[name].cpu().numpy()
        rw = G[name][0]
        gb = net.gb[name].cpu().numpy()
        rb = G[name][1]
        if name == "e0a":
            gw, rw = gw[:, :, :2], rw[:, :, :2]
        if name == "out":
            gw, rw, gb, rb = gw[:1], rw[:1], gb[:1], rb[:1]
        errs[name] = (np.linalg.norm(gw - rw) / max(np.linalg.norm(rw), 1e-30),
                      np.linalg.norm(gb - rb) / max(np.linalg.norm(rb), 1e-30))
    worst = max(max(e) for e in errs.values())
    median = float(np.median([e[0] for e in errs.values()]))
    assert worst < 0.1 and median < 0.03, errs


@pytest.mark.gpu
def test_trained_network_saves_iterations(gpu):
    """Train on solver-generated solutions of a 32^3 family for a few epochs;
    on held-out systems the network's guess is within half of the solution's
    norm and the solve to 1e-8 (relative to ||b||) needs fewer inner
    iterations than from a zero guess, with the same converged answer."""
    import learned
    n, nv = 32, 8
    net = learned.Net(seed=1)
    data = learned.generate(list(range(1, 49)), n, nv)
    assert all(c for _, _, c in data["stats"])
    hist, _ = learned.train(net, data, epochs=12, batch=8, lr=1e-3)
    assert hist[-1] < 0.5 * hist[0]
    ev = learned.evaluate(net, [900001, 900002, 900003, 900004, 900005, 900006], n, nv)
    assert all(e["converged"] for e in ev)
    assert np.mean([e["guess_rel_err"] for e in ev]) < 0.3
    assert np.mean([e["its_x0"] for e in ev]) < np.mean([e["its_zero"] for e in ev])
    assert max(e["rel_diff"] for e in ev) < 1e-6
