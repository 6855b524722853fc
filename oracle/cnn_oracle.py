"""CPU oracle of the learned initial guess's network (test infrastructure only).

The learned form has no counterpart in the reference: this file restates, in
numpy, the encoder-decoder that xamg-test_b200/csrc/cnn.cu and
xamg-test_b200/learned.py run on the GPU, so that the GPU forward pass and its
gradients can be checked against an independent implementation.  With
`bf16=True` every tensor is rounded to BF16 (round to nearest even) at the
points where the GPU stores BF16 (activations except the FP32 prediction,
activation gradients, weights);
products are accumulated in float64 (the GPU accumulates in FP32, so results
agree to FP32 accumulation error plus the occasional one-ulp BF16 rounding
difference).  With `bf16=False` it is a plain float64 network whose gradients
are pinned by finite differences in the CPU tests.

Layout: volumes [nb, d, h, w, c] (channels last), weights [cout, 27, cin] with
tap t = (dz+1)*9 + (dy+1)*3 + (dx+1), zero padding outside the volume.
"""
import numpy as np

LAYERS = [
    ("e0a", 16, 16, True), ("e0b", 16, 16, True),
    ("e1a", 16, 32, True), ("e1b", 32, 32, True),
    ("e2a", 32, 64, True), ("e2b", 64, 64, True),
    ("b1", 64, 128, True), ("b2", 128, 128, True),
    ("d2a", 192, 64, True), ("d2b", 64, 64, True),
    ("d1a", 96, 32, True), ("d1b", 32, 32, True),
    ("d0a", 48, 16, True), ("d0b", 16, 16, True),
    ("out", 16, 16, False),
]
SPEC = {l[0]: l for l in LAYERS}


def to_bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


def _shift(x, t):
    """y[v] = x[v + off(t)] with zeros outside (x: [nb, d, h, w, c])."""
    dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
    p = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    d, h, w = x.shape[1:4]
    return p[:, 1 + dz:1 + dz + d, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w, :]


def _unshift_add(acc, g, t):
    """acc[v + off(t)] += g[v] (the adjoint of _shift)."""
    dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
    d, h, w = g.shape[1:4]
    p = np.zeros((g.shape[0], d + 2, h + 2, w + 2, g.shape[4]))
    p[:, 1 + dz:1 + dz + d, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w, :] += g
    acc += p[:, 1:-1, 1:-1, 1:-1, :]


def conv3d(x, w, b=None):
    """sum_t shift(x, t) @ w[:, t, :].T (+ b), float64."""
    out = np.zeros(x.shape[:4] + (w.shape[0],))
    for t in range(27):
        out += _shift(x, t).astype(np.float64) @ w[:, t, :].T.astype(np.float64)
    if b is not None:
        out += b
    return out


def conv3d_bwd_data(g, w):
    """d/dx of conv3d: sum_t unshift(g @ w[:, t, :])."""
    out = np.zeros(g.shape[:4] + (w.shape[2],))
    for t in range(27):
        _unshift_add(out, g.astype(np.float64) @ w[:, t, :].astype(np.float64), t)
    return out


def conv3d_wgrad(x, g):
    """dW[co, t, ci] = sum_v g[v, co] x[v + off(t), ci]."""
    co, ci = g.shape[4], x.shape[4]
    dw = np.zeros((co, 27, ci))
    G = g.reshape(-1, co).astype(np.float64)
    for t in range(27):
        dw[:, t, :] = G.T @ _shift(x, t).reshape(-1, ci).astype(np.float64)
    return dw


def pool2(x):
    nb, d, h, w, c = x.shape
    return x.reshape(nb, d // 2, 2, h // 2, 2, w // 2, 2, c).astype(np.float64).mean(axis=(2, 4, 6))


def up2(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def up2_bwd(g):
    nb, d, h, w, c = g.shape
    return g.reshape(nb, d // 2, 2, h // 2, 2, w // 2, 2, c).astype(np.float64).sum(axis=(2, 4, 6))


class Net:
    """weights: {name: (w [cout, 27, cin], b [cout])}."""

    def __init__(self, weights, bf16=True):
        self.bf = bf16
        self.w = {k: (self.r(np.asarray(w, np.float64)), np.asarray(b, np.float64)) for k, (w, b) in weights.items()}

    def r(self, a):
        return to_bf16(a).astype(np.float64) if self.bf else np.asarray(a, np.float64)

    def layer(self, name, x, rounded=True):
        _, ci, co, relu = SPEC[name]
        w, b = self.w[name]
        y = conv3d(x, w, b)
        if relu:
            y = np.maximum(y, 0.0)
        return self.r(y) if rounded else y

    def forward(self, x0):
        """x0: [nb, n, n, n, 16]; returns the activations dictionary."""
        A = {"X0": self.r(x0)}
        A["e0a"] = self.layer("e0a", A["X0"])
        A["e0b"] = self.layer("e0b", A["e0a"])
        A["P1"] = self.r(pool2(A["e0b"]))
        A["e1a"] = self.layer("e1a", A["P1"])
        A["e1b"] = self.layer("e1b", A["e1a"])
        A["P2"] = self.r(pool2(A["e1b"]))
        A["e2a"] = self.layer("e2a", A["P2"])
        A["e2b"] = self.layer("e2b", A["e2a"])
        A["P3"] = self.r(pool2(A["e2b"]))
        A["b1"] = self.layer("b1", A["P3"])
        A["b2"] = self.layer("b2", A["b1"])
        A["C2"] = np.concatenate([up2(A["b2"]), A["e2b"]], axis=4)
        A["d2a"] = self.layer("d2a", A["C2"])
        A["d2b"] = self.layer("d2b", A["d2a"])
        A["C1"] = np.concatenate([up2(A["d2b"]), A["e1b"]], axis=4)
        A["d1a"] = self.layer("d1a", A["C1"])
        A["d1b"] = self.layer("d1b", A["d1a"])
        A["C0"] = np.concatenate([up2(A["d1b"]), A["e0b"]], axis=4)
        A["d0a"] = self.layer("d0a", A["C0"])
        A["d0b"] = self.layer("d0b", A["d0a"])
        A["out"] = self.layer("out", A["d0b"], rounded=False)  # FP32 prediction
        return A

    def loss(self, A, target):
        return float(np.mean((A["out"][..., 0] - target) ** 2))

    def backward(self, A, target):
        """Gradients {name: (dW, db)} of the mean squared error of channel 0."""
        r = self.r
        G = {}
        nvox = target.size
        gout = np.zeros_like(A["out"])
        gout[..., 0] = r(2.0 * (A["out"][..., 0] - target) / nvox)

        def lb(name, g, act, inp, need_in=True):
            _, ci, co, relu = SPEC[name]
            if relu:
                g = g * (act > 0)
            G[name] = (conv3d_wgrad(inp, g), g.reshape(-1, co).sum(axis=0))
            return r(conv3d_bwd_data(g, self.w[name][0])) if need_in else None

        g = lb("out", gout, None, A["d0b"])
        g = lb("d0b", g, A["d0b"], A["d0a"])
        gc0 = lb("d0a", g, A["d0a"], A["C0"])
        g = r(up2_bwd(gc0[..., :32]))
        g = lb("d1b", g, A["d1b"], A["d1a"])
        gc1 = lb("d1a", g, A["d1a"], A["C1"])
        g = r(up2_bwd(gc1[..., :64]))
        g = lb("d2b", g, A["d2b"], A["d2a"])
        gc2 = lb("d2a", g, A["d2a"], A["C2"])
        g = r(up2_bwd(gc2[..., :128]))
        g = lb("b2", g, A["b2"], A["b1"])
        gp3 = lb("b1", g, A["b1"], A["P3"])
        ge2b = r(gc2[..., 128:] + up2(gp3) * 0.125)
        g = lb("e2b", ge2b, A["e2b"], A["e2a"])
        gp2 = lb("e2a", g, A["e2a"], A["P2"])
        ge1b = r(gc1[..., 64:] + up2(gp2) * 0.125)
        g = lb("e1b", ge1b, A["e1b"], A["e1a"])
        gp1 = lb("e1a", g, A["e1a"], A["P1"])
        ge0b = r(gc0[..., 32:] + up2(gp1) * 0.125)
        g = lb("e0b", ge0b, A["e0b"], A["e0a"])
        lb("e0a", g, A["e0a"], A["X0"], need_in=False)
        return G
