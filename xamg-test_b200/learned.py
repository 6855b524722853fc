"""Learned initial guess for families of 3-D diffusion problems.

A convolutional encoder-decoder (4 levels, 16/32/64/128 channels, 1.47 M
parameters, BF16 weights and activations, FP32 accumulation) maps the
coefficient field and the right-hand side of a 7-point diffusion system to an
initial guess x0.  Training and inference run on the GPU through the
hand-written kernels of csrc/cnn.cu (include/xamg_learned.h); torch provides
device memory only.  The solver's own residual check still decides
convergence, so the network can only change the iteration count, never the
accuracy of the result; a zero guess is the fallback.

Problem family (one system = one coefficient field, nv right-hand sides):
  k(x)  = exp(sum of 8 Gaussian bumps), centres uniform in the unit cube,
          widths uniform in [0.05, 0.2], amplitudes uniform in [-2, 2];
          faces carry the harmonic mean of their two cells (the cell value on
          the Dirichlet boundary);
  b     = white noise smoothed by a Gaussian filter of sigma = 3 cells.

Network input (16 channels, channels-last): log(k)/4 and b/rms(b); output
channel 0 is x/(rms(b)*S) with S a data-set constant (mean rms(x)/rms(b)).
"""
import ctypes as C
import os

import numpy as np

import xamg

# (name, input channels, output channels, ReLU)
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
IN_CH = 2  # real input channels (the rest of the 16 are zero)


def n_params():
    return sum(27 * ci * co + co for _, ci, co, _ in LAYERS)


# resolution level of each layer (0: n^3 cells, l: (n / 2^l)^3 cells)
LEVEL = {"e0a": 0, "e0b": 0, "e1a": 1, "e1b": 1, "e2a": 2, "e2b": 2, "b1": 3, "b2": 3,
         "d2a": 2, "d2b": 2, "d1a": 1, "d1b": 1, "d0a": 0, "d0b": 0, "out": 0}


def conv_shapes():
    """(level, input channels, output channels) of every convolution of a
    forward pass; its multiply-adds per volume are 27 ci co (n >> level)^3."""
    return [(LEVEL[name], ci, co) for name, ci, co, _ in LAYERS]


_SIGS = {
    "xcnn_conv3d": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "xcnn_conv3d_wgrad": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                          C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "xcnn_weight_flip": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "xcnn_relu_bwd": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_void_p],
    "xcnn_bias_grad": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_void_p, C.c_void_p],
    "xcnn_pool2": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                   C.c_int, C.c_void_p],
    "xcnn_up2": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                 C.c_int, C.c_int, C.c_void_p],
    "xcnn_up2_bwd": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                     C.c_int, C.c_void_p],
    "xcnn_mse": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p],
    "xcnn_adam": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float,
                  C.c_float, C.c_float, C.c_int, C.c_void_p],
    "xcnn_pack2": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p],
    "xcnn_unpack": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p],
    "xcnn_set_box_conv": [C.c_int],
    "xcnn_set_tc_conv": [C.c_int],
    "xcnn_tc_error": [],
    "xcnn_unpack_x0": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p],
}


def klib():
    L = xamg.lib()
    if not getattr(L, "_xcnn_sigs", False):
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L._xcnn_sigs = True
    return L


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed with code %d" % (what, rc))


class View:
    """Channel window (c0, c) of a channels-last BF16 buffer t [nb, d, h, w, cs]."""

    def __init__(self, t, c0=0, c=None):
        self.t, self.cs = t, t.shape[-1]
        self.c0, self.c = c0, (t.shape[-1] - c0 if c is None else c)

    @property
    def dims(self):
        return tuple(self.t.shape[:4])


class Net:
    """The encoder-decoder with its FP32 master weights, BF16 copies, the
    flipped copies for the backward-data convolutions, gradients and Adam
    state, all on the current CUDA device."""

    def __init__(self, seed=0):
        import torch
        self.torch = torch
        self.L = klib()
        g = torch.Generator().manual_seed(seed)
        self.w32, self.b32, self.wbf, self.wflip = {}, {}, {}, {}
        self.gw, self.gb, self.m, self.v = {}, {}, {}, {}
        for name, ci, co, relu in LAYERS:
            fan = 27 * (IN_CH if name == "e0a" else ci)
            std = (2.0 / fan) ** 0.5 if relu else (1.0 / fan) ** 0.5
            w = torch.randn((co, 27, ci), generator=g) * std
            if name == "e0a":
                w[:, :, IN_CH:] = 0
            if name == "out":
                w[1:] = 0
            self.w32[name] = w.cuda().contiguous()
            self.b32[name] = torch.zeros(co, device="cuda")
            self.wbf[name] = self.w32[name].to(torch.bfloat16)
            self.wflip[name] = torch.empty((ci, 27, co), dtype=torch.bfloat16, device="cuda")
            for d in (self.gw, self.m, self.v):
                d[name] = torch.zeros_like(self.w32[name])
            for d in (self.gb,):
                d[name] = torch.zeros_like(self.b32[name])
        self.mb = {k: torch.zeros_like(v) for k, v in self.b32.items()}
        self.vb = {k: torch.zeros_like(v) for k, v in self.b32.items()}
        self.step = 0
        self.scale = 1.0  # S: x/(rms(b) S) is the network's target
        self._buf = {}

    # ---------------------------------------------------------------- buffers
    def _bufs(self, nb, n):
        key = (nb, n)
        if key in self._buf:
            return self._buf[key]
        torch = self.torch
        assert n % 8 == 0, "grid side must be a multiple of 8"

        def T(s, c):
            return torch.zeros((nb, s, s, s, c), dtype=torch.bfloat16, device="cuda")

        s0, s1, s2, s3 = n, n // 2, n // 4, n // 8
        B = dict(
            X0=T(s0, 16), e0a=T(s0, 16), C0=T(s0, 48), P1=T(s1, 16), e1a=T(s1, 32), C1=T(s1, 96),
            P2=T(s2, 32), e2a=T(s2, 64), C2=T(s2, 192), P3=T(s3, 64), b1=T(s3, 128), b2=T(s3, 128),
            d2a=T(s2, 64), d2b=T(s2, 64), d1a=T(s1, 32), d1b=T(s1, 32), d0a=T(s0, 16), d0b=T(s0, 16),
            out=torch.zeros((nb, s0, s0, s0, 16), dtype=torch.float32, device="cuda"),
            # gradients
            Gout=T(s0, 16), G0a=T(s0, 16), G0b=T(s0, 16), GC0=T(s0, 48), G1a=T(s1, 32), G1b=T(s1, 32),
            GC1=T(s1, 96), GP1=T(s1, 16), G2a=T(s2, 64), G2b=T(s2, 64), GC2=T(s2, 192), GP2=T(s2, 32),
            G3a=T(s3, 128), G3b=T(s3, 128), GP3=T(s3, 64),
        )
        self._buf = {key: B}  # keep one shape at a time
        return B

    # --------------------------------------------------------------- kernels
    def _conv(self, name, src, dst, flags=None, w=None):
        _, ci, co, relu = dict((l[0], l) for l in LAYERS)[name]
        nb, d, h, wd = src.dims
        if w is None:
            w, bias, cin, cout = self.wbf[name], self.b32[name], ci, co
            fl = (1 if relu else 0) if flags is None else flags
        else:
            bias, cin, cout, fl = None, co, ci, (0 if flags is None else flags)
        assert src.c == cin and dst.c == cout, (name, src.c, cin, dst.c, cout)
        _ok(self.L.xcnn_conv3d(_p(src.t), src.cs, src.c0, cin, _p(w), _p(bias), _p(dst.t), dst.cs, dst.c0, cout,
                               nb, d, h, wd, fl, None), "conv3d " + name)

    def _pool(self, src, dst):
        nb, d, h, w = src.dims
        _ok(self.L.xcnn_pool2(_p(src.t), src.cs, src.c0, _p(dst.t), dst.cs, dst.c0, src.c, nb, d, h, w, None), "pool2")

    def _up(self, src, dst, mode=0):
        nb, d, h, w = dst.dims
        _ok(self.L.xcnn_up2(_p(src.t), src.cs, src.c0, _p(dst.t), dst.cs, dst.c0, src.c, nb, d, h, w, mode, None),
            "up2")

    def _up_bwd(self, gfine, gin):
        nb, d, h, w = gfine.dims
        _ok(self.L.xcnn_up2_bwd(_p(gfine.t), gfine.cs, gfine.c0, _p(gin.t), gin.cs, gin.c0, gin.c, nb, d, h, w, None),
            "up2_bwd")

    def _layer_bwd(self, name, g, act, inp, gin=None, gin_flags=0):
        """g: gradient of the layer output (post-activation), modified in place
        to the pre-activation gradient; accumulates dW, db; writes dIn."""
        _, ci, co, relu = dict((l[0], l) for l in LAYERS)[name]
        nb, d, h, w = g.dims
        nvox = nb * d * h * w
        if relu:
            _ok(self.L.xcnn_relu_bwd(_p(g.t), g.cs, g.c0, _p(act.t), act.cs, act.c0, co, nvox, None), "relu_bwd")
        _ok(self.L.xcnn_conv3d_wgrad(_p(inp.t), inp.cs, inp.c0, ci, _p(g.t), g.cs, g.c0, co, _p(self.gw[name]),
                                     nb, d, h, w, None), "wgrad " + name)
        _ok(self.L.xcnn_bias_grad(_p(g.t), g.cs, g.c0, co, nvox, _p(self.gb[name]), None), "bias_grad")
        if gin is not None:
            self._conv(name, g, gin, flags=gin_flags, w=self.wflip[name])

    # ---------------------------------------------------------------- passes
    def forward(self, B):
        V = View
        self._conv("e0a", V(B["X0"]), V(B["e0a"]))
        self._conv("e0b", V(B["e0a"]), V(B["C0"], 32, 16))
        self._pool(V(B["C0"], 32, 16), V(B["P1"]))
        self._conv("e1a", V(B["P1"]), V(B["e1a"]))
        self._conv("e1b", V(B["e1a"]), V(B["C1"], 64, 32))
        self._pool(V(B["C1"], 64, 32), V(B["P2"]))
        self._conv("e2a", V(B["P2"]), V(B["e2a"]))
        self._conv("e2b", V(B["e2a"]), V(B["C2"], 128, 64))
        self._pool(V(B["C2"], 128, 64), V(B["P3"]))
        self._conv("b1", V(B["P3"]), V(B["b1"]))
        self._conv("b2", V(B["b1"]), V(B["b2"]))
        self._up(V(B["b2"]), V(B["C2"], 0, 128))
        self._conv("d2a", V(B["C2"]), V(B["d2a"]))
        self._conv("d2b", V(B["d2a"]), V(B["d2b"]))
        self._up(V(B["d2b"]), V(B["C1"], 0, 64))
        self._conv("d1a", V(B["C1"]), V(B["d1a"]))
        self._conv("d1b", V(B["d1a"]), V(B["d1b"]))
        self._up(V(B["d1b"]), V(B["C0"], 0, 32))
        self._conv("d0a", V(B["C0"]), V(B["d0a"]))
        self._conv("d0b", V(B["d0a"]), V(B["d0b"]))
        self._conv("out", V(B["d0b"]), V(B["out"]), flags=4)

    def backward(self, B):
        """Gradients of the loss whose output gradient is in B['Gout']."""
        V = View
        for name, *_ in LAYERS:
            _ok(self.L.xcnn_weight_flip(_p(self.wbf[name]), _p(self.wflip[name]), self.wbf[name].shape[0],
                                        self.wbf[name].shape[2], None), "weight_flip")
        self._layer_bwd("out", V(B["Gout"]), None, V(B["d0b"]), V(B["G0a"]))
        self._layer_bwd("d0b", V(B["G0a"]), V(B["d0b"]), V(B["d0a"]), V(B["G0b"]))
        self._layer_bwd("d0a", V(B["G0b"]), V(B["d0a"]), V(B["C0"]), V(B["GC0"]))
        self._up_bwd(V(B["GC0"], 0, 32), V(B["G1a"]))
        self._layer_bwd("d1b", V(B["G1a"]), V(B["d1b"]), V(B["d1a"]), V(B["G1b"]))
        self._layer_bwd("d1a", V(B["G1b"]), V(B["d1a"]), V(B["C1"]), V(B["GC1"]))
        self._up_bwd(V(B["GC1"], 0, 64), V(B["G2a"]))
        self._layer_bwd("d2b", V(B["G2a"]), V(B["d2b"]), V(B["d2a"]), V(B["G2b"]))
        self._layer_bwd("d2a", V(B["G2b"]), V(B["d2a"]), V(B["C2"]), V(B["GC2"]))
        self._up_bwd(V(B["GC2"], 0, 128), V(B["G3a"]))
        self._layer_bwd("b2", V(B["G3a"]), V(B["b2"]), V(B["b1"]), V(B["G3b"]))
        self._layer_bwd("b1", V(B["G3b"]), V(B["b1"]), V(B["P3"]), V(B["GP3"]))
        self._up(V(B["GP3"]), V(B["GC2"], 128, 64), mode=1)
        self._layer_bwd("e2b", V(B["GC2"], 128, 64), V(B["C2"], 128, 64), V(B["e2a"]), V(B["G2a"]))
        self._layer_bwd("e2a", V(B["G2a"]), V(B["e2a"]), V(B["P2"]), V(B["GP2"]))
        self._up(V(B["GP2"]), V(B["GC1"], 64, 32), mode=1)
        self._layer_bwd("e1b", V(B["GC1"], 64, 32), V(B["C1"], 64, 32), V(B["e1a"]), V(B["G1a"]))
        self._layer_bwd("e1a", V(B["G1a"]), V(B["e1a"]), V(B["P1"]), V(B["GP1"]))
        self._up(V(B["GP1"]), V(B["GC0"], 32, 16), mode=1)
        self._layer_bwd("e0b", V(B["GC0"], 32, 16), V(B["C0"], 32, 16), V(B["e0a"]), V(B["G0a"]))
        self._layer_bwd("e0a", V(B["G0a"]), V(B["e0a"]), V(B["X0"]))

    # ------------------------------------------------------------ user calls
    def pack(self, B, a, b):
        """Fill the network input from FP32 device tensors a (log-coefficient
        feature) and b (normalised right-hand side), both [nb, n, n, n]."""
        a, b = a.contiguous(), b.contiguous()  # the kernel reads dense [nb, n, n, n] arrays
        nvox = a.numel()
        assert b.numel() == nvox and a.dtype == b.dtype == self.torch.float32
        _ok(self.L.xcnn_pack2(_p(a), _p(b), _p(B["X0"]), nvox, None), "pack2")

    def loss_and_grad(self, B, target):
        torch = self.torch
        loss = torch.zeros(1, device="cuda")
        target = target.contiguous()
        nvox = target.numel()
        _ok(self.L.xcnn_mse(_p(B["out"]), 16, 0, _p(target), _p(B["Gout"]), 16, nvox, _p(loss), None), "mse")
        return loss

    def zero_grad(self):
        for d in (self.gw, self.gb):
            for t in d.values():
                t.zero_()

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        for name, *_ in LAYERS:
            _ok(self.L.xcnn_adam(_p(self.w32[name]), _p(self.gw[name]), _p(self.m[name]), _p(self.v[name]),
                                 _p(self.wbf[name]), self.w32[name].numel(), lr, b1, b2, eps, self.step, None), "adam")
            _ok(self.L.xcnn_adam(_p(self.b32[name]), _p(self.gb[name]), _p(self.mb[name]), _p(self.vb[name]),
                                 None, self.b32[name].numel(), lr, b1, b2, eps, self.step, None), "adam")

    def train_step(self, a, b, target, lr=1e-3):
        nb, n = a.shape[0], a.shape[1]
        B = self._bufs(nb, n)
        self.pack(B, a, b)
        self.forward(B)
        loss = self.loss_and_grad(B, target)
        self.zero_grad()
        self.backward(B)
        self.adam(lr)
        return loss

    def predict(self, a, b):
        """FP32 [nb, n, n, n] prediction of the network (output channel 0)."""
        torch = self.torch
        nb, n = a.shape[0], a.shape[1]
        B = self._bufs(nb, n)
        self.pack(B, a, b)
        self.forward(B)
        out = torch.empty(a.shape, dtype=torch.float32, device="cuda")
        _ok(self.L.xcnn_unpack(_p(B["out"]), 16, 0, None, 1, _p(out), a.numel(), None), "unpack")
        return out

    def save(self, path):
        """Weights as used by the forward pass (BF16 bits) and FP32 biases."""
        torch = self.torch
        d = {"scale": np.array([self.scale])}
        for name, *_ in LAYERS:
            d["wb_" + name] = self.wbf[name].view(torch.int16).cpu().numpy()
            d["b_" + name] = self.b32[name].cpu().numpy()
        np.savez_compressed(path, **d)

    def load(self, path):
        torch = self.torch
        z = np.load(path)
        self.scale = float(z["scale"][0])
        for name, *_ in LAYERS:
            wb = torch.from_numpy(z["wb_" + name]).view(torch.bfloat16).cuda()
            self.wbf[name].copy_(wb)
            self.w32[name].copy_(wb.float())
            self.b32[name].copy_(torch.from_numpy(z["b_" + name]))


# ------------------------------------------------------------------ family
def bump_field(rng, n):
    """Cell coefficients exp(sum of 8 Gaussian bumps) on an n^3 grid ([z, y, x])."""
    c = (np.arange(n) + 0.5) / n
    f = np.zeros((n, n, n))
    for _ in range(8):
        cz, cy, cx = rng.uniform(0.0, 1.0, 3)
        w = rng.uniform(0.05, 0.2)
        a = rng.uniform(-2.0, 2.0)
        gz = np.exp(-(c - cz) ** 2 / (2 * w * w))
        gy = np.exp(-(c - cy) ** 2 / (2 * w * w))
        gx = np.exp(-(c - cx) ** 2 / (2 * w * w))
        f += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return np.exp(f)


def face_coefficients(k):
    """Harmonic means on interior faces, the cell value on boundary faces."""
    def hm(a, b):
        return 2.0 * a * b / (a + b)
    kx = np.concatenate([k[:, :, :1], hm(k[:, :, 1:], k[:, :, :-1]), k[:, :, -1:]], axis=2)
    ky = np.concatenate([k[:, :1, :], hm(k[:, 1:, :], k[:, :-1, :]), k[:, -1:, :]], axis=1)
    kz = np.concatenate([k[:1], hm(k[1:], k[:-1]), k[-1:]], axis=0)
    return kx, ky, kz


def smooth_rhs(rng, n, nv, sigma=3.0):
    """nv fields of white noise filtered by a periodic Gaussian of sigma cells,
    as an [n^3, nv] array (row = x + n (y + n z))."""
    w = rng.standard_normal((nv, n, n, n))
    f = np.fft.fftfreq(n)
    g1 = np.exp(-2.0 * (np.pi * f * sigma) ** 2)
    G = g1[:, None, None] * g1[None, :, None] * g1[None, None, :]
    out = np.real(np.fft.ifftn(np.fft.fftn(w, axes=(1, 2, 3)) * G, axes=(1, 2, 3)))
    return np.ascontiguousarray(out.reshape(nv, -1).T)


def make_system(seed, n):
    """(matrix, log-coefficient feature [n,n,n] float32) of family member `seed`."""
    rng = np.random.default_rng(seed)
    k = bump_field(rng, n)
    kx, ky, kz = face_coefficients(k)
    A = xamg.CsrMatrix.faces7(n, n, n, kx, ky, kz)
    return A, (np.log(k) / 4.0).astype(np.float32), rng


def solver_spec(rel_tol=1e-8, base="rhs", blocks=296, mixed=False):
    """AMG-PBiCGStab with the relative tolerance measured against ||b|| (so
    that a good x0 pays off) and hybrid SGS on `blocks` blocks per level.
    mixed = True wraps an FP32 solver in FP64 iterative refinement."""
    sp = {
        "solver": {"method": "PBiCGStab", "max_iters": 200, "abs_tolerance": 0.0, "rel_tolerance": rel_tol,
                   "rel_tolerance_base": base, "convergence_details": "check-L2,noprint"},
        "preconditioner": {"method": "MultiGrid", "mg_coarsening_type": 10, "mg_interpolation_type": 6,
                           "mg_strength_threshold": 0.25, "mg_max_levels": 6, "mg_agg_num_levels": 0},
        "pre_smoother": {"method": "HSGS", "max_iters": 1, "hybrid_blocks": blocks},
        "post_smoother": {"method": "HSGS", "max_iters": 1, "hybrid_blocks": blocks},
        "coarse_grid_solver": {"method": "Direct"},
    }
    if mixed:
        sp["meta_solver"] = {"method": "IterativeRefinement", "max_iters": 30, "abs_tolerance": 0.0,
                             "rel_tolerance": rel_tol, "rel_tolerance_base": base,
                             "subsolver_reduced_precision": True, "inner_rel_tolerance": 1e-4,
                             "convergence_details": "check-L2,noprint"}
        sp["solver"].pop("rel_tolerance_base")
    return sp


def smoother_spec(sweeps=2, blocks=296):
    """Symmetric Gauss-Seidel sweeps applied to the network's guess before the
    solve: they remove the guess's high-frequency error, which otherwise
    dominates its residual."""
    return {"solver": {"method": "HSGS", "max_iters": sweeps, "hybrid_blocks": blocks,
                       "convergence_details": "nocheck,noprint"}}


# ------------------------------------------------------- data and training
def _rms(B):
    return np.sqrt(np.mean(B * B, axis=0))


def generate(seeds, n, nv, log=None):
    """Solve the family members `seeds` with the GPU solver (tolerance 1e-8
    relative to ||b||).  Returns device tensors: a [S, n, n, n] (log-coefficient
    feature per system), b and x [S*nv, n, n, n] (right-hand side and solution,
    both divided by rms(b) of their column), and the solve statistics."""
    import torch
    S = len(seeds)
    a = torch.empty((S, n, n, n), dtype=torch.float32, device="cuda")
    b = torch.empty((S * nv, n, n, n), dtype=torch.float32, device="cuda")
    x = torch.empty((S * nv, n, n, n), dtype=torch.float32, device="cuda")
    stats = []
    xamg.set_nv(nv)
    for i, seed in enumerate(seeds):
        A, feat, rng = make_system(seed, n)
        Bm = smooth_rhs(rng, n, nv)
        M = xamg.Matrix(A)
        xv, bv = xamg.Vector(A.nrows, nv), xamg.Vector(A.nrows, nv)
        bv.upload(Bm)
        s = xamg.Solver(M, xamg.Params(solver_spec()), xv, bv)
        s.solve()
        X = xv.download()
        r = _rms(Bm)
        a[i] = torch.from_numpy(feat)
        b[i * nv:(i + 1) * nv] = torch.from_numpy((Bm / r).T.reshape(nv, n, n, n).astype(np.float32))
        x[i * nv:(i + 1) * nv] = torch.from_numpy((X / r).T.reshape(nv, n, n, n).astype(np.float32))
        stats.append((s.iters(), s.last_ms(), all(s.converged())))
        if log and (i + 1) % 32 == 0:
            log("generated %d/%d systems" % (i + 1, S))
    return {"a": a, "b": b, "x": x, "nv": nv, "stats": stats}


def train(net, data, epochs, batch=8, lr=1e-3, seed=0, log=None):
    """Adam on the mean squared error of x/(rms(b) S), cosine learning-rate
    decay; batches mix samples of different systems.  Returns the loss history
    (mean per epoch) and the device time of the training steps (ms)."""
    import torch
    nv = data["nv"]
    N = data["b"].shape[0]
    sc = float(torch.sqrt(torch.mean(data["x"] ** 2)).item())
    net.scale = sc
    g = torch.Generator().manual_seed(seed)
    steps = epochs * (N // batch)
    hist = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(N, generator=g).cuda()
        tot = torch.zeros(1, device="cuda")
        for q in range(N // batch):
            idx = perm[q * batch:(q + 1) * batch]
            aa = data["a"].index_select(0, idx // nv)
            bb = data["b"].index_select(0, idx)
            tt = data["x"].index_select(0, idx) / sc
            cur = lr * 0.5 * (1.0 + np.cos(np.pi * k / max(steps, 1)))
            tot += net.train_step(aa, bb, tt, lr=cur)
            k += 1
        hist.append(float(tot.item()) / max(N // batch, 1))
        if log:
            log("epoch %d loss %.4e" % (ep + 1, hist[-1]))
    ev1.record()
    torch.cuda.synchronize()
    return hist, ev0.elapsed_time(ev1)


def evaluate(net, seeds, n, nv, log=None, sweeps=2, mixed=False):
    """Per held-out system: Krylov iterations and device time to 1e-8
    (relative to ||b||) from a zero guess and from the network's guess
    smoothed by `sweeps` symmetric Gauss-Seidel sweeps (inference and
    smoothing time included), the guess's relative error before smoothing and
    relative residual after it, and the difference of the two solutions."""
    import torch
    L = klib()
    out = []
    xamg.set_nv(nv)
    per = n * n * n
    for seed in seeds:
        A, feat, rng = make_system(seed, n)
        Bm = smooth_rhs(rng, n, nv)
        r = _rms(Bm)
        M = xamg.Matrix(A)
        xv, bv = xamg.Vector(A.nrows, nv), xamg.Vector(A.nrows, nv)
        bv.upload(Bm)
        s = xamg.Solver(M, xamg.Params(solver_spec(mixed=mixed)), xv, bv)
        sm = xamg.Solver(M, xamg.Params(smoother_spec(sweeps)), xv, bv) if sweeps > 0 else None
        # zero guess (run twice: the first solve also warms up the plan)
        for _ in range(2):
            xv.set(0.0)
            s.solve()
        it0, ms0 = s.iters(), s.last_ms()
        X0 = xv.download()
        h0 = s.history()
        # network guess
        aa = torch.from_numpy(np.broadcast_to(feat, (nv, n, n, n)).copy()).cuda()
        bb = torch.from_numpy(np.ascontiguousarray((Bm / r).T.reshape(nv, n, n, n), dtype=np.float32)).cuda()
        scale = torch.from_numpy((r * net.scale).astype(np.float32)).cuda()
        xv.set(0.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B = net._bufs(nv, n)
        net.pack(B, aa, bb)
        net.forward(B)
        _ok(L.xcnn_unpack_x0(_p(B["out"]), 16, 0, _p(scale), nv, per, xamg.lib().XAMG_b200_vector_device_ptr(xv.h),
                             None), "unpack_x0")
        e1.record()
        torch.cuda.synchronize()
        ms_inf = e0.elapsed_time(e1)
        G = xv.download()
        err0 = float(np.linalg.norm(G - X0) / np.linalg.norm(X0))
        ms_sm = 0.0
        if sm is not None:
            sm.solve()
            ms_sm = sm.last_ms()
        s.solve()
        it1, ms1 = s.iters(), s.last_ms()
        X1 = xv.download()
        h1 = s.history()
        # relative residual of the guess: first history entry over ||b||^2
        bb2 = np.sum(Bm * Bm, axis=0)
        rel0 = float(np.sqrt(np.mean(h1[0] / bb2)))
        diff = float(np.linalg.norm(X1 - X0) / np.linalg.norm(X0))
        # Krylov iterations (the inner FP32 ones under iterative refinement)
        out.append({"seed": seed, "its_zero": it0[1] if mixed else it0[0], "its_x0": it1[1] if mixed else it1[0],
                    "ms_zero": ms0, "ms_x0": ms1 + ms_inf + ms_sm, "ms_infer": ms_inf, "ms_smooth": ms_sm,
                    "guess_rel_res": rel0, "guess_rel_err": err0, "rel_diff": diff,
                    "converged": bool(all(s.converged()))})
        if log:
            log("seed %d: zero %d it %.2f ms | x0 %d it %.2f ms (infer %.2f smooth %.2f) | res %.3e err %.3e" %
                (seed, out[-1]["its_zero"], ms0, out[-1]["its_x0"], ms1 + ms_inf + ms_sm, ms_inf, ms_sm, rel0, err0))
    return out


def main():
    import argparse
    import json
    import sys
    import time
    import torch
    ap = argparse.ArgumentParser(description="train and evaluate the learned initial guess")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--nv", type=int, default=8)
    ap.add_argument("--train-systems", type=int, default=512)
    ap.add_argument("--eval-systems", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--weights", default="")
    ap.add_argument("--load", default="")
    ap.add_argument("--forward-only", type=int, default=0, metavar="K",
                    help="time K forward passes (inference) of the network on random inputs of nv volumes of n^3 "
                         "cells and exit; --tcgen05 selects the tcgen05 convolution")
    ap.add_argument("--tcgen05", action="store_true")
    args = ap.parse_args()
    log = lambda m: print(m, file=sys.stderr, flush=True)
    if args.forward_only:
        L = klib()
        L.xcnn_set_tc_conv(int(args.tcgen05))
        net = Net(seed=1)
        if args.load:
            net.load(args.load)
        g = torch.Generator().manual_seed(3)
        a = torch.randn((args.nv, args.n, args.n, args.n), generator=g).cuda()
        b = torch.randn((args.nv, args.n, args.n, args.n), generator=g).cuda()
        B = net._bufs(args.nv, args.n)
        net.pack(B, a, b)
        net.forward(B)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.forward_only):
            net.forward(B)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.forward_only
        flops = 2.0 * args.nv * sum(27 * ci * co * (args.n >> lev) ** 3 for lev, ci, co in conv_shapes())
        print(json.dumps({"n": args.n, "nv": args.nv, "tcgen05": bool(args.tcgen05), "ms_forward": round(ms, 3),
                          "conv_tflops": round(flops / ms / 1e9, 1), "tc_error": int(L.xcnn_tc_error())}),
              flush=True)
        return
    xamg.init(args.nv)
    net = Net(seed=1)
    res = {"n": args.n, "nv": args.nv, "params": n_params()}
    if args.load:
        net.load(args.load)
    else:
        t0 = time.time()
        data = generate(list(range(1, args.train_systems + 1)), args.n, args.nv, log=log)
        res["generate_s"] = round(time.time() - t0, 1)
        res["train_samples"] = int(data["b"].shape[0])
        hist, ms = train(net, data, args.epochs, batch=args.batch, lr=args.lr, log=log)
        res.update(loss_history=[round(h, 5) for h in hist], train_ms=round(ms, 1))
        del data
        torch.cuda.empty_cache()
        if args.weights:
            net.save(args.weights)
    ev = evaluate(net, list(range(100001, 100001 + args.eval_systems)), args.n, args.nv, log=log)
    for k in ("its_zero", "its_x0", "ms_zero", "ms_x0", "ms_infer", "ms_smooth", "guess_rel_res",
              "guess_rel_err", "rel_diff"):
        res["mean_" + k] = float(np.mean([e[k] for e in ev]))
    res["all_converged"] = all(e["converged"] for e in ev)
    res["eval_samples"] = args.eval_systems * args.nv
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
