"""The warm-start U-Net on the project's own BF16 kernels.

Four levels (channels c1..c4, 2x2 average pooling down, nearest 2x
upsampling up, skip connections by channel concatenation), 3x3
convolutions with ReLU, and a linear 3x3 head to one channel.  With the
default channels (24, 48, 96, 192) it has 1.1M parameters.

Tensors are NHWC bfloat16 on the GPU; torch only allocates them.  Every
layer, its gradient and the Adam update run in ``libsmili_unet.so``
(smili_b200/csrc/unet.cu).  The concatenation buffers are written in place
by their two producers (upsampled path at channel 0, encoder skip after it),
so there is no copy.
"""
from __future__ import annotations

import numpy as np

from . import kernels as K

CHANNELS = (24, 48, 96, 192)


def layer_specs(c=CHANNELS, cin=1, cout=1):
    """(name, Cin, Cout, relu) of every 3x3 convolution in forward order."""
    c1, c2, c3, c4 = c
    return [("e1a", cin, c1, True), ("e1b", c1, c1, True),
            ("e2a", c1, c2, True), ("e2b", c2, c2, True),
            ("e3a", c2, c3, True), ("e3b", c3, c3, True),
            ("ba", c3, c4, True), ("bb", c4, c4, True),
            ("d3a", c4 + c3, c3, True), ("d3b", c3, c3, True),
            ("d2a", c3 + c2, c2, True), ("d2b", c2, c2, True),
            ("d1a", c2 + c1, c1, True), ("d1b", c1, c1, True),
            ("head", c1, cout, False)]


class _Layer:
    def __init__(self, name, cin, cout, relu):
        self.name, self.cin, self.cout, self.relu = name, cin, cout, relu
        self.nw = cout * 9 * cin


class UNet:
    """Parameters, activations and optimiser state of one U-Net on one GPU."""

    def __init__(self, channels=CHANNELS, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.c = tuple(channels)
        self.layers = [_Layer(*s) for s in layer_specs(self.c)]
        n = sum(L.nw + L.cout for L in self.layers)
        self.nparam = n
        f32 = dict(dtype=torch.float32, device=self.device)
        self.master = torch.zeros(n, **f32)
        self.grad = torch.zeros(n, **f32)
        self.m = torch.zeros(n, **f32)
        self.v = torch.zeros(n, **f32)
        self.w16 = torch.zeros(n, dtype=torch.bfloat16, device=self.device)
        o = 0
        for L in self.layers:
            L.w32 = self.master[o:o + L.nw]
            L.w = self.w16[o:o + L.nw]
            L.dw = self.grad[o:o + L.nw]
            o += L.nw
            L.b = self.master[o:o + L.cout]
            L.db = self.grad[o:o + L.cout]
            o += L.cout
            L.wt = torch.zeros(L.nw, dtype=torch.bfloat16, device=self.device)
        self.by = {L.name: L for L in self.layers}
        self.step_count = 0
        self.shape = None
        rng = np.random.default_rng(seed)
        params = {}
        for L in self.layers:
            std = np.sqrt(2.0 / (9 * L.cin)) * (1.0 if L.relu else 0.1)
            params[L.name] = (rng.standard_normal((L.cout, 3, 3, L.cin)) * std, np.zeros(L.cout))
        self.set_params(params)

    # ------------------------------------------------------------ parameters
    def set_params(self, params):
        """Load {name: (w [Cout,3,3,Cin], b [Cout])}; the bf16 copy is the
        rounded master (what the kernels use)."""
        torch = self.torch
        for L in self.layers:
            w, b = params[L.name]
            L.w32.copy_(torch.as_tensor(np.asarray(w, np.float32).reshape(-1), device=self.device))
            L.b.copy_(torch.as_tensor(np.asarray(b, np.float32), device=self.device))
        K.f32_to_bf16(self.master, self.w16, self.nparam)
        self._flip_all()

    def params(self):
        """{name: (w, b)} as float32 numpy arrays (the master copy)."""
        out = {}
        for L in self.layers:
            out[L.name] = (L.w32.detach().cpu().numpy().reshape(L.cout, 3, 3, L.cin).copy(),
                           L.b.detach().cpu().numpy().copy())
        return out

    def params_bf16(self):
        """{name: (w as used by the kernels, b)} as float32 numpy arrays."""
        out = {}
        for L in self.layers:
            out[L.name] = (L.w.float().cpu().numpy().reshape(L.cout, 3, 3, L.cin).copy(),
                           L.b.detach().cpu().numpy().copy())
        return out

    def save(self, path, bf16=True):
        """Weights (bf16 bit patterns as uint16 when ``bf16``, else float32)
        and float32 biases."""
        p = self.params_bf16() if bf16 else self.params()

        def enc(w):
            w = np.ascontiguousarray(w, np.float32)
            return (w.view(np.uint32) >> 16).astype(np.uint16) if bf16 else w

        np.savez(path, channels=np.array(self.c), bf16=np.array(bool(bf16)),
                 **{f"{k}_w": enc(v[0]) for k, v in p.items()}, **{f"{k}_b": v[1] for k, v in p.items()})

    @classmethod
    def load(cls, path, device="cuda"):
        z = np.load(path)
        net = cls(tuple(int(c) for c in z["channels"]), device=device)

        def dec(w):
            if w.dtype == np.uint16:
                return (w.astype(np.uint32) << 16).view(np.float32)
            return w

        net.set_params({L.name: (dec(z[f"{L.name}_w"]), z[f"{L.name}_b"]) for L in net.layers})
        return net

    def _flip_all(self):
        for L in self.layers:
            K.flip_weights(L.w, L.wt, L.cout, L.cin)

    # ------------------------------------------------------------ buffers
    def _alloc(self, B, H, W):
        if self.shape == (B, H, W):
            return
        if H % 8 or W % 8:
            raise ValueError("image sides must be multiples of 8")
        torch = self.torch
        c1, c2, c3, c4 = self.c
        H2, W2, H3, W3, H4, W4 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8

        def buf(h, w, c):
            return torch.zeros((B, h, w, c), dtype=torch.bfloat16, device=self.device)

        A = {"x": buf(H, W, 1), "e1a": buf(H, W, c1), "cat1": buf(H, W, c2 + c1), "p1": buf(H2, W2, c1),
             "e2a": buf(H2, W2, c2), "cat2": buf(H2, W2, c3 + c2), "p2": buf(H3, W3, c2),
             "e3a": buf(H3, W3, c3), "cat3": buf(H3, W3, c4 + c3), "p3": buf(H4, W4, c3),
             "ba": buf(H4, W4, c4), "bb": buf(H4, W4, c4), "d3a": buf(H3, W3, c3), "d3b": buf(H3, W3, c3),
             "d2a": buf(H2, W2, c2), "d2b": buf(H2, W2, c2), "d1a": buf(H, W, c1), "d1b": buf(H, W, c1),
             "out": buf(H, W, 1)}
        D = {"out": buf(H, W, 1), "d1b": buf(H, W, c1), "d1a": buf(H, W, c1), "cat1": buf(H, W, c2 + c1),
             "d2b": buf(H2, W2, c2), "d2a": buf(H2, W2, c2), "cat2": buf(H2, W2, c3 + c2),
             "d3b": buf(H3, W3, c3), "d3a": buf(H3, W3, c3), "cat3": buf(H3, W3, c4 + c3),
             "bb": buf(H4, W4, c4), "ba": buf(H4, W4, c4), "p3": buf(H4, W4, c3), "e3a": buf(H3, W3, c3),
             "p2": buf(H3, W3, c2), "e2a": buf(H2, W2, c2), "p1": buf(H2, W2, c1), "e1a": buf(H, W, c1)}
        self.A, self.D = A, D
        # weight-gradient split partials: enough for the largest layer's split
        self.nsplit = {}
        need = 1
        sizes = {"e1a": (H, W), "e1b": (H, W), "d1a": (H, W), "d1b": (H, W), "head": (H, W),
                 "e2a": (H2, W2), "e2b": (H2, W2), "d2a": (H2, W2), "d2b": (H2, W2),
                 "e3a": (H3, W3), "e3b": (H3, W3), "d3a": (H3, W3), "d3b": (H3, W3),
                 "ba": (H4, W4), "bb": (H4, W4)}
        self.hw = sizes
        for L in self.layers:
            h, w = sizes[L.name]
            tiles = B * ((h + 7) // 8) * ((w + 15) // 16)
            blocks = ((L.cout + 63) // 64) * ((L.cin + 15) // 16)
            ns = int(max(1, min(tiles, 296 // blocks)))
            self.nsplit[L.name] = ns
            need = max(need, ns * L.nw)
        self.partial = torch.zeros(need, dtype=torch.float32, device=self.device)
        self.loss_part = torch.zeros(256, dtype=torch.float32, device=self.device)
        self.shape = (B, H, W)

    # ------------------------------------------------------------ forward
    def _conv(self, name, x, ldx, y, ldy):
        L = self.by[name]
        B = self.shape[0]
        h, w = self.hw[name]
        K.conv3x3(x, B, h, w, L.cin, ldx, L.w, L.b, y, ldy, L.cout, L.relu)

    def forward(self, x):
        """x: (B, H, W) float array or tensor (normalised dirty images).
        Returns the (B, H, W, 1) bf16 output tensor (kept for backward)."""
        torch = self.torch
        x = torch.as_tensor(x, device=self.device)
        B, H, W = x.shape
        self._alloc(B, H, W)
        A = self.A
        c1, c2, c3, c4 = self.c
        A["x"].copy_(x.reshape(B, H, W, 1).to(torch.bfloat16))
        H2, W2, H3, W3, H4, W4 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        self._conv("e1a", A["x"], 1, A["e1a"], c1)
        self._conv("e1b", A["e1a"], c1, (A["cat1"], c2), c2 + c1)
        K.avgpool2((A["cat1"], c2), c2 + c1, A["p1"], c1, B, H, W, c1)
        self._conv("e2a", A["p1"], c1, A["e2a"], c2)
        self._conv("e2b", A["e2a"], c2, (A["cat2"], c3), c3 + c2)
        K.avgpool2((A["cat2"], c3), c3 + c2, A["p2"], c2, B, H2, W2, c2)
        self._conv("e3a", A["p2"], c2, A["e3a"], c3)
        self._conv("e3b", A["e3a"], c3, (A["cat3"], c4), c4 + c3)
        K.avgpool2((A["cat3"], c4), c4 + c3, A["p3"], c3, B, H3, W3, c3)
        self._conv("ba", A["p3"], c3, A["ba"], c4)
        self._conv("bb", A["ba"], c4, A["bb"], c4)
        K.upsample2(A["bb"], c4, (A["cat3"], 0), c4 + c3, B, H4, W4, c4)
        self._conv("d3a", A["cat3"], c4 + c3, A["d3a"], c3)
        self._conv("d3b", A["d3a"], c3, A["d3b"], c3)
        K.upsample2(A["d3b"], c3, (A["cat2"], 0), c3 + c2, B, H3, W3, c3)
        self._conv("d2a", A["cat2"], c3 + c2, A["d2a"], c2)
        self._conv("d2b", A["d2a"], c2, A["d2b"], c2)
        K.upsample2(A["d2b"], c2, (A["cat1"], 0), c2 + c1, B, H2, W2, c2)
        self._conv("d1a", A["cat1"], c2 + c1, A["d1a"], c1)
        self._conv("d1b", A["d1a"], c1, A["d1b"], c1)
        self._conv("head", A["d1b"], c1, A["out"], 1)
        return A["out"]

    # ------------------------------------------------------------ backward
    def _back(self, name, x, ldx, dy, lddy, yout, ldyout, dx, lddx, need_dx=True):
        L = self.by[name]
        B = self.shape[0]
        h, w = self.hw[name]
        npix = B * h * w
        if L.relu:
            K.relu_mask(yout, ldyout, dy, lddy, npix, L.cout)
        K.conv3x3_wgrad(x, ldx, dy, lddy, B, h, w, L.cin, L.cout, self.partial, self.nsplit[name], L.dw)
        K.bias_grad(dy, lddy, npix, L.cout, L.db)
        if need_dx:
            K.conv3x3(dy, B, h, w, L.cout, lddy, L.wt, None, dx, lddx, L.cin, False)

    def backward(self, dout=None):
        """Gradients of every parameter into ``self.grad``.  ``dout`` is the
        output gradient (B, H, W); None uses the one ``loss`` wrote."""
        torch = self.torch
        A, D = self.A, self.D
        B, H, W = self.shape
        c1, c2, c3, c4 = self.c
        H2, W2, H3, W3, H4, W4 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        if dout is not None:
            D["out"].copy_(torch.as_tensor(dout, device=self.device).reshape(B, H, W, 1).to(torch.bfloat16))
        self._back("head", A["d1b"], c1, D["out"], 1, None, 0, D["d1b"], c1)
        self._back("d1b", A["d1a"], c1, D["d1b"], c1, A["d1b"], c1, D["d1a"], c1)
        self._back("d1a", A["cat1"], c2 + c1, D["d1a"], c1, A["d1a"], c1, D["cat1"], c2 + c1)
        K.upsample2_bwd((D["cat1"], 0), c2 + c1, D["d2b"], c2, B, H2, W2, c2)
        self._back("d2b", A["d2a"], c2, D["d2b"], c2, A["d2b"], c2, D["d2a"], c2)
        self._back("d2a", A["cat2"], c3 + c2, D["d2a"], c2, A["d2a"], c2, D["cat2"], c3 + c2)
        K.upsample2_bwd((D["cat2"], 0), c3 + c2, D["d3b"], c3, B, H3, W3, c3)
        self._back("d3b", A["d3a"], c3, D["d3b"], c3, A["d3b"], c3, D["d3a"], c3)
        self._back("d3a", A["cat3"], c4 + c3, D["d3a"], c3, A["d3a"], c3, D["cat3"], c4 + c3)
        K.upsample2_bwd((D["cat3"], 0), c4 + c3, D["bb"], c4, B, H4, W4, c4)
        self._back("bb", A["ba"], c4, D["bb"], c4, A["bb"], c4, D["ba"], c4)
        self._back("ba", A["p3"], c3, D["ba"], c4, A["ba"], c4, D["p3"], c3)
        K.avgpool2_bwd(D["p3"], c3, (D["cat3"], c4), c4 + c3, B, H3, W3, c3, accumulate=True)
        self._back("e3b", A["e3a"], c3, (D["cat3"], c4), c4 + c3, (A["cat3"], c4), c4 + c3, D["e3a"], c3)
        self._back("e3a", A["p2"], c2, D["e3a"], c3, A["e3a"], c3, D["p2"], c2)
        K.avgpool2_bwd(D["p2"], c2, (D["cat2"], c3), c3 + c2, B, H2, W2, c2, accumulate=True)
        self._back("e2b", A["e2a"], c2, (D["cat2"], c3), c3 + c2, (A["cat2"], c3), c3 + c2, D["e2a"], c2)
        self._back("e2a", A["p1"], c1, D["e2a"], c2, A["e2a"], c2, D["p1"], c1)
        K.avgpool2_bwd(D["p1"], c1, (D["cat1"], c2), c2 + c1, B, H, W, c1, accumulate=True)
        self._back("e1b", A["e1a"], c1, (D["cat1"], c2), c2 + c1, (A["cat1"], c2), c2 + c1, D["e1a"], c1)
        self._back("e1a", A["x"], 1, D["e1a"], c1, A["e1a"], c1, None, 1, need_dx=False)

    # ------------------------------------------------------------ training
    def loss(self, target):
        """MSE of the last forward output against target (B, H, W) float32;
        writes the output gradient for ``backward``.  Returns the loss tensor
        (mean of squares) without synchronising."""
        torch = self.torch
        B, H, W = self.shape
        t = torch.as_tensor(target, dtype=torch.float32, device=self.device).reshape(-1).contiguous()
        n = B * H * W
        K.mse(self.A["out"], 1, t, n, self.D["out"], 1, self.loss_part, self.loss_part.numel())
        return self.loss_part.sum() / n

    def adam_step(self, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        self.step_count += 1
        K.adam(self.master, self.w16, self.grad, self.m, self.v, self.nparam, lr, b1, b2, eps, wd,
               self.step_count)
        self._flip_all()

    def predict(self, x, batch=64):
        """Output images (N, H, W) float32 numpy for inputs (N, H, W)."""
        torch = self.torch
        x = np.asarray(x, np.float32)
        out = []
        for i in range(0, len(x), batch):
            xb = x[i:i + batch]
            y = self.forward(torch.as_tensor(xb, device=self.device))
            out.append(y[:len(xb), :, :, 0].float().cpu().numpy())
        return np.concatenate(out)
