"""Learned warm start for the to-tolerance pressure solve.

A small 3-D U-Net maps the normalised divergence and the cell classes of a
pot scene to a first guess of the pressure; the multigrid-preconditioned CG
solve then starts from it (``warm_start``) and finishes to the same FP64
tolerance, so the network can only save iterations, never change the answer.
The plain solve generates the training targets and judges the network's
error.

Architecture (4 levels, channels 16/32/64/128, BF16 activations and weights,
FP32 accumulate and master weights): two 3x3x3 convolutions with ReLU per
level, 2x2x2 average pooling down, nearest-neighbour x2 upsampling up with an
additive skip from the encoder, a 16 -> 1 linear head.  Every layer runs in
the library's own kernels (``csrc/unet.cu``: tensor-core implicit-GEMM
convolutions for the forward pass, the data gradient and the weight
gradient; pooling, upsampling, head, loss and Adam); torch tensors are only
device buffers.  Grid dimensions must be multiples of 8 (three poolings).

Scaling.  A p = b is linear, so the network sees div / s (s = RMS of the
divergence over fluid cells) and predicts p / S with
S = -(rho dx^2 / dt) s H^2, H the water depth in cells; the Dirichlet free
surface makes p grow with H^2.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream_handle

CH = (16, 32, 64, 128)
# (name, cin, cout): encoder levels 1-3, bottom, decoder levels 3-1
LAYERS = [("e1a", 16, 16), ("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32),
          ("e3a", 32, 64), ("e3b", 64, 64), ("bta", 64, 128), ("btb", 128, 128),
          ("u3a", 128, 64), ("u3b", 64, 64), ("u2a", 64, 32), ("u2b", 32, 32),
          ("u1a", 32, 16), ("u1b", 16, 16)]
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                            "unet_warmstart.npz")
HEAD_BLOCKS = 512


def _bf16(shape, device):
    return torch.empty(shape, dtype=torch.bfloat16, device=device)


@dataclass
class Layer:
    name: str
    cin: int
    cout: int
    w: torch.Tensor        # FP32 master [27][cout][cin]
    wb: torch.Tensor       # BF16 copy
    b: torch.Tensor        # FP32 [cout]
    gw: torch.Tensor | None = None
    gb: torch.Tensor | None = None
    mw: torch.Tensor | None = None
    vw: torch.Tensor | None = None
    mb: torch.Tensor | None = None
    vb: torch.Tensor | None = None


def scene_scales(div: torch.Tensor, mask: torch.Tensor, dx: float, dt: float, rho: float):
    """(s, S): input scale (RMS divergence on fluid cells) and output scale."""
    fl = (mask & 0x80) != 0
    nfl = int(fl.sum().item())
    s = float(torch.sqrt((div[fl].double() ** 2).sum() / max(nfl, 1)).item()) if nfl else 1.0
    s = s if s > 0 else 1.0
    depth = float(fl.sum(dim=2).max().item()) if nfl else 1.0
    S = -(rho * dx * dx / dt) * s * depth * depth
    return s, S, nfl


class UNet:
    def __init__(self, seed: int = 0, device="cuda"):
        self.device = torch.device(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.layers: list[Layer] = []
        for name, cin, cout in LAYERS:
            std = math.sqrt(2.0 / (27 * cin))
            w = (torch.randn((27, cout, cin), generator=g) * std).to(self.device)
            self.layers.append(Layer(name, cin, cout, w, w.to(torch.bfloat16),
                                     torch.zeros(cout, device=self.device)))
        self.hw = (torch.randn(16, generator=g) * 0.25).to(self.device)
        self.hb = torch.zeros(1, device=self.device)
        self.by = {L.name: L for L in self.layers}
        self.step = 0
        self._ws = {}

    # ---- parameters -------------------------------------------------------------------
    def state(self) -> dict:
        d = {f"{L.name}.w": L.w.cpu().numpy() for L in self.layers}
        d.update({f"{L.name}.b": L.b.cpu().numpy() for L in self.layers})
        d["head.w"] = self.hw.cpu().numpy()
        d["head.b"] = self.hb.cpu().numpy()
        return d

    def save(self, path: str = WEIGHTS_PATH):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez_compressed(path, **{k: v.astype(np.float32) for k, v in self.state().items()})

    @classmethod
    def load(cls, path: str = WEIGHTS_PATH, device="cuda") -> "UNet":
        net = cls(device=device)
        d = np.load(path)
        for L in net.layers:
            L.w.copy_(torch.as_tensor(d[f"{L.name}.w"]))
            L.wb.copy_(L.w.to(torch.bfloat16))
            L.b.copy_(torch.as_tensor(d[f"{L.name}.b"]))
        net.hw.copy_(torch.as_tensor(d["head.w"]))
        net.hb.copy_(torch.as_tensor(d["head.b"]))
        return net

    # ---- building blocks ------------------------------------------------------------------
    def _conv(self, x, L: Layer, dims, relu=True, w=None, cin=None, cout=None, bias=True):
        nx, ny, nz = dims
        cin = L.cin if cin is None else cin
        cout = L.cout if cout is None else cout
        out = _bf16((nx * ny * nz, cout), self.device)
        call("bsp_unet_conv3_fwd", ptr(out), ptr(x), ptr(L.wb if w is None else w),
             ptr(L.b) if bias else None, nx, ny, nz, cin, cout, 1 if relu else 0, stream_handle())
        return out

    def _pool(self, x, dims, c):
        nx, ny, nz = dims
        out = _bf16((nx * ny * nz // 8, c), self.device)
        call("bsp_unet_pool", ptr(out), ptr(x), nx, ny, nz, c, 0, 0, stream_handle())
        return out

    def _up(self, x, dims, c):
        nx, ny, nz = dims
        out = _bf16((nx * ny * nz, c), self.device)
        call("bsp_unet_up", ptr(out), ptr(x), nx, ny, nz, c, 0, stream_handle())
        return out

    def _add(self, a, b):
        out = a.clone()
        call("bsp_unet_add", ptr(out), ptr(b), out.numel(), stream_handle())
        return out

    # ---- forward ----------------------------------------------------------------------------
    def forward(self, div, mask, dims, dx, dt, rho, scales=None):
        """Returns (p [nx,ny,nz] FP32, cache for backward)."""
        nx, ny, nz = dims
        if nx % 8 or ny % 8 or nz % 8:
            raise ValueError("U-Net grids need dimensions divisible by 8")
        n1 = nx * ny * nz
        d1, d2, d3, d4 = dims, (nx // 2, ny // 2, nz // 2), (nx // 4, ny // 4, nz // 4), \
            (nx // 8, ny // 8, nz // 8)
        s, S, nfl = scales if scales is not None else scene_scales(div, mask, dx, dt, rho)
        st = stream_handle()
        x0 = _bf16((n1, 16), self.device)
        call("bsp_unet_pack_input", ptr(x0), ptr(div), ptr(mask), n1, 1.0 / s, st)
        c = {"x0": x0, "dims": (d1, d2, d3, d4), "scales": (s, S, nfl)}
        B = self.by
        c["a1"] = self._conv(x0, B["e1a"], d1)
        c["e1"] = self._conv(c["a1"], B["e1b"], d1)
        c["p1"] = self._pool(c["e1"], d1, 16)
        c["a2"] = self._conv(c["p1"], B["e2a"], d2)
        c["e2"] = self._conv(c["a2"], B["e2b"], d2)
        c["p2"] = self._pool(c["e2"], d2, 32)
        c["a3"] = self._conv(c["p2"], B["e3a"], d3)
        c["e3"] = self._conv(c["a3"], B["e3b"], d3)
        c["p3"] = self._pool(c["e3"], d3, 64)
        c["a4"] = self._conv(c["p3"], B["bta"], d4)
        c["b4"] = self._conv(c["a4"], B["btb"], d4)
        c["q3"] = self._up(c["b4"], d3, 128)
        c["c3"] = self._conv(c["q3"], B["u3a"], d3)
        c["s3"] = self._add(c["c3"], c["e3"])
        c["u3"] = self._conv(c["s3"], B["u3b"], d3)
        c["q2"] = self._up(c["u3"], d2, 64)
        c["c2"] = self._conv(c["q2"], B["u2a"], d2)
        c["s2"] = self._add(c["c2"], c["e2"])
        c["u2"] = self._conv(c["s2"], B["u2b"], d2)
        c["q1"] = self._up(c["u2"], d1, 32)
        c["c1"] = self._conv(c["q1"], B["u1a"], d1)
        c["s1"] = self._add(c["c1"], c["e1"])
        c["u1"] = self._conv(c["s1"], B["u1b"], d1)
        p = torch.empty(dims, dtype=torch.float32, device=self.device)
        call("bsp_unet_head_fwd", ptr(p), ptr(c["u1"]), ptr(self.hw), ptr(self.hb), ptr(mask), n1,
             S, st)
        c["mask"] = mask
        return p, c

    def predict(self, div, mask, dx, dt, rho) -> torch.Tensor:
        with torch.no_grad():
            p, _ = self.forward(div, mask, tuple(div.shape), dx, dt, rho)
        return p

    # ---- backward -----------------------------------------------------------------------------
    def _wgrad_ws(self, dims, cin, cout):
        nx, ny, nz = dims
        nb = int(_lib.lib().bsp_unet_wgrad_workspace_bytes(nx, ny, nz, cin, cout))
        key = "wg"
        if key not in self._ws or self._ws[key].numel() * 4 < nb:
            self._ws[key] = torch.empty((nb + 3) // 4, dtype=torch.float32, device=self.device)
        return self._ws[key], nb

    def _conv_bwd(self, g, x, out, L: Layer, dims, need_dx=True):
        """g: gradient of the conv's ReLU output (modified in place to the
        pre-activation gradient); x: its input.  Accumulates L.gw, L.gb;
        returns the gradient of x."""
        nx, ny, nz = dims
        st = stream_handle()
        call("bsp_unet_relu_bwd", ptr(g), ptr(out), g.numel(), st)
        ws, nb = self._wgrad_ws(dims, L.cin, L.cout)
        gw = torch.empty_like(L.w)
        gb = torch.empty_like(L.b)
        call("bsp_unet_conv3_wgrad", ptr(gw), ptr(gb), ptr(g), ptr(x), nx, ny, nz, L.cin, L.cout,
             ptr(ws), nb, st)
        L.gw = gw if L.gw is None else L.gw + gw
        L.gb = gb if L.gb is None else L.gb + gb
        if not need_dx:
            return None
        wt = _bf16(L.wb.shape[:1] + (L.cin, L.cout), self.device)
        call("bsp_unet_flip_weights", ptr(wt), ptr(L.wb), L.cin, L.cout, st)
        return self._conv(g, L, dims, relu=False, w=wt, cin=L.cout, cout=L.cin, bias=False)

    def backward(self, c, target):
        """Loss (mean squared error of p / S on fluid cells) and gradients."""
        d1, d2, d3, d4 = c["dims"]
        s, S, nfl = c["scales"]
        n1 = d1[0] * d1[1] * d1[2]
        st = stream_handle()
        B = self.by
        gx = _bf16((n1, 16), self.device)
        parts = torch.empty((18, HEAD_BLOCKS), dtype=torch.float32, device=self.device)
        pred = c["pred"]
        call("bsp_unet_head_loss", ptr(gx), ptr(parts), HEAD_BLOCKS, ptr(pred), ptr(target),
             ptr(c["u1"]), ptr(self.hw), ptr(c["mask"]), n1, 1.0 / S, 1.0 / max(nfl, 1), st)
        sums = torch.empty(18, dtype=torch.float32, device=self.device)
        call("bsp_unet_sum_partials", ptr(sums), ptr(parts), HEAD_BLOCKS, 18, st)
        self.g_hb = sums[1:2].clone()
        self.g_hw = sums[2:18].clone()
        # decoder level 1
        g = self._conv_bwd(gx, c["s1"], c["u1"], B["u1b"], d1)          # d s1
        g_e1 = g.clone()                                                  # skip
        g = self._conv_bwd(g, c["q1"], c["c1"], B["u1a"], d1)            # d q1
        g_u2 = _bf16((d2[0] * d2[1] * d2[2], 32), self.device)
        call("bsp_unet_up", ptr(g_u2), ptr(g), *d1, 32, 1, st)
        g = self._conv_bwd(g_u2, c["s2"], c["u2"], B["u2b"], d2)
        g_e2 = g.clone()
        g = self._conv_bwd(g, c["q2"], c["c2"], B["u2a"], d2)
        g_u3 = _bf16((d3[0] * d3[1] * d3[2], 64), self.device)
        call("bsp_unet_up", ptr(g_u3), ptr(g), *d2, 64, 1, st)
        g = self._conv_bwd(g_u3, c["s3"], c["u3"], B["u3b"], d3)
        g_e3 = g.clone()
        g = self._conv_bwd(g, c["q3"], c["c3"], B["u3a"], d3)
        g_b4 = _bf16((d4[0] * d4[1] * d4[2], 128), self.device)
        call("bsp_unet_up", ptr(g_b4), ptr(g), *d3, 128, 1, st)
        g = self._conv_bwd(g_b4, c["a4"], c["b4"], B["btb"], d4)
        g = self._conv_bwd(g, c["p3"], c["a4"], B["bta"], d4)
        call("bsp_unet_pool", ptr(g_e3), ptr(g), *d3, 64, 1, 1, st)      # g_e3 += pool'(g)
        g = self._conv_bwd(g_e3, c["a3"], c["e3"], B["e3b"], d3)
        g = self._conv_bwd(g, c["p2"], c["a3"], B["e3a"], d3)
        call("bsp_unet_pool", ptr(g_e2), ptr(g), *d2, 32, 1, 1, st)
        g = self._conv_bwd(g_e2, c["a2"], c["e2"], B["e2b"], d2)
        g = self._conv_bwd(g, c["p1"], c["a2"], B["e2a"], d2)
        call("bsp_unet_pool", ptr(g_e1), ptr(g), *d1, 16, 1, 1, st)
        g = self._conv_bwd(g_e1, c["a1"], c["e1"], B["e1b"], d1)
        self._conv_bwd(g, c["x0"], c["a1"], B["e1a"], d1, need_dx=False)
        return sums[0]

    def zero_grad(self):
        for L in self.layers:
            L.gw = L.gb = None

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        st = stream_handle()
        for L in self.layers:
            if L.mw is None:
                L.mw, L.vw = torch.zeros_like(L.w), torch.zeros_like(L.w)
                L.mb, L.vb = torch.zeros_like(L.b), torch.zeros_like(L.b)
            call("bsp_unet_adam", ptr(L.w), ptr(L.wb), ptr(L.mw), ptr(L.vw), ptr(L.gw), L.w.numel(),
                 lr, b1, b2, eps, self.step, st)
            call("bsp_unet_adam", ptr(L.b), None, ptr(L.mb), ptr(L.vb), ptr(L.gb), L.b.numel(), lr,
                 b1, b2, eps, self.step, st)
        if not hasattr(self, "mhw"):
            self.mhw, self.vhw = torch.zeros_like(self.hw), torch.zeros_like(self.hw)
            self.mhb, self.vhb = torch.zeros_like(self.hb), torch.zeros_like(self.hb)
        call("bsp_unet_adam", ptr(self.hw), None, ptr(self.mhw), ptr(self.vhw), ptr(self.g_hw), 16,
             lr, b1, b2, eps, self.step, st)
        call("bsp_unet_adam", ptr(self.hb), None, ptr(self.mhb), ptr(self.vhb), ptr(self.g_hb), 1,
             lr, b1, b2, eps, self.step, st)

    def train_step(self, div, mask, target, dx, dt, rho, lr=1e-3) -> float:
        dims = tuple(div.shape)
        pred, c = self.forward(div, mask, dims, dx, dt, rho)
        c["pred"] = pred
        self.zero_grad()
        loss = self.backward(c, target)
        self.adam_step(lr)
        return loss
