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
divergence over fluid cells) and predicts p / S with S = -(rho dx^2 / dt) s,
the solution of A (p / S) = div / s.  The loss is the relative squared error
sum (y - t)^2 / sum t^2 over fluid cells, so every scene weighs the same.
"""
from __future__ import annotations

import ctypes
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
    """(s, S, n_fluid): input scale s (RMS divergence on fluid cells) and
    output scale S = -(rho dx^2 / dt) s, so that the target p / S solves
    A (p / S) = div / s: dimensionless, O(1) per unit input."""
    fl = (mask & 0x80) != 0
    nfl = int(fl.sum().item())
    s = float(torch.sqrt((div[fl].double() ** 2).sum() / max(nfl, 1)).item()) if nfl else 1.0
    s = s if s > 0 else 1.0
    S = -(rho * dx * dx / dt) * s
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
        """Convolution weights as BF16 bit patterns (the inference copy), biases
        and head in FP32."""
        os.makedirs(os.path.dirname(path), exist_ok=True)
        out = {}
        for k, v in self.state().items():
            if k.endswith(".w") and not k.startswith("head"):
                b = torch.as_tensor(v).to(torch.bfloat16).view(torch.int16).numpy()
                out[k + ".bf16"] = b
            else:
                out[k] = v.astype(np.float32)
        np.savez_compressed(path, **out)

    @classmethod
    def load(cls, path: str = WEIGHTS_PATH, device="cuda") -> "UNet":
        net = cls(device=device)
        d = np.load(path)
        for L in net.layers:
            if f"{L.name}.w.bf16" in d:
                w = torch.as_tensor(d[f"{L.name}.w.bf16"]).view(torch.bfloat16).float()
            else:
                w = torch.as_tensor(d[f"{L.name}.w"])
            L.w.copy_(w)
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

    def predict(self, div, mask, dx, dt, rho, backend: str = "tc") -> torch.Tensor:
        """The network's pressure for ``div``.  ``backend="tc"``: inference on
        the fifth-generation tensor cores (tcgen05 kernels, padded layout,
        buffers kept per grid shape); ``"mma"``: the training forward pass
        (mma.sync kernels), which also keeps the activations for backward."""
        if backend == "tc":
            return self.tc_plan(tuple(div.shape)).run(div, mask, dx, dt, rho)
        with torch.no_grad():
            p, _ = self.forward(div, mask, tuple(div.shape), dx, dt, rho)
        return p

    def tc_plan(self, dims) -> "TcPlan":
        plans = self.__dict__.setdefault("_tc_plans", {})
        if dims not in plans:
            plans[dims] = TcPlan(self, dims)
        plan = plans[dims]
        if plan.version != self.step:
            plan.refresh_weights()
        return plan

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

    def _spmv(self, x, mask):
        out = torch.empty_like(x)
        nx, ny, nz = x.shape
        call("bsp_spmv", ptr(out), ptr(x), ptr(mask), nx, ny, nz, stream_handle())
        return out

    def backward(self, c, target, loss: str = "energy"):
        """Loss and gradients.  With y = prediction / S and t = target / S on
        fluid cells: ``l2``: sum (y - t)^2 / sum t^2; ``energy``: the error in
        the operator's energy norm, (y - t)^T A (y - t) / t^T A t -- the norm
        the conjugate-gradient finish is sensitive to (A symmetric positive
        definite on the fluid cells, so dL/dy = 2 A (y - t) / t^T A t);
        ``residual``: ||A (y - t)||^2 / ||A t||^2, the starting residual
        relative to ||b|| (dL/dy = 2 A A (y - t) / ||A t||^2)."""
        d1, d2, d3, d4 = c["dims"]
        s, S, nfl = c["scales"]
        n1 = d1[0] * d1[1] * d1[2]
        st = stream_handle()
        B = self.by
        gx = _bf16((n1, 16), self.device)
        pred = c["pred"]
        mask = c["mask"]
        fl = (mask & 0x80) != 0
        sums = torch.empty(18, dtype=torch.float32, device=self.device)
        if loss == "l2":
            parts = torch.empty((18, HEAD_BLOCKS), dtype=torch.float32, device=self.device)
            norm = float(((target[fl].double() / S) ** 2).sum().item()) or 1.0
            c["norm"] = norm
            call("bsp_unet_head_loss", ptr(gx), ptr(parts), HEAD_BLOCKS, ptr(pred), ptr(target),
                 ptr(c["u1"]), ptr(self.hw), ptr(mask), n1, 1.0 / S, 1.0 / norm, st)
            call("bsp_unet_sum_partials", ptr(sums), ptr(parts), HEAD_BLOCKS, 18, st)
            self.g_hb = sums[1:2].clone()
            self.g_hw = sums[2:18].clone()
            lval = sums[0]
        else:
            zero = torch.zeros((), dtype=torch.float32, device=self.device)
            d = torch.where(fl, (pred - target) / S, zero).contiguous()
            t = torch.where(fl, target / S, zero).contiguous()
            Ad = self._spmv(d, mask)
            At = self._spmv(t, mask)
            if loss == "residual":
                # ||A (y - t)||^2 / ||A t||^2: the starting residual relative to
                # ||b||, the quantity the solve's stopping test measures
                normA = float((At.double() ** 2).sum().item()) or 1.0
                lval = ((Ad.double() ** 2).sum() / normA).float()
                gy = (2.0 / normA) * self._spmv(Ad.contiguous(), mask)
            else:
                normA = float((t.double() * At.double()).sum().item()) or 1.0
                lval = ((d.double() * Ad.double()).sum() / normA).float()
                gy = (2.0 / normA) * Ad
            c["norm"] = normA
            parts = torch.empty((17, HEAD_BLOCKS), dtype=torch.float32, device=self.device)
            call("bsp_unet_head_bwd", ptr(gx), ptr(parts), HEAD_BLOCKS, ptr(gy), ptr(c["u1"]),
                 ptr(self.hw), ptr(mask), n1, st)
            call("bsp_unet_sum_partials", ptr(sums), ptr(parts), HEAD_BLOCKS, 17, st)
            self.g_hb = sums[0:1].clone()
            self.g_hw = sums[1:17].clone()
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
        return lval

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

    def train_step(self, div, mask, target, dx, dt, rho, lr=1e-3, loss: str = "residual"):
        dims = tuple(div.shape)
        pred, c = self.forward(div, mask, dims, dx, dt, rho)
        c["pred"] = pred
        self.zero_grad()
        loss = self.backward(c, target, loss)
        self.adam_step(lr)
        return loss


class TcPlan:
    """Inference of the network on one grid shape with the tensor-core
    kernels (``bsp_unet_tc_*``): activations on the padded layout (a one-cell
    zero halo per level), every buffer allocated and zero-filled once, the
    weight images rebuilt when the weights change.  The skip additions of the
    decoder are fused into the epilogue of the convolution before them."""

    def __init__(self, net: UNet, dims):
        nx, ny, nz = dims
        if nx % 8 or ny % 8 or nz % 8:
            raise ValueError("U-Net grids need dimensions divisible by 8")
        self.net = net
        self.dims = (dims, (nx // 2, ny // 2, nz // 2), (nx // 4, ny // 4, nz // 4),
                     (nx // 8, ny // 8, nz // 8))
        lib = _lib.lib()
        dev = net.device

        def buf(level, c):
            rows = int(lib.bsp_unet_tc_rows(*self.dims[level]))
            return torch.zeros((rows, c), dtype=torch.bfloat16, device=dev)

        # level-indexed activations (names as in UNet.forward)
        spec = {"x0": (0, 16), "a1": (0, 16), "e1": (0, 16), "p1": (1, 16), "a2": (1, 32),
                "e2": (1, 32), "p2": (2, 32), "a3": (2, 64), "e3": (2, 64), "p3": (3, 64),
                "a4": (3, 128), "b4": (3, 128), "q3": (2, 128), "c3": (2, 64), "u3": (2, 64),
                "q2": (1, 64), "c2": (1, 32), "u2": (1, 32), "q1": (0, 32), "c1": (0, 16),
                "u1": (0, 16)}
        self.a = {k: buf(lv, c) for k, (lv, c) in spec.items()}
        self.wimg = {L.name: torch.empty(27 * L.cin * L.cout, dtype=torch.bfloat16, device=dev)
                     for L in net.layers}
        self.s_dev = torch.ones(1, dtype=torch.float32, device=dev)  # input scale s
        nb = int(lib.bsp_unet_scale_workspace_bytes())
        self.scale_ws = torch.empty((nb + 7) // 8, dtype=torch.float64, device=dev)
        self.version = None
        self.refresh_weights()

    def refresh_weights(self):
        st = stream_handle()
        for L in self.net.layers:
            call("bsp_unet_tc_weights", ptr(self.wimg[L.name]), ptr(L.wb), L.cin, L.cout, st)
        self.version = self.net.step

    # the convolutions of one forward pass: (output, input, layer, level, skip)
    CONVS = (("a1", "x0", "e1a", 0, None), ("e1", "a1", "e1b", 0, None),
             ("a2", "p1", "e2a", 1, None), ("e2", "a2", "e2b", 1, None),
             ("a3", "p2", "e3a", 2, None), ("e3", "a3", "e3b", 2, None),
             ("a4", "p3", "bta", 3, None), ("b4", "a4", "btb", 3, None),
             ("c3", "q3", "u3a", 2, "e3"), ("u3", "c3", "u3b", 2, None),
             ("c2", "q2", "u2a", 1, "e2"), ("u2", "c2", "u2b", 1, None),
             ("c1", "q1", "u1a", 0, "e1"), ("u1", "c1", "u1b", 0, None))

    def conv_timings(self, layers=None, reps: int = 10, warmup: int = 2, trace: bool = False):
        """Per-layer device time of the tensor-core convolutions on this plan's
        current activations (run() first): CUDA events around ``reps``
        back-to-back launches after ``warmup`` untimed ones; with ``trace`` the
        cycle accounting of one more launch (bsp_unet_tc_trace) as fractions
        of the CTA lifetime."""
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        rows = []
        for dst, src, name, level, skip in self.CONVS:
            if layers and name not in layers:
                continue
            L = self.net.by[name]
            for _ in range(warmup):
                self._conv(dst, src, name, level, skip)
            row = {"layer": name, "dims": list(self.dims[level]), "cin": L.cin, "cout": L.cout}
            if reps > 0:
                e0.record()
                for _ in range(reps):
                    self._conv(dst, src, name, level, skip)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                n = self.dims[level][0] * self.dims[level][1] * self.dims[level][2]
                row.update(ms=round(ms, 4), TFLOPs=round(2.0 * 27 * L.cin * L.cout * n / ms / 1e9, 1))
            if trace:
                tr = np.zeros(8, np.uint64)
                call("bsp_unet_tc_trace", None, 1)
                self._conv(dst, src, name, level, skip)
                torch.cuda.synchronize()
                call("bsp_unet_tc_trace", tr.ctypes.data, 0)
                life = max(float(tr[5]), 1.0)
                keys = ("producer_wait", "mma_wait_stage", "mma_wait_accumulator",
                        "epilogue_wait", "epilogue_busy", None, None, "mma_busy")
                row["trace"] = {k: round(float(tr[i]) / life, 3) for i, k in enumerate(keys) if k}
                row["trace"]["cycles_per_item"] = round(life / max(float(tr[6]), 1.0), 1)
            rows.append(row)
        return rows

    def _conv(self, dst, src, name, level, skip=None):
        L = self.net.by[name]
        call("bsp_unet_tc_conv3", ptr(self.a[dst]), ptr(self.a[src]), ptr(self.wimg[name]),
             ptr(L.b), ptr(self.a[skip]) if skip else None, *self.dims[level], L.cin, L.cout, 1,
             stream_handle())

    def run(self, div, mask, dx, dt, rho, out=None) -> torch.Tensor:
        """Network pressure for ``div`` (no host synchronisation: the input
        scale s is computed and applied on the device, S = -(rho dx^2/dt) s)."""
        st = stream_handle()
        d = self.dims
        call("bsp_unet_input_scale", ptr(self.s_dev), ptr(div), ptr(mask), *d[0],
             ptr(self.scale_ws), self.scale_ws.numel() * 8, st)
        call("bsp_unet_tc_pack", ptr(self.a["x0"]), ptr(div), ptr(mask), *d[0], ptr(self.s_dev),
             st)
        cv = self.CONVS
        for c in cv[0:2]:
            self._conv(*c)
        call("bsp_unet_tc_pool", ptr(self.a["p1"]), ptr(self.a["e1"]), *d[0], 16, st)
        for c in cv[2:4]:
            self._conv(*c)
        call("bsp_unet_tc_pool", ptr(self.a["p2"]), ptr(self.a["e2"]), *d[1], 32, st)
        for c in cv[4:6]:
            self._conv(*c)
        call("bsp_unet_tc_pool", ptr(self.a["p3"]), ptr(self.a["e3"]), *d[2], 64, st)
        for c in cv[6:8]:
            self._conv(*c)
        call("bsp_unet_tc_up", ptr(self.a["q3"]), ptr(self.a["b4"]), *d[2], 128, st)
        for c in cv[8:10]:   # c3 = relu(conv) + e3, then u3
            self._conv(*c)
        call("bsp_unet_tc_up", ptr(self.a["q2"]), ptr(self.a["u3"]), *d[1], 64, st)
        for c in cv[10:12]:
            self._conv(*c)
        call("bsp_unet_tc_up", ptr(self.a["q1"]), ptr(self.a["u2"]), *d[0], 32, st)
        for c in cv[12:14]:
            self._conv(*c)
        p = out if out is not None else torch.empty(d[0], dtype=torch.float32,
                                                    device=self.net.device)
        call("bsp_unet_tc_head", ptr(p), ptr(self.a["u1"]), ptr(self.net.hw), ptr(self.net.hb),
             ptr(mask), *d[0], ptr(self.s_dev), -(rho * dx * dx / dt), st)
        return p


def coarse_materials(mat_t: torch.Tensor) -> torch.Tensor:
    """Material grid coarsened 2x (once per geometry): fluid where at least
    half of the 8 children are fluid, else air where any child is air, else
    solid -- the free surface stays a Dirichlet boundary on the coarse grid."""
    nx, ny, nz = mat_t.shape
    m = mat_t.view(nx // 2, 2, ny // 2, 2, nz // 2, 2)
    nf = (m == 0).sum(dim=(1, 3, 5))
    na = (m == 2).sum(dim=(1, 3, 5))
    return torch.where(nf >= 4, 0, torch.where(na > 0, 2, 1)).to(torch.int32).contiguous()


class WarmStart:
    """The network's starting pressure for one grid.

    ``mode="full"``: the network at the grid's own resolution.  ``"coarse"``:
    the network on the grid coarsened 2x (divergence averaged over the fluid
    children, classes by coarse_materials), its pressure interpolated back
    onto the fine fluid cells (bsp_unet_restrict_div / bsp_unet_prolong) --
    an eighth of the network's work, for grids large enough that a full-size
    prediction would cost more than the iterations it saves.  ``"coarse4"``:
    the same through two coarsenings (a 64th of the work; the network then
    sees the pot at 4x the cell size, where its receptive field spans more of
    the domain).

    ``scale=True`` (default) multiplies the prediction by the energy-optimal
    gamma = (b . p) / (p . A p) (bsp_unet_energy_scale_keep), so the guess
    handed to the solve is never farther from the solution than zero in the
    A-norm: the plain solve stays the judge of the network's error.  With
    ``keep_below`` > 0 the scaled guess is kept only when its relative
    residual ||b - A p|| / ||b|| is below that value, else the solve starts
    from zero (decided on the device, no host synchronisation; the residual
    of the last guess is in ``relres``).  The default 0.1: measured on the
    384x384x256 pot, guesses with relative residuals 1.01 and 0.60 took 34
    and 35 inner iterations and one at 0.10 took 31, against 31 from zero."""

    def __init__(self, net: UNet, mat_t: torch.Tensor, mask: torch.Tensor, mode: str = "auto",
                 scale: bool = True, keep_below: float = 0.1):
        from .fluid import cell_mask

        self.net = net
        self.dims = tuple(mat_t.shape)
        self.mask = mask
        self.scale = scale
        self.keep_below = float(keep_below)
        if scale:
            self.Ap = torch.empty(self.dims, dtype=torch.float32, device=mat_t.device)
            nb = int(_lib.lib().bsp_unet_scale_workspace_bytes())
            self.ws = torch.empty((nb + 7) // 8, dtype=torch.float64, device=mat_t.device)
            self.gamma = torch.zeros(1, dtype=torch.float32, device=mat_t.device)
            self.relres = torch.zeros(1, dtype=torch.float32, device=mat_t.device)
        nx, ny, nz = self.dims
        if mode == "auto":
            # large grids: the network two coarsenings down when the
            # dimensions allow (measured at 384x384x256: a 1.0 ms guess against
            # 2.5 ms one coarsening down, and no more solve iterations after
            # it), else one coarsening down
            big = nx * ny * nz >= 16_000_000
            if big and nx % 32 == 0 and ny % 32 == 0 and nz % 32 == 0:
                mode = "coarse4"
            elif big and nx % 16 == 0 and ny % 16 == 0 and nz % 16 == 0:
                mode = "coarse"
            else:
                mode = "full"
        self.mode = mode
        # coarse levels 1 .. nlev: masks, divergence and pressure buffers
        self.nlev = {"full": 0, "coarse": 1, "coarse4": 2}[mode]
        self.maskc, self.divc, self.pc = [], [], []
        m = mat_t
        for lv in range(1, self.nlev + 1):
            m = coarse_materials(m)
            self.maskc.append(cell_mask(m))
            f = 1 << lv
            self.divc.append(torch.zeros((nx // f, ny // f, nz // f), dtype=torch.float32,
                                         device=mat_t.device))
            self.pc.append(torch.zeros_like(self.divc[-1]))

    def guess(self, div, dx, dt, rho, out: torch.Tensor, graph: bool = True) -> torch.Tensor:
        """Writes the starting pressure into ``out``.  With ``graph`` the
        launches of one guess (about 25 kernels) are captured once into a CUDA
        graph per (div, out, dx, dt, rho) and replayed afterwards."""
        if not graph:
            return self._launch(div, dx, dt, rho, out)
        key = (div.data_ptr(), out.data_ptr(), float(dx), float(dt), float(rho),
               self.net.step)
        g = self.__dict__.get("_graph")
        if g is None or g[0] != key:
            self._launch(div, dx, dt, rho, out)  # first run: plans, weights, opt-ins
            cg = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(cg, stream=s):
                    self._launch(div, dx, dt, rho, out)
            torch.cuda.current_stream().wait_stream(s)
            self._graph = g = (key, cg)
        g[1].replay()
        return out

    def _launch(self, div, dx, dt, rho, out: torch.Tensor) -> torch.Tensor:
        nx, ny, nz = self.dims
        st = stream_handle()
        if self.nlev == 0:
            self.net.tc_plan(self.dims).run(div, self.mask, dx, dt, rho, out=out)
        else:
            # restrict level by level, the network on the coarsest, prolong back
            fine_d, fine_m, dims = div, self.mask, self.dims
            for lv in range(self.nlev):
                call("bsp_unet_restrict_div", ptr(self.divc[lv]), ptr(self.maskc[lv]), ptr(fine_d),
                     ptr(fine_m), *dims, st)
                fine_d, fine_m = self.divc[lv], self.maskc[lv]
                dims = tuple(self.divc[lv].shape)
            k = self.nlev - 1
            self.net.tc_plan(dims).run(self.divc[k], self.maskc[k], float(1 << self.nlev) * dx,
                                       dt, rho, out=self.pc[k])
            for lv in range(k, -1, -1):
                dst = out if lv == 0 else self.pc[lv - 1]
                dmask = self.mask if lv == 0 else self.maskc[lv - 1]
                ddims = self.dims if lv == 0 else tuple(self.pc[lv - 1].shape)
                call("bsp_unet_prolong", ptr(dst), ptr(self.pc[lv]), ptr(dmask), *ddims, st)
        if self.scale:
            call("bsp_spmv", ptr(self.Ap), ptr(out), ptr(self.mask), nx, ny, nz, st)
            call("bsp_unet_energy_scale_keep", ptr(out), ptr(self.Ap), ptr(div), ptr(self.mask),
                 nx, ny, nz, -(rho * dx * dx / dt), self.keep_below, ptr(self.ws),
                 self.ws.numel() * 8, ptr(self.gamma), ptr(self.relres), st)
        return out


# ---- training data: the plain solver on seeded pot variants ----------------------------------
def training_specs(count: int, seed: int = 11):
    """Pot variants of the batched configuration (48^3 .. 128x128x96 cells,
    wall 2-4 cells, radius filling the box minus the wall and a 2-cell pad,
    water level 0.6-0.85 of the height, carrot radius 4-10 cells) with every
    dimension a multiple of 8 (the network pools three times)."""
    from .scenes import PotSpec

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nxy = int(rng.integers(6, 17)) * 8          # 48 .. 128
        nz = int(rng.integers(6, 13)) * 8           # 48 .. 96
        t_w = int(rng.integers(2, 5))
        r_in = nxy / 2.0 - t_w - 2
        level = float(rng.uniform(0.6, 0.85))
        water = t_w + level * (nz - t_w)
        cr = min(float(rng.integers(4, 11)), 0.45 * (water - t_w))
        out.append(PotSpec(nxy, nxy, nz, r_in=r_in, t_w=t_w, water_line=water, carrot_r=cr,
                           carrot_len=min(1.2 * r_in, 5.0 * cr)))
    return out


class SceneSource:
    """Divergence fields of one pot geometry on the GPU: seeded N(0, 0.05)
    face velocities, box-smoothed three times (edge-replicated 3x3x3 mean),
    a Gaussian plume of amplitude A on fluid z-faces, no-slip; the divergence
    of that field.  The same rules as scenes.velocity_field, drawn with torch's
    generator so a new field costs no host work."""

    def __init__(self, mat: np.ndarray, device="cuda", sigma: float = 3.0):
        from .fluid import cell_mask

        self.mat = mat
        self.shape = mat.shape
        self.device = torch.device(device)
        self.mat_t = torch.as_tensor(np.ascontiguousarray(mat, np.int32)).to(self.device)
        self.mask = cell_mask(self.mat_t)
        nx, ny, nz = mat.shape
        ci = torch.arange(nx, device=self.device, dtype=torch.float32)[:, None] + 0.5
        cj = torch.arange(ny, device=self.device, dtype=torch.float32)[None, :] + 0.5
        r2 = (ci - nx / 2.0) ** 2 + (cj - ny / 2.0) ** 2
        self.gauss = torch.exp(-r2 / (2.0 * sigma * sigma))
        f = torch.as_tensor(mat == 0, device=self.device)
        ff = torch.zeros((nx, ny, nz + 1), dtype=torch.bool, device=self.device)
        ff[:, :, 1:-1] = f[:, :, :-1] & f[:, :, 1:]
        self.zface_fluid = ff

    @staticmethod
    def _box3(a):
        import torch.nn.functional as Fn

        x = a[None, None]
        for _ in range(3):
            x = Fn.avg_pool3d(Fn.pad(x, (1, 1, 1, 1, 1, 1), mode="replicate"), 3, stride=1)
        return x[0, 0]

    def draw(self, seed: int, plume: float, dx: float):
        from .fluid import compute_divergence
        from ._lib import call as _call

        nx, ny, nz = self.shape
        g = torch.Generator(device=self.device).manual_seed(int(seed))
        U = []
        for shp in ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)):
            U.append(self._box3(torch.randn(shp, generator=g, device=self.device) * 0.05)
                     .contiguous())
        U[2] += torch.where(self.zface_fluid, plume * self.gauss[:, :, None], 0.0)
        _call("bsp_enforce_no_slip", ptr(U[0]), ptr(U[1]), ptr(U[2]), ptr(self.mask), nx, ny, nz,
              stream_handle())
        div = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        compute_divergence(div, *U, self.mask, dx)
        return div


def train(steps: int = 20000, n_geometries: int = 64, seed: int = 11, lr: float = 1e-3,
          dx: float = 0.002, dt: float = 0.01, rho: float = 997.0, log_every: int = 500,
          net: UNet | None = None, log=print, loss: str = "residual") -> UNet:
    """Train on ``steps`` fresh (divergence, mask, pressure) triples: geometry
    ``step % n_geometries``, velocity seed ``step``, plume amplitude drawn in
    [0.02, 0.3] m/s; the target is the plain solve to FP64 rel-residual 1e-6.
    Adam with a cosine learning-rate decay to lr / 10; ``loss`` as in
    UNet.backward.  The default, the starting residual, is what the
    multigrid-preconditioned finish gains from: its passes stop on the
    residual, and the V-cycle removes smooth error cheaply, so a prediction
    with a small residual saves more iterations than one with a small L2
    error."""
    from .scenes import pot_mat
    from .solver import TolSolver

    net = net or UNet(seed=seed)
    specs = training_specs(n_geometries, seed)
    sources = [SceneSource(pot_mat(s)) for s in specs]
    solvers = [TolSolver(src.mask, "fp32") for src in sources]
    rng = np.random.default_rng(seed + 1)
    running = None
    for step in range(steps):
        q = step % n_geometries
        src = sources[q]
        div = src.draw(seed * 1000003 + step, float(rng.uniform(0.02, 0.3)), dx)
        p = torch.zeros_like(div)
        solvers[q].solve(div, dx, dt, rho, tol=1e-6, p=p)
        cur_lr = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * step / max(steps, 1))))
        loss_v = float(net.train_step(div, src.mask, p, dx, dt, rho, lr=cur_lr, loss=loss).item())
        running = loss_v if running is None else 0.98 * running + 0.02 * loss_v
        if log and (step % log_every == 0 or step == steps - 1):
            log(f"step {step} loss {loss_v:.4g} running {running:.4g} lr {cur_lr:.2g}")
    return net


def evaluate(net: UNet, spec, seeds=(101, 102, 103), plume: float = 0.1, dx: float = 0.002,
             dt: float = 0.01, rho: float = 997.0, storage: str = "fp32", tol: float = 1e-6):
    """Cold and warm-started solves of held-out scenes: inner iterations of
    each; before the finishing solve, the network's relative error against the
    converged pressure and its relative residual ||b - A p|| / ||b|| (fluid
    cells); the times of the prediction and of both solves (CUDA events)."""
    from .scenes import pot_mat
    from .solver import TolSolver

    src = SceneSource(pot_mat(spec))
    solver = TolSolver(src.mask, storage)
    fl = (src.mask & 0x80) != 0
    rows = []
    for sd in seeds:
        div = src.draw(sd, plume, dx)
        p_cold = torch.zeros_like(div)
        solver.solve(div, dx, dt, rho, tol=tol, p=p_cold)  # setup and warm-up
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        p_cold.zero_()
        ev[0].record()
        rc = solver.solve(div, dx, dt, rho, tol=tol, p=p_cold)
        ev[1].record()
        net.predict(div, src.mask, dx, dt, rho)  # first-call allocations out of the timing
        ev[2].record()
        p_net = net.predict(div, src.mask, dx, dt, rho)
        ev[3].record()
        p_warm = p_net.clone()
        ev[4].record()
        rw = solver.solve(div, dx, dt, rho, tol=tol, p=p_warm, warm_start=True)
        ev[5].record()
        torch.cuda.synchronize()
        ref = p_cold[fl].double()
        err = float(torch.linalg.norm(p_net[fl].double() - ref) / torch.linalg.norm(ref))
        b = (-(rho * dx * dx / dt) * div.double())[fl]
        r0 = b - net._spmv(p_net.contiguous(), src.mask).double()[fl]
        res0 = float(torch.linalg.norm(r0) / torch.linalg.norm(b))
        rows.append({"seed": sd, "cold_inner": rc.inner_iterations,
                     "warm_inner": rw.inner_iterations, "net_rel_error": err,
                     "net_rel_residual": res0,
                     "cold_ms": ev[0].elapsed_time(ev[1]), "predict_ms": ev[2].elapsed_time(ev[3]),
                     "warm_ms": ev[4].elapsed_time(ev[5]),
                     "cold_rel_residual": rc.rel_residual, "warm_rel_residual": rw.rel_residual})
    return rows


def main(argv=None):
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(description="train / evaluate the learned warm start; time "
                                 "its tensor-core convolutions")
    ap.add_argument("cmd", choices=["train", "eval", "convs"])
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--out", default=WEIGHTS_PATH)
    ap.add_argument("--weights", default=WEIGHTS_PATH)
    ap.add_argument("--layers", default="", help="convs: comma-separated layer names (all)")
    ap.add_argument("--reps", type=int, default=10, help="convs: timed launches per layer")
    ap.add_argument("--warmup", type=int, default=2, help="convs: untimed launches per layer")
    ap.add_argument("--trace", action="store_true", help="convs: cycle accounting per layer")
    ap.add_argument("--epilogue", type=int, default=0,
                    help="convs: epilogue warpgroups of the convolution kernel (2-4; 0 default)")
    args = ap.parse_args(argv)
    if args.cmd == "convs":
        if args.epilogue:
            call("bsp_set_tuning", 16, args.epilogue)
        # one forward pass on the 192x192x128 pot (synthetic divergence), then
        # the convolutions one layer at a time on its activations
        from .scenes import pot_192, pot_mat

        net = UNet.load(args.weights)
        src = SceneSource(pot_mat(pot_192(2)))
        div = src.draw(5, 0.1, 0.002)
        plan = net.tc_plan(tuple(div.shape))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        plan.run(div, src.mask, 0.002, 0.01, 997.0)
        e0.record()
        plan.run(div, src.mask, 0.002, 0.01, 997.0)
        e1.record()
        torch.cuda.synchronize()
        layers = [x for x in args.layers.split(",") if x]
        rows = plan.conv_timings(layers, args.reps, args.warmup, args.trace)
        flag = ctypes.c_int(0)
        call("bsp_unet_tc_error", ctypes.addressof(flag))
        print(json.dumps({"dims": list(plan.dims[0]), "forward_ms": round(e0.elapsed_time(e1), 4),
                          "conv_total_ms": round(sum(r.get("ms", 0.0) for r in rows), 4),
                          "convs": rows, "timeout_flag": flag.value}))
        return
    if args.cmd == "train":
        t0 = time.time()
        net = train(args.steps)
        torch.cuda.synchronize()
        net.save(args.out)
        print(json.dumps({"trained_steps": args.steps, "seconds": round(time.time() - t0, 1),
                          "weights": args.out}))
    else:
        from .scenes import pot_192

        net = UNet.load(args.weights)
        for tw in (2, 3, 4):
            print(json.dumps({"wall": tw, "rows": evaluate(net, pot_192(tw))}))


if __name__ == "__main__":
    main()
