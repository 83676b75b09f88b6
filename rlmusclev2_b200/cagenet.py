"""Per-cage-vertex MLP of the learned coarse correction, on the library's
tensor-core kernels (xpbd_gemm_bf16 and friends).

Network: 64 features -> 4 hidden layers of width 256 with GELU -> 3 outputs
(the cage correction in millimetres).  Weights live as FP32 masters with BF16
copies (row-major [out][in] for the forward GEMM, transposed [in][out] for
the backward GEMM); activations and deltas are BF16, every product
accumulates in FP32.  One sample per cage vertex; the batch is the cage
(padded to a multiple of 128 rows, padded rows carry zero loss gradient).

Forward of layer l:  Z_l = H_l W_l^T + b_l,  H_{l+1} = gelu(Z_l)
Backward:            dZ_4 = dL/dY,  dW_l = dZ_l^T H_l,  db_l = sum_s dZ_l,
                     dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1})
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi as capi

DIMS = (64, 256, 256, 256, 256, 3)
OUT_PAD_FWD = 16   # rows of the last layer's weight (n of its GEMM, a multiple of 16)
OUT_PAD_BWD = 64   # k of the last layer's backward GEMM (a multiple of 64)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def gemm(lib, stream, a, b, m, n, k, *, lda=None, ldb=None, bias=None, act=0, gelu_grad_of=None, out_pre=None,
         out_f32=None, out_bf16=None, out_bf16_t=None, status=None, n_tile=None, flags=0):
    """C = A B^T (+ epilogue) through xpbd_gemm_bf16; tensors are CUDA, BF16
    operands row-major along k.  Output row strides are the tensors' own.
    ``flags``: XpbdGemm.flags (1: thread-staged operands instead of TMA)."""
    g = capi.XpbdGemm()
    g.a, g.b = a.data_ptr(), b.data_ptr()
    g.lda = lda if lda is not None else a.shape[-1]
    g.ldb = ldb if ldb is not None else b.shape[-1]
    g.m, g.n, g.k, g.act = int(m), int(n), int(k), int(act)
    g.bias = None if bias is None else bias.data_ptr()
    if gelu_grad_of is not None:
        g.gelu_grad_of, g.ld_g = gelu_grad_of.data_ptr(), gelu_grad_of.shape[-1]
    if out_pre is not None:
        g.out_pre, g.ld_pre = out_pre.data_ptr(), out_pre.shape[-1]
    if out_f32 is not None:
        g.out_f32, g.ld_f32 = out_f32.data_ptr(), out_f32.shape[-1]
    if out_bf16 is not None:
        g.out_bf16, g.ld_bf16 = out_bf16.data_ptr(), out_bf16.shape[-1]
    if out_bf16_t is not None:
        g.out_bf16_t, g.ld_bf16_t = out_bf16_t.data_ptr(), out_bf16_t.shape[-1]
    g.status = None if status is None else status.data_ptr()
    g.flags = int(flags)
    if n_tile is None:
        # 64-column tiles: four times the CTAs of a 256-column tile on the
        # MLP's 256-wide layers, each with a quarter of the epilogue (measured
        # 12.4 against 16.5 (128) and 24.9 us (256) at 9472 x 256 x 64)
        n_tile = min(64, ((int(n) + 15) // 16) * 16)
    capi.check(lib.xpbd_gemm_bf16(C.byref(g), int(n_tile), stream))


class CageMLP:
    """The MLP, its training buffers for a batch of up to ``m_max`` samples,
    and Adam state."""

    def __init__(self, device, m_max: int, seed: int = 0, stream=None):
        self.lib = capi.load()
        self.device = torch.device(device)
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._sp = C.c_void_p(self.stream.cuda_stream)
        self.m_pad = ((int(m_max) + 127) // 128) * 128
        dev, f32, bf = self.device, torch.float32, torch.bfloat16
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []          # FP32 masters [out][in], [out]
        self.Wb, self.Wt = [], []        # BF16 [out_pad][in], [in][out_pad_k]
        self.mW, self.vW, self.mb, self.vb = [], [], [], []
        for l in range(5):
            fi, fo = DIMS[l], DIMS[l + 1]
            lim = np.sqrt(6.0 / fi) if l < 4 else np.sqrt(6.0 / (fi + fo))
            w = rng.uniform(-lim, lim, (fo, fi)).astype(np.float32)
            self.W.append(torch.from_numpy(w).to(dev))
            self.b.append(torch.zeros(fo, dtype=f32, device=dev))
            op_f = OUT_PAD_FWD if l == 4 else fo
            op_b = OUT_PAD_BWD if l == 4 else fo
            self.Wb.append(torch.zeros((op_f, fi), dtype=bf, device=dev))
            self.Wt.append(torch.zeros((fi, op_b), dtype=bf, device=dev))
            for lst in (self.mW, self.vW):
                lst.append(torch.zeros((fo, fi), dtype=f32, device=dev))
            for lst in (self.mb, self.vb):
                lst.append(torch.zeros(fo, dtype=f32, device=dev))
        self.bpad4 = torch.zeros(OUT_PAD_FWD, dtype=f32, device=dev)
        self.refresh_copies()
        M = self.m_pad
        self.X = torch.zeros((M, 64), dtype=bf, device=dev)
        self.Xt = torch.zeros((64, M), dtype=bf, device=dev)
        self.Z = [torch.zeros((M, 256), dtype=f32, device=dev) for _ in range(4)]
        self.H = [None] + [torch.zeros((M, 256), dtype=bf, device=dev) for _ in range(4)]
        self.Ht = [self.Xt] + [torch.zeros((256, M), dtype=bf, device=dev) for _ in range(4)]
        self.Y = torch.zeros((M, OUT_PAD_FWD), dtype=f32, device=dev)
        self.dY = torch.zeros((M, OUT_PAD_BWD), dtype=bf, device=dev)
        self.dYt = torch.zeros((OUT_PAD_BWD, M), dtype=bf, device=dev)
        self.dZ = [torch.zeros((M, 256), dtype=bf, device=dev) for _ in range(2)]
        self.dZt = [torch.zeros((256, M), dtype=bf, device=dev) for _ in range(2)]
        self.gW = [torch.zeros((DIMS[l + 1], DIMS[l]), dtype=f32, device=dev) for l in range(5)]
        self.gb = [torch.zeros(DIMS[l + 1], dtype=f32, device=dev) for l in range(5)]
        self.loss = torch.zeros(1, dtype=f32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.step_count = 0

    # ------------------------------------------------------------- weights
    def refresh_copies(self) -> None:
        with torch.cuda.stream(self.stream):
            for l in range(5):
                fo = DIMS[l + 1]
                self.Wb[l][:fo].copy_(self.W[l].to(torch.bfloat16))
                self.Wt[l][:, :fo].copy_(self.W[l].t().to(torch.bfloat16))
            self.bpad4[:3].copy_(self.b[4])

    def state_dict(self) -> dict:
        return {f"W{l}": self.W[l].cpu().numpy() for l in range(5)} | {f"b{l}": self.b[l].cpu().numpy()
                                                                       for l in range(5)}

    def load_state_dict(self, sd: dict) -> None:
        with torch.cuda.stream(self.stream):
            for l in range(5):
                self.W[l].copy_(torch.from_numpy(np.asarray(sd[f"W{l}"], np.float32)).to(self.device))
                self.b[l].copy_(torch.from_numpy(np.asarray(sd[f"b{l}"], np.float32)).to(self.device))
        self.refresh_copies()

    # ------------------------------------------------------------ forward
    def forward(self, m: int, train: bool = True) -> torch.Tensor:
        """Forward of the first m rows of X (Xt must hold X's transpose when a
        backward follows).  train=False stores only what the next layer reads
        (no pre-activations, no transposed copies) and splits each layer over
        four 64-column tiles.  Returns Y[:m, :3] (a view)."""
        lib, sp = self.lib, self._sp
        H = [self.X] + self.H[1:]
        for l in range(4):
            if train:
                gemm(lib, sp, H[l], self.Wb[l], self.m_pad, 256, DIMS[l], bias=self.b[l], act=1, out_pre=self.Z[l],
                     out_bf16=self.H[l + 1], out_bf16_t=self.Ht[l + 1], status=self.status)
            else:
                gemm(lib, sp, H[l], self.Wb[l], self.m_pad, 256, DIMS[l], bias=self.b[l], act=1,
                     out_bf16=self.H[l + 1], status=self.status, n_tile=64)
        gemm(lib, sp, self.H[4], self.Wb[4], self.m_pad, 3, 256, bias=self.bpad4, act=0, out_f32=self.Y,
             status=self.status, n_tile=16)
        return self.Y[:m, :3]

    # ----------------------------------------------------------- backward
    def backward(self, m: int, target: torch.Tensor) -> None:
        """Gradients of the mean squared error of Y[:m, :3] against target
        (m x 3, FP32) into gW, gb; adds sum of squared errors to loss."""
        lib, sp, M = self.lib, self._sp, self.m_pad
        tgt = target.contiguous()
        capi.check(lib.xpbd_mse_grad(int(m), M, 3, OUT_PAD_BWD, _p(self.Y), OUT_PAD_FWD, _p(tgt), 3, _p(self.dY),
                                     _p(self.dYt), M, _p(self.loss), sp))
        # last layer
        gemm(lib, sp, self.dYt, self.Ht[4], 3, 256, M, out_f32=self.gW[4], status=self.status)
        capi.check(lib.xpbd_colsum_bf16(3, int(m), _p(self.dYt), M, _p(self.gb[4]), sp))
        gemm(lib, sp, self.dY, self.Wt[4], M, 256, OUT_PAD_BWD, gelu_grad_of=self.Z[3], out_bf16=self.dZ[0],
             out_bf16_t=self.dZt[0], status=self.status)
        cur = 0
        for l in range(3, -1, -1):
            gemm(lib, sp, self.dZt[cur], self.Ht[l], 256, DIMS[l], M, out_f32=self.gW[l], status=self.status)
            capi.check(lib.xpbd_colsum_bf16(256, int(m), _p(self.dZt[cur]), M, _p(self.gb[l]), sp))
            if l > 0:
                nxt = 1 - cur
                gemm(lib, sp, self.dZ[cur], self.Wt[l], M, 256, 256, gelu_grad_of=self.Z[l - 1],
                     out_bf16=self.dZ[nxt], out_bf16_t=self.dZt[nxt], status=self.status)
                cur = nxt

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step_count += 1
        lib, sp, t = self.lib, self._sp, self.step_count
        for l in range(5):
            fo, fi = DIMS[l + 1], DIMS[l]
            capi.check(lib.xpbd_adam(fo, fi, _p(self.W[l]), _p(self.gW[l]), fi, _p(self.mW[l]), _p(self.vW[l]),
                                     C.c_float(lr), C.c_float(beta1), C.c_float(beta2), C.c_float(eps), t,
                                     _p(self.Wb[l]), _p(self.Wt[l]), self.Wt[l].shape[1], sp))
            capi.check(lib.xpbd_adam(1, fo, _p(self.b[l]), _p(self.gb[l]), fo, _p(self.mb[l]), _p(self.vb[l]),
                                     C.c_float(lr), C.c_float(beta1), C.c_float(beta2), C.c_float(eps), t, None, None,
                                     1, sp))
        with torch.cuda.stream(self.stream):
            self.bpad4[:3].copy_(self.b[4])
