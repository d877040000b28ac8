"""Learned walk-length bracket (host side of csrc/ht_bracket.cu).

A 12 -> 64 -> 64 -> 64 -> 2 MLP with BF16 weights predicts the 10 % and 90 % quantiles of
the radius (lattice units) at which a peak's radial-shell walk stops.  The prediction only
orders the collapse work (HT_MODE_LEARNED: peaks with similar predicted walks share a warp,
longest first); the catalog is identical to the plain path whatever the model says.

Training runs on the device with the library's own kernels: ht_bracket_grad (forward and
backward GEMMs on the tensor cores, BF16 inputs, FP32 accumulation, pinball loss) and
ht_bracket_adam.  `reference_grad` restates the same forward/backward in torch FP32 on the
CPU (rounding every GEMM input to BF16 exactly where the device does) for the gradient
check.  Nothing here has a counterpart in the reference.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import HT_BRACKET_NPARAMS, HtBracketModel, HtPeakBatch, check

NIN, NHID = 16, 64
# packed FP32 layout: W1 [64x16] W2 [64x64] W3 [64x64] W4 [8x64] b1 b2 b3 [64] b4 [8]
LAYOUT = (("W1", (64, 16)), ("W2", (64, 64)), ("W3", (64, 64)), ("W4", (8, 64)),
          ("b1", (64,)), ("b2", (64,)), ("b3", (64,)), ("b4", (8,)))
OFFSETS = {}
_o = 0
for _n, _s in LAYOUT:
    OFFSETS[_n] = (_o, _s)
    _o += int(np.prod(_s))
assert _o == HT_BRACKET_NPARAMS
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bracket_box512.npz")
QUANTILES = (0.1, 0.9)


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream(stream):
    return (stream if stream is not None else torch.cuda.current_stream()).cuda_stream


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised packed FP32 parameters (W4 rows 2..7 and padding inputs zero)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(HT_BRACKET_NPARAMS, np.float32)
    for name, fan_in, rows in (("W1", 12, 64), ("W2", 64, 64), ("W3", 64, 64), ("W4", 64, 2)):
        o, shape = OFFSETS[name]
        w = np.zeros(shape, np.float32)
        w[:rows, :fan_in] = rng.standard_normal((rows, fan_in)) * np.sqrt(2.0 / fan_in)
        p[o:o + w.size] = w.reshape(-1)
    return p


class BracketModel:
    """Device copy of the model: BF16 weights, FP32 biases and feature standardisation,
    plus (for training) the packed FP32 master parameters."""

    def __init__(self, params: np.ndarray, mean: np.ndarray, istd: np.ndarray, device="cuda"):
        self.device = torch.device(device)
        self.params = torch.as_tensor(np.asarray(params, np.float32), device=self.device).clone()
        self.mean = torch.as_tensor(np.asarray(mean, np.float32), device=self.device).clone()
        self.istd = torch.as_tensor(np.asarray(istd, np.float32), device=self.device).clone()
        self.W = {}
        self.b = {}
        self.sync_from_params()

    def sync_from_params(self):
        for name, (o, shape) in OFFSETS.items():
            v = self.params[o:o + int(np.prod(shape))].view(shape)
            if name.startswith("W"):
                self.W[name] = v.to(torch.bfloat16).contiguous()
            else:
                self.b[name] = v.clone().contiguous()

    def struct(self) -> HtBracketModel:
        return HtBracketModel(*[self.W[n].data_ptr() for n in ("W1", "W2", "W3", "W4")],
                              *[self.b[n].data_ptr() for n in ("b1", "b2", "b3", "b4")],
                              self.mean.data_ptr(), self.istd.data_ptr())

    def save(self, path: str):
        np.savez(path, params=self.params.cpu().numpy(), mean=self.mean.cpu().numpy(),
                 istd=self.istd.cpu().numpy())

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device="cuda") -> "BracketModel":
        d = np.load(path)
        return cls(d["params"], d["mean"], d["istd"], device)


def features(finder, pi, pj, pk, Rf, ir2min, ZZon, fcrit, alatt: float,
             peak_delta: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
    """[n x 16] float32 features of the peaks on the finder's bound tile."""
    n = int(pi.numel())
    F = torch.zeros((max(n, 1), NIN), dtype=torch.float32, device=pi.device)
    b = HtPeakBatch(pi.data_ptr(), pj.data_ptr(), pk.data_ptr(), Rf.data_ptr(),
                    ir2min.data_ptr(), ZZon.data_ptr(), fcrit.data_ptr(), n)
    check(_lib.load().ht_bracket_features(finder.handle, C.byref(b), _ptr(peak_delta),
                                          float(alatt), F.data_ptr(), _stream(stream)))
    return F[:n]


def predict(finder, model: BracketModel, F: torch.Tensor, stream=None) -> torch.Tensor:
    """[n x 2] float32 (low, high) quantiles of the walk's stop radius."""
    n = int(F.shape[0])
    Y = torch.empty((max(n, 1), 2), dtype=torch.float32, device=F.device)
    m = model.struct()
    check(_lib.load().ht_bracket_predict(finder.handle, C.byref(m), F.contiguous().data_ptr(),
                                         n, Y.data_ptr(), _stream(stream)))
    return Y[:n]


def grad(finder, model: BracketModel, F: torch.Tensor, target: torch.Tensor):
    """(packed FP32 gradient, mean pinball loss) on the device."""
    g = torch.empty(HT_BRACKET_NPARAMS, dtype=torch.float32, device=F.device)
    loss = torch.empty(1, dtype=torch.float32, device=F.device)
    m = model.struct()
    check(_lib.load().ht_bracket_grad(finder.handle, C.byref(m), F.contiguous().data_ptr(),
                                      target.contiguous().data_ptr(), int(F.shape[0]),
                                      g.data_ptr(), loss.data_ptr(), _stream(None)))
    return g, loss


def train(finder, F: torch.Tensor, target: torch.Tensor, *, epochs: int = 4,
          batch: int = 65536, lr: float = 2e-3, seed: int = 0, log=None) -> BracketModel:
    """Adam on the pinball loss with the library's kernels; returns the trained model."""
    Fh = F.double()
    mean = Fh.mean(0).float()
    std = Fh.std(0).float()
    istd = torch.where(std > 1e-6, 1.0 / std, torch.zeros_like(std))
    model = BracketModel(init_params(seed), mean.cpu().numpy(), istd.cpu().numpy(), F.device)
    mom = torch.zeros_like(model.params)
    vel = torch.zeros_like(model.params)
    gen = torch.Generator(device=F.device)
    gen.manual_seed(seed)
    n = int(F.shape[0])
    step = 0
    L = _lib.load()
    for ep in range(epochs):
        perm = torch.randperm(n, device=F.device, generator=gen)
        tot, cnt = 0.0, 0
        for s in range(0, n, batch):
            idx = perm[s:s + batch]
            g, loss = grad(finder, model, F[idx], target[idx])
            step += 1
            m = model.struct()
            check(L.ht_bracket_adam(finder.handle, model.params.data_ptr(), g.data_ptr(),
                                    mom.data_ptr(), vel.data_ptr(), step, float(lr),
                                    C.byref(m), _stream(None)))
            tot += float(loss.item()) * len(idx)
            cnt += len(idx)
        if log:
            log(f"epoch {ep}: pinball loss {tot / max(cnt, 1):.4f}")
    return model


# ------------------------------------------------------ CPU reference (tests) ----

def reference_forward(params: np.ndarray, mean, istd, F: np.ndarray, bf16: bool = True):
    """FP32 forward on the CPU with every GEMM input rounded to BF16 as on the device
    (bf16=False: plain FP32, for checking the backward formulas against autograd).
    Returns (Y, cache)."""
    _bf16 = (lambda x: x.to(torch.bfloat16).to(torch.float32)) if bf16 else (lambda x: x)
    p = torch.as_tensor(np.asarray(params, np.float32))
    W = {n: _bf16(p[o:o + int(np.prod(s))].view(s)) for n, (o, s) in OFFSETS.items()
         if n.startswith("W")}
    b = {n: p[o:o + int(np.prod(s))].view(s) for n, (o, s) in OFFSETS.items()
         if n.startswith("b")}
    X = _bf16((torch.as_tensor(F) - torch.as_tensor(mean)) * torch.as_tensor(istd))
    Z, H = [], [X]
    for l, (wn, bn) in enumerate((("W1", "b1"), ("W2", "b2"), ("W3", "b3"))):
        z = H[-1] @ W[wn].T + b[bn]
        Z.append(z)
        H.append(_bf16(torch.clamp(z, min=0.0)))
    Y = H[-1] @ W["W4"][:2].T + b["b4"][:2]
    return Y, (W, b, Z, H)


def reference_grad(params: np.ndarray, mean, istd, F: np.ndarray, target: np.ndarray,
                   bf16: bool = True):
    """Packed FP32 gradient of the mean pinball loss, restating ht_bracket_grad."""
    _bf16 = (lambda x: x.to(torch.bfloat16).to(torch.float32)) if bf16 else (lambda x: x)
    Y, (W, b, Z, H) = reference_forward(params, mean, istd, F, bf16)
    t = torch.as_tensor(np.asarray(target, np.float32))
    n = Y.shape[0]
    dY = torch.zeros_like(Y)
    for q, tau in enumerate(QUANTILES):
        d = t - Y[:, q]
        dY[:, q] = torch.where(d > 0, torch.full_like(d, -tau), torch.full_like(d, 1.0 - tau)) / n
    g = torch.zeros(HT_BRACKET_NPARAMS, dtype=torch.float32)

    def put(name, v):
        o, s = OFFSETS[name]
        full = torch.zeros(s)
        full[tuple(slice(0, k) for k in v.shape)] = v
        g[o:o + full.numel()] = full.reshape(-1)

    dYb = _bf16(dY)
    put("W4", dYb.T @ H[3])
    put("b4", dY.sum(0))
    dH = dYb @ W["W4"][:2]
    for l in (2, 1, 0):
        dZ = torch.where(Z[l] > 0, dH, torch.zeros_like(dH))
        put(f"b{l + 1}", dZ.sum(0))
        dZb = _bf16(dZ)
        put(f"W{l + 1}", dZb.T @ H[l])
        if l > 0:
            dH = dZb @ W[f"W{l + 1}"]
    return g.numpy()
