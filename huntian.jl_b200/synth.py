"""Seeded synthetic inputs for the halo-finding path (not part of the hot path).

No public dataset is involved: the reference runs on Gaussian random fields it generates
itself.  This module produces fields of the same kind with torch on the GPU:

* P(k): BBKS transfer function (Bardeen, Bond, Kaiser & Szalay 1986, eq. G3) with shape
  Gamma = Omega_m h, tilt n_s, normalised to sigma_8 with a real-space top-hat of
  8 Mpc/h; the amplitude convention of RandomField.jl:134-170 (P / (2 pi)^3 per mode,
  amp = sqrt(P dk^3 n^3)).
* white noise: Threefry-2x64-20 (Salmon et al. 2011, the Random123 counter-based
  generator RandomField.jl:45-53 uses) with key (seed, 0) and counter (pair, 0),
  Box-Muller on 53-bit uniforms in (0, 1].  Its bit-level agreement with Random123.jl is
  not pinned by any reference test; the shell walk and the peak finder are checked on
  whatever field is generated, so this does not affect parity.
* displacements: 1LPT psi = i k / k^2 delta_k and 2LPT from the sum of principal minors
  of phi_ij (LPT.jl:21-180), Nyquist planes zeroed; the k^2-weighted "Laplacian"
  irfft(k^2 delta_k) / n^3 (Pipeline.jl:36-52).
* a periodic box becomes a tile with `nbuff` cells of periodic wrap on every side
  (one tile with periodic cores, Parameters.jl:418-422).

Arrays are (n3, n2, n1) C-order float32 tensors (Julia column-major bytes).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

_PARITY = 0x1BD11BDAA9FC1A22
_ROT = (16, 42, 12, 31, 16, 32, 24, 21)


def _i64(v: int) -> int:
    v &= (1 << 64) - 1
    return v - (1 << 64) if v >= (1 << 63) else v


def _lsr(x: torch.Tensor, s: int) -> torch.Tensor:
    return (x >> s) & ((1 << (64 - s)) - 1)


def _rotl(x: torch.Tensor, r: int) -> torch.Tensor:
    return (x << r) | _lsr(x, 64 - r)


def threefry2x64_20(k0: int, k1: int, c0: torch.Tensor, c1: torch.Tensor):
    """Threefry-2x64 with 20 rounds on int64 tensors (two's-complement wrap = mod 2^64)."""
    ks = [_i64(k0), _i64(k1), _i64(_PARITY ^ k0 ^ k1)]
    x0 = c0 + ks[0]
    x1 = c1 + ks[1]
    for r in range(20):
        x0 = x0 + x1
        x1 = _rotl(x1, _ROT[r % 8])
        x1 = x1 ^ x0
        if r % 4 == 3:
            s = (r + 1) // 4
            x0 = x0 + ks[s % 3]
            x1 = x1 + _i64(ks[(s + 1) % 3] + s)
    return x0, x1


def threefry_noise(n: int, seed: int, device, planes_per_chunk: int = 32) -> torch.Tensor:
    """Unit Gaussian white noise on an n^3 grid: cell with 1-based column-major index idx
    takes member (idx-1) % 2 of pair (idx-1) >> 1 (RandomField.jl:74-88)."""
    out = torch.empty((n, n, n), dtype=torch.float32, device=device)
    cells_per_plane = n * n
    for k0 in range(0, n, planes_per_chunk):
        k1 = min(n, k0 + planes_per_chunk)
        first = k0 * cells_per_plane
        cnt = (k1 - k0) * cells_per_plane
        lin = torch.arange(first, first + cnt, device=device, dtype=torch.int64)
        pair = lin >> 1
        a, b = threefry2x64_20(seed, 0, pair, torch.zeros_like(pair))
        u1 = (_lsr(a, 11).to(torch.float64) + 1.0) * 1.1102230246251565e-16
        u2 = (_lsr(b, 11).to(torch.float64) + 1.0) * 1.1102230246251565e-16
        r = torch.sqrt(-2.0 * torch.log(u1))
        th = 2.0 * math.pi * u2
        g = torch.where((lin & 1) == 0, r * torch.cos(th), r * torch.sin(th))
        out[k0:k1] = g.to(torch.float32).view(k1 - k0, n, n)
        del lin, pair, a, b, u1, u2, r, th, g
    return out


@dataclass
class Cosmology:
    Om: float = 0.31
    h: float = 0.68
    sigma8: float = 0.81
    ns: float = 0.965


def bbks_transfer(k, Om, h):
    q = np.asarray(k) / (Om * h)
    q = np.maximum(q, 1e-30)
    return (np.log(1.0 + 2.34 * q) / (2.34 * q) *
            (1.0 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3 + (6.71 * q) ** 4) ** -0.25)


def pk_table(cosmo: Cosmology, kmin=1e-5, kmax=1e3, nk=4000):
    """(k [h/Mpc], P(k)/(2 pi)^3) on a log grid, sigma_8-normalised (pk_websky.dat units)."""
    k = np.exp(np.linspace(np.log(kmin), np.log(kmax), nk))
    P = k ** cosmo.ns * bbks_transfer(k, cosmo.Om, cosmo.h) ** 2
    x = k * 8.0
    W = 3.0 * (np.sin(x) - x * np.cos(x)) / x ** 3
    lnk = np.log(k)
    s2 = np.trapezoid(P * W ** 2 * k ** 3 / (2.0 * math.pi ** 2), lnk)
    P = P * cosmo.sigma8 ** 2 / s2
    return k, P / (2.0 * math.pi) ** 3


def _kgrid(n: int, boxsize: float, device):
    dk = 2.0 * math.pi / boxsize
    kf = torch.fft.fftfreq(n, d=1.0 / n, device=device).to(torch.float32) * dk
    kx = torch.arange(n // 2 + 1, device=device, dtype=torch.float32) * dk
    return kf.view(-1, 1, 1), kf.view(1, -1, 1), kx.view(1, 1, -1), dk


def _nyq_mask(n: int, device):
    """1 on modes off the Nyquist planes (LPT.jl:48-54), broadcastable to the rfft grid."""
    iz = torch.arange(n, device=device)
    ok_f = (iz != n // 2).to(torch.float32)
    ok_x = (torch.arange(n // 2 + 1, device=device) != n // 2).to(torch.float32)
    return ok_f.view(-1, 1, 1), ok_f.view(1, -1, 1), ok_x.view(1, 1, -1)


def gaussian_box(n: int, boxsize: float, seed: int, cosmo: Cosmology, device):
    """delta_k of a Gaussian random field on the periodic n^3 box (RandomField.jl:134-170)."""
    noise = threefry_noise(n, seed, device)
    dk_ = torch.fft.rfftn(noise, dim=(0, 1, 2))
    del noise
    kz, ky, kx, dk = _kgrid(n, boxsize, device)
    ktab, ptab = pk_table(cosmo)
    lk = torch.as_tensor(np.log(ktab), device=device, dtype=torch.float32)
    lp = torch.as_tensor(np.log(ptab), device=device, dtype=torch.float32)
    for z0 in range(0, n, 64):
        z1 = min(n, z0 + 64)
        k = torch.sqrt(kz[z0:z1] ** 2 + ky ** 2 + kx ** 2)
        lnk = torch.log(torch.clamp(k, min=1e-30))
        idx = torch.clamp(torch.searchsorted(lk, lnk.reshape(-1)).view_as(lnk), 1, len(lk) - 1)
        t = (lnk - lk[idx - 1]) / (lk[idx] - lk[idx - 1])
        lnp = lp[idx - 1] + t * (lp[idx] - lp[idx - 1])
        amp = torch.sqrt(torch.exp(lnp) * (dk ** 3) * float(n) ** 3)
        amp = torch.where(k == 0, torch.zeros_like(amp), amp)
        dk_[z0:z1] *= amp
        del k, lnk, idx, t, lnp, amp
    return dk_.contiguous()


def _irfft(a: torch.Tensor, n: int) -> torch.Tensor:
    return torch.fft.irfftn(a, s=(n, n, n), dim=(0, 1, 2)).contiguous()


def displacements(delta_k: torch.Tensor, n: int, boxsize: float, ilpt: int = 2):
    """(psi1 x/y/z, psi2 x/y/z or None) per LPT.jl:21-180."""
    device = delta_k.device
    kz, ky, kx, _ = _kgrid(n, boxsize, device)
    nz, ny, nx = _nyq_mask(n, device)
    k2 = kz ** 2 + ky ** 2 + kx ** 2
    inv = torch.where(k2 == 0, torch.zeros_like(k2), 1.0 / k2)
    ks = (kx, ky, kz)
    psi1 = []
    for L in range(3):
        psi1.append(_irfft(delta_k * (1j * ks[L] * inv * nz * ny * nx), n))
    psi2 = None
    if ilpt >= 2:
        phi = {}
        src = None
        for (a, b) in ((0, 0), (1, 1), (2, 2)):
            phi[a] = _irfft(delta_k * (-ks[a] * ks[b] * inv), n)
        src = phi[0] * phi[1] + phi[0] * phi[2] + phi[1] * phi[2]
        del phi
        for (a, b) in ((0, 1), (0, 2), (1, 2)):
            p = _irfft(delta_k * (-ks[a] * ks[b] * inv), n)
            src -= p * p
            del p
        src_k = torch.fft.rfftn(src, dim=(0, 1, 2))
        del src
        psi2 = [_irfft(src_k * (-1j * ks[L] * inv * nz * ny * nx), n) for L in range(3)]
        del src_k
    return psi1, psi2


def laplacian(delta_k: torch.Tensor, n: int, boxsize: float) -> torch.Tensor:
    kz, ky, kx, _ = _kgrid(n, boxsize, delta_k.device)
    return _irfft(delta_k * (kz ** 2 + ky ** 2 + kx ** 2), n) / float(n) ** 3


def wrap_pad(f: torch.Tensor, nbuff: int) -> torch.Tensor:
    """Periodic box (n^3) -> tile (n + 2 nbuff)^3 with periodic wrap in every direction."""
    if nbuff == 0:
        return f.contiguous()
    import torch.nn.functional as F
    return F.pad(f[None, None], (nbuff,) * 6, mode="circular")[0, 0].contiguous()
