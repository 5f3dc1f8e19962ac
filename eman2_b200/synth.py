"""Seeded synthetic particles: a Gaussian-blob phantom, analytic projections,
CTF, translations and noise.

Stand-in for real data (no dataset is available).  Phantom: 50 3-D Gaussians
with centres uniform in a ball of radius 0.3*box, sigma U(1.5, 3) px,
amplitude U(0.5, 1).  A 3-D Gaussian projects to a 2-D Gaussian of amplitude
a*sigma*sqrt(2*pi) centred at (R c)[0:2], R the orientation block: the
insertion maps slice frequency (kx, ky) to kx*R[0] + ky*R[1], so by the
projection-slice theorem the image is the integral of the volume along R[2].
Orientations are uniform SO(3) quaternions.  The particle content is displaced
by its xform.projection translation (the reference undoes it with the
inverted translation, programs/e2spa_make3d.py:339-342).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Phantom:
    centres: np.ndarray      # (G, 3) in (x, y, z) pixels about the box centre
    sigmas: np.ndarray       # (G,)
    amps: np.ndarray         # (G,)


def make_phantom(box: int, rng: np.random.Generator, nblobs: int = 50) -> Phantom:
    r = 0.3 * box
    c = rng.normal(size=(nblobs, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    c *= (r * rng.uniform(0, 1, nblobs) ** (1.0 / 3.0))[:, None]
    return Phantom(c, rng.uniform(1.5, 3.0, nblobs), rng.uniform(0.5, 1.0, nblobs))


def phantom_volume(ph: Phantom, n: int) -> np.ndarray:
    """Real-space phantom on an n^3 grid centred at n/2 ([z][y][x])."""
    ax = np.arange(n) - n // 2
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    v = np.zeros((n, n, n))
    for (cx, cy, cz), s, a in zip(ph.centres, ph.sigmas, ph.amps):
        v += a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2 * s * s))
    return v.astype(np.float32)


def random_quaternions(n: int, rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def quaternion_blocks(q: np.ndarray) -> np.ndarray:
    """Transform::set_rotation "quaternion" (libEM/transform.cpp:667-678): double
    arithmetic, each element rounded to float."""
    e0, e1, e2, e3 = (q[:, i].astype(np.float64) for i in range(4))
    m = np.empty((q.shape[0], 3, 3), np.float64)
    m[:, 0, 0] = e0 * e0 + e1 * e1 - e2 * e2 - e3 * e3
    m[:, 0, 1] = 2.0 * (e1 * e2 + e0 * e3)
    m[:, 0, 2] = 2.0 * (e1 * e3 - e0 * e2)
    m[:, 1, 0] = 2.0 * (e2 * e1 - e0 * e3)
    m[:, 1, 1] = e0 * e0 - e1 * e1 + e2 * e2 - e3 * e3
    m[:, 1, 2] = 2.0 * (e2 * e3 + e0 * e1)
    m[:, 2, 0] = 2.0 * (e3 * e1 + e0 * e2)
    m[:, 2, 1] = 2.0 * (e3 * e2 - e0 * e1)
    m[:, 2, 2] = e0 * e0 - e1 * e1 - e2 * e2 + e3 * e3
    return m.astype(np.float32)


def ctf_curve(s, defocus_um, voltage=300.0, cs=2.7, ampcont=10.0, bfactor=50.0):
    """EMAN2-convention CTF amplitude cos(gamma - acac) * exp(-B s^2/4) at
    spatial frequency s (1/A) (libEM/ctf.cpp:1000-1012 CTF_AMP)."""
    lam = 12.2639 / math.sqrt(voltage * 1000.0 + 0.97845 * voltage * voltage)
    g1 = math.pi / 2.0 * cs * 1.0e7 * lam ** 3
    g2 = math.pi * lam * 10000.0
    acac = math.pi / 2.0 - math.asin(ampcont / 100.0)
    gam = -g1 * s ** 4 + g2 * defocus_um * s ** 2
    return np.cos(gam - acac) * np.exp(-(bfactor / 4.0) * s * s)


@dataclass
class ParticleSet:
    box: int
    images: np.ndarray       # (n, box, box) float32
    rots: np.ndarray         # (n, 3, 3) float32
    shifts: np.ndarray       # (n, 2) float32
    weights: np.ndarray      # (n,) float32
    defocus: np.ndarray      # (n,) float32 (0: no CTF)
    phantom: Phantom
    meta: dict = field(default_factory=dict)


def make_particles(box: int, n: int, seed: int, snr: float = 0.1, shift: float = 2.0,
                   weights: tuple | None = None, ctf: bool = False, defocus=(0.8, 2.5),
                   apix: float = 1.0, bfactor: float = 50.0, phantom: Phantom | None = None,
                   device: str | None = None) -> ParticleSet:
    """n seeded particles.  ``device`` = a torch device renders on the GPU
    (float64), else numpy renders on the CPU."""
    rng = np.random.default_rng(seed)
    ph = phantom if phantom is not None else make_phantom(box, rng)
    q = random_quaternions(n, rng)
    rots = quaternion_blocks(q)
    shifts = rng.uniform(-shift, shift, (n, 2)).astype(np.float32)
    w = (np.ones(n, np.float32) if weights is None
         else rng.uniform(weights[0], weights[1], n).astype(np.float32))
    dfs = (rng.uniform(defocus[0], defocus[1], n).astype(np.float32) if ctf
           else np.zeros(n, np.float32))
    noise_seed = int(rng.integers(0, 2 ** 31 - 1))
    if device is not None:
        imgs = _render_torch(box, ph, rots, shifts, dfs, ctf, snr, apix, bfactor, noise_seed, device)
    else:
        imgs = _render_numpy(box, ph, rots, shifts, dfs, ctf, snr, apix, bfactor, noise_seed)
    return ParticleSet(box, imgs, rots, shifts, w, dfs, ph,
                       {"seed": seed, "snr": snr, "apix": apix, "ctf": ctf})


def _centres_2d(ph, rots, shifts):
    c = np.einsum("nij,gj->ngi", rots[:, :2, :].astype(np.float64), ph.centres)  # (n, G, 2)
    return c + shifts[:, None, :].astype(np.float64)


def _render_numpy(box, ph, rots, shifts, dfs, ctf, snr, apix, bfactor, noise_seed):
    n = rots.shape[0]
    ax = np.arange(box) - box // 2
    yy, xx = np.meshgrid(ax, ax, indexing="ij")
    uv = _centres_2d(ph, rots, shifts)
    amp = ph.amps * ph.sigmas * math.sqrt(2 * math.pi)
    out = np.zeros((n, box, box), np.float64)
    for i in range(n):
        img = np.zeros((box, box))
        for g in range(len(ph.amps)):
            s2 = 2 * ph.sigmas[g] ** 2
            img += amp[g] * np.exp(-((xx - uv[i, g, 0]) ** 2 + (yy - uv[i, g, 1]) ** 2) / s2)
        out[i] = img
    if ctf:
        out = _apply_ctf_numpy(out, dfs, apix, bfactor)
    rng = np.random.default_rng(noise_seed)
    sig_var = out.var(axis=(1, 2), keepdims=True)
    out += rng.normal(size=out.shape) * np.sqrt(sig_var / snr)
    return out.astype(np.float32)


def _apply_ctf_numpy(imgs, dfs, apix, bfactor):
    box = imgs.shape[-1]
    f = np.fft.fftfreq(box, d=apix)
    fx = np.fft.rfftfreq(box, d=apix)
    s = np.sqrt(fx[None, :] ** 2 + f[:, None] ** 2)
    out = np.empty_like(imgs)
    for i in range(imgs.shape[0]):
        F = np.fft.rfft2(np.fft.ifftshift(imgs[i]))
        F *= ctf_curve(s, float(dfs[i]), bfactor=bfactor)
        out[i] = np.fft.fftshift(np.fft.irfft2(F, s=(box, box)))
    return out


def _render_torch(box, ph, rots, shifts, dfs, ctf, snr, apix, bfactor, noise_seed, device):
    import torch
    dev = torch.device(device)
    n = rots.shape[0]
    uv = torch.as_tensor(_centres_2d(ph, rots, shifts), device=dev)           # (n, G, 2)
    sig = torch.as_tensor(ph.sigmas, device=dev, dtype=torch.float64)
    amp = torch.as_tensor(ph.amps * ph.sigmas * math.sqrt(2 * math.pi), device=dev)
    ax = torch.arange(box, device=dev, dtype=torch.float64) - box // 2
    out = torch.empty((n, box, box), device=dev, dtype=torch.float32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(noise_seed)
    chunk = max(1, int(2 ** 26 // (box * box * len(ph.amps))))
    if ctf:
        f = torch.fft.fftfreq(box, d=apix, device=dev, dtype=torch.float64)
        fx = torch.fft.rfftfreq(box, d=apix, device=dev, dtype=torch.float64)
        s = torch.sqrt(fx[None, :] ** 2 + f[:, None] ** 2).cpu().numpy()
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        dx = ax[None, None, :] - uv[a:b, :, 0, None]          # (m, G, box)
        dy = ax[None, None, :] - uv[a:b, :, 1, None]
        ex = torch.exp(-dx * dx / (2 * sig[None, :, None] ** 2))
        ey = torch.exp(-dy * dy / (2 * sig[None, :, None] ** 2))
        img = torch.einsum("mgy,mgx,g->myx", ey, ex, amp)
        if ctf:
            cur = np.stack([ctf_curve(s, float(d), bfactor=bfactor) for d in dfs[a:b]])
            F = torch.fft.rfft2(torch.fft.ifftshift(img, dim=(-2, -1)))
            F = F * torch.as_tensor(cur, device=dev)
            img = torch.fft.fftshift(torch.fft.irfft2(F, s=(box, box)), dim=(-2, -1))
        var = img.var(dim=(1, 2), keepdim=True)
        noise = torch.randn(img.shape, generator=gen, device=dev, dtype=torch.float64)
        out[a:b] = (img + noise * torch.sqrt(var / snr)).float()
    return out
