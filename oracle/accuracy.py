"""Accuracy at the configurations' own sizes: the oracle's side.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/`` and by ``bench.py``'s
accuracy leg, where it is the checker; the product never imports it.

* ``slices_from_particles`` -- the reference caller's per-particle pipeline
  (``oracle.particle_to_slice``, programs/e2spa_make3d.py:300-342) over many
  particles, the FFTs batched over chunks and the chunks run on threads
  (numpy's FFT and the oracle's C calls release the GIL).  Identical in
  float32 to calling ``particle_to_slice`` per particle.
* ``insert_tasks`` -- the insertion of many particles the way the
  reference's parallel make3d runs it (programs/e2spa_make3d.py:154-188):
  the particles are dealt into T tasks (``data[i::T]``), each task inserts its
  share sequentially into its own (complex, weight) volume, and the volumes
  are added in task order.  T = 1 is a single sequential reconstructor.  The
  FP32 build gives the reference's own FP32 result for that split; the FP64
  build the FP64 oracle (where the split does not matter).  The reference
  normalises each task's volume and multiplies it back by its weights before
  the sum; the oracle adds the un-normalised accumulators directly.
* ``fsc`` -- EMData::calc_fourier_shell_correlation
  (libEM/sparx/emdata_sparx.cpp:867-990) with ring width 1: the shell index
  is formed in single precision as the reference forms it, the sums in
  double.
* ``compare`` -- relative L2 of the normalised complex volumes (finish(False))
  and of the weight volumes (normout), the FSC of the complex volumes in
  every shell, and per-cell checks of the weights.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import oracle


def host_threads(cap: int = 16) -> int:
    """Threads for the oracle: the host's cores, at most ``cap``."""
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        n = os.cpu_count() or 1
    return max(1, min(cap, n))


# ------------------------------------------------------------------ prologue

def _clip_pad_batch(imgs: np.ndarray, N: int) -> np.ndarray:
    """oracle.clip_pad for a stack: clip_inplace(Region((nx-N)//2, (ny-N)//2, N, N))
    with zero fill."""
    n, ny, nx = imgs.shape
    x0, y0 = (nx - N) // 2, (ny - N) // 2
    out = np.zeros((n, N, N), np.float32)
    ys, ye = max(0, -y0), min(N, ny - y0)
    xs, xe = max(0, -x0), min(N, nx - x0)
    out[:, ys:ye, xs:xe] = imgs[:, ys + y0:ye + y0, xs + x0:xe + x0]
    return out


def _prologue_chunk(imgs, N, shifts, defocus, ctf):
    """particle_to_slice for a chunk of particles (same operations, same order)."""
    n = imgs.shape[0]
    work = np.array(imgs, np.float32, copy=True)
    for i in range(n):
        work[i] -= oracle.edge_mean(work[i])
    work = _clip_pad_batch(work, N)
    flip = [i for i in range(n) if defocus is not None and abs(float(defocus[i])) > 1e-4]
    if flip:
        F = np.fft.rfft2(work[flip].astype(np.float64)).astype(np.complex64)
        c = dict(ctf or {})
        for k, i in enumerate(flip):
            s = oracle.ctf_sign(N, float(defocus[i]), c.get("voltage", 300.0), c.get("cs", 2.7),
                                c.get("apix", 1.0), c.get("ampcont", 10.0), c.get("dfdiff", 0.0),
                                c.get("dfang", 0.0))
            F[k] = (F[k].real * s + 1j * (F[k].imag * s)).astype(np.complex64)
        r = np.fft.irfft2(F.astype(np.complex128), s=(N, N), norm="forward").astype(np.float32)
        work[flip] = r * np.float32(1.0 / (N * N))
    for i in range(n):
        work[i] -= oracle.edge_mean(work[i])
        tx, ty = float(np.float32(shifts[i][0])), float(np.float32(shifts[i][1]))
        if not (oracle._near_int(-tx) == 0 and oracle._near_int(-ty) == 0):
            work[i] = oracle.translate(work[i], tx, ty)
    work = np.roll(work, (-(N // 2), -(N // 2)), axis=(1, 2))
    F = np.fft.rfft2(work.astype(np.float64)).astype(np.complex64)
    scale = np.sqrt(np.float32(1.0) / np.float32(N) * np.float32(N + 2)).astype(np.float32)
    out = np.empty((n, N, N + 2), np.float32)
    out[:, :, 0::2] = F.real * scale
    out[:, :, 1::2] = F.imag * scale
    return out


def slices_from_particles(images, N: int, shifts, defocus=None, ctf: dict | None = None,
                          threads: int | None = None, chunk: int = 64) -> np.ndarray:
    """(n, N, N+2) float32 preprocessed slices of n raw particles (n, box, box):
    edge mean, clip to N, CTF phase flip where |defocus| > 1e-4, edge mean,
    inverse shift, phase origin to corner, r2c, x sqrt((N+2)/N)."""
    images = np.asarray(images, np.float32)
    n = images.shape[0]
    shifts = np.asarray(shifts, np.float32).reshape(n, 2)
    out = np.empty((n, N, N + 2), np.float32)
    threads = threads or host_threads()

    def run(a):
        b = min(n, a + chunk)
        out[a:b] = _prologue_chunk(images[a:b], N, shifts[a:b],
                                   None if defocus is None else defocus[a:b], ctf)

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, range(0, n, chunk)))
    return out


# ------------------------------------------------------------------ insertion

def insert_tasks(N: int, slices, rots, weights, mode: str, sym: str, precision: str = "fp32",
                 tasks: int = 1) -> oracle.OracleVolume:
    """Un-normalised accumulators of n slices inserted as ``tasks`` private
    reconstructions (particle p to task p % tasks), added in task order."""
    slices = np.asarray(slices, np.float32)
    rots = np.asarray(rots, np.float32).reshape(-1, 3, 3)
    weights = np.asarray(weights, np.float32).reshape(-1)
    n = slices.shape[0]
    tasks = max(1, min(int(tasks), n))

    def one(t):
        v = oracle.OracleVolume(N, precision)
        idx = np.arange(t, n, tasks)
        v.insert(np.ascontiguousarray(slices[idx]), np.ascontiguousarray(rots[idx]),
                 np.ascontiguousarray(weights[idx]), mode, sym)
        return v

    if tasks == 1:
        return one(0)
    with ThreadPoolExecutor(tasks) as ex:
        parts = list(ex.map(one, range(tasks)))
    total = parts[0]
    for v in parts[1:]:
        total.data += v.data
        total.norm += v.norm
    return total


def normalized(vol: oracle.OracleVolume, sqrtnorm: bool = False):
    """finish(False) + normout of a copy: (normalised complex, weights)."""
    v = vol.copy()
    v.normalize(sqrtnorm)
    return v.data, v.norm


# ------------------------------------------------------------------ metrics

def fsc(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """FSC of two complex half volumes (N, N, N+2), one value per shell
    0..N/2 (EMData::calc_fourier_shell_correlation, w = 1).  Shells where
    either volume has no power are reported as 1 (both empty) or 0."""
    N = a.shape[0]
    n2 = N // 2
    f32 = np.float32
    dx2 = f32(1.0) / f32(n2) / f32(n2)
    inc = n2                                      # Util::round(nx2 / w), w = 1
    k = np.arange(N)
    k = np.where(k > n2, k - N, k)
    kk = (k * k).astype(f32)
    argz = kk * dx2                               # float(kz*kz)*dz2
    argy = argz[:, None] + kk[None, :] * dx2      # argz + float(ky*ky)*dy2
    ix = np.arange(0, N + 2, 2)                   # interleaved x index, kx = ix/2
    tx = (ix * ix).astype(f32) * f32(0.25) * dx2  # float(ix*ix)*0.25f*dx2
    argx = f32(0.5) * np.sqrt(argy[:, :, None] + tx[None, None, :])
    t = f32(inc * 2) * argx
    r = np.where(t < 0, (t - f32(0.5)).astype(np.int64), (t + f32(0.5)).astype(np.int64))
    kz = k[:, None, None]
    ky = k[None, :, None]
    keep = (ix[None, None, :] > 0) | ((kz >= 0) & ((ky >= 0) | (kz != 0)))
    keep = keep & (r <= inc)
    rr = r[keep]
    ca = a.astype(np.float64).reshape(N, N, N // 2 + 1, 2)[keep]
    cb = b.astype(np.float64).reshape(N, N, N // 2 + 1, 2)[keep]
    num = np.bincount(rr, ca[:, 0] * cb[:, 0] + ca[:, 1] * cb[:, 1], inc + 1)
    n1 = np.bincount(rr, ca[:, 0] ** 2 + ca[:, 1] ** 2, inc + 1)
    n2s = np.bincount(rr, cb[:, 0] ** 2 + cb[:, 1] ** 2, inc + 1)
    out = np.zeros(inc + 1)
    ok = (n1 > 0) & (n2s > 0)
    out[ok] = num[ok] / np.sqrt(n1[ok] * n2s[ok])
    out[(n1 <= 0) & (n2s <= 0)] = 1.0
    return out


def compare(data, norm, ref_data, ref_norm) -> dict:
    """Distances of a normalised (complex, weight) pair from a reference pair:
    relative L2 of each, the FSC's minimum over shells, and per voxel the
    cells whose weight is zero in one and not the other (a tap that went
    missing or appeared) and the largest relative weight difference over the
    cells the reference reaches."""
    norm = np.asarray(norm)
    ref_norm = np.asarray(ref_norm)
    f = fsc(np.asarray(data), np.asarray(ref_data))
    m = ref_norm != 0
    rw = np.abs(norm[m].astype(np.float64) - ref_norm[m]) / np.abs(ref_norm[m].astype(np.float64))
    return {"rel_l2_complex": oracle.rel_l2(data, ref_data),
            "rel_l2_weight": oracle.rel_l2(norm, ref_norm),
            "fsc_min": float(f.min()), "fsc_min_shell": int(f.argmin()),
            "support_mismatch": int(np.count_nonzero((norm != 0) != m)),
            "max_rel_weight_voxel": float(rw.max()) if rw.size else 0.0}


def report(gpu: dict, o32, o64, oacc=None) -> dict:
    """Per GPU form (name -> normalised (data, norm)): distances from the FP32
    oracle (the reference's own arithmetic), from the FP64 oracle and, when
    given, from the FP32-taps/FP64-sums oracle (the same taps added exactly:
    what is left against it is summation order), beside the FP32 oracle's
    own distances from those."""
    out = {"fp32_oracle_vs_fp64": compare(o32[0], o32[1], o64[0], o64[1])}
    if oacc is not None:
        out["fp32_oracle_vs_exact_sums"] = compare(o32[0], o32[1], oacc[0], oacc[1])
    for name, (d, n) in gpu.items():
        out[name] = {"vs_fp32_oracle": compare(d, n, o32[0], o32[1]),
                     "vs_fp64_oracle": compare(d, n, o64[0], o64[1])}
        if oacc is not None:
            out[name]["vs_exact_sums"] = compare(d, n, oacc[0], oacc[1])
    return out
