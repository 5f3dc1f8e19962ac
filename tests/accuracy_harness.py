"""Accuracy of the GPU reconstruction at the configurations' own sizes.

Test infrastructure (used by ``tests/test_gpu_accuracy.py`` and by the
accuracy leg of ``bench.py``).  Each case renders seeded particles of one
configuration on the GPU, runs them through the public API in the plain form
(one ``insert_particles`` call per particle, scatter insertion: the drop-in
``insert_slice`` loop) and the batched form (chunks of 2048 particles, the
library's gather kernels; or several reconstructions in one CUDA-graph
replay), and compares ``finish(False)`` and ``normout`` with the oracle fed
the same raw particles: the FP32-faithful restatement (the reference's own
arithmetic, particles dealt into tasks as the reference's parallel make3d
deals them) and the FP64 restatement.  Reported per form: relative L2 of the
normalised complex volume and of the weight volume, and the minimum FSC over
all shells (the reference's shell rule), against both oracles, beside the
FP32 oracle's own distance from the FP64 one.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

# The configurations (seeded synthetic stand-ins for data: Gaussian-blob
# phantom projections, CTF, noise), at their own sizes unless `n` is reduced.
CASES = {
    # box 64 padded to 96, 2,000 particles, gauss_2, c1, no CTF, SNR 0.1
    "c1": dict(box=64, N=96, mode="gauss_2", sym="c1", n=2000, ctf=False, snr=0.1, shift=2.0,
               weights=None, seed=101, tasks=1),
    # box 128 padded to 192, 20,000 particles, gauss_2, c1, CTF, SNR 0.05,
    # weights U(0.5, 1), shifts U(-4, 4), plus the agreement pass
    "c2": dict(box=128, N=192, mode="gauss_2", sym="c1", n=20000, ctf=True, snr=0.05, shift=4.0,
               weights=(0.5, 1.0), seed=102, tasks=0, agree=512),
    # box 256 padded to 384, d7, gauss_5, CTF, SNR 0.02: a seeded subsample of
    # the 200,000-particle job (the oracle needs ~2.5 core-s per particle)
    "c4": dict(box=256, N=384, mode="gauss_5", sym="d7", n=64, ctf=True, snr=0.02, shift=4.0,
               weights=(0.5, 1.0), seed=104, tasks=8, agree=32, full_n=200_000),
    # box 256 padded to 384, d7, gauss_2: 320 particles = 4,480 slices, more
    # than one 4,096-slice bucket of the gather kernels' work order; both
    # gather kernels (pixel-major, column) are run
    "c4g2": dict(box=256, N=384, mode="gauss_2", sym="d7", n=320, ctf=True, snr=0.02, shift=4.0,
                 weights=(0.5, 1.0), seed=105, tasks=8, kernels=(6, 5), full_n=200_000),
}

CHUNK = 2048


def _threads(t):
    from oracle.accuracy import host_threads
    return host_threads() if not t else min(int(t), host_threads())


def _meta_view(meta, a, b):
    """Entries a..b-1 of an fr_particle array, without a copy."""
    from eman2_b200 import _lib
    sz = ctypes.sizeof(_lib.fr_particle)
    return (_lib.fr_particle * (b - a)).from_address(ctypes.addressof(meta) + a * sz)


def _finish(r):
    """finish(False) and normout of a reconstructor, as numpy arrays."""
    from eman2_b200 import EMData
    nout = EMData()
    r.params["normout"] = nout
    out = r.finish(False).numpy()
    del r.params["normout"]
    return out, nout.numpy()


def _recon(c):
    from eman2_b200 import FourierReconstructor
    r = FourierReconstructor({"size": [c["N"]] * 3, "sym": c["sym"], "mode": c["mode"]})
    r.setup()
    return r


def gpu_plain(c, imgs, meta):
    """One insert call per particle (scatter insertion)."""
    r = _recon(c)
    for i in range(imgs.shape[0]):
        r.insert_particles(imgs[i:i + 1], _meta_view(meta, i, i + 1), schedule="scatter")
    res = _finish(r)
    r.close()
    return res


def gpu_batched(c, imgs, meta, tile=-1, agree=None):
    """Chunks of CHUNK particles per call through the gather kernels (tile:
    pin one; -1 the library's choice).  agree = (slices, rots, weights): the
    agreement pass against the volume before finish."""
    from eman2_b200.batch import set_tile
    from oracle.oracle import sym_ops
    nsym = len(sym_ops(c["sym"]))
    r = _recon(c)
    if tile != -1:
        set_tile(c["N"], c["mode"], nsym, tile)
    try:
        n = imgs.shape[0]
        for a in range(0, n, CHUNK):
            b = min(n, a + CHUNK)
            r.insert_particles(imgs[a:b], _meta_view(meta, a, b), schedule="gather")
    finally:
        if tile != -1:
            set_tile(c["N"], c["mode"], nsym, -1)
    ag = r.slice_agreement(*agree) if agree is not None else None
    res = _finish(r)
    r.close()
    return res, ag


def render(c, dev, n=None):
    """Seeded particles of case c (rendered on the GPU) and their metadata."""
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    n = int(n or c["n"])
    ps = make_particles(c["box"], n, seed=c["seed"], snr=c["snr"], shift=c["shift"],
                        weights=c["weights"], ctf=c["ctf"], device=dev)
    meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
    return ps, meta


def oracle_volumes(c, host_imgs, shifts, defocus, rots, weights, tasks=None):
    """The oracle's slices of the same raw particles and its FP32 and FP64
    volumes (un-normalised)."""
    from oracle import accuracy
    N = c["N"]
    t0 = time.perf_counter()
    sl = accuracy.slices_from_particles(host_imgs, N, shifts, defocus if c["ctf"] else None)
    t1 = time.perf_counter()
    T = _threads(c["tasks"] if tasks is None else tasks)
    o32 = accuracy.insert_tasks(N, sl, rots, weights, c["mode"], c["sym"], "fp32", T)
    t2 = time.perf_counter()
    o64 = accuracy.insert_tasks(N, sl, rots, weights, c["mode"], c["sym"], "fp64", T)
    t3 = time.perf_counter()
    oacc = accuracy.insert_tasks(N, sl, rots, weights, c["mode"], c["sym"], "fp32acc64", T)
    t4 = time.perf_counter()
    return sl, (o32, o64, oacc), {"tasks": T, "prologue_s": t1 - t0, "fp32_s": t2 - t1,
                                  "fp64_s": t3 - t2, "exact_sums_s": t4 - t3}


def _report(gpu, vols):
    from oracle import accuracy
    o32, o64, oacc = vols
    return accuracy.report(gpu, accuracy.normalized(o32), accuracy.normalized(o64),
                           accuracy.normalized(oacc))


def agreement_check(ag, o32, sym, sl, rots, weights, apix=1.0):
    """Largest relative difference of the agreement statistics (reconstruct_norm,
    absqual, absqual_lowres, qual, weight) from the oracle's, over the slices."""
    worst = 0.0
    for i in range(ag.shape[0]):
        want = o32.compare(sl[i], rots[i], float(weights[i]), sym=sym, apix=apix)
        d = np.abs(ag[i].astype(np.float64) - want) / np.maximum(np.abs(want), 1e-6)
        worst = max(worst, float(d.max()))
    return worst


def run_case(name: str, dev, n=None, forms=("plain", "batched"), tasks=None) -> dict:
    """GPU forms of case `name` against the FP32 and FP64 oracles."""
    import torch
    c = dict(CASES[name])
    ps, meta = render(c, dev, n)
    imgs = ps.images
    n = int(imgs.shape[0])
    gpu, timing = {}, {}
    sl_agree = None
    host = imgs.cpu().numpy() if isinstance(imgs, torch.Tensor) else np.asarray(imgs)
    sl, vols, ot = oracle_volumes(c, host, ps.shifts, ps.defocus, ps.rots, ps.weights, tasks)
    o32 = vols[0]
    agree_worst = None
    if "plain" in forms:
        t = time.perf_counter()
        gpu["plain"] = gpu_plain(c, imgs, meta)
        timing["plain_s"] = time.perf_counter() - t
    if "batched" in forms:
        na = int(c.get("agree", 0))
        if na:
            sl_agree = (torch.as_tensor(sl[:na], device=dev),
                        torch.as_tensor(np.ascontiguousarray(ps.rots[:na]), device=dev),
                        torch.as_tensor(np.ascontiguousarray(ps.weights[:na]), device=dev))
        for tile in c.get("kernels", (-1,)):
            key = "batched" if tile == -1 else {5: "batched_column", 6: "batched_pixel"}[tile]
            t = time.perf_counter()
            gpu[key], ag = gpu_batched(c, imgs, meta, tile, sl_agree)
            timing[key + "_s"] = time.perf_counter() - t
            if ag is not None and agree_worst is None:
                agree_worst = agreement_check(ag, o32, c["sym"], sl, ps.rots, ps.weights)
    rep = _report(gpu, vols)
    rep["case"] = {"name": name, "box": c["box"], "N": c["N"], "mode": c["mode"], "sym": c["sym"],
                   "particles": n, "ctf": c["ctf"], "snr": c["snr"],
                   "subsample_of": c.get("full_n") if c.get("full_n", n) != n else None}
    rep["oracle"] = ot
    rep["gpu_s"] = timing
    if agree_worst is not None:
        rep["agreement_max_rel_diff"] = agree_worst
        rep["agreement_slices"] = int(c["agree"])
    return rep


def graph_case(dev, seed: int = 103, pairs=((64, "gauss_5", "d7", 500), (160, "gauss_2", "c1", 700)),
               tasks=None) -> dict:
    """Batched form of the 64-job configuration, sampled: even/odd half-map
    pairs of distinct phantoms (box x1.5 padding, CTF, SNR 0.05, shifts
    U(-4, 4), weights U(0.5, 1)), all jobs inserted by ONE replay of a CUDA
    graph of the round; each job's finish(False) against the oracles."""
    import torch

    from eman2_b200.batch import BatchReconstructor
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    params, boxes, counts, imgs, metas, jobs = [], [], [], [], [], []
    for k, (box, mode, sym, n2) in enumerate(pairs):
        ps = make_particles(box, 2 * n2, seed=seed + k, snr=0.05, shift=4.0, weights=(0.5, 1.0),
                            ctf=True, device=dev)
        for half in range(2):
            idx = np.arange(half, 2 * n2, 2)
            c = dict(box=box, N=box * 3 // 2, mode=mode, sym=sym, ctf=True, tasks=tasks or 0)
            params.append({"size": [c["N"]] * 3, "sym": sym, "mode": mode})
            boxes.append(box)
            counts.append(len(idx))
            imgs.append(ps.images[torch.as_tensor(idx, device=ps.images.device)].contiguous())
            metas.append(particle_meta(ps.rots[idx], ps.shifts[idx], ps.weights[idx],
                                       defocus=ps.defocus[idx]))
            jobs.append((c, ps, idx))
    b = BatchReconstructor(params)
    g = b.capture(boxes, counts, [True] * len(params))
    g.launch(imgs, metas)
    g.close()
    out = {"jobs": []}
    for j, (c, ps, idx) in enumerate(jobs):
        d, nm = _finish(b.recons[j])
        host = imgs[j].cpu().numpy()
        _, vols, ot = oracle_volumes(c, host, ps.shifts[idx], ps.defocus[idx], ps.rots[idx],
                                     ps.weights[idx])
        rep = _report({"graph": (d, nm)}, vols)
        rep["job"] = {"box": c["box"], "N": c["N"], "mode": c["mode"], "sym": c["sym"],
                      "particles": int(len(idx)), "half": j % 2}
        rep["oracle"] = ot
        out["jobs"].append(rep)
    b.close()
    return out


def worst(rep: dict, against: str = "vs_fp32_oracle") -> dict:
    """Worst figures over the GPU forms of a report."""
    forms = [v[against] for k, v in rep.items()
             if isinstance(v, dict) and against in v]
    return {"rel_l2_complex": max(f["rel_l2_complex"] for f in forms),
            "rel_l2_weight": max(f["rel_l2_weight"] for f in forms),
            "fsc_min": min(f["fsc_min"] for f in forms)}
