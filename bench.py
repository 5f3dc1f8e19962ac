"""Benchmark of the direct Fourier inversion hot path (FourierReconstructor
insert_slice pipeline) on B200.

One step = one batch of particles through the reference caller's per-particle
pipeline (edge-mean, pad, CTF phase flip, shift, r2c) and the insertion of all
symmetry copies into the resident volume.  Default workload: box 256 padded to
384, gauss_5, d7, CTF, SNR 0.02 (the large single job of the reference's
make3d use), synthetic seeded particles.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

Prints one JSON line.  Multi-GPU runs are independent replicas (one
reconstruction per GPU, no collective on the data path): value is the sum of
particle-slices over ranks divided by the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: box, pad, mode, sym, ctf, snr, shift, weights, particles in the full job
    "c4": dict(box=256, N=384, mode="gauss_5", sym="d7", ctf=True, snr=0.02, shift=4.0,
               weights=(0.5, 1.0), job=200_000,
               desc="box 256 pad 384, gauss_5, d7, CTF, SNR 0.02 (200k-particle job)"),
    "c4g2": dict(box=256, N=384, mode="gauss_2", sym="d7", ctf=True, snr=0.02, shift=4.0,
                 weights=(0.5, 1.0), job=200_000,
                 desc="box 256 pad 384, gauss_2, d7, CTF, SNR 0.02 (the targets' configuration)"),
    "c2": dict(box=128, N=192, mode="gauss_2", sym="c1", ctf=True, snr=0.05, shift=4.0,
               weights=(0.5, 1.0), job=20_000,
               desc="box 128 pad 192, gauss_2, c1, CTF, SNR 0.05 (20k-particle job)"),
    "c1": dict(box=64, N=96, mode="gauss_2", sym="c1", ctf=False, snr=0.1, shift=2.0,
               weights=None, job=2_000, desc="box 64 pad 96, gauss_2, c1 (2k-particle job)"),
}


def nsym_of(sym: str) -> int:
    sym = sym.lower()
    platonic = {"tet": 12, "oct": 24, "icos": 60, "icos5": 60}
    if sym in platonic:
        return platonic[sym]
    k, n = sym[0], int(sym[1:] or 1)
    return n if k == "c" else 2 * n


def pixels_per_slice(N: int) -> int:
    """p(N): pixels kept by do_insert_slice_work (round(hypot) <= N/2)."""
    n2 = N // 2
    c = 0
    for y in range(-n2, n2):
        for x in range(0, n2 + 1):
            if int(float(np.float32(np.hypot(x, y))) + 0.5) <= n2:
                c += 1
    return c


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index),
                                      f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ------------------------------------------------------------------ helpers
def dist_setup():
    from eman2_b200 import replicas
    return replicas.init("nccl")


def barrier(ws):
    from eman2_b200 import replicas
    replicas.barrier(ws)


def max_over_ranks(v: float, ws: int) -> float:
    from eman2_b200 import replicas
    return replicas.max_over_ranks(v, ws)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(workload: str, batch: int):
    """DRAM bytes (read + write) of one insertion launch of this workload and
    batch, from the committed ncu capture of the same bench command; None
    when no capture of that size exists."""
    path = os.path.join(ROOT, "profiles", "k_column3_dram.json")
    try:
        with open(path) as f:
            e = json.load(f)[workload]
        if int(e["particles_per_launch"]) != batch:
            return None
        return float(e["dram_bytes_read"]) + float(e["dram_bytes_write"])
    except Exception:
        return None


def update_peaks():
    """Measured scattered-update roofs on this device (taps/s): shared-memory
    float4 read-modify-write, shared-memory atomics, L2 reductions."""
    from eman2_b200 import _lib
    lib = _lib.load()
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    if lib.fr_update_peaks(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) != 0:
        return None
    return {"smem_rmw": a.value, "smem_atom": b.value, "l2_red": c.value}


# ------------------------------------------------------------------ CPU baseline
def cpu_sample(wl: dict, seed: int, budget_s: float = 15.0, max_n: int = 64, threads: int = 0):
    """The oracle's FP32 restatement (-O3 -ffast-math, OpenMP with private
    volumes) on a bounded sample of the workload: prologue (numpy FFTs over
    batches of particles on the host threads, the same slices as the
    per-particle restatement) and insertion.  Returns (particle-slices/s,
    sample size, threads, seconds)."""
    from eman2_b200.synth import make_particles
    from oracle import accuracy, oracle
    threads = threads or os.cpu_count() or 1
    N, box = wl["N"], wl["box"]
    n = max(1, min(max_n, threads))
    total_n, total_t = 0, 0.0
    vol = oracle.OracleVolume(N, "omp")
    k = 0
    while total_t < budget_s and total_n < max_n:
        ps = make_particles(box, n, seed=seed + k, snr=wl["snr"], shift=wl["shift"],
                            weights=wl["weights"], ctf=wl["ctf"])
        t0 = time.perf_counter()
        sl = accuracy.slices_from_particles(ps.images, N, ps.shifts,
                                            ps.defocus if wl["ctf"] else None, threads=threads,
                                            chunk=max(1, -(-n // threads)))
        vol.insert_omp(sl, ps.rots, ps.weights, wl["mode"], wl["sym"], threads=threads)
        total_t += time.perf_counter() - t0
        total_n += n
        k += 1
        if total_t < budget_s / 4:
            n = min(max_n - total_n, n * 2) or n
    return total_n / total_t, total_n, threads, total_t


def cpu_sample_reference(wl: dict, seed: int, budget_s: float = 15.0, max_n: int = 64,
                         threads: int = 0):
    """The reference's own CPU insertion on a bounded sample of the workload:
    every pixel of every symmetry copy through FourierPixelInserter3D
    (libEM/reconstructor_tools.cpp, built from the reference tree with its
    release flags -O3 -ffast-math into oracle/_ref by oracle/build_ref.sh),
    fed the pixel stream of do_insert_slice_work as the oracle restates it,
    one private volume per host thread; the prologue as in cpu_sample.
    Returns (particle-slices/s, sample size, threads, seconds), or None when
    the reference could not be built."""
    from eman2_b200.synth import make_particles
    from oracle import accuracy, oracle
    if not oracle.ref_available():
        return None
    threads = threads or os.cpu_count() or 1
    N, box = wl["N"], wl["box"]
    n = max(1, min(max_n, threads))
    total_n, total_t = 0, 0.0
    k = 0
    while total_t < budget_s and total_n < max_n:
        ps = make_particles(box, n, seed=seed + k, snr=wl["snr"], shift=wl["shift"],
                            weights=wl["weights"], ctf=wl["ctf"])
        t0 = time.perf_counter()
        sl = accuracy.slices_from_particles(ps.images, N, ps.shifts,
                                            ps.defocus if wl["ctf"] else None, threads=threads,
                                            chunk=max(1, -(-n // threads)))
        oracle.ref_insert_threaded(N, sl, ps.rots, ps.weights, wl["mode"], wl["sym"], threads)
        total_t += time.perf_counter() - t0
        total_n += n
        k += 1
        if total_t < budget_s / 4:
            n = min(max_n - total_n, n * 2) or n
    return total_n / total_t, total_n, threads, total_t


def cpu_baseline_sample(wl: dict, seed: int, budget_s: float = 15.0, max_n: int = 64,
                        threads: int = 0):
    """(rate, sample, threads, seconds, kind, what): the reference's own
    inserter when oracle/_ref was built, else the oracle's restatement."""
    r = cpu_sample_reference(wl, seed, budget_s, max_n, threads)
    if r is not None:
        return (*r, "reference",
                "reference FourierPixelInserter3D (libEM/reconstructor_tools.cpp, -O3 "
                "-ffast-math) fed by the restated do_insert_slice_work pixel loop; numpy "
                "prologue")
    r = cpu_sample(wl, seed, budget_s, max_n, threads)
    return (*r, "port", "the oracle's OpenMP restatement; numpy prologue")


# ------------------------------------------------------------------ serving
SERVE_BOXES = (64, 128, 192, 256, 320)


def _meta_view(meta, a, b):
    """Entries a..b-1 of an fr_particle array, without a copy."""
    from eman2_b200 import _lib
    sz = ctypes.sizeof(_lib.fr_particle)
    return (_lib.fr_particle * (b - a)).from_address(ctypes.addressof(meta) + a * sz)


def particle_pools(dev, boxes, n: int, seed: int):
    """Per box, n seeded particles on the device (CTF, SNR 0.05, shifts U(-4, 4),
    weights U(0.5, 1)) and their metadata.  Requests and jobs take views of
    these, so their particles repeat every n."""
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    out = {}
    for box in boxes:
        ps = make_particles(box, n, seed=seed + box, snr=0.05, shift=4.0, weights=(0.5, 1.0),
                            ctf=True, device=dev)
        out[box] = (ps.images, particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus))
    return out


def serving_requests(pools, seed: int, nreq: int, rate: float, chunk: int,
                     pmin: int = 1000, pmax: int = 100_000):
    """A seeded stream of reconstruction requests of the serving configuration:
    box uniform over SERVE_BOXES padded x1.5, particle count log-uniform over
    [pmin, pmax], sym c1/c4/d7, gauss_2, CTF, chunks of `chunk`, Poisson
    arrivals at `rate`/s."""
    from eman2_b200.server import Request
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    for k in range(nreq):
        box = int(rng.choice(SERVE_BOXES))
        n = int(np.exp(rng.uniform(np.log(pmin), np.log(pmax))))
        sym = str(rng.choice(["c1", "c4", "d7"]))
        imgs, meta = pools[box]
        chunks = []
        for a in range(0, n, chunk):
            m = min(chunk, n - a)
            chunks.append((imgs[:m], _meta_view(meta, 0, m)))
        t += float(rng.exponential(1.0 / rate))
        reqs.append(Request(k, {"size": [box * 3 // 2] * 3, "sym": sym, "mode": "gauss_2"},
                            chunks, arrival=t, particles=n))
    return reqs


def fifo_latency(arrivals, service):
    """Latencies of a single server taking requests one at a time in arrival order."""
    free, lat = 0.0, []
    for a, s in sorted(zip(arrivals, service)):
        done = max(free, a) + s
        lat.append(done - a)
        free = done
    return lat


def run_serving(dev, seed: int = 4242, nreq: int = 128, rate: float = 4.0, chunk: int = 2048,
                plain_sample: int = 24, plain_every: int = 4, plain: bool = True):
    """The served form against the plain per-job GPU path on one request stream
    of the serving configuration (boxes 64-320 x1.5, 1,000-100,000 particles
    log-uniform, c1/c4/d7, gauss_2, CTF, chunks of 2048, Poisson arrivals).
    Served: continuous batching (one fr_insert_particles_multi per tick over
    every active job; finishes on their own streams), p50/p99 latency and
    throughput over the stream.  Plain: each request through its own
    FourierReconstructor with one insert call per particle (the drop-in
    insert_slice form), timed on `plain_sample` particles of every
    `plain_every`-th request and scaled to its count; its latency is that of
    a single FIFO server given those service times and the same arrivals."""
    import dataclasses

    import torch

    from eman2_b200 import FourierReconstructor
    from eman2_b200.server import GpuExecutor, Scheduler, Server
    pools = particle_pools(dev, SERVE_BOXES, chunk, seed)
    reqs = serving_requests(pools, seed, nreq, rate, chunk)
    parts = sum(r.particles for r in reqs)
    budget = int(torch.cuda.mem_get_info()[0] * 0.5)
    exe = GpuExecutor(doift=False)
    warm = [dataclasses.replace(r, arrival=0.0) for r in reqs[:6]]
    Server(Scheduler(budget, max_active=16), exe).run(warm)            # warm-up (untimed)
    torch.cuda.synchronize()
    srv = Server(Scheduler(budget, max_active=16), exe)
    poi = srv.run(reqs)
    torch.cuda.synchronize()
    exe.close()
    lat = sorted(j.done - j.req.arrival for j in srv.sched.done)
    stream = (f"{nreq} requests, Poisson {rate}/s, boxes {'/'.join(map(str, SERVE_BOXES))} x1.5, "
              f"1,000-100,000 particles log-uniform, c1/c4/d7, gauss_2, CTF, chunks of {chunk}; "
              f"particles repeat within a box's pool of {chunk}")
    served = {"p50_s": poi["p50_s"], "p99_s": poi["p99_s"], "p90_s": percentile(lat, 90),
              "max_s": lat[-1] if lat else None, "particle_slices_per_s": parts / poi["wall_s"],
              "wall_s": poi["wall_s"], "ticks": poi["ticks"], "requests": poi["requests"],
              "particles": parts}
    if not plain:
        return {"served": served, "stream": stream}

    def per_job(r, k=None, schedule="scatter"):
        """Seconds for request r alone: setup, insert (k particles one per
        call, or every chunk whole when k is None), finish."""
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rec = FourierReconstructor(r.params)
        rec.setup()
        t1 = time.perf_counter()
        if k is None:
            for img, meta in r.chunks:
                rec.insert_particles(img, meta, schedule=schedule)
        else:
            img, meta = r.chunks[0]
            for i in range(min(k, len(meta))):
                rec.insert_particles(img[i:i + 1], _meta_view(meta, i, i + 1), schedule=schedule)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        rec.finish(False)
        t3 = time.perf_counter()
        rec.close()
        return (t1 - t0) + (t3 - t2), t2 - t1

    sample = reqs[::plain_every]
    for r in sample[:3]:
        per_job(r, 4)                                                  # warm-up
    service, s_parts = [], 0
    for r in sample:
        fixed, ins = per_job(r, plain_sample)
        service.append(fixed + ins * r.particles / min(plain_sample, r.particles))
        s_parts += r.particles
    plain_rate = s_parts / sum(service)
    # the plain path's latency on the whole stream: each request's service
    # time from the sampled rate of its (box, sym) class or, failing that,
    # the overall rate
    rate_of = {}
    for r, sv in zip(sample, service):
        rate_of.setdefault((r.params["size"][0], r.params["sym"]), []).append(r.particles / sv)
    est = [r.particles / float(np.mean(rate_of.get((r.params["size"][0], r.params["sym"]),
                                                   [plain_rate])))
           for r in reqs]
    plain_lat = fifo_latency([r.arrival for r in reqs], est)
    served_rate = parts / poi["wall_s"]
    return {
        "served": served,
        "plain_per_particle": {"particle_slices_per_s": plain_rate,
                               "p50_s": percentile(plain_lat, 50), "p99_s": percentile(plain_lat, 99),
                               "sample": f"{plain_sample} particles of every {plain_every}th request, "
                                         "scaled to its count; latency from a FIFO single server "
                                         "under the same arrivals"},
        "speedup_served_vs_plain": served_rate / plain_rate,
        "stream": stream,
    }


def percentile(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


# ------------------------------------------------------------------ finish
def run_finish(dev, wl: dict, reps: int = 3):
    """finish(True) + math.gausskernelfix + centred clip to the box (what
    e2make3dpar does after the last insert) on a seeded N^3 volume: the fused
    fr_finish_corrected against finish, the processor and the clip as three
    device passes.  Device-timed with CUDA events, outputs in HBM."""
    import torch

    from eman2_b200 import FourierReconstructor, _lib
    lib = _lib.load()
    N, box = wl["N"], wl["box"]
    width = FourierReconstructor.KERNEL_FIX_WIDTH.get(wl["mode"], 0.0)
    g = torch.Generator(device=dev).manual_seed(5)
    seed = torch.randn((N, N, N + 2), device=dev, generator=g)
    wts = torch.rand((N, N, N // 2 + 1), device=dev, generator=g) + 0.5
    stream = torch.cuda.Stream(device=dev)
    full = torch.empty((N, N, N), device=dev)
    out = torch.empty((box, box, box), device=dev)
    torch.cuda.synchronize()
    r = FourierReconstructor({"size": [N] * 3, "sym": wl["sym"], "mode": wl["mode"]})
    r.setup()
    _lib.check(lib.fr_set_stream(r.handle, ctypes.c_void_p(stream.cuda_stream)))
    x0 = (N - box) // 2

    def fused():
        r.setup_seedandweights(seed, wts)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(lib.fr_finish_corrected(r.handle, width, box, box, box, out.data_ptr(), None))
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def separate():
        r.setup_seedandweights(seed, wts)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(lib.fr_finish(r.handle, 1, full.data_ptr(), None))
        _lib.check(lib.fr_kernel_fix(full.data_ptr(), N, N, N, width,
                                     ctypes.c_void_p(stream.cuda_stream)))
        with torch.cuda.stream(stream):
            out.copy_(full[x0:x0 + box, x0:x0 + box, x0:x0 + box])
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for f in (fused, separate):
        f()
    t_fused = min(fused() for _ in range(reps))
    t_sep = min(separate() for _ in range(reps))
    r.close()
    return {"N": N, "out": box, "gauss_width": width, "fused_ms": t_fused, "separate_ms": t_sep,
            "note": "normalize + c2r 3-D + depad/centre/scale + kernel fix + clip"}


# ------------------------------------------------------------------ I/O
def run_io(dev, wl: dict, n: int = 16384, chunk: int = 4096):
    """Particles streamed from a .mrcs stack on local disk (page cache) into a
    reconstruction of the workload, stored as float32 and as float16, against
    the same particles already in HBM; one warmed reconstructor for all three
    (setup() re-zeroes it).  The files are written to a temporary directory
    and removed afterwards."""
    import shutil
    import tempfile

    import torch

    from eman2_b200 import FourierReconstructor, io
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    B, N = wl["box"], wl["N"]
    ps = make_particles(B, n, seed=77, snr=wl["snr"], shift=wl["shift"], weights=wl["weights"],
                        ctf=wl["ctf"], device=dev)
    meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
    sz = ctypes.sizeof(type(meta[0]))
    d_imgs = ps.images if isinstance(ps.images, torch.Tensor) else torch.as_tensor(ps.images, device=dev)
    host = d_imgs.cpu().numpy()
    tmp = tempfile.mkdtemp(prefix="fr_io_")
    out = {"particles": n, "chunk": chunk, "box": B, "pad": N}
    r = FourierReconstructor({"size": [N] * 3, "sym": wl["sym"], "mode": wl["mode"]})
    r.setup()

    def from_hbm():
        for a in range(0, n, chunk):
            m = (type(meta[0]) * min(chunk, n - a)).from_address(ctypes.addressof(meta) + a * sz)
            r.insert_particles(d_imgs[a:a + chunk], m)

    def timed(fn):
        r.setup()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    try:
        from_hbm()                                           # warm-up: plans, scratch
        out["hbm_resident_particle_slices_per_s"] = n / timed(from_hbm)
        for mode, name in ((2, "float32"), (12, "float16")):
            path = os.path.join(tmp, f"ptcl_{name}.mrcs")
            io.write_mrc(path, host, mode=mode)
            io.insert_stack(r, path, meta, chunk=chunk)      # warm-up: page cache, pinned buffers
            dt = timed(lambda: io.insert_stack(r, path, meta, chunk=chunk))
            fbytes = n * B * B * (4 if mode == 2 else 2)
            out[name] = {"particle_slices_per_s": n / dt, "file_gbs": fbytes / dt / 1e9,
                         "file_bytes": fbytes}
    finally:
        r.close()
        shutil.rmtree(tmp, ignore_errors=True)
    out["source"] = "page cache of local disk; file read by 16 threads into pinned buffers"
    return out


# ------------------------------------------------------------------ batched
BATCH_BOXES = (64, 96, 128, 160)


def config3_jobs(seed: int = 33, pairs: int = 32):
    """The batched configuration's 64 reconstructions: 32 even/odd half-map
    pairs, each pair a box from BATCH_BOXES (padded x1.5), sym c1 or d7, mode
    gauss_2 or gauss_5 (each 50/50); a pair's particle count is log-uniform
    over [1,000, 100,000] and split evenly, so each reconstruction's count is
    log-uniform over [500, 50,000]."""
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(pairs):
        b = int(rng.choice(BATCH_BOXES))
        sym, mode = str(rng.choice(["c1", "d7"])), str(rng.choice(["gauss_2", "gauss_5"]))
        n = int(np.exp(rng.uniform(np.log(1000), np.log(100_000))))
        for half in range(2):
            jobs.append({"params": {"size": [b * 3 // 2] * 3, "sym": sym, "mode": mode},
                         "box": b, "count": (n + 1 - half) // 2})
    return jobs


def run_batched(dev, seed: int = 33, chunk: int = 2048, graph_chunk: int = 512, reps: int = 3,
                plain_sample: int = 16):
    """The batched form on the batched configuration's draw of 64
    reconstructions (config3_jobs): every particle of every job, inserted in
    rounds of up to `chunk` particles per job (one multi-job launch sequence
    per round, schedules from the autotuner), device-timed; and one round of
    the first `graph_chunk` particles of every job captured as a CUDA graph
    and replayed.  Beside them the plain per-particle path, sampled."""
    import torch

    from eman2_b200 import FourierReconstructor
    from eman2_b200.batch import BatchReconstructor, autotune, insert_particles_multi, set_tile
    jobs = config3_jobs(seed)
    params = [j["params"] for j in jobs]
    boxes = [j["box"] for j in jobs]
    counts = [j["count"] for j in jobs]
    total = sum(counts)
    pools = particle_pools(dev, BATCH_BOXES, chunk, seed)
    combos = {}
    for p, n in zip(params, counts):
        key = (p["size"][0], p["mode"], nsym_of(p["sym"]))
        combos[key] = max(combos.get(key, 0), min(n, chunk))
    tuned = {f"N{k[0]} {k[1]} nsym{k[2]}": autotune(k[0], k[1], k[2], nparticles=n)[0]
             for k, n in combos.items()}
    stream = torch.cuda.Stream(device=dev)

    def rounds(recons, upto=None):
        """Every job's particles (or its first `upto`), round by round."""
        left = list(counts) if upto is None else [min(c, upto) for c in counts]
        while any(left):
            act = [j for j in range(len(jobs)) if left[j] > 0]
            m = [min(chunk, left[j]) for j in act]
            insert_particles_multi([recons[j] for j in act],
                                   [pools[boxes[j]][0][:k] for j, k in zip(act, m)],
                                   [_meta_view(pools[boxes[j]][1], 0, k) for j, k in zip(act, m)],
                                   stream)
            for j, k in zip(act, m):
                left[j] -= k

    def timed(fn, n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    try:
        b1 = BatchReconstructor(params)
        rounds(b1.recons, upto=chunk)                                   # warm-up: scratch, plans
        ms_full = timed(lambda: rounds(b1.recons), 1)
        b1.close()
        gcounts = [min(c, graph_chunk) for c in counts]
        b2 = BatchReconstructor(params)
        t0 = time.perf_counter()
        g = b2.capture(boxes, gcounts, [True] * len(params), stream=stream)
        capture_s = time.perf_counter() - t0
        gimgs = [pools[b][0][:k] for b, k in zip(boxes, gcounts)]
        gmetas = [_meta_view(pools[b][1], 0, k) for b, k in zip(boxes, gcounts)]
        g.launch(gimgs, gmetas)
        ms_graph = timed(lambda: g.launch(gimgs, gmetas), reps)
        ms_multi = timed(lambda: insert_particles_multi(b2.recons, gimgs, gmetas, stream), reps)
        g.close()
        b2.close()
    finally:
        for k in combos:
            set_tile(k[0], k[1], k[2], -1)
    spent, done = 0.0, 0
    for j in range(0, len(params), 4):
        rec = FourierReconstructor(params[j])
        rec.setup()
        imgs, meta = pools[boxes[j]]
        rec.insert_particles(imgs[:1], _meta_view(meta, 0, 1), schedule="scatter")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(plain_sample):
            rec.insert_particles(imgs[i:i + 1], _meta_view(meta, i, i + 1), schedule="scatter")
        torch.cuda.synchronize()
        spent += time.perf_counter() - t0
        done += plain_sample
        rec.close()
    plain = done / spent
    full_rate = total / (ms_full / 1e3)
    gparts = sum(gcounts)
    graph_rate = gparts / (ms_graph / 1e3)
    overhead = per_job_overhead(params, boxes, [pools[b][0] for b in boxes],
                                [pools[b][1] for b in boxes], stream, reps)
    return {"jobs": len(params), "particles": total,
            "counts": {"min": min(counts), "median": float(np.median(counts)), "max": max(counts)},
            "all_particles": {"ms": ms_full, "particle_slices_per_s": full_rate,
                              "rounds_of": chunk},
            "graph_round": {"ms_per_round": ms_graph, "particles_per_round": gparts,
                            "particle_slices_per_s": graph_rate, "capture_s": capture_s,
                            "no_graph_ms_per_round": ms_multi},
            "plain_per_particle": {"particle_slices_per_s": plain,
                                   "sample": f"{plain_sample} particles of every 4th job"},
            "speedup_batched_vs_plain": full_rate / plain,
            "per_job_overhead": overhead,
            "autotuned": tuned,
            "draw": "32 even/odd pairs, boxes 64/96/128/160 x1.5, c1/d7, gauss_2/gauss_5, "
                    "500-50,000 particles per job log-uniform, CTF; particles repeat within a "
                    f"box's pool of {chunk}"}


def per_job_overhead(params, boxes, pool_imgs, pool_metas, stream, reps: int = 5):
    """Per-job latency overhead of the plain path against the batched form, on
    the 64 jobs with ONE particle each, under one rule for both arms: every
    call is enqueued and the round is waited for once at its end (what a
    drop-in insert_slice loop does: the ABI returns once work is enqueued).
    "empty": the particle has weight 0, so every stage runs (host call,
    metadata, prologue launches, insertion launch) but no tap is added, so
    the time is all fixed cost; "one_particle": weight as drawn, schedules
    autotuned for one particle.  Plain: one insert call per job.  Batched: one
    replay of a graph of all jobs (and one multi-job call without the
    graph).  Wall-clock per round divided by the job count, since the
    overhead is host and launch time."""
    import torch

    from eman2_b200 import _lib
    from eman2_b200.batch import BatchReconstructor, autotune, insert_particles_multi, set_tile
    nj = len(params)
    combos = {(p["size"][0], p["mode"], nsym_of(p["sym"])) for p in params}
    tuned = {f"N{k[0]} {k[1]} nsym{k[2]}": autotune(k[0], k[1], k[2], nparticles=1)[0]
             for k in combos}
    one_imgs = [im[:1] for im in pool_imgs]

    def first(m, weight=None):
        a = (_lib.fr_particle * 1)()
        ctypes.memmove(a, ctypes.addressof(m), ctypes.sizeof(_lib.fr_particle))
        if weight is not None:
            a[0].weight = weight
        return a

    def wall(fn, n):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / n

    def measure(one_metas):
        bp = BatchReconstructor(params)
        try:
            for r in bp.recons:
                _lib.check(_lib.load().fr_set_stream(r.handle, ctypes.c_void_p(stream.cuda_stream)))

            def plain_round():
                for j in range(nj):
                    bp.recons[j].insert_particles(one_imgs[j], one_metas[j], schedule="scatter")
            plain_s = wall(plain_round, reps)
            multi_s = wall(lambda: insert_particles_multi(bp.recons, one_imgs, one_metas, stream),
                           reps * 8)
        finally:
            bp.close()
        bg = BatchReconstructor(params)
        try:
            g = bg.capture(boxes, [1] * nj, [True] * nj, stream=stream)
            # a replay lasts ~0.1 ms: enough of them that the closing wait
            # and the clock ramp do not weigh on the per-replay time
            graph_s = wall(lambda: g.launch(one_imgs, one_metas), reps * 40)
            g.close()
        finally:
            bg.close()
        ms = lambda t: t * 1e3 / nj
        return {"plain_ms_per_job": ms(plain_s), "no_graph_ms_per_job": ms(multi_s),
                "graph_ms_per_job": ms(graph_s), "removed_x": plain_s / graph_s}

    try:
        empty = measure([first(m, 0.0) for m in pool_metas])
        one = measure([first(m) for m in pool_metas])
    finally:
        for k in combos:
            set_tile(k[0], k[1], k[2], -1)
    return {"jobs": nj, "rule": "every call enqueued, the round waited for once at its end",
            "empty": empty, "one_particle": one, "autotuned_one_particle": tuned}


# ------------------------------------------------------------------ accuracy
def run_accuracy(dev):
    """Accuracy at the configurations' sizes (the harness of
    tests/test_gpu_accuracy.py): box 64 -> 96, 2,000 particles and box 128 ->
    192, 20,000 particles in full, and a 16-particle sample of the box 256 ->
    384, gauss_5, d7 job, each through the plain and the batched form against
    the FP32-faithful, exact-sum and FP64 oracles."""
    from tests import accuracy_harness as H
    out = {}
    for name, kw in (("c1", {}), ("c2", {}), ("c4", {"n": 16, "tasks": 16})):
        t0 = time.perf_counter()
        rep = H.run_case(name, dev, **kw)
        summary = {"particles": rep["case"]["particles"], "box": rep["case"]["box"],
                   "pad": rep["case"]["N"], "mode": rep["case"]["mode"], "sym": rep["case"]["sym"],
                   "fp32_oracle_vs_fp64": {k: rep["fp32_oracle_vs_fp64"][k]
                                           for k in ("rel_l2_complex", "rel_l2_weight", "fsc_min")}}
        for form in ("plain", "batched"):
            summary[form] = {against: {k: rep[form][against][k]
                                       for k in ("rel_l2_complex", "rel_l2_weight", "fsc_min",
                                                 "support_mismatch")}
                             for against in ("vs_fp32_oracle", "vs_exact_sums", "vs_fp64_oracle")}
        if "agreement_max_rel_diff" in rep:
            summary["agreement_max_rel_diff"] = rep["agreement_max_rel_diff"]
        summary["seconds"] = time.perf_counter() - t0
        out[name] = summary
    out["bar"] = ("relative L2 <= 1e-5 of finish(False) and normout against the FP32 oracle, "
                  "FSC >= 0.9999 in every shell (the reference's shell rule)")
    return out


# ------------------------------------------------------------------ target configuration
def run_target(dev, steps: int = 3, plain_n: int = 64):
    """Box 256 padded to 384, gauss_2, d7 (the targets' configuration): the
    batched form (2,048 particles per call through the pixel-major gather
    kernel) against the plain form (one insert call per particle, scatter),
    both device-timed on the library stream with particles in HBM, and
    the pixel kernel's update roofline against the shared-atomic peak."""
    import torch

    from eman2_b200 import Reconstructors, _lib
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    lib = _lib.load()
    wl = WORKLOADS["c4g2"]
    N, B = wl["N"], wl["box"]
    ps = make_particles(B, 2048, seed=1300, snr=wl["snr"], shift=wl["shift"], weights=wl["weights"],
                        ctf=True, device=dev)
    meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
    r = Reconstructors.get("fourier", {"size": [N] * 3, "sym": wl["sym"], "mode": wl["mode"]})
    r.setup()
    stream = torch.cuda.Stream(device=dev)
    _lib.check(lib.fr_set_stream(r.handle, ctypes.c_void_p(stream.cuda_stream)))
    for _ in range(2):
        r.insert_particles(ps.images, meta)
    torch.cuda.synchronize()
    _lib.check(lib.fr_profile(1))
    _lib.check(lib.fr_stats_reset())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        r.insert_particles(ps.images, meta)
    e1.record(stream)
    e1.synchronize()
    st = _lib.stats()
    _lib.check(lib.fr_profile(0))
    batched = steps * 2048 / (e0.elapsed_time(e1) / 1e3)
    for i in range(3):
        r.insert_particles(ps.images[i:i + 1], _meta_view(meta, i, i + 1), schedule="scatter")
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(plain_n):
        r.insert_particles(ps.images[i:i + 1], _meta_view(meta, i, i + 1), schedule="scatter")
    e1.record(stream)
    e1.synchronize()
    plain = plain_n / (e0.elapsed_time(e1) / 1e3)
    r.close()
    gms = st["gather_ms"] / max(1, st["gather_launches"])
    taps = nsym_of(wl["sym"]) * pixels_per_slice(N) * 8 * 2048 / (gms / 1e3)
    upd = update_peaks()
    out = {"workload": wl["desc"], "batched": {"value": batched, "unit": "particle-slices/s",
                                               "particles_per_call": 2048, "kernel": "k_pixel",
                                               "avg_launch_ms": gms},
           "plain": {"value": plain, "unit": "particle-slices/s", "sample": plain_n,
                     "kernel": "k_scatter"},
           "batched_vs_plain": batched / plain}
    if upd is not None:
        out["update_roofline"] = {"bound": "shared-memory FP32 atomics (3 per tap)",
                                  "achieved": taps, "peak": upd["smem_atom"], "unit": "taps/s",
                                  "frac": taps / upd["smem_atom"]}
    # the HBM roofline of the same launch, as the main line's (algorithmic
    # bytes over the launch time) with its committed DRAM traffic
    peak, peak_kind = load_peaks()
    V = (N // 2 + 1) * N * N
    alg = 2048 * (8 * (N // 2 + 1) * N + 64) + 24 * V
    achieved = alg / (gms / 1e3) / 1e9
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "traffic": load_traffic("c4g2", 2048),
                       "peak_source": peak_kind, "alg_bytes_per_launch": alg}
    return out


# ------------------------------------------------------------------ GPU run
def run_gpu(args, wl, ws, rank, local):
    import torch

    from eman2_b200 import Reconstructors, _lib
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _lib.load()
    B, N, batch = wl["box"], wl["N"], args.batch
    ps = make_particles(B, batch, seed=1000 + rank, snr=wl["snr"], shift=wl["shift"],
                        weights=wl["weights"], ctf=wl["ctf"], device=dev)
    d_imgs = ps.images if isinstance(ps.images, torch.Tensor) else torch.as_tensor(ps.images, device=dev)
    meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
    r = Reconstructors.get("fourier", {"size": [N] * 3, "sym": wl["sym"], "mode": wl["mode"]})
    r.setup()
    if args.tile != -1:
        _lib.check(lib.fr_set_tile(N, _lib.MODE_IDS[wl["mode"]], nsym_of(wl["sym"]), args.tile))
    stream = torch.cuda.Stream(device=dev)
    _lib.check(lib.fr_set_stream(r.handle, ctypes.c_void_p(stream.cuda_stream)))

    def step(src):
        r.insert_particles(src, meta)

    for _ in range(args.warmup):
        step(d_imgs)
    torch.cuda.synchronize()
    _lib.check(lib.fr_profile(1))
    _lib.check(lib.fr_stats_reset())
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")      # ncu --nvtx --nvtx-include timed/
        e0.record(stream)
        for _ in range(args.steps):
            step(d_imgs)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    st = _lib.stats()
    _lib.check(lib.fr_profile(0))
    ms_max = max_over_ranks(ms, ws)

    # e2e: the same steps through the public API from pinned host memory
    h_imgs = d_imgs.cpu().pin_memory()
    for _ in range(max(2, args.warmup)):      # both staging buffers allocated
        step(h_imgs)
    torch.cuda.synchronize()
    barrier(ws)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        step(h_imgs)
    f1.record(stream)
    f1.synchronize()
    barrier(ws)
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), ws)

    # plain per-call path: one particle per call (scatter insertion)
    plain = None
    if rank == 0 and args.plain > 0:
        m1 = [particle_meta(ps.rots[i:i + 1], ps.shifts[i:i + 1], ps.weights[i:i + 1],
                            defocus=ps.defocus[i:i + 1]) for i in range(args.plain)]
        for i in range(3):
            r.insert_particles(d_imgs[i:i + 1], m1[i], schedule="scatter")
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for i in range(args.plain):
            r.insert_particles(d_imgs[i:i + 1], m1[i], schedule="scatter")
        g1.record(stream)
        g1.synchronize()
        plain = args.plain / (g0.elapsed_time(g1) / 1e3)
    # agreement pass (determine_slice_agreement, sub=False) against the volume
    # just built: n slices through the batched call, device-timed
    agree = None
    if rank == 0 and args.agree > 0:
        g = torch.Generator(device=dev).manual_seed(11)
        na = args.agree
        sl = torch.randn((na, N, N + 2), device=dev, generator=g)
        rots = torch.as_tensor(ps.rots[:na], device=dev) if not isinstance(ps.rots, torch.Tensor) \
            else ps.rots[:na].contiguous()
        wts = torch.ones(na, device=dev)
        torch.cuda.synchronize()
        r.slice_agreement(sl[:4], rots[:4], wts[:4])
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        r.slice_agreement(sl, rots, wts)
        a1.record(stream)
        a1.synchronize()
        ams = a0.elapsed_time(a1)
        agree = {"slices": na, "ms": ams, "particle_slices_per_s": na / (ams / 1e3),
                 "note": "sub=False, FP64 sums, every symmetry copy of every slice"}
    return ms_max, e2e_ms, st, clk.summary(), plain, agree


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOADS))
    ap.add_argument("--batch", type=int, default=2048, help="particles per step")
    ap.add_argument("--plain", type=int, default=64, help="particles timed on the plain path")
    ap.add_argument("--agree", type=int, default=256,
                    help="slices timed through the agreement pass (0: skip)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true",
                    help="skip the target, finish, I/O, batched and serving legs")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the accuracy leg (GPU forms against the oracles)")
    ap.add_argument("--tile", type=int, default=-1,
                    help="pin the insertion kernel (0-3 register tiles, 4 staged column, 6 pixel-major, "
                         "5 barrier-free column, -2 scatter); default: library choice")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    ws, rank, local = dist_setup()
    S = nsym_of(wl["sym"])
    N = wl["N"]
    metric = "particle-slices inserted/s"
    config = {"workload": f"{args.workload}: {wl['desc']}", "box": wl["box"], "pad": N,
              "mode": wl["mode"], "sym": wl["sym"], "particles_per_step": args.batch,
              "l2": "inputs larger than L2 (particles + volume > 126 MB)",
              "parallelism": f"replicas x{ws}"}

    if args.impl == "reference":
        if rank != 0:
            return
        from eman2_b200.synth import make_particles  # noqa: F401
        vals = []
        for k in range(args.warmup + args.steps):
            v, n, thr, secs, kind, what = cpu_baseline_sample(wl, seed=5000 + k, budget_s=8.0,
                                                              max_n=32)
            if k >= args.warmup:
                vals.append((v, n, thr, secs))
        val = float(np.mean([v for v, *_ in vals]))
        line = {"impl": "reference", "metric": metric, "value": val, "unit": "particle-slices/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": float(np.mean([s for *_, s in vals])) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": val, "unit": "particle-slices/s", "cores": vals[0][2],
                                 "kind": kind,
                                 "sample": f"{vals[0][1]} particles per step of the workload; "
                                           f"{what}"},
                "e2e": {"value": val, "unit": "particle-slices/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    ms, e2e_ms, st, clk, plain, agree = run_gpu(args, wl, ws, rank, local)
    if rank != 0:
        return
    value = ws * args.steps * args.batch / (ms / 1e3)
    e2e = ws * args.steps * args.batch / (e2e_ms / 1e3)
    V = (N // 2 + 1) * N * N
    alg_bytes = args.batch * (8 * (N // 2 + 1) * N + 64) + 24 * V
    if st["gather_launches"] > 0:
        # the library's default: k_column3 for gauss_5, k_pixel for the narrow windows
        tile = args.tile if args.tile != -1 else (5 if wl["mode"] == "gauss_5" else 6)
        kname = {6: "k_pixel", 5: "k_column3", 4: "k_column"}.get(tile, "k_gather") + \
            " (gather schedule)"
        gms = st["gather_ms"] / st["gather_launches"]
    else:
        kname, gms = "k_scatter", st["insert_ms"] / max(1, st["insert_launches"])
    achieved = alg_bytes / (gms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    traffic = load_traffic(args.workload, args.batch)
    p = pixels_per_slice(N)
    taps_per = S * p * (216 if wl["mode"] == "gauss_5" else 8 if wl["mode"] == "gauss_2" else 1)
    taps_s = taps_per * args.batch / (gms / 1e3)
    upd = update_peaks()
    line = {
        "metric": metric, "value": value, "unit": "particle-slices/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian-blob phantom projections, CTF, noise)",
        "config": config,
        "e2e": {"value": e2e, "unit": "particle-slices/s",
                "h2d_bytes_per_step": args.batch * wl["box"] * wl["box"] * 4 + args.batch * 76,
                "d2h_bytes_per_step": 4},
        "gpu_launches": int(st["kernel_launches"]),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "kernel": kname,
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": gms},
        "taps": {"per_particle_upper": taps_per, "per_s_upper": taps_s},
        "clocks": clk,
    }
    if upd is not None:
        # the binding roof: the rate of the accumulator update the kernel
        # uses (the column kernel: one shared float4 read-modify-write per
        # tap; the pixel kernel: three shared FP32 atomics; the scatter:
        # three L2 reductions)
        key = ("l2_red" if st["gather_launches"] == 0 else
               "smem_atom" if kname.startswith("k_pixel") else "smem_rmw")
        line["update_roofline"] = {
            "bound": {"smem_rmw": "shared-memory float4 read-modify-write",
                      "smem_atom": "shared-memory FP32 atomics (3 per tap)",
                      "l2_red": "L2 red.global.add.f32 (3 per tap)"}[key],
            "achieved": taps_s, "peak": upd[key], "unit": "taps/s", "frac": taps_s / upd[key],
            "peaks_measured": upd, "taps": "upper bound S*p(N)*window"}
    if agree is not None:
        line["agreement"] = agree
    if plain is not None:
        line["plain_gpu"] = {"value": plain, "unit": "particle-slices/s", "sample": args.plain,
                             "speedup_batched_vs_plain": value / plain}
    if not args.no_serve and ws == 1:
        import torch
        dev = torch.device("cuda", local)
        line["target_c4g2"] = run_target(dev)
        line["finish"] = run_finish(dev, wl)
        line["io"] = run_io(dev, WORKLOADS["c2"])
        line["batched"] = run_batched(dev)
        line["serving"] = run_serving(dev)
        # the same configuration at the low end of its arrival rates, where
        # the stream does not saturate the device: latency without queueing
        line["serving_1rps"] = run_serving(dev, seed=4343, nreq=48, rate=1.0, plain=False)
    if not args.no_accuracy and ws == 1:
        import torch
        line["accuracy"] = run_accuracy(torch.device("cuda", local))
    if not args.no_cpu and ws == 1:
        v, n, thr, secs, kind, what = cpu_baseline_sample(wl, seed=7000)
        line["cpu_baseline"] = {"value": v, "unit": "particle-slices/s", "cores": thr,
                                "kind": kind,
                                "sample": f"{n} particles of the workload, {secs:.1f} s; {what}"}
        # the same code on one host core (a per-core figure beside the all-core one)
        v1, n1, _, secs1, _, _ = cpu_baseline_sample(wl, seed=7100, budget_s=6.0, max_n=8,
                                                     threads=1)
        line["cpu_baseline"]["single_thread"] = {
            "value": v1, "unit": "particle-slices/s", "cores": 1,
            "sample": f"{n1} particles, {secs1:.1f} s"}
    print(json.dumps(line))


if __name__ == "__main__":
    try:
        main()
    finally:
        from eman2_b200 import replicas
        replicas.finalize(int(os.environ.get("WORLD_SIZE", "1")))
