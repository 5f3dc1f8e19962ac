"""Batched and served forms change execution, not arithmetic: every job's
volume equals the one the plain per-job path gives it (alone vs in the mix),
within the FP32 summation-order tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

# Two GPU runs of the same job differ only in the order of their FP32 atomic
# adds; for gauss_5 with symmetry copies (216 taps per pixel, several slices
# per particle) that order alone moves the volumes by up to ~2e-6 relative L2.
RTOL = 5e-6


def _jobs():
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    specs = [(32, 48, "gauss_2", "c1", 40), (40, 60, "gauss_5", "d2", 25),
             (32, 48, "gauss_5", "c1", 30), (24, 36, "nearest_neighbor", "c3", 50)]
    jobs = []
    for k, (box, N, mode, sym, n) in enumerate(specs):
        ps = make_particles(box, n, seed=300 + k, snr=0.5, shift=2.0, weights=(0.5, 1.0),
                            ctf=(k % 2 == 0))
        meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
        jobs.append(({"size": [N] * 3, "sym": sym, "mode": mode}, ps, meta))
    return jobs


def _alone(params, images, meta):
    from eman2_b200 import FourierReconstructor
    r = FourierReconstructor(params)
    r.setup()
    r.insert_particles(images, meta)
    return r.get_accumulators()


def test_batch_equals_each_job_alone(gpu):
    from eman2_b200.batch import BatchReconstructor
    jobs = _jobs()
    b = BatchReconstructor([p for p, _, _ in jobs])
    b.insert_particles([ps.images for _, ps, _ in jobs], [m for _, _, m in jobs])
    for j, (params, ps, meta) in enumerate(jobs):
        d, n = b.get_accumulators(j)
        d0, n0 = _alone(params, ps.images, meta)
        assert oracle.rel_l2(d, d0) < RTOL and oracle.rel_l2(n, n0) < RTOL
    # one job against the oracle's restatement of the whole caller loop
    params, ps, meta = jobs[1]
    N = params["size"][0]
    sl = np.stack([oracle.particle_to_slice(ps.images[i], N, ps.shifts[i],
                                            {"defocus": float(ps.defocus[i])})
                   for i in range(len(ps.images))])
    o = oracle.OracleVolume(N, "fp32")
    o.insert(sl, ps.rots, ps.weights, params["mode"], params["sym"])
    d, n = b.get_accumulators(1)
    assert oracle.rel_l2(n, o.norm) < RTOL and oracle.rel_l2(d, o.data) < 2e-5


def test_autotune_and_mixed_schedules_in_one_batch(gpu):
    """The autotuner times every schedule; with each job pinned to a
    different one, the batch still gives every job its alone result."""
    from eman2_b200.batch import BatchReconstructor, autotune, set_tile
    tile, ms = autotune(48, "gauss_2", 1, nparticles=64)
    assert tile in (0, 1, 2, 3, 4, 5, 6, -2) and len(ms) == 8 and all(v > 0 for v in ms.values())
    set_tile(48, "gauss_2", 1, -1)
    jobs = _jobs()
    nsym = {"c1": 1, "d2": 4, "c3": 3}
    pins = [6, 1, 5, -2]
    try:
        for (params, _, _), t in zip(jobs, pins):
            set_tile(params["size"][0], params["mode"], nsym[params["sym"]], t)
        b = BatchReconstructor([p for p, _, _ in jobs])
        b.insert_particles([ps.images for _, ps, _ in jobs], [m for _, _, m in jobs])
        got = [b.get_accumulators(j) for j in range(len(jobs))]
    finally:
        for (params, _, _) in jobs:
            set_tile(params["size"][0], params["mode"], nsym[params["sym"]], -1)
    for j, (params, ps, meta) in enumerate(jobs):
        d0, n0 = _alone(params, ps.images, meta)
        assert oracle.rel_l2(got[j][0], d0) < RTOL and oracle.rel_l2(got[j][1], n0) < RTOL


def _split(ps, meta_fn, a, b):
    return ps.images[a:b], meta_fn(ps.rots[a:b], ps.shifts[a:b], ps.weights[a:b],
                                   defocus=ps.defocus[a:b])


def test_graph_replays_equal_batched_rounds(gpu):
    """Replays of a captured round (device images, host images, the slots as
    filled, then a mix of device and host images) give each job what the same
    batched calls give it."""
    import torch

    from eman2_b200.batch import BatchReconstructor
    from eman2_b200.particles import particle_meta
    jobs = _jobs()
    half = [len(ps.images) // 2 for _, ps, _ in jobs]
    first = [_split(ps, particle_meta, 0, h) for (_, ps, _), h in zip(jobs, half)]
    second = [_split(ps, particle_meta, h, 2 * h) for (_, ps, _), h in zip(jobs, half)]
    ctf = [bool(np.any(np.abs(ps.defocus) > 1e-4)) for _, ps, _ in jobs]
    boxes = [ps.images.shape[-1] for _, ps, _ in jobs]
    b1 = BatchReconstructor([p for p, _, _ in jobs])
    for part in (first, second, second, first):
        b1.insert_particles([im for im, _ in part], [m for _, m in part])
    b2 = BatchReconstructor([p for p, _, _ in jobs])
    g = b2.capture(boxes, half, ctf)
    g.launch([torch.as_tensor(im, device="cuda") for im, _ in first], [m for _, m in first])
    g.launch([im for im, _ in second], [m for _, m in second])      # host images
    g.launch(None, [m for _, m in second])                           # the slots as filled
    mixed = [torch.as_tensor(im, device="cuda") if j % 2 else im for j, (im, _) in enumerate(first)]
    g.launch(mixed, [m for _, m in first])          # device images in place, host ones copied
    torch.cuda.synchronize()
    for j in range(len(jobs)):
        d1, n1 = b1.get_accumulators(j)
        d2, n2 = b2.get_accumulators(j)
        assert oracle.rel_l2(d2, d1) < RTOL and oracle.rel_l2(n2, n1) < RTOL
    g.close()


def _grouped_jobs():
    """Jobs that share (N, box) and so one prologue launch per stage: with
    and without a CTF, different inserters (so different schedules),
    different symmetries, beside a job of its own group."""
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    specs = [(32, 48, "gauss_2", "c1", 20, True), (32, 48, "gauss_2", "c1", 14, False),
             (32, 48, "gauss_5", "c1", 9, True), (32, 48, "nearest_neighbor", "c1", 17, False),
             (32, 48, "gauss_2", "d3", 8, True), (40, 60, "gauss_2", "d2", 11, True)]
    jobs = []
    for k, (box, N, mode, sym, n, ctf) in enumerate(specs):
        ps = make_particles(box, n, seed=700 + k, snr=0.5, shift=2.0, weights=(0.5, 1.0), ctf=ctf)
        meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
        jobs.append(({"size": [N] * 3, "sym": sym, "mode": mode}, ps, meta, ctf))
    return jobs


def test_grouped_prologue_equals_each_job_alone(gpu):
    """Jobs of equal (N, box) run one prologue over their concatenated
    particles (mixed CTF, schedules and symmetries): each job still gets
    its alone result, batched and through a graph reading device images in
    place."""
    import torch

    from eman2_b200.batch import BatchReconstructor
    jobs = _grouped_jobs()
    params = [p for p, _, _, _ in jobs]
    b = BatchReconstructor(params)
    b.insert_particles([ps.images for _, ps, _, _ in jobs], [m for _, _, m, _ in jobs])
    alone = [_alone(p, ps.images, m) for p, ps, m, _ in jobs]
    for j in range(len(jobs)):
        d, n = b.get_accumulators(j)
        assert oracle.rel_l2(d, alone[j][0]) < RTOL and oracle.rel_l2(n, alone[j][1]) < RTOL
    g_b = BatchReconstructor(params)
    g = g_b.capture([ps.images.shape[-1] for _, ps, _, _ in jobs],
                    [len(ps.images) for _, ps, _, _ in jobs], [c for _, _, _, c in jobs])
    dev = [torch.as_tensor(ps.images, device="cuda") for _, ps, _, _ in jobs]
    g.launch(dev, [m for _, _, m, _ in jobs])
    torch.cuda.synchronize()
    for j in range(len(jobs)):
        d, n = g_b.get_accumulators(j)
        assert oracle.rel_l2(d, alone[j][0]) < RTOL and oracle.rel_l2(n, alone[j][1]) < RTOL
    g.close()


def test_graph_of_one_particle_jobs_scatter(gpu):
    """One particle per job, every job pinned to the scatter schedule: the
    round's insertion is one multi-job scatter launch, and replays equal the
    jobs inserted alone."""
    import torch

    from eman2_b200.batch import BatchReconstructor, set_tile
    from eman2_b200.particles import particle_meta
    jobs = _grouped_jobs()
    nsym = {"c1": 1, "d2": 4, "d3": 6}
    keys = {(p["size"][0], p["mode"], nsym[p["sym"]]) for p, _, _, _ in jobs}
    try:
        for k in keys:
            set_tile(k[0], k[1], k[2], -2)
        b = BatchReconstructor([p for p, _, _, _ in jobs])
        g = b.capture([ps.images.shape[-1] for _, ps, _, _ in jobs], [1] * len(jobs),
                      [c for _, _, _, c in jobs])
        for i in range(3):
            imgs = [torch.as_tensor(ps.images[i:i + 1], device="cuda") for _, ps, _, _ in jobs]
            metas = [particle_meta(ps.rots[i:i + 1], ps.shifts[i:i + 1], ps.weights[i:i + 1],
                                   defocus=ps.defocus[i:i + 1]) for _, ps, _, _ in jobs]
            g.launch(imgs, metas)
        torch.cuda.synchronize()
        got = [b.get_accumulators(j) for j in range(len(jobs))]
        g.close()
    finally:
        for k in keys:
            set_tile(k[0], k[1], k[2], -1)
    for j, (params, ps, meta, _) in enumerate(jobs):
        d0, n0 = _alone(params, ps.images[:3], particle_meta(
            ps.rots[:3], ps.shifts[:3], ps.weights[:3], defocus=ps.defocus[:3]))
        assert oracle.rel_l2(got[j][0], d0) < RTOL and oracle.rel_l2(got[j][1], n0) < RTOL


def test_graph_rejects_ctf_mismatch(gpu):
    from eman2_b200.batch import BatchReconstructor
    from eman2_b200.exceptions import InvalidParameterException
    from eman2_b200.particles import particle_meta
    params, ps, meta = _jobs()[0]                 # particles with a CTF
    b = BatchReconstructor([params])
    g = b.capture([ps.images.shape[-1]], [8], [False])
    im, m = _split(ps, particle_meta, 0, 8)
    with pytest.raises(InvalidParameterException):
        g.launch([im], [m])
    g.close()


def test_served_result_equals_alone(gpu):
    """Requests arriving at different times, split into chunks, admitted by
    footprint and batched together: each result equals the job run alone."""
    from eman2_b200.server import GpuExecutor, Request, Scheduler, Server
    from eman2_b200.particles import particle_meta
    jobs = _jobs()
    reqs = []
    for k, (params, ps, meta) in enumerate(jobs):
        n = len(ps.images)
        cut = list(range(0, n, 12)) + [n]
        chunks = [(ps.images[a:b], particle_meta(ps.rots[a:b], ps.shifts[a:b], ps.weights[a:b],
                                                  defocus=ps.defocus[a:b]))
                  for a, b in zip(cut[:-1], cut[1:])]
        reqs.append(Request(k, params, chunks, arrival=0.02 * k))
    # a late request with job 0's parameters takes job 0's pooled reconstructor
    reqs.append(Request(4, jobs[0][0], reqs[0].chunks, arrival=1.0))
    sched = Scheduler(hbm_budget=8 << 30, max_active=3)
    exe = GpuExecutor(doift=False)
    res = Server(sched, exe).run(reqs)
    assert res["requests"] == 5 and res["p99_s"] >= res["p50_s"] > 0
    assert exe.reused >= 1
    exe.close()
    by_id = {j.req.rid: j for j in sched.done}
    for k, (params, ps, meta) in enumerate(jobs + [jobs[0]]):
        want = _alone(params, ps.images, meta)
        from eman2_b200 import FourierReconstructor
        r = FourierReconstructor(params)
        r.setup_seedandweights(*want)
        want_final = r.finish(False).numpy()
        got = by_id[k].result.numpy()
        assert oracle.rel_l2(got, want_final) < 1e-5


def test_large_finish_does_not_hold_small_request(gpu):
    """A retiring job's finish (normalise, 480^3 inverse FFT, a 442 MB map
    copied out) runs on a finish stream of its own: the scheduler issues the
    small request's next chunks while it is in flight, and on the device those
    chunks are inserted before it lands.  Both results equal the jobs alone."""
    import torch

    from eman2_b200 import FourierReconstructor
    from eman2_b200.particles import particle_meta
    from eman2_b200.server import GpuExecutor, Request, Scheduler, Server
    from eman2_b200.synth import make_particles

    class Timed(GpuExecutor):
        """Timing events around each tick and each finish."""
        def __init__(self, **kw):
            super().__init__(**kw)
            self.ticks, self.finishes = [], {}

        def insert(self, items):
            super().insert(items)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(self.stream)
            self.ticks.append(({id(h) for h, _ in items}, ev))

        def finish_async(self, handle):
            if not self.finish_streams:
                self.finish_streams = [torch.cuda.Stream() for _ in range(self.nfinish)]
            fs = self.finish_streams[self._next_fs % self.nfinish]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(fs)
            p = super().finish_async(handle)
            e1.record(fs)
            self.finishes[id(handle)] = (e0, e1)
            return p

    def chunks(ps, size):
        n = len(ps.images)
        cut = list(range(0, n, size)) + [n]
        return [(ps.images[a:b], particle_meta(ps.rots[a:b], ps.shifts[a:b], ps.weights[a:b]))
                for a, b in zip(cut[:-1], cut[1:])]

    big = make_particles(320, 16, seed=401, snr=0.5, device=gpu)
    small = make_particles(64, 48, seed=402, snr=0.5, device=gpu)
    pb = {"size": [480] * 3, "sym": "c1", "mode": "gauss_2"}
    psm = {"size": [96] * 3, "sym": "c1", "mode": "gauss_2"}
    reqs = [Request(0, pb, chunks(big, 16), 0.0), Request(1, psm, chunks(small, 12), 0.0)]
    exe = Timed(doift=True)
    # warm-up with the same requests: plans, scratch and the pooled volumes
    Server(Scheduler(hbm_budget=16 << 30, max_active=4), exe).run(reqs)
    torch.cuda.synchronize()
    exe.ticks.clear()
    exe.finishes.clear()
    sched = Scheduler(hbm_budget=16 << 30, max_active=4)
    srv = Server(sched, exe)
    srv.run(reqs)
    torch.cuda.synchronize()
    by = {j.req.rid: j for j in sched.done}
    assert set(by) == {0, 1}
    # host: small chunks issued after the big finish started, before it landed
    t0 = next(t for t, kind, ids in srv.trace if kind == "finish_start" and 0 in ids)
    t1 = next(t for t, kind, ids in srv.trace if kind == "done" and 0 in ids)
    late = [t for t, kind, ids in srv.trace if kind == "tick" and 1 in ids and t0 < t < t1]
    assert late
    # device: a small-job tick issued in that window ran while the big finish
    # was in flight
    hbig, hsmall = by[0].handle, by[1].handle
    e0, e1 = exe.finishes[id(hbig)]
    small_ticks = [ev for ids, ev in exe.ticks if id(hsmall) in ids]
    first_late = small_ticks[-len([t for t, kind, ids in srv.trace
                                   if kind == "tick" and 1 in ids and t > t0])]
    finish_ms = e0.elapsed_time(e1)
    tick_ms = e0.elapsed_time(first_late)
    print(f"\nbig finish {finish_ms:.2f} ms; the small job's first tick after it started done "
          f"{tick_ms:.2f} ms after it began")
    assert tick_ms < finish_ms
    exe.close()
    for rid, params, ps in ((0, pb, big), (1, psm, small)):
        r = FourierReconstructor(params)
        r.setup()
        r.insert_particles(ps.images, particle_meta(ps.rots, ps.shifts, ps.weights))
        want = r.finish(True).numpy()
        r.close()
        assert oracle.rel_l2(by[rid].result.numpy(), want) < 1e-5
