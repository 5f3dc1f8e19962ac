"""Served form: a request loop that admits reconstruction jobs by HBM
footprint, keeps their accumulating volumes resident on the device across
insertion ticks, and batches the chunks of every active job into one
persistent insertion launch per tick (continuous batching: a request that
arrives while others are on the GPU joins at the next tick once a slot and
its memory are free).

A job whose chunks are all inserted leaves the active set at once: with an
executor that finishes asynchronously (``finish_async``), its normalise,
inverse FFT and copy-out run on a stream of their own while the tick loop
keeps inserting the other jobs, and the job completes (its memory is
released) when that work has landed.

The scheduler is plain Python (testable without a GPU through any executor
with the same methods); ``GpuExecutor`` runs it on the device.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    """A reconstruction request: parameters plus particle chunks."""
    rid: int
    params: dict                   # {"size": [N]*3, "sym": ..., "mode": ...}
    chunks: list                   # [(images (n, box, box), meta fr_particle array), ...]
    arrival: float = 0.0           # seconds, on the server clock
    particles: int = 0

    def __post_init__(self):
        if not self.particles:
            self.particles = sum(int(np.shape(c[0])[0]) for c in self.chunks)


@dataclass
class Job:
    req: Request
    handle: object = None
    next_chunk: int = 0
    admitted: float = 0.0
    done: float = 0.0
    footprint: int = 0
    result: object = None
    pending: object = None         # an asynchronous finish in flight

    @property
    def finished_inserting(self) -> bool:
        return self.next_chunk >= len(self.req.chunks)


def footprint_bytes(params: dict, box: int, chunk: int) -> int:
    """Device bytes a job holds: the (complex, weight) accumulators
    (12*(N/2+1)*N^2 bytes, as libEM/reconstructor.cpp:782,800 allocate) plus
    the per-chunk prologue and slice scratch (~5 N^2 floats per particle and
    the raw images)."""
    N = int(params["size"][0]) if not np.isscalar(params["size"]) else int(params["size"])
    vol = 4 * (N * N * (N + 2) + N * N * (N // 2 + 1))
    return vol + chunk * (20 * N * N + 4 * box * box)


class Scheduler:
    """FIFO admission by HBM footprint and slot count; one chunk per active job
    per tick."""

    def __init__(self, hbm_budget: int, max_active: int = 16, chunks_per_tick: int = 1):
        self.budget = int(hbm_budget)
        self.max_active = max_active
        self.chunks_per_tick = chunks_per_tick
        self.waiting: list[Request] = []
        self.active: list[Job] = []
        self.finishing: list[Job] = []    # finish enqueued, memory still held
        self.done: list[Job] = []
        self.used = 0
        self.rejected: list[Request] = []

    def submit(self, req: Request):
        self.waiting.append(req)

    def _need(self, req: Request) -> int:
        box = int(np.shape(req.chunks[0][0])[-1]) if req.chunks else 0
        chunk = max((int(np.shape(c[0])[0]) for c in req.chunks), default=0)
        return footprint_bytes(req.params, box, chunk)

    def admit(self, now: float, executor) -> list[Job]:
        out = []
        while self.waiting and self.waiting[0].arrival <= now and len(self.active) < self.max_active:
            req = self.waiting[0]
            need = self._need(req)
            if need > self.budget:          # can never fit: refuse instead of blocking the queue
                self.rejected.append(self.waiting.pop(0))
                continue
            if self.used + need > self.budget:
                break                       # wait for memory to free up
            self.waiting.pop(0)
            job = Job(req, footprint=need, admitted=now)
            job.handle = executor.create(req.params)
            self.used += need
            self.active.append(job)
            out.append(job)
        return out

    def tick_work(self) -> list[tuple[Job, object]]:
        """The chunks of this tick: up to chunks_per_tick from every active job."""
        work = []
        for job in self.active:
            for _ in range(self.chunks_per_tick):
                if job.finished_inserting:
                    break
                work.append((job, job.req.chunks[job.next_chunk]))
                job.next_chunk += 1
        return work

    def retire(self, now: float, executor) -> list[Job]:
        """Jobs with every chunk inserted leave the active set (freeing their
        slot).  An asynchronous executor's finish is only started here; the
        job completes in collect().  Returns the jobs completed now."""
        out = []
        for job in list(self.active):
            if job.finished_inserting:
                self.active.remove(job)
                if hasattr(executor, "finish_async"):
                    job.pending = executor.finish_async(job.handle)
                    self.finishing.append(job)
                else:
                    job.result = executor.finish(job.handle)
                    self._complete(job, now)
                    out.append(job)
        return out + self.collect(now, executor)

    def collect(self, now: float, executor, wait: bool = False) -> list[Job]:
        """Completes the jobs whose asynchronous finish has landed (all of
        them, waiting, when ``wait``)."""
        out = []
        for job in list(self.finishing):
            if wait or executor.finish_ready(job.pending):
                job.result = executor.finish_result(job.pending)
                job.pending = None
                self.finishing.remove(job)
                self._complete(job, now)
                out.append(job)
        return out

    def _complete(self, job: Job, now: float):
        job.done = now
        self.used -= job.footprint
        self.done.append(job)

    def idle(self) -> bool:
        return not self.waiting and not self.active and not self.finishing


def percentile(v, q):
    if not v:
        return None
    return float(np.percentile(np.asarray(v, np.float64), q))


class Server:
    """Runs a scheduler against an executor on a wall clock.  Requests with
    arrival times in the future are held until their time comes."""

    def __init__(self, scheduler: Scheduler, executor, clock=time.perf_counter):
        self.sched = scheduler
        self.exe = executor
        self.clock = clock
        self.trace: list[tuple] = []    # (time, "tick" | "finish_start" | "done", job ids)

    def run(self, requests: list[Request], timeout: float = 3600.0) -> dict:
        for r in sorted(requests, key=lambda r: r.arrival):
            self.sched.submit(r)
        t0 = self.clock()
        ticks = 0
        while not self.sched.idle():
            now = self.clock() - t0
            if now > timeout:
                raise TimeoutError("server did not drain its queue")
            self.sched.admit(now, self.exe)
            work = self.sched.tick_work()
            if work:
                self.exe.insert([(job.handle, chunk) for job, chunk in work])
                ticks += 1
                self.trace.append((self.clock() - t0, "tick", [job.req.rid for job, _ in work]))
            before = {id(j) for j in self.sched.finishing}
            done = self.sched.retire(self.clock() - t0, self.exe)
            started = [j.req.rid for j in self.sched.finishing if id(j) not in before]
            if started:
                self.trace.append((self.clock() - t0, "finish_start", started))
            if done:
                self.trace.append((self.clock() - t0, "done", [j.req.rid for j in done]))
            if not work and not self.sched.active:
                if self.sched.finishing:
                    time.sleep(0.0002)          # poll the finishes in flight
                elif self.sched.waiting:
                    nxt = self.sched.waiting[0].arrival
                    wait = nxt - (self.clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
        wall = self.clock() - t0
        lat = [j.done - j.req.arrival for j in self.sched.done]
        parts = sum(j.req.particles for j in self.sched.done)
        return {"requests": len(self.sched.done), "rejected": len(self.sched.rejected),
                "ticks": ticks, "wall_s": wall, "p50_s": percentile(lat, 50),
                "p99_s": percentile(lat, 99), "particles": parts,
                "particles_per_s": parts / wall if wall > 0 else math.nan}


class GpuExecutor:
    """Device execution for the scheduler: a resident FourierReconstructor per
    job; each tick's chunks go through one fr_insert_particles_multi call on
    the insertion stream; a retiring job's finish is enqueued
    (fr_finish_async) on one of a few finish streams, into page-locked host
    buffers, so it overlaps the next ticks.

    Finished jobs' reconstructors return to a pool keyed by their parameters;
    a later job with the same parameters takes one (setup() zeroes its
    accumulators) and so reuses its volumes, FFT plans and scratch instead of
    allocating them.  At most ``pool_bytes`` of idle volumes are kept."""

    def __init__(self, doift: bool = False, stream=None, pool_bytes: int = 8 << 30,
                 finish_streams: int = 4):
        self.doift = doift
        self.stream = stream
        self.nfinish = max(1, int(finish_streams))
        self.finish_streams: list = []
        self._next_fs = 0
        self.pool_bytes = int(pool_bytes)
        self.pool: dict = {}            # key -> [FourierReconstructor]
        self.pooled = 0
        self.reused = 0

    @staticmethod
    def _key(params: dict):
        return tuple(sorted((k, tuple(v) if isinstance(v, (list, tuple)) else v)
                            for k, v in params.items()))

    def create(self, params: dict):
        from .reconstructor import FourierReconstructor
        key = self._key(params)
        free = self.pool.get(key)
        if free:
            r = free.pop()
            self.pooled -= r._pool_bytes
            self.reused += 1
        else:
            r = FourierReconstructor(params)
            r._pool_key, r._pool_bytes = key, footprint_bytes(params, 0, 0)
        r.setup()
        return r

    def insert(self, items):
        from .batch import insert_particles_multi
        if self.stream is None:
            # one stream for every tick: the ticks' launches queue back to back
            import torch
            self.stream = torch.cuda.Stream()
        recons = [h for h, _ in items]
        # a handle may appear once per call: group repeated jobs into rounds
        while items:
            seen, now, later = set(), [], []
            for h, c in items:
                (later if id(h) in seen else now).append((h, c))
                seen.add(id(h))
            insert_particles_multi([h for h, _ in now], [c[0] for _, c in now],
                                   [c[1] for _, c in now], self.stream)
            items = later
        del recons

    def finish_async(self, handle):
        """Enqueues the job's finish on the next finish stream."""
        import torch
        if not self.finish_streams:
            self.finish_streams = [torch.cuda.Stream() for _ in range(self.nfinish)]
        fs = self.finish_streams[self._next_fs % self.nfinish]
        self._next_fs += 1
        return handle.finish_async(self.doift, stream=fs)

    def finish_ready(self, pending) -> bool:
        return pending.ready()

    def finish_result(self, pending):
        out = pending.result()
        self._release(pending.owner)
        return out

    def finish(self, handle):
        out = handle.finish(self.doift)
        self._release(handle)
        return out

    def _release(self, handle):
        vol = handle._pool_bytes
        if self.pooled + vol <= self.pool_bytes:
            self.pool.setdefault(handle._pool_key, []).append(handle)
            self.pooled += vol
        else:
            handle.close()

    def close(self):
        for free in self.pool.values():
            for r in free:
                r.close()
        self.pool.clear()
        self.pooled = 0
