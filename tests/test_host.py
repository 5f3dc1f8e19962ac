"""Host-side logic without a GPU: the C ABI loads and exports every declared
entry point, parameter validation and exception mapping, Transform and
symmetry conventions against the oracle, particle metadata layout, the
serving scheduler (fake executor) and the bench's pixel counts."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from eman2_b200 import _lib
    from eman2_b200 import build as b
    b.build()
    return _lib.load()


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "eman2_b200.h")).read()
    return sorted(set(re.findall(r"FR_API\s+[\w\s\*]*?\b(fr_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    from eman2_b200 import _lib
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_abi_errors_without_touching_the_device(lib):
    from eman2_b200 import _lib
    h = ctypes.c_void_p()
    assert lib.fr_create(None, ctypes.byref(h)) == 3          # FR_ENULL
    p = _lib.fr_params()
    p.nx = p.ny = p.nz = 33
    p.mode = 2
    p.sym = b"c1"
    assert lib.fr_create(ctypes.byref(p), ctypes.byref(h)) == 7   # odd size unsupported
    assert b"odd" in lib.fr_last_error()
    p.nx, p.ny, p.nz = 32, 24, 32
    assert lib.fr_create(ctypes.byref(p), ctypes.byref(h)) == 7   # slices must be square
    p.nx, p.ny, p.nz = 32, 32, 17
    assert lib.fr_create(ctypes.byref(p), ctypes.byref(h)) == 7   # odd z size
    p.nx = p.ny = p.nz = 32
    p.mode = 3
    assert lib.fr_create(ctypes.byref(p), ctypes.byref(h)) == 7   # gauss_3 not built
    p.mode = 2
    p.sym = b"h3"                                                   # helical: not built
    assert lib.fr_create(ctypes.byref(p), ctypes.byref(h)) == 7
    p.sym = b"c2000000000"                                          # beyond the operator limit
    assert lib.fr_create(ctypes.byref(p), ctypes.byref(h)) == 7
    assert lib.fr_version().startswith(b"eman2_b200")


@pytest.mark.parametrize("sym", ["c1", "c4", "c7", "d1", "d2", "d7", "D3", "C2", "tet", "oct",
                                 "icos", "ICOS5", "c1000", "d500"])
def test_library_symmetry_matches_oracle(lib, sym):
    out = np.zeros(9 * 1000, np.float32)
    n = lib.fr_sym_ops(sym.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 1000)
    want = oracle.sym_ops(sym)
    assert n == len(want)
    assert np.array_equal(out[: 9 * n].reshape(n, 3, 3), want)


def test_platonic_groups_are_groups():
    """tet, oct and icos: 12, 24 and 60 distinct rotations closed under products."""
    for sym, count in (("tet", 12), ("oct", 24), ("icos", 60)):
        ops = oracle.sym_ops(sym).astype(np.float64)
        assert len(ops) == count
        np.testing.assert_allclose(np.linalg.det(ops), 1.0, atol=1e-6)
        for a in ops:
            prod = np.einsum("ij,njk->nik", a, ops)
            d = np.abs(prod[:, None] - ops[None]).max(axis=(2, 3)).min(axis=1)
            assert d.max() < 1e-5


def test_symmetry_order_limits(lib):
    out = np.zeros(9, np.float32)
    P = ctypes.POINTER(ctypes.c_float)
    for bad in (b"c1001", b"d501", b"c2000000000", b"c99999999999", b"c-3", b"c0", b"x2", b"h4"):
        assert lib.fr_sym_ops(bad, out.ctypes.data_as(P), 1) == -1, bad


def test_params_and_exceptions():
    from eman2_b200 import (InvalidParameterException, NotExistingObjectException,
                            Reconstructors, UnsupportedParameterException)
    assert Reconstructors.get_list() == ["fourier", "wiener_fourier", "fourier_iter"]
    with pytest.raises(NotExistingObjectException):
        Reconstructors.get("nn4")                 # SPARX reconstructors are not built
    with pytest.raises(InvalidParameterException):
        Reconstructors.get("fourier", {"size": [32] * 3, "bogus": 1})
    r = Reconstructors.get("fourier", {"size": [32] * 3, "sym": "d7"})
    # the reference's TypeDict keys (libEM/reconstructor.h:501-516)
    assert sorted(r.get_param_types()) == sorted(
        ["size", "sym", "mode", "corners", "sqrtnorm", "usessnr", "verbose", "quiet",
         "subvolume", "savenorm", "normout"])
    assert r.get_name() == "fourier" and "direct Fourier" in r.get_desc()
    r.insert_params({"mode": "gauss_5"})
    assert r.get_params()["sym"] == "d7" and r.get_params()["mode"] == "gauss_5"
    r.set_params({"size": [16] * 3})
    assert "sym" not in r.get_params()
    r.set_params({"size": [16] * 3, "mode": "gauss_3"})
    with pytest.raises(UnsupportedParameterException):
        r.setup()


def test_transform_conventions_match_oracle():
    from eman2_b200 import Transform
    rng = np.random.default_rng(1)
    for _ in range(20):
        az, alt, phi = rng.uniform(-360, 360, 3)
        t = Transform({"type": "eman", "az": az, "alt": alt, "phi": phi})
        assert np.array_equal(t.rotation_block(), oracle.eman_matrix(az, alt, phi))
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        tq = Transform({"type": "quaternion", "e0": q[0], "e1": q[1], "e2": q[2], "e3": q[3]})
        assert np.array_equal(tq.rotation_block(), oracle.quaternion_matrix(q))
        # product in float, the reference's order
        assert np.array_equal((t * tq).rotation_block(),
                              oracle.compose(t.rotation_block(), tq.rotation_block()))
    tr = Transform({"type": "eman", "az": 10, "alt": 20, "phi": 30, "tx": 1.5, "ty": -2.25})
    inv = tr.inverse()
    assert np.allclose((tr * inv).matrix, np.eye(3, 4), atol=1e-6)
    e = Transform({"type": "eman", "az": 10, "alt": 20, "phi": 30}).get_rotation("eman")
    assert np.allclose([e["az"], e["alt"], e["phi"]], [10, 20, 30], atol=1e-4)


def test_synth_quaternion_blocks_match_oracle():
    from eman2_b200.synth import quaternion_blocks, random_quaternions
    q = random_quaternions(10, np.random.default_rng(4))
    m = quaternion_blocks(q)
    for i in range(10):
        assert np.array_equal(m[i], oracle.quaternion_matrix(q[i]))


def test_particle_meta_layout():
    from eman2_b200 import _lib
    from eman2_b200.particles import particle_meta
    assert ctypes.sizeof(_lib.fr_particle) == 19 * 4
    m = particle_meta(np.eye(3, dtype=np.float32)[None].repeat(2, 0), [[1, 2], [3, 4]],
                      [0.5, 1.0], defocus=[1.5, 0.0])
    assert m[1].tx == 3 and m[0].weight == 0.5 and m[0].defocus == 1.5 and m[1].voltage == 300


def test_bench_pixel_counts():
    import bench
    assert [bench.pixels_per_slice(N) for N in (96, 192)] == [3738, 14711]
    assert bench.nsym_of("d7") == 14 and bench.nsym_of("c4") == 4


class FakeExecutor:
    def __init__(self):
        self.created, self.inserted, self.finished = 0, [], 0

    def create(self, params):
        self.created += 1
        return {"params": params, "chunks": 0}

    def insert(self, items):
        self.inserted.append(len(items))
        for h, _ in items:
            h["chunks"] += 1

    def finish(self, h):
        self.finished += 1
        return h["chunks"]


def _req(rid, N, nchunks, arrival=0.0, chunk=8, box=None):
    from eman2_b200.server import Request
    box = box or N * 2 // 3
    return Request(rid, {"size": [N] * 3, "sym": "c1", "mode": "gauss_2"},
                   [(np.zeros((chunk, box, box), np.float32), None)] * nchunks, arrival)


def test_scheduler_admits_by_footprint_and_batches_continuously():
    from eman2_b200.server import Scheduler, Server, footprint_bytes
    one = footprint_bytes({"size": [96] * 3}, 64, 8)
    sched = Scheduler(hbm_budget=int(2.5 * one), max_active=8)
    exe = FakeExecutor()
    reqs = [_req(i, 96, 3 + i % 2) for i in range(5)] + [_req(9, 400, 1)]   # last never fits
    res = Server(sched, exe).run(reqs)
    assert res["requests"] == 5 and res["rejected"] == 1
    # never more than two 96^3 jobs resident: batches of at most 2 chunks
    assert max(exe.inserted) == 2
    # every job got all its chunks, each exactly once
    assert sorted(j.result for j in sched.done) == sorted(len(r.chunks) for r in reqs[:5])
    assert sched.used == 0 and res["p99_s"] >= res["p50_s"] >= 0


def test_scheduler_joins_late_arrivals_at_next_tick():
    from eman2_b200.server import Scheduler
    sched = Scheduler(hbm_budget=1 << 40, max_active=4)
    exe = FakeExecutor()
    sched.submit(_req(0, 64, 4, arrival=0.0))
    sched.submit(_req(1, 64, 2, arrival=0.5))
    sched.admit(0.0, exe)
    assert len(sched.tick_work()) == 1
    sched.admit(0.6, exe)                  # arrived while job 0 was on the GPU
    assert len(sched.tick_work()) == 2     # both in the same tick now


class FakeAsyncExecutor(FakeExecutor):
    """Finishes land only after `delay` polls, as a finish enqueued on its own
    stream lands some ticks later."""

    def __init__(self, delay=3):
        super().__init__()
        self.delay = delay

    def finish_async(self, h):
        return {"h": h, "polls": 0}

    def finish_ready(self, p):
        p["polls"] += 1
        return p["polls"] > self.delay

    def finish_result(self, p):
        self.finished += 1
        return p["h"]["chunks"]


def test_scheduler_keeps_ticking_while_a_finish_is_in_flight():
    """A retiring job's asynchronous finish does not hold the tick loop: the
    other job's chunks are inserted while it is in flight, and its memory is
    released only once it has landed."""
    from eman2_b200.server import Scheduler, Server, footprint_bytes
    big, small = _req(0, 192, 1), _req(1, 96, 4)
    sched = Scheduler(hbm_budget=1 << 40, max_active=4)
    exe = FakeAsyncExecutor(delay=5)
    srv = Server(sched, exe)
    res = srv.run([big, small])
    assert res["requests"] == 2 and sched.used == 0
    t_big_start = next(t for t, kind, ids in srv.trace if kind == "finish_start" and 0 in ids)
    t_big_done = next(t for t, kind, ids in srv.trace if kind == "done" and 0 in ids)
    small_ticks = [t for t, kind, ids in srv.trace if kind == "tick" and 1 in ids]
    assert any(t_big_start < t < t_big_done for t in small_ticks)
    assert sorted(j.result for j in sched.done) == [1, 4]
    # while in flight the big job still holds its memory
    sched2 = Scheduler(hbm_budget=1 << 40, max_active=4)
    sched2.submit(_req(0, 192, 1))
    sched2.admit(0.0, exe)
    sched2.tick_work()
    sched2.retire(0.0, exe)
    assert not sched2.active and len(sched2.finishing) == 1
    assert sched2.used == footprint_bytes({"size": [192] * 3}, 128, 8)
    sched2.collect(0.1, exe, wait=True)
    assert sched2.used == 0 and sched2.idle()


def test_batched_call_argument_marshalling():
    """The batched calls hand the library contiguous float32 particles and the
    addresses of fr_particle arrays: float32 contiguous tensors pass through
    untouched, other arrays are converted, None stays None."""
    import torch

    from eman2_b200.batch import _meta_address, _particles
    from eman2_b200.particles import particle_meta
    t32 = torch.zeros(2, 4, 4)
    a64 = np.arange(32, dtype=np.float64).reshape(2, 4, 4)
    strided = torch.zeros(2, 4, 8)[:, :, ::2]
    keep, ptrs = _particles([t32, a64, None, strided])
    assert keep[0] is t32 and ptrs[0] == t32.data_ptr()
    assert keep[1].dtype == np.float32 and keep[1].flags["C_CONTIGUOUS"]
    assert np.array_equal(keep[1], a64.astype(np.float32)) and ptrs[1] == keep[1].ctypes.data
    assert keep[2] is None and ptrs[2] is None
    assert keep[3].is_contiguous() and ptrs[3] == keep[3].data_ptr()
    meta = particle_meta(np.eye(3, dtype=np.float32)[None], np.zeros((1, 2), np.float32),
                         np.ones(1, np.float32))
    assert _meta_address(meta) == ctypes.cast(meta, ctypes.c_void_p).value
    assert _meta_address(None) is None


def test_bench_workload_draws_follow_the_configurations():
    """The batched and served legs' seeded draws have the configurations'
    shapes: 64 jobs as 32 even/odd pairs over boxes 64-160 x1.5 with
    500-50,000 particles each; requests over boxes 64-320 x1.5 with
    1,000-100,000 particles in chunks of 2048 and Poisson arrivals."""
    import ctypes

    import bench
    from eman2_b200 import _lib
    jobs = bench.config3_jobs(33)
    assert len(jobs) == 64
    for a, b in zip(jobs[0::2], jobs[1::2]):
        assert a["params"] == b["params"] and a["box"] == b["box"]
        assert abs(a["count"] - b["count"]) <= 1
    for j in jobs:
        assert j["box"] in bench.BATCH_BOXES
        assert j["params"]["size"] == [j["box"] * 3 // 2] * 3
        assert j["params"]["sym"] in ("c1", "d7") and j["params"]["mode"] in ("gauss_2", "gauss_5")
        assert 500 <= j["count"] <= 50_000
    meta = (_lib.fr_particle * 2048)()
    pools = {b: (np.zeros((2048, 1, 1), np.float32), meta) for b in bench.SERVE_BOXES}
    reqs = bench.serving_requests(pools, 4242, 200, 4.0, 2048)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and 0.15 < np.mean(np.diff(arr)) < 0.35
    for r in reqs:
        assert 1000 <= r.particles <= 100_000
        assert r.params["size"][0] in [b * 3 // 2 for b in bench.SERVE_BOXES]
        assert r.params["sym"] in ("c1", "c4", "d7") and r.params["mode"] == "gauss_2"
        assert sum(c[0].shape[0] for c in r.chunks) == r.particles
        assert all(c[0].shape[0] <= 2048 for c in r.chunks)
    assert ctypes.sizeof(meta) > 0


def test_bench_fifo_latency():
    """A single FIFO server: waits when busy, starts at arrival when idle."""
    import bench
    assert bench.fifo_latency([0.0, 1.0, 10.0], [2.0, 2.0, 1.0]) == [2.0, 3.0, 1.0]
    assert bench.percentile([], 50) is None
    assert bench.percentile([1.0, 2.0, 3.0], 50) == 2.0
