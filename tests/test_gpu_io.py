"""Particle stacks from disk on the GPU: the device decode of every MRC mode
equals the host decode, streamed chunks equal the stack, and a streamed
insertion equals the insertion of the same particles from memory."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from eman2_b200 import io
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 17, 1, 6, 12, 2, 101])
@pytest.mark.parametrize("swap", [False, True])
def test_device_decode_equals_host(gpu, mode, swap):
    import torch
    from eman2_b200 import _lib
    rng = np.random.default_rng(mode + 10 * swap)
    nbytes = 4096 if mode != 101 else 2048
    raw = rng.integers(0, 256, nbytes, dtype=np.uint8)
    if mode == 12:      # keep float16 values finite
        raw.view(np.uint16)[:] &= 0x7BFF
    if mode == 2:
        raw.view(np.uint32)[:] = np.frombuffer(rng.normal(size=1024).astype(np.float32).tobytes(),
                                               np.uint32).byteswap() if swap else \
            np.frombuffer(rng.normal(size=1024).astype(np.float32).tobytes(), np.uint32)
    info = type("I", (), {"mode": mode, "swap": swap})()
    want = io._decode_host(raw, info)
    d_raw = torch.as_tensor(raw, device="cuda")
    out = torch.empty(want.size, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().fr_decode_images(ctypes.c_void_p(d_raw.data_ptr()), mode, int(swap),
                                            want.size, ctypes.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), want)


@pytest.mark.parametrize("mode,chunk", [(2, 7), (12, 16), (1, 50)])
def test_stack_stream_chunks(gpu, tmp_path, mode, chunk):
    import torch
    rng = np.random.default_rng(chunk)
    a = (rng.normal(size=(45, 24, 24)) * 100).astype(np.float32)
    p = str(tmp_path / "s.mrcs")
    io.write_mrc(p, a, mode=mode)
    want = io.read_mrc_stack(p)
    seen = 0
    for first, d in io.StackStream(p, chunk):
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d.cpu().numpy(), want[first:first + d.shape[0]])
        seen += d.shape[0]
    assert seen == 45


def test_streamed_insertion_equals_memory(gpu, tmp_path):
    from eman2_b200 import FourierReconstructor
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    ps = make_particles(32, 100, seed=21, snr=0.5, shift=2.0, weights=(0.5, 1.0), ctf=True)
    meta = particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus)
    p = str(tmp_path / "ptcl.mrcs")
    io.write_mrc(p, ps.images)
    params = {"size": [48] * 3, "sym": "d2", "mode": "gauss_2"}
    a = FourierReconstructor(params)
    a.setup()
    a.insert_particles(np.ascontiguousarray(ps.images, np.float32), meta)
    b = FourierReconstructor(params)
    b.setup()
    assert io.insert_stack(b, p, meta, chunk=32) == 100
    (da, na), (db, nb) = a.get_accumulators(), b.get_accumulators()
    assert oracle.rel_l2(db, da) < 2e-6 and oracle.rel_l2(nb, na) < 2e-6


def test_reconstruct_from_lst(gpu, tmp_path):
    """An #LSX list over two stacks, in shuffled order: the streamed
    reconstruction equals inserting the same particles, in list order, from
    memory."""
    import os

    from eman2_b200 import FourierReconstructor, Transform
    from eman2_b200.synth import make_particles
    ps = make_particles(32, 40, seed=31, snr=0.5, shift=2.0, weights=None, ctf=False)
    a, b = str(tmp_path / "a.mrcs"), str(tmp_path / "b.mrcs")
    io.write_mrc(a, ps.images[:25])
    io.write_mrc(b, ps.images[25:])
    order = [3, 4, 5, 6, 30, 31, 32, 10, 0, 1, 2, 39, 38, 20, 21]
    lst = io.LSXFile(str(tmp_path / "set.lst"))
    for i in order:
        m34 = np.zeros((3, 4), np.float32)
        m34[:, :3] = ps.rots[i]
        m34[:2, 3] = ps.shifts[i]
        f, n = (a, i) if i < 25 else (b, i - 25)
        lst.write(-1, n, f, {"xform.projection": Transform(m34), "score": -1.0 - 0.01 * i})
    lst.close()
    params = {"size": [48] * 3, "sym": "c2", "mode": "gauss_2"}
    r = FourierReconstructor(params)
    r.setup()
    assert io.reconstruct_lst(r, str(tmp_path / "set.lst"), chunk=4) == len(order)
    # the same records (matrices as the list stores them, 6 significant
    # digits), the images from memory
    m = io.records_to_meta(io.load_lst_params(str(tmp_path / "set.lst")))
    r0 = FourierReconstructor(params)
    r0.setup()
    r0.insert_particles(np.ascontiguousarray(ps.images[order], np.float32), m)
    (d, nr), (d0, n0) = r.get_accumulators(), r0.get_accumulators()
    assert oracle.rel_l2(d, d0) < 2e-6 and oracle.rel_l2(nr, n0) < 2e-6
    assert os.path.exists(a)
