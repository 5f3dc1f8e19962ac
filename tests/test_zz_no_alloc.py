"""The allocation-free insertion entry point (fr_insert_slices_noalloc).

It exists for callers that cannot let a library call cudaMalloc -- a process
that has reserved all of its HBM for its own pool allocator, or a path that
cannot afford an allocation's stall or implicit device synchronisation.  This
test calls it through the C ABI with device buffers the test owns, twice in a
row, and checks each result against the regular entry point (fr_insert_slices)
fed the same slices.  The file is named to be collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_ACC = 2e-6   # FP32 summation order only (both paths add with atomics)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("mode,sym", [("gauss_2", "c1"), ("gauss_5", "d2"),
                                      ("nearest_neighbor", "c3"), ("trilinear", "c1"),
                                      ("gauss_2", "tet")])
def test_noalloc_matches_regular_insert_twice(gpu, mode, sym):
    import torch

    from eman2_b200 import Reconstructors, _lib
    from eman2_b200.synth import quaternion_blocks, random_quaternions
    lib = _lib.load()
    N, n = 32, 20
    rng = np.random.default_rng(2024)
    batches = []
    for _ in range(2):
        sl = rng.normal(size=(n, N, N + 2)).astype(np.float32)
        rt = quaternion_blocks(random_quaternions(n, rng))
        w = rng.uniform(0.5, 1.0, n).astype(np.float32)
        batches.append((sl, rt, w))

    dev = torch.device("cuda:0")
    data = torch.zeros((N, N, N + 2), dtype=torch.float32, device=dev)
    norm = torch.zeros((N, N, N // 2 + 1), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    ref = Reconstructors.get("fourier", {"size": [N] * 3, "sym": sym, "mode": mode})
    ref.setup()
    for sl, rt, w in batches:
        d_sl = torch.as_tensor(sl, device=dev)
        d_rt = torch.as_tensor(rt, device=dev)
        d_w = torch.as_tensor(w, device=dev)
        rc = lib.fr_insert_slices_noalloc(
            ctypes.c_void_p(d_sl.data_ptr()), n, N, _lib.MODE_IDS[mode], sym.encode(),
            ctypes.c_void_p(d_rt.data_ptr()), ctypes.c_void_p(d_w.data_ptr()),
            ctypes.c_void_p(data.data_ptr()), ctypes.c_void_p(norm.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.fr_last_error().decode()
        torch.cuda.synchronize()
        ref.insert_slices(sl, rt, w, schedule="scatter")
        want_d, want_n = ref.get_accumulators()
        got_d, got_n = data.cpu().numpy(), norm.cpu().numpy()
        assert _rel(got_d, want_d) < RTOL_ACC
        assert _rel(got_n, want_n) < RTOL_ACC
        assert np.array_equal(got_n != 0, want_n != 0)


def test_noalloc_rejects_oversized_requests(gpu):
    import torch

    from eman2_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda:0")
    buf = torch.zeros(16, device=dev)
    p = ctypes.c_void_p(buf.data_ptr())
    # size above the static scratch's limit
    assert lib.fr_insert_slices_noalloc(p, 1, 2048, 2, b"c1", p, p, p, p, None) == 1
    assert b"1024" in lib.fr_last_error()
    # too many slices x symmetry copies for one call
    assert lib.fr_insert_slices_noalloc(p, 2000, 32, 2, b"d7", p, p, p, p, None) == 1
    assert b"16384" in lib.fr_last_error()
    # a symmetry order beyond the operator limit is refused before any operator is built
    assert lib.fr_insert_slices_noalloc(p, 1, 32, 2, b"c2000000000", p, p, p, p, None) != 0
    assert lib.fr_insert_slices_noalloc(p, 1, 32, 2, b"c99999999999", p, p, p, p, None) != 0
    # a host buffer is refused (the kernels would read it from the device)
    host = (ctypes.c_float * 16)()
    hp = ctypes.cast(host, ctypes.c_void_p)
    assert lib.fr_insert_slices_noalloc(hp, 1, 32, 2, b"c1", p, p, p, p, None) == 1
    assert b"current device" in lib.fr_last_error()
