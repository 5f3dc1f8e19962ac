"""Pins the oracle's insert_pixel / add_complex_at restatement against the
reference's own inserter source (libEM/reconstructor_tools.cpp with
libEM/emdata_core.h), compiled from the reference tree into oracle/_ref by
oracle/build_ref.sh.  Bitwise: both are built with strict IEEE flags."""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.skipif(not os.path.exists(oracle.REF_SO),
                                reason="reference tree not present, oracle/_ref not built")

_F = ctypes.POINTER(ctypes.c_float)


def _ref():
    lib = ctypes.CDLL(oracle.REF_SO)
    lib.ref_insert_pixels.argtypes = [ctypes.c_char_p, _F, _F, ctypes.c_int, _F, ctypes.c_long]
    lib.ref_add_complex_at_fast.argtypes = [_F, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_float, ctypes.c_float]
    lib.ref_add_complex_at_fast.restype = ctypes.c_long
    return lib


def _pixels(N, n, rng, spread=1.0):
    """Random insert_pixel calls covering the whole cube, its faces and beyond."""
    h = N / 2
    xyz = rng.uniform(-(h + 4) * spread, (h + 4) * spread, (n, 3))
    # plus points snapped near integers and half-integers, where windows flip
    k = n // 4
    xyz[:k] = np.round(xyz[:k] * 2) / 2 + rng.choice([-1e-6, 0, 1e-6], (k, 3))
    # plus points on the x=0 and x=N/2 planes and the axes
    xyz[k:2 * k, 0] = rng.choice([0.0, h, -h, 0.49, -0.51], k)
    px = np.empty((n, 6), np.float32)
    px[:, :3] = xyz
    px[:, 3:5] = rng.normal(size=(n, 2))
    px[:, 5] = rng.uniform(0.2, 1.5, n)
    return px


@pytest.mark.parametrize("mode", ["nearest_neighbor", "gauss_2", "gauss_5", "trilinear"])
@pytest.mark.parametrize("N", [8, 16, 22])
def test_insert_pixel_matches_reference_bitwise(mode, N):
    rng = np.random.default_rng(100 + N)
    px = _pixels(N, 4000, rng)
    lib = _ref()
    d_ref = np.zeros((N, N, N + 2), np.float32)
    n_ref = np.zeros((N, N, N // 2 + 1), np.float32)
    lib.ref_insert_pixels(mode.encode(), d_ref.ctypes.data_as(_F), n_ref.ctypes.data_as(_F), N,
                          px.ctypes.data_as(_F), px.shape[0])
    v = oracle.OracleVolume(N, "fp32")
    v.insert_pixels(mode, px)
    assert np.array_equal(v.data, d_ref), np.abs(v.data - d_ref).max()
    assert np.array_equal(v.norm, n_ref), np.abs(v.norm - n_ref).max()
    assert np.abs(d_ref).sum() > 0


def test_add_complex_at_fast_indices_and_hermitian_rules():
    """The reference's add_complex_at_fast on its own: the reported index and
    the duplicated conjugate adds on the x=0 and x=+-N/2 planes."""
    lib = _ref()
    N = 8
    h = N // 2
    nxyz = (N + 2) * N * N
    for x in range(-h - 1, h + 2):
        for y in range(-h - 1, h + 2):
            for z in (-h, -1, 0, 1, h):
                d = np.zeros((N, N, N + 2), np.float32)
                idx = lib.ref_add_complex_at_fast(d.ctypes.data_as(_F), N, x, y, z, 1.0, 2.0)
                v = oracle.OracleVolume(N, "fp32")
                px = np.array([[0, 0, 0, 0, 0, 0]], np.float32)
                del px
                if abs(x) > h or abs(y) > h or abs(z) > h:
                    assert idx == nxyz
                    assert not d.any()
                    continue
                flat = d.reshape(-1)
                # the value lands where the index says (plus conjugates)
                if (x, y, z) == (0, 0, 0):
                    assert idx == 0 and flat[0] == 1.0 and flat[1] == 0.0
                elif abs(x) == h and y == 0 and z == 0:
                    assert idx == N and flat[N] == 1.0 and flat[N + 1] == 0.0
                else:
                    assert flat[idx] >= 1.0
                del v


@pytest.mark.parametrize("mode,sym", [("gauss_5", "d2"), ("gauss_2", "c3"), ("nearest_neighbor", "c1")])
def test_reference_arm_matches_restatement(mode, sym):
    """The timed CPU reference arm: the restatement's pixel stream of
    do_insert_slice_work (or_slice_pixels) through the reference's own
    inserter.  With the strict build and one thread it is bitwise the
    restatement's insert_slice; with the release build on several threads it
    stays within FP32 order noise of it."""
    N, n = 24, 6
    rng = np.random.default_rng(7)
    sl = rng.normal(size=(n, N, N + 2)).astype(np.float32)
    rots = np.stack([oracle.quaternion_matrix(q / np.linalg.norm(q))
                     for q in rng.normal(size=(n, 4))]).astype(np.float32)
    w = rng.uniform(0.5, 1.0, n).astype(np.float32)
    want = oracle.OracleVolume(N, "fp32")
    ops = oracle.sym_ops(sym).reshape(-1, 3, 3)
    want.insert(sl, rots, w, mode=mode, sym=sym)
    d, m = oracle.ref_insert_threaded(N, sl, rots, w, mode, sym, 1, lib_path=oracle.REF_SO)
    assert np.array_equal(d, want.data) and np.array_equal(m, want.norm)
    if oracle.ref_available():
        d, m = oracle.ref_insert_threaded(N, sl, rots, w, mode, sym, 3)
        assert oracle.rel_l2(d, want.data) < 1e-5 and oracle.rel_l2(m, want.norm) < 1e-5
    assert ops.shape[0] >= 1
