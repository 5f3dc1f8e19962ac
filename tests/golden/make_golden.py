"""Generates tests/golden/insert_*.npz: small insertions computed with the
reference's own pixel inserters and add_complex_at_fast
(libEM/reconstructor_tools.cpp, libEM/emdata_core.h, compiled from the
reference tree by oracle/build_ref.sh into oracle/_ref/libfr_ref.so).  The
per-slice loop of do_insert_slice_work (libEM/reconstructor.cpp:1164-1207)
that feeds them pixels is restated here in float32 numpy arithmetic.

Run from the repository root (needs the reference tree, i.e. this container):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

F32 = np.float32
_F = ctypes.POINTER(ctypes.c_float)
CASES = [("nearest_neighbor", 12, "c1"), ("gauss_2", 12, "d1"), ("gauss_5", 14, "c2"),
         ("trilinear", 12, "c1"), ("gauss_2", 18, "c3")]


def slice_pixels(sl, t3d, N, weight):
    """(xx, yy, zz, re, im, w) for every kept pixel of one slice and one
    symmetry operator, in the loop order of do_insert_slice_work."""
    inx, iny = F32(N + 2), F32(N)
    out = []
    M = t3d.astype(np.float32)
    for y in range(-N // 2, N // 2):
        for x in range(0, N // 2 + 1):
            r = oracle._lib().or_hypot_int(x, y)
            if r > N / 2:
                continue
            rx = F32(x) / (inx - F32(2.0))
            ry = F32(y) / iny
            xx = F32(F32(rx * M[0, 0]) + F32(ry * M[1, 0])) * F32(N)
            yy = F32(F32(rx * M[0, 1]) + F32(ry * M[1, 1])) * F32(N)
            zz = F32(F32(rx * M[0, 2]) + F32(ry * M[1, 2])) * F32(N)
            if x == 0 and y < 0:   # EMData::get_complex_at(x,y), libEM/emdata_core.cpp:126-132
                re, im = sl[-y, 0], -sl[-y, 1]
            else:
                row = y if y >= 0 else N + y
                re, im = sl[row, 2 * x], sl[row, 2 * x + 1]
            out.append((xx, yy, zz, re, im, weight))
    return out


def main():
    ref = ctypes.CDLL(oracle.REF_SO)
    ref.ref_insert_pixels.argtypes = [ctypes.c_char_p, _F, _F, ctypes.c_int, _F, ctypes.c_long]
    here = os.path.dirname(os.path.abspath(__file__))
    for k, (mode, N, sym) in enumerate(CASES):
        rng = np.random.default_rng(700 + k)
        n = 3
        slices = rng.normal(size=(n, N, N + 2)).astype(np.float32)
        from eman2_b200.synth import quaternion_blocks, random_quaternions
        rots = quaternion_blocks(random_quaternions(n, rng))
        weights = rng.uniform(0.5, 1.0, n).astype(np.float32)
        ops = oracle.sym_ops(sym)
        px = []
        for i in range(n):
            for op in ops:
                px += slice_pixels(slices[i], oracle.compose(rots[i], op), N, weights[i])
        px = np.ascontiguousarray(np.array(px, np.float32))
        data = np.zeros((N, N, N + 2), np.float32)
        norm = np.zeros((N, N, N // 2 + 1), np.float32)
        ref.ref_insert_pixels(mode.encode(), data.ctypes.data_as(_F), norm.ctypes.data_as(_F), N,
                              px.ctypes.data_as(_F), px.shape[0])
        path = os.path.join(here, f"insert_{k}_{mode}_N{N}_{sym}.npz")
        np.savez_compressed(path, mode=mode, N=N, sym=sym, slices=slices, rots=rots,
                            weights=weights, data=data, norm=norm)
        print("wrote", path, px.shape[0], "pixel inserts")


if __name__ == "__main__":
    main()
