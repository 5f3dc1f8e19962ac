"""Particle I/O on the host: MRC headers, modes, byte order and stacks
(libEM/io/mrcio.cpp), the #LSX particle list (libEM/io/lstfastio.cpp,
libpyEM/EMAN2.py LSXFile), and particle metadata from list records."""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from eman2_b200 import io
from eman2_b200.transform import Transform


def _raw_mrc(path, arr, mode, big=False, nsymbt=0, stamp=True):
    """An MRC file written field by field with numpy, independent of io.write_mrc."""
    e = ">" if big else "<"
    nz, ny, nx = arr.shape
    hdr = np.zeros(256, e + "i4")
    hdr[0:4] = nx, ny, nz, mode
    hdr[7:10] = nx, ny, nz
    hdr.view(e + "f4")[10:13] = 2.0 * nx, 2.0 * ny, 2.0 * nz
    hdr[16:19] = 1, 2, 3
    hdr[23] = nsymbt
    raw = bytearray(hdr.tobytes())
    raw[208:212] = b"MAP "
    if stamp:
        raw[212:214] = b"\x11\x11" if big else b"\x44\x44"
    if mode == 101:
        flat = arr.reshape(-1).astype(np.uint8)
        body = (flat[0::2] | (flat[1::2] << 4)).astype(np.uint8).tobytes()
    else:
        body = arr.astype(np.dtype(io.MODE_DTYPE[mode]).newbyteorder(e)).tobytes()
    with open(path, "wb") as f:
        f.write(bytes(raw) + b"\x07" * nsymbt + body)


@pytest.mark.parametrize("mode", [0, 17, 1, 6, 12, 2, 101])
@pytest.mark.parametrize("big", [False, True])
def test_mrc_modes_and_byte_order(tmp_path, mode, big):
    rng = np.random.default_rng(mode)
    lo, hi = {0: (0, 255), 17: (-128, 127), 1: (-3000, 3000), 6: (0, 60000), 12: (-4, 4),
              2: (-4, 4), 101: (0, 15)}[mode]
    a = rng.uniform(lo, hi, (3, 6, 8))
    a = a if mode in (2, 12) else np.rint(a)
    if mode == 12:
        a = a.astype(np.float16).astype(np.float32)
    p = str(tmp_path / "s.mrcs")
    _raw_mrc(p, a.astype(np.float32), mode, big=big, nsymbt=40, stamp=not big)
    info = io.mrc_info(p)
    assert (info.nx, info.ny, info.nz, info.mode, info.swap) == (8, 6, 3, mode, big)
    assert info.nimg == 3 and info.data_offset == 1064 and info.apix == 2.0
    np.testing.assert_array_equal(io.read_mrc_stack(p), a.astype(np.float32))
    np.testing.assert_array_equal(io.read_mrc(p, 2).numpy(), a[2].astype(np.float32))


def test_mrc_volume_is_not_a_stack(tmp_path):
    a = np.arange(4 * 5 * 6, dtype=np.float32).reshape(4, 5, 6)
    p = str(tmp_path / "v.mrc")
    io.write_mrc(p, a, apix=1.5)
    e = io.read_mrc(p)
    assert e.numpy().shape == (4, 5, 6) and e.get_attr("apix_x") == pytest.approx(1.5)
    with pytest.raises(Exception):
        io.read_mrc(p, 1)


@pytest.mark.parametrize("mode", [2, 12, 1])
def test_write_read_round_trip(tmp_path, mode):
    rng = np.random.default_rng(5)
    a = rng.normal(size=(7, 16, 16)).astype(np.float32) * 50
    p = str(tmp_path / "r.mrcs")
    io.write_mrc(p, a, mode=mode)
    want = {2: a, 12: a.astype(np.float16).astype(np.float32), 1: np.rint(a)}[mode]
    np.testing.assert_array_equal(io.read_mrc_stack(p, 2, 3), want[2:5])
    hdr = np.fromfile(p, "<i4", 256)
    assert hdr[3] == mode and bytes(np.fromfile(p, np.uint8, 4, offset=208)) == b"MAP "


def test_lsx_round_trip_and_rewrite(tmp_path):
    p = str(tmp_path / "p.lst")
    lsx = io.LSXFile(p)
    xf = Transform({"type": "eman", "az": 10.0, "alt": 20.0, "phi": 30.0, "tx": 1.5, "ty": -2.0})
    lsx.write(-1, 5, "stack.mrcs", {"xform.projection": xf, "score": -0.5})
    lsx.write(-1, 6, "stack.mrcs")
    long_note = "x" * 200
    lsx.write(-1, 7, "stack.mrcs", {"note": long_note})      # longer than the line: rewrite
    lsx.close()
    with open(p) as f:
        lines = f.read().split("\n")
    assert lines[0] == "#LSX" and lines[2].startswith("# ")
    L = int(lines[2][1:])
    assert all(len(x) + 1 == L for x in lines[3:-1])
    r = io.LSXFile(p, True)
    assert len(r) == 3
    n, f, d = r.read(0)
    assert (n, f, d["score"]) == (5, "stack.mrcs", -0.5)
    np.testing.assert_allclose(d["xform.projection"].matrix, xf.matrix, atol=2e-5)
    assert r.read(1)[2] == {} and r.read(2)[2]["note"] == long_note
    r.close()


def test_weights_from_scores_rule():
    """initialize_data (programs/e2spa_make3d.py:248-292): no scores -> 1;
    negative similarity scores -> -score / max(-score)."""
    assert io.weights_from_scores([{}, {}]).tolist() == [1.0, 1.0]
    w = io.weights_from_scores([{"score": -2.0}, {"score": -1.0}, {"score": 0.5}])
    np.testing.assert_allclose(w, [1.0, 0.5, 0.0])
    np.testing.assert_allclose(io.weights_from_scores([{"score": 0.3}, {"score": 0.6}]), [0.3, 0.6])


def test_records_to_meta(tmp_path):
    xf = Transform({"type": "eman", "az": 30.0, "alt": 40.0, "phi": 50.0, "tx": 3.0, "ty": 1.0})
    recs = [{"src": "a.mrcs", "idx": 0, "xform.projection": xf, "score": -1.0,
             "ctf": {"defocus": 1.8, "voltage": 300.0, "cs": 2.7, "ampcont": 10.0, "apix": 1.1,
                     "dfdiff": 0.0, "dfang": 0.0}}]
    m = io.records_to_meta(recs)
    p = m[0]
    np.testing.assert_allclose(np.array(p.rot[:]).reshape(3, 3), xf.rotation_block(), atol=1e-6)
    assert (p.tx, p.ty, p.weight) == (3.0, 1.0, 1.0)
    assert math.isclose(p.defocus, 1.8, rel_tol=1e-6) and math.isclose(p.apix, 1.1, rel_tol=1e-6)
