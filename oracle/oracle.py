"""CPU oracle for EMAN2's direct Fourier inversion (FourierReconstructor).

TEST INFRASTRUCTURE ONLY.  The product (the ``eman2_b200`` package) never
imports this module.  It is imported by ``tests/``, by the smoke check in
``__graft_entry__.py`` and by the ``cpu_baseline`` / ``--impl reference`` legs
of ``bench.py``, where it is the checker or the timed CPU baseline.

Three builds of one restatement (``fr_oracle.c``):

* ``fp32`` -- FP32-faithful: the reference's operation order and rounding
  points in strict IEEE single precision.  This is the stand-in for the
  reference's own FourierReconstructor, which cannot be built here.
* ``fp32acc64`` -- FP32 tap arithmetic (identical taps) with FP64 sums: the
  yardstick for summation-order noise.
* ``fp64`` -- the same algorithm in double precision (coordinates, weights,
  accumulators); the FP64 oracle both GPU forms state their error against.

The FFTs (numpy/pocketfft, float64) replace FFTW, which is not present; the
FP32 path rounds each FFT result to float32, so it differs from an FFTW float
transform at the 1e-7 level.  The restatement's insert_pixel/add_complex_at
arithmetic is pinned bitwise against the reference's own inserter source
(``build_ref.sh`` -> ``_ref/libfr_ref.so``; ``tests/test_oracle_ref.py``).
The same source built with the reference's release flags
(``_ref/libfr_ref_fast.so``) is the timed CPU reference arm
(``ref_insert_threaded``): the reference's own inserter fed the restatement's
pixel stream.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_SO = os.path.join(HERE, "_ref", "libfr_ref.so")
# the same reference source built with its default release flags (-O3
# -ffast-math, CMakeLists.txt): the timed CPU reference arm
REF_FAST_SO = os.path.join(HERE, "_ref", "libfr_ref_fast.so")

MODES = {"nearest_neighbor": 1, "gauss_2": 2, "gauss_5": 5, "trilinear": 6}

_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_libs: dict = {}


def build(ref: bool = True, reference: str | None = None) -> None:
    """Compile the oracle libraries and, when ``ref`` and a reference tree is
    given (``reference`` or $EMAN2_REFERENCE), the reference pin."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    tree = reference or os.environ.get("EMAN2_REFERENCE")
    if ref and tree:
        subprocess.run(["sh", os.path.join(HERE, "build_ref.sh"), tree], check=True,
                       stdout=subprocess.DEVNULL)


def _lib(kind: str = "fp32"):
    if kind in _libs:
        return _libs[kind]
    name = {"fp32": "liborfp32.so", "fp64": "liborfp64.so", "omp": "liborfp32_omp.so",
            "fp32acc64": "liborfp32acc64.so"}[kind]
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build(ref=False)
    lib = ctypes.CDLL(path)
    R = _F if kind in ("fp32", "omp") else _D   # accumulator pointer type
    lib.or_insert_slice.argtypes = [R, R, ctypes.c_int, ctypes.c_int, _F, _F, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_int, _F, ctypes.c_int]
    lib.or_insert_batch.argtypes = [R, R, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, _F, _F,
                                    ctypes.c_int, _F, ctypes.c_int]
    lib.or_insert_pixels.argtypes = [ctypes.c_int, R, R, ctypes.c_int, _F, ctypes.c_long]
    lib.or_normalize.argtypes = [R, R, ctypes.c_int, ctypes.c_int]
    lib.or_normalize_w.argtypes = [R, R, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.or_normalize_nz.argtypes = [R, R, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.or_insert_batch_nz.argtypes = [R, R, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F,
                                       ctypes.c_int, _F, _F, ctypes.c_int, _F]
    lib.or_insert_slice_iter.argtypes = [R, R, ctypes.c_int, _F, _F, ctypes.c_int, ctypes.c_float,
                                         _F]
    lib.or_insert_slice_wiener.argtypes = [R, R, ctypes.c_int, ctypes.c_int, _F, _F, ctypes.c_int,
                                           ctypes.c_float, _F, ctypes.c_int, ctypes.c_int]
    lib.or_compare_slice.argtypes = [R, R, ctypes.c_int, _F, _F, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_float, _F]
    lib.or_sym_ops.argtypes = [ctypes.c_char, ctypes.c_int, _F, ctypes.c_int]
    lib.or_projection.argtypes = [R, R, ctypes.c_int, _F, ctypes.c_float, ctypes.c_float, _F]
    lib.or_eman_matrix.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, _F]
    lib.or_quaternion_matrix.argtypes = [ctypes.c_double] * 4 + [_F]
    lib.or_compose.argtypes = [_F, _F, _F]
    lib.or_edge_mean.argtypes = [_F, ctypes.c_int, ctypes.c_int]
    lib.or_edge_mean.restype = ctypes.c_float
    lib.or_ctf_sign.argtypes = [_F, ctypes.c_int] + [ctypes.c_float] * 7
    lib.or_translate_bilinear.argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                          ctypes.c_float]
    lib.or_fast_exp_value.argtypes = [ctypes.c_float]
    lib.or_fast_exp_value.restype = ctypes.c_float
    lib.or_hypot_int.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.or_kernel_fix.argtypes = [_F, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
    if kind == "omp":
        lib.or_insert_batch_omp.argtypes = [R, R, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, _F,
                                            _F, ctypes.c_int, _F, ctypes.c_int]
    _libs[kind] = lib
    return lib


def ref_available() -> bool:
    """Whether the reference's own inserter was built (``build_ref.sh``)."""
    return os.path.exists(REF_FAST_SO)


def ref_insert_threaded(N: int, slices, rots, weights, mode: str, sym: str, threads: int,
                        lib_path: str = REF_FAST_SO):
    """The reference's own pixel inserter (FourierPixelInserter3D::insert_pixel,
    libEM/reconstructor_tools.cpp, compiled from the reference tree with its
    release flags) on every pixel of every symmetry copy of n slices, the
    pixels formed by the restatement of do_insert_slice_work
    (``or_slice_pixels``).  Particle p runs on host thread p % threads into
    that thread's own volume, as parallel reconstructors do, and the volumes
    are added at the end.  ``lib_path``: the release build (timing) or
    ``REF_SO``, the strict build (bitwise checks).  Returns (data, norm)."""
    from concurrent.futures import ThreadPoolExecutor
    slices = np.ascontiguousarray(slices, np.float32).reshape(-1, N, N + 2)
    n = slices.shape[0]
    rots = np.asarray(rots, np.float32).reshape(n, 3, 3)
    weights = np.asarray(weights, np.float32).reshape(n)
    ops = sym_ops(sym).reshape(-1, 3, 3)
    nsym = ops.shape[0]
    ref = ctypes.CDLL(lib_path)
    ref.ref_insert_pixels.argtypes = [ctypes.c_char_p, _F, _F, ctypes.c_int, _F, ctypes.c_long]
    lib = _lib("fp32")
    lib.or_slice_pixels.argtypes = [ctypes.c_int, _F, _F, ctypes.c_int, ctypes.c_float, _F,
                                    ctypes.c_long]
    lib.or_slice_pixels.restype = ctypes.c_long
    cap = nsym * N * (N // 2 + 1)
    threads = max(1, min(int(threads), n))

    def run(t):
        data = np.zeros((N, N, N + 2), np.float32)
        norm = np.zeros((N, N, N // 2 + 1), np.float32)
        px = np.empty(cap * 6, np.float32)
        for p in range(t, n, threads):
            if weights[p] == 0:
                continue
            t3d = np.ascontiguousarray(
                np.stack([compose(rots[p], o) for o in ops]).astype(np.float32).reshape(-1))
            k = lib.or_slice_pixels(N, _fp(slices[p]), _fp(t3d), nsym, float(weights[p]),
                                    _fp(px), cap)
            if k < 0:
                raise RuntimeError("pixel stream overflow")
            if ref.ref_insert_pixels(mode.encode(), _fp(data), _fp(norm), N, _fp(px), k):
                raise RuntimeError(f"reference inserter refused mode {mode}")
        return data, norm

    with ThreadPoolExecutor(threads) as ex:
        parts = list(ex.map(run, range(threads)))
    data, norm = parts[0]
    for d, m in parts[1:]:
        data += d
        norm += m
    return data, norm


def _fp(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_F)


def _rp(a: np.ndarray):
    if a.dtype == np.float32:
        return a.ctypes.data_as(_F)
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


# ----------------------------------------------------------------- transforms

def eman_matrix(az: float, alt: float, phi: float) -> np.ndarray:
    m = np.zeros(9, np.float32)
    _lib().or_eman_matrix(az, alt, phi, _fp(m))
    return m.reshape(3, 3)


def quaternion_matrix(q) -> np.ndarray:
    m = np.zeros(9, np.float32)
    _lib().or_quaternion_matrix(float(q[0]), float(q[1]), float(q[2]), float(q[3]), _fp(m))
    return m.reshape(3, 3)


def sym_ops(sym: str) -> np.ndarray:
    """Symmetry operators of ``c<n>`` / ``d<n>`` / ``tet`` / ``oct`` / ``icos``
    (``icos5``) as (nsym, 3, 3) float32."""
    sym = sym.lower()
    platonic = {"tet": ("t", 12), "oct": ("o", 24), "icos": ("i", 60), "icos5": ("i", 60)}
    if sym in platonic:
        kind, n = platonic[sym]
    else:
        kind, n = sym[0], int(sym[1:] or 1)
    out = np.zeros(9 * 2 * n, np.float32)
    k = _lib().or_sym_ops(kind.encode(), n, _fp(out), 2 * n)
    if k < 0:
        raise ValueError(f"unsupported symmetry {sym}")
    return out[: 9 * k].reshape(k, 3, 3)


def compose(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, np.float32).reshape(9)
    b = np.ascontiguousarray(b, np.float32).reshape(9)
    out = np.zeros(9, np.float32)
    _lib().or_compose(_fp(a), _fp(b), _fp(out))
    return out.reshape(3, 3)


# ------------------------------------------------------------------ the volume

class OracleVolume:
    """Un-normalised (complex, weight) accumulators in the reference layout."""

    def __init__(self, N: int, precision: str = "fp32", NZ: int | None = None):
        self.N = N
        self.NZ = N if NZ is None else int(NZ)    # the volume's z size (square N x N slices)
        self.kind = precision
        dt = np.float32 if precision in ("fp32", "omp") else np.float64   # accumulators
        self.data = np.zeros((self.NZ, N, N + 2), dt)
        self.norm = np.zeros((self.NZ, N, N // 2 + 1), dt)

    @property
    def lib(self):
        return _lib(self.kind)

    def insert(self, slices, rots, weights, mode="gauss_2", sym="c1", corners=False):
        """insert_slice for n preprocessed slices (n, N, N+2) float32 with
        orientation blocks rots (n, 3, 3) and weights (n,)."""
        slices = np.ascontiguousarray(slices, np.float32).reshape(-1, self.N, self.N + 2)
        n = slices.shape[0]
        rots = np.ascontiguousarray(rots, np.float32).reshape(n, 9)
        weights = np.ascontiguousarray(weights, np.float32).reshape(n)
        ops = np.ascontiguousarray(sym_ops(sym)).reshape(-1, 9)
        if self.NZ != self.N:
            rc = self.lib.or_insert_batch_nz(_rp(self.data), _rp(self.norm), self.N, self.NZ,
                                             MODES[mode], _fp(slices), n, _fp(rots), _fp(ops),
                                             ops.shape[0], _fp(weights))
        else:
            rc = self.lib.or_insert_batch(_rp(self.data), _rp(self.norm), self.N, MODES[mode],
                                          _fp(slices), n, _fp(rots), _fp(ops), ops.shape[0],
                                          _fp(weights), int(bool(corners)))
        if rc:
            raise RuntimeError(f"oracle insert failed rc={rc}")

    def insert_wiener(self, slices, rots, weights, snr, undo=None, mode="gauss_2", sym="c1"):
        """WienerFourierReconstructor insert_slice for n slices with their
        ctf_snr_total curves snr (n, nsnr) and Wiener-filtered flags undo (n,)."""
        slices = np.ascontiguousarray(slices, np.float32).reshape(-1, self.N, self.N + 2)
        n = slices.shape[0]
        rots = np.ascontiguousarray(rots, np.float32).reshape(n, 9)
        snr = np.ascontiguousarray(snr, np.float32).reshape(n, -1)
        ops = np.ascontiguousarray(sym_ops(sym)).reshape(-1, 9)
        t3d = np.empty((ops.shape[0], 9), np.float32)
        for p in range(n):
            for s in range(ops.shape[0]):
                t3d[s] = compose(rots[p].reshape(3, 3), ops[s].reshape(3, 3)).reshape(9)
            rc = self.lib.or_insert_slice_wiener(
                _rp(self.data), _rp(self.norm), self.N, MODES[mode], _fp(slices[p]), _fp(t3d),
                ops.shape[0], float(weights[p]), _fp(snr[p]), snr.shape[1],
                int(bool(undo[p])) if undo is not None else 0)
            if rc:
                raise RuntimeError(f"oracle insert failed rc={rc}")

    def insert_iter(self, slices, rots, weights, sym="c1", ref=None):
        """FourierIterReconstructor insert_slice for n slices; ref: the
        reference volume (N, N, N+2) float32 or None."""
        slices = np.ascontiguousarray(slices, np.float32).reshape(-1, self.N, self.N + 2)
        n = slices.shape[0]
        rots = np.ascontiguousarray(rots, np.float32).reshape(n, 9)
        ops = np.ascontiguousarray(sym_ops(sym)).reshape(-1, 9)
        refp = None if ref is None else np.ascontiguousarray(ref, np.float32)
        t3d = np.empty((ops.shape[0], 9), np.float32)
        for p in range(n):
            for s in range(ops.shape[0]):
                t3d[s] = compose(rots[p].reshape(3, 3), ops[s].reshape(3, 3)).reshape(9)
            self.lib.or_insert_slice_iter(_rp(self.data), _rp(self.norm), self.N, _fp(slices[p]),
                                          _fp(t3d), ops.shape[0], float(weights[p]),
                                          _fp(refp) if refp is not None else None)

    def insert_omp(self, slices, rots, weights, mode="gauss_2", sym="c1", threads=0):
        assert self.kind == "omp"
        slices = np.ascontiguousarray(slices, np.float32).reshape(-1, self.N, self.N + 2)
        n = slices.shape[0]
        rots = np.ascontiguousarray(rots, np.float32).reshape(n, 9)
        weights = np.ascontiguousarray(weights, np.float32).reshape(n)
        ops = np.ascontiguousarray(sym_ops(sym)).reshape(-1, 9)
        rc = self.lib.or_insert_batch_omp(_rp(self.data), _rp(self.norm), self.N, MODES[mode],
                                          _fp(slices), n, _fp(rots), _fp(ops), ops.shape[0],
                                          _fp(weights), int(threads))
        if rc:
            raise RuntimeError(f"oracle insert failed rc={rc}")

    def insert_pixels(self, mode: str, px: np.ndarray):
        px = np.ascontiguousarray(px, np.float32).reshape(-1, 6)
        self.lib.or_insert_pixels(MODES[mode], _rp(self.data), _rp(self.norm), self.N,
                                  _fp(px), px.shape[0])

    def compare(self, slice_, rot, weight=1.0, sym="c1", apix=1.0):
        """determine_slice_agreement(sub=False) statistics for one slice:
        (norm, absqual, absqual_lowres, qual, weight)."""
        s = np.ascontiguousarray(slice_, np.float32).reshape(self.N, self.N + 2)
        ops = sym_ops(sym)
        t3d = np.stack([compose(rot, o) for o in ops]).astype(np.float32).reshape(-1, 9)
        out = np.zeros(5, np.float32)
        self.lib.or_compare_slice(_rp(self.data), _rp(self.norm), self.N, _fp(s),
                                  _fp(np.ascontiguousarray(t3d)), t3d.shape[0], float(weight),
                                  float(apix), _fp(out))
        return out

    def projection(self, rot, tx: float = 0.0, ty: float = 0.0, ret_fourier: bool = True):
        """FourierReconstructor::projection (libEM/reconstructor.cpp:1383-1445)
        of the current accumulators for rotation block rot (3, 3) and
        translation (tx, ty): the complex slice (N, N+2), or with
        ret_fourier False the phase origin moved to the centre
        (center_origin_fft, libEM/sparx/emdata_sparx.cpp:8420-8462) and the
        inverse FFT x 1/N^2 (do_ift, libEM/emdata_transform.cpp:330-375):
        a real (N, N) image."""
        N = self.N
        out = np.zeros((N, N + 2), np.float32)
        r = np.ascontiguousarray(rot, np.float32).reshape(9)
        self.lib.or_projection(_rp(self.data), _rp(self.norm), N, _fp(r), float(tx), float(ty),
                               _fp(out))
        if ret_fourier:
            return out
        c = out[:, 0::2] + 1j * out[:, 1::2].astype(np.float64)
        kx = np.arange(N // 2 + 1)[None, :]
        row = np.arange(N)[:, None]
        c = np.where((kx + row) % 2 == 1, -c, c)
        return _ift_f32(c.astype(np.complex64), N)

    def copy(self):
        o = OracleVolume.__new__(OracleVolume)
        o.N, o.NZ, o.kind = self.N, self.NZ, self.kind
        o.data, o.norm = self.data.copy(), self.norm.copy()
        return o

    def normalize(self, sqrtnorm=False, wiener=False):
        self.lib.or_normalize_nz(_rp(self.data), _rp(self.norm), self.N, self.NZ,
                                 int(bool(sqrtnorm)), int(bool(wiener)))

    def finish(self, doift=True, sqrtnorm=False, wiener=False):
        """FourierReconstructor::finish (libEM/reconstructor.cpp:1552-1641):
        normalise; optionally inverse FFT (x 1/N^3), depad, phase-origin to
        centre.  Returns (volume, norm) like finish() + normout."""
        self.normalize(sqrtnorm, wiener)
        if not doift:
            return self.data, self.norm
        N, NZ = self.N, self.NZ
        c = self.data.astype(np.float64).view(np.complex128)
        real = np.fft.irfftn(c, s=(NZ, N, N), axes=(0, 1, 2), norm="forward")
        if self.data.dtype == np.float64:
            real = real * (1.0 / (N * N * NZ))
        else:
            real = real.astype(np.float32) * np.float32(1.0 / (N * N * NZ))
        real = np.roll(real, (NZ // 2, N // 2, N // 2), axis=(0, 1, 2))
        return real, self.norm


def kernel_fix(vol: np.ndarray, gauss_width: float) -> np.ndarray:
    """math.gausskernelfix on a real volume (a copy)."""
    v = np.ascontiguousarray(vol, np.float32).copy()
    nz, ny, nx = v.shape
    _lib().or_kernel_fix(_fp(v), nx, ny, nz, float(gauss_width))
    return v


def clip_centre(vol: np.ndarray, outsize) -> np.ndarray:
    """clip_inplace(Region((nx-ox)//2, (ny-oy)//2, (nz-oz)//2, ox, oy, oz))
    (programs/e2make3dpar.py:430-431) for a region inside the volume."""
    nz, ny, nx = vol.shape
    ox, oy, oz = outsize
    x0, y0, z0 = (nx - ox) // 2, (ny - oy) // 2, (nz - oz) // 2
    return np.ascontiguousarray(vol[z0:z0 + oz, y0:y0 + oy, x0:x0 + ox])


# ------------------------------------------------------------------- prologue

def edge_mean(img: np.ndarray) -> np.float32:
    img = np.ascontiguousarray(img, np.float32)
    return np.float32(_lib().or_edge_mean(_fp(img), img.shape[1], img.shape[0]))


def clip_pad(img: np.ndarray, N: int) -> np.ndarray:
    """clip_inplace(Region((nx-N)//2, (ny-N)//2, N, N)) with zero fill
    (libEM/emdata.cpp:350)."""
    ny, nx = img.shape
    x0, y0 = (nx - N) // 2, (ny - N) // 2
    out = np.zeros((N, N), np.float32)
    for y in range(N):
        sy = y + y0
        if 0 <= sy < ny:
            xs = np.arange(N) + x0
            ok = (xs >= 0) & (xs < nx)
            out[y, ok] = img[sy, xs[ok]]
    return out


def ctf_sign(N: int, defocus, voltage=300.0, cs=2.7, apix=1.0, ampcont=10.0, dfdiff=0.0,
             dfang=0.0) -> np.ndarray:
    out = np.zeros((N, N // 2 + 1), np.float32)
    _lib().or_ctf_sign(_fp(out), N, float(defocus), float(dfdiff), float(dfang), float(voltage),
                       float(cs), float(apix), float(ampcont))
    return out


def _fft_f32(img: np.ndarray) -> np.ndarray:
    """Unnormalised r2c of a float32 image, rounded to complex64 (FFTW stand-in)."""
    return np.fft.rfft2(img.astype(np.float64)).astype(np.complex64)


def _ift_f32(spec: np.ndarray, N: int) -> np.ndarray:
    """do_ift (libEM/emdata_transform.cpp:392-425): unnormalised c2r, then x 1/N^2."""
    r = np.fft.irfft2(spec.astype(np.complex128), s=(N, N), norm="forward").astype(np.float32)
    return r * np.float32(1.0 / (N * N))


def ctf_flip(img: np.ndarray, ctf: dict) -> np.ndarray:
    """FFT -> x CTF_SIGN -> IFT (programs/e2spa_make3d.py:316-326, one flip)."""
    N = img.shape[0]
    F = _fft_f32(img)
    s = ctf_sign(N, ctf["defocus"], ctf.get("voltage", 300.0), ctf.get("cs", 2.7),
                 ctf.get("apix", 1.0), ctf.get("ampcont", 10.0), ctf.get("dfdiff", 0.0),
                 ctf.get("dfang", 0.0))
    F = (F.real * s + 1j * (F.imag * s)).astype(np.complex64)
    return _ift_f32(F, N)


def translate(img: np.ndarray, tx: float, ty: float) -> np.ndarray:
    img = np.ascontiguousarray(img, np.float32)
    out = np.zeros_like(img)
    _lib().or_translate_bilinear(_fp(img), _fp(out), img.shape[1], img.shape[0], float(tx),
                                 float(ty))
    return out


def _near_int(v: float) -> float:
    c, f = np.ceil(np.float32(v)), np.floor(np.float32(v))
    if abs(v - c) < 1e-6:
        return c
    if abs(v - f) < 1e-6:
        return f
    return v


def preprocess_slice(img: np.ndarray, inv_tx: float = 0.0, inv_ty: float = 0.0) -> np.ndarray:
    """FourierReconstructor::preprocess_slice (libEM/reconstructor.cpp:1022-1061)
    for a translation-only transform whose inverse translates by
    (inv_tx, inv_ty): bilinear xform (identity -> copy), phase origin to corner,
    r2c, x sqrt((N+2)/N).  Returns the (N, N+2) float32 interleaved slice."""
    N = img.shape[0]
    img = np.ascontiguousarray(img, np.float32)
    if _near_int(-inv_tx) == 0 and _near_int(-inv_ty) == 0:
        work = img.copy()
    else:
        work = translate(img, inv_tx, inv_ty)
    work = np.roll(work, (-(N // 2), -(N // 2)), axis=(0, 1))
    F = _fft_f32(work)
    scale = np.sqrt(np.float32(1.0) / np.float32(N) * np.float32(N + 2)).astype(np.float32)
    out = np.empty((N, N + 2), np.float32)
    out[:, 0::2] = F.real * scale
    out[:, 1::2] = F.imag * scale
    return out


def particle_to_slice(raw: np.ndarray, N: int, shift=(0.0, 0.0), ctf: dict | None = None):
    """The reference caller's per-particle pipeline (programs/e2spa_make3d.py:300-342):
    edge-mean subtract, clip to N, optional CTF phase flip, edge-mean subtract,
    then preprocess_slice with the inverted translation of xform.projection."""
    img = np.asarray(raw, np.float32)
    img = img - edge_mean(img)
    img = clip_pad(img, N)
    if ctf is not None and abs(ctf.get("defocus", 0.0)) > 1e-4:
        img = ctf_flip(img, ctf)
    img = img - edge_mean(img)
    return preprocess_slice(img, float(np.float32(shift[0])), float(np.float32(shift[1])))


# ------------------------------------------------------------------- metrics

def fsc(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Fourier shell correlation of two complex half volumes (N, N, N+2)
    following EMData::calc_fourier_shell_correlation
    (libEM/sparx/emdata_sparx.cpp:867-990) with ring width 1."""
    N = a.shape[0]
    ca = a.astype(np.float64).view(np.complex128)
    cb = b.astype(np.float64).view(np.complex128)
    k = np.fft.fftfreq(N, 1.0 / N)
    kz, ky, kx = np.meshgrid(k, k, np.arange(N // 2 + 1), indexing="ij")
    r = np.floor(np.sqrt(kx ** 2 + ky ** 2 + kz ** 2) + 0.5).astype(int)
    keep = (kx > 0) | ((kz >= 0) & ((ky >= 0) | (kz != 0)))
    keep &= r <= N // 2
    rr = r[keep]
    num = np.bincount(rr, (ca[keep] * np.conj(cb[keep])).real, N // 2 + 1)
    n1 = np.bincount(rr, np.abs(ca[keep]) ** 2, N // 2 + 1)
    n2 = np.bincount(rr, np.abs(cb[keep]) ** 2, N // 2 + 1)
    with np.errstate(invalid="ignore", divide="ignore"):
        out = num / np.sqrt(n1 * n2)
    out[(n1 <= 0) | (n2 <= 0)] = 1.0
    return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)
