"""GPU parity: libeman2_b200 against the CPU oracle on identical seeded inputs.

Tolerances: the GPU reproduces every tap selection and exp-table index of the
reference bit for bit; only the order of FP32 additions differs (atomics in
the scatter schedule, FP64 partial sums in the gather schedule), so the
accumulators agree with the FP32-faithful oracle to a relative L2 of
RTOL_ACC = 2e-6 and to the FP64 oracle likewise.  Anything that moves a
window or a table index shows up as an error of order 1e-3 or more.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL_ACC = 2e-6      # accumulators, FP32 summation-order noise only
RTOL_FFT = 2e-5      # paths through cuFFT vs pocketfft (float64 rounded to float32)
# versus the FP64 oracle: within 3x the FP32-faithful oracle's own distance


def rand_slices(N, n, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, N, N + 2)).astype(np.float32)


def rand_rots(n, seed):
    from eman2_b200.synth import quaternion_blocks, random_quaternions
    return quaternion_blocks(random_quaternions(n, np.random.default_rng(seed)))


def use_tile(N, mode, sym, tile):
    """Pin the gather schedule's kernel for (N, mode, sym): 0-3 the per-voxel
    register tiles, 4 the staged column-owner kernel, 5 the barrier-free
    column kernel, 6 the pixel-major kernel (gauss_5: 5), -1 back to the
    default."""
    from eman2_b200 import _lib
    from oracle.oracle import sym_ops
    _lib.check(_lib.load().fr_set_tile(N, _lib.MODE_IDS[mode], len(sym_ops(sym)), tile))


def recon(N, mode="gauss_2", sym="c1", **kw):
    from eman2_b200 import Reconstructors
    p = {"size": [N, N, N], "sym": sym, "mode": mode}
    p.update(kw)
    r = Reconstructors.get("fourier", p)
    r.setup()
    return r


def oracle_insert(N, slices, rots, weights, mode, sym, prec="fp32", corners=False):
    v = oracle.OracleVolume(N, prec)
    v.insert(slices, rots, weights, mode, sym, corners=corners)
    return v


def rel(a, b):
    return oracle.rel_l2(a, b)


@pytest.mark.parametrize("sched", ["scatter", "gather_v1", "gather_column", "gather_column3",
                                   "gather_pixel"])
@pytest.mark.parametrize("mode", ["nearest_neighbor", "gauss_2", "gauss_5", "trilinear"])
@pytest.mark.parametrize("N,sym", [(16, "c1"), (22, "d2"), (32, "c3"), (40, "d1")])
def test_insert_schedules_match_oracle(gpu, sched, mode, N, sym):
    n = 24
    sl, rt = rand_slices(N, n, N), rand_rots(n, N + 1)
    w = np.random.default_rng(N + 2).uniform(0.5, 1.0, n).astype(np.float32)
    r = recon(N, mode, sym)
    if sched != "scatter":
        use_tile(N, mode, sym, {"gather_v1": 0, "gather_column": 4, "gather_column3": 5,
                                "gather_pixel": 6}[sched])
    try:
        st = r.insert_slices(sl, rt, w, schedule="scatter" if sched == "scatter" else "gather")
    finally:
        use_tile(N, mode, sym, -1)
    assert st == [0] * n
    d, nm = r.get_accumulators()
    o = oracle_insert(N, sl, rt, w, mode, sym)
    assert rel(nm, o.norm) < RTOL_ACC
    assert rel(d, o.data) < RTOL_ACC
    # same support: no tap went missing or appeared
    assert np.array_equal(nm != 0, o.norm != 0)
    # every cell's weight (a sum of positive taps) to FP32 summation noise: a
    # missing far tap (gauss_5's weights reach 1e-9) shows here, not in the L2
    m = o.norm != 0
    assert np.max(np.abs(nm[m] - o.norm[m]) / o.norm[m]) < 1e-4
    # Same taps summed in FP64: what is left is summation-order noise only.
    oa = oracle_insert(N, sl, rt, w, mode, sym, "fp32acc64")
    assert rel(d, oa.data) < RTOL_ACC and rel(nm, oa.norm) < RTOL_ACC
    # Against the FP64 oracle the distance is the FP32 path's own rounding
    # (coordinates, weights, a rare exp-table index): the GPU sits as close to
    # it as the FP32-faithful oracle does.
    o64 = oracle_insert(N, sl, rt, w, mode, sym, "fp64")
    assert rel(d, o64.data) < 3 * rel(o.data, o64.data) + 1e-6


def test_plain_insert_slice_path(gpu):
    """One insert_slice call per particle (the plain per-call path)."""
    from eman2_b200 import EMData, Transform
    N, n = 24, 12
    sl, rt = rand_slices(N, n, 5), rand_rots(n, 6)
    r = recon(N, "gauss_2", "c1")
    for i in range(n):
        img = EMData(sl[i], is_complex=True, attrs={"reconstruct_preproc": 1})
        assert r.insert_slice(img, Transform(rt[i]), 0.75) == 0
    assert r.insert_slice(EMData(sl[0], is_complex=True, attrs={"reconstruct_preproc": 1}),
                          Transform(rt[0]), 0.0) == -1
    d, nm = r.get_accumulators()
    o = oracle_insert(N, sl, rt, np.full(n, 0.75, np.float32), "gauss_2", "c1")
    assert rel(d, o.data) < RTOL_ACC and rel(nm, o.norm) < RTOL_ACC


def interior(N):
    """Cells with |x|,|y|,|z| < N/2 (the gather kernel's own cells): every
    cell except the x=N/2 column and the y=-N/2 row and z=-N/2 slab."""
    m = np.ones((N, N, N // 2 + 1), bool)
    m[:, :, N // 2] = False
    m[:, N // 2, :] = False
    m[N // 2, :, :] = False
    return m


def test_gather_is_deterministic_and_matches_scatter(gpu):
    """The gather schedule owns every interior cell: bitwise reproducible
    there.  Cube-face cells come from the atomic face-tap kernel."""
    N, n = 48, 64
    sl, rt = rand_slices(N, n, 11), rand_rots(n, 12)
    w = np.ones(n, np.float32)
    outs = []
    use_tile(N, "gauss_5", "d3", 0)
    try:
        for sched in ("gather", "gather", "scatter"):
            r = recon(N, "gauss_5", "d3")
            r.insert_slices(sl, rt, w, schedule=sched)
            outs.append(r.get_accumulators())
    finally:
        use_tile(N, "gauss_5", "d3", -1)
    m = interior(N)
    c0 = outs[0][0].view(np.complex64)
    c1 = outs[1][0].view(np.complex64)
    assert np.array_equal(c0[m], c1[m]) and np.array_equal(outs[0][1][m], outs[1][1][m])
    assert rel(outs[0][0], outs[1][0]) < RTOL_ACC
    assert rel(outs[0][0], outs[2][0]) < RTOL_ACC


def test_zero_and_negative_weights(gpu):
    """weight 0 inserts nothing (-1); a negative weight selects the SSNR path,
    which needs class_ssnr (NotExistingObjectException without it)."""
    from eman2_b200 import EMData, NotExistingObjectException, Transform
    N, n = 20, 10
    sl, rt = rand_slices(N, n, 21), rand_rots(n, 22)
    w = np.ones(n, np.float32)
    w[3] = 0.0
    r = recon(N, "gauss_2", "c1")
    st = r.insert_slices(sl, rt, w, schedule="scatter")
    assert st[3] == -1 and st.count(-1) == 1
    img = EMData(sl[0], is_complex=True, attrs={"reconstruct_preproc": 1})
    with pytest.raises(NotExistingObjectException):
        r.insert_slice(img, Transform(rt[0]), -1.0)


def test_ssnr_weighted_insertion(gpu):
    """usessnr: per-pixel weights max(0, ssnr[int(r*sscale)]) from class_ssnr
    (libEM/reconstructor.cpp:1158-1184), against the oracle fed the same
    per-pixel weights through its inserter."""
    from eman2_b200 import EMData, Transform
    N = 16
    sl, rt = rand_slices(N, 1, 23), rand_rots(1, 24)
    ssnr = np.linspace(2.0, -0.5, 12).astype(np.float32)
    r = recon(N, "gauss_2", "c1", usessnr=True)
    img = EMData(sl[0], is_complex=True, attrs={"reconstruct_preproc": 1, "class_ssnr": ssnr})
    assert r.insert_slice(img, Transform(rt[0]), 1.0) == 0
    d, nm = r.get_accumulators()
    # oracle: the same loop with the SSNR weight per pixel
    import ctypes
    v = oracle.OracleVolume(N, "fp32")
    lib = v.lib
    F = ctypes.POINTER(ctypes.c_float)
    rc = lib.or_insert_slice(v.data.ctypes.data_as(F), v.norm.ctypes.data_as(F), N, 2,
                             np.ascontiguousarray(sl[0]).ctypes.data_as(F),
                             np.ascontiguousarray(rt[0]).ctypes.data_as(F), 1, -1.0, 0,
                             ssnr.ctypes.data_as(F), ssnr.size)
    assert rc == 0
    assert rel(d, v.data) < RTOL_ACC and rel(nm, v.norm) < RTOL_ACC


def test_corners_mode(gpu):
    N, n = 16, 8
    sl, rt = rand_slices(N, n, 31), rand_rots(n, 32)
    w = np.ones(n, np.float32)
    for sched in ("scatter", "gather"):
        r = recon(N, "gauss_2", "c1", corners=True)
        r.insert_slices(sl, rt, w, schedule=sched)
        d, nm = r.get_accumulators()
        o = oracle_insert(N, sl, rt, w, "gauss_2", "c1", corners=True)
        assert rel(d, o.data) < RTOL_ACC and rel(nm, o.norm) < RTOL_ACC


def test_preprocess_matches_oracle(gpu):
    from eman2_b200 import EMData, Transform
    N = 32
    rng = np.random.default_rng(41)
    r = recon(N)
    for t in [(0.0, 0.0), (1.25, -2.5), (3.0, 0.75)]:
        img = rng.normal(size=(N, N)).astype(np.float32)
        xf = Transform({"type": "eman", "az": 10.0, "alt": 20.0, "phi": 30.0, "tx": t[0], "ty": t[1]})
        got = r.preprocess_slice(EMData(img), xf).numpy()
        want = oracle.preprocess_slice(img, -t[0], -t[1])
        assert rel(got, want) < RTOL_FFT


def test_particle_pipeline_matches_oracle(gpu):
    """fr_insert_particles (edge mean, pad, CTF flip, shift, r2c, insert) vs
    the oracle's restatement of the caller loop."""
    from eman2_b200.particles import particle_meta
    from eman2_b200.synth import make_particles
    box, N, n = 32, 48, 24
    ps = make_particles(box, n, seed=51, snr=0.5, shift=3.0, weights=(0.5, 1.0), ctf=True)
    r = recon(N, "gauss_2", "c1")
    r.insert_particles(ps.images, particle_meta(ps.rots, ps.shifts, ps.weights, defocus=ps.defocus))
    d, nm = r.get_accumulators()
    slices = np.stack([oracle.particle_to_slice(ps.images[i], N, ps.shifts[i],
                                                {"defocus": float(ps.defocus[i])})
                       for i in range(n)])
    o = oracle_insert(N, slices, ps.rots, ps.weights, "gauss_2", "c1")
    assert rel(nm, o.norm) < RTOL_ACC
    assert rel(d, o.data) < RTOL_FFT


def test_finish_matches_oracle(gpu):
    N, n = 32, 40
    sl, rt = rand_slices(N, n, 61), rand_rots(n, 62)
    w = np.ones(n, np.float32)
    for doift in (False, True):
        r = recon(N, "gauss_2", "c1")
        r.insert_slices(sl, rt, w)
        out = r.finish(doift).numpy()
        o = oracle_insert(N, sl, rt, w, "gauss_2", "c1")
        want, _ = o.finish(doift)
        assert rel(out, want) < (RTOL_FFT if doift else RTOL_ACC)


def test_kernel_fix_matches_oracle(gpu):
    """math.gausskernelfix on host and device volumes, cubic and not, equals
    the oracle's restatement (same float distance, double quotient)."""
    import torch
    from eman2_b200 import EMData
    rng = np.random.default_rng(81)
    for shape, wdt in [((24, 24, 24), 10.4), ((10, 14, 18), 4.0)]:
        v = rng.normal(size=shape).astype(np.float32)
        want = oracle.kernel_fix(v, wdt)
        e = EMData(v.copy())
        e.process_inplace("math.gausskernelfix", {"gauss_width": wdt})
        np.testing.assert_array_max_ulp(e.numpy(), want, maxulp=1)
        d = torch.as_tensor(v, device="cuda")
        from eman2_b200 import _lib
        nz, ny, nx = shape
        _lib.check(_lib.load().fr_kernel_fix(d.data_ptr(), nx, ny, nz, wdt, None))
        np.testing.assert_array_max_ulp(d.cpu().numpy(), want, maxulp=1)


@pytest.mark.parametrize("mode,width,outsize", [("gauss_5", None, 36), ("gauss_2", 4.0, (30, 32, 34)),
                                                ("nearest_neighbor", None, 40)])
def test_finish_corrected_matches_oracle(gpu, mode, width, outsize):
    """finish(True) + math.gausskernelfix + centred clip (programs/e2make3dpar.py:421-431)
    in one pass equals the oracle's finish, kernel fix and clip, and the
    GPU's own unfused sequence bit for bit."""
    from eman2_b200 import Region
    N, n = 40, 30
    sl, rt = rand_slices(N, n, 91), rand_rots(n, 92)
    w = np.ones(n, np.float32)
    widths = {"gauss_5": 10.4, "gauss_2": 4.0, "nearest_neighbor": 0.0}
    wd = widths[mode] if width is None else width
    osz = (outsize,) * 3 if np.isscalar(outsize) else outsize
    r = recon(N, mode, "d2")
    r.insert_slices(sl, rt, w)
    got = r.finish_corrected(width, outsize).numpy()
    assert got.shape == (osz[2], osz[1], osz[0])
    o = oracle_insert(N, sl, rt, w, mode, "d2")
    real, _ = o.finish(True)
    want = oracle.clip_centre(oracle.kernel_fix(real, wd) if wd > 0 else real, osz)
    assert rel(got, want) < RTOL_FFT
    r2 = recon(N, mode, "d2")
    r2.insert_slices(sl, rt, w)
    e = r2.finish(True)
    if wd > 0:
        e.process_inplace("math.gausskernelfix", {"gauss_width": wd})
    e.clip_inplace(Region((N - osz[0]) // 2, (N - osz[1]) // 2, (N - osz[2]) // 2, *osz))
    assert rel(got, e.numpy()) < RTOL_ACC


@pytest.mark.parametrize("mode,sym", [("gauss_2", "c1"), ("nearest_neighbor", "d2"),
                                      ("gauss_5", "c2"), ("trilinear", "d1")])
def test_wiener_matches_oracle(gpu, mode, sym):
    """wiener_fourier: SNR-weighted pixels on the rn < 0.5 disk, some slices
    Wiener filtered (undone), one subtracted, and the (weight + 1) finish."""
    from eman2_b200 import EMData, Reconstructors
    from eman2_b200.exceptions import NotExistingObjectException
    N, n = 24, 12
    sl, rt = rand_slices(N, n, 101), rand_rots(n, 102)
    rng = np.random.default_rng(103)
    snr = rng.uniform(0.2, 5.0, (n, 13)).astype(np.float32)
    undo = (np.arange(n) % 3 == 0).astype(np.int32)
    w = np.ones(n, np.float32)
    w[5] = -1.0
    r = Reconstructors.get("wiener_fourier", {"size": [N] * 3, "sym": sym, "mode": mode})
    r.setup()
    r.insert_slices_wiener(sl, rt, w, snr, undo)
    d, nrm = r.get_accumulators()
    o = oracle.OracleVolume(N, "fp32")
    o.insert_wiener(sl, rt, w, snr, undo, mode, sym)
    assert rel(nrm, o.norm) < RTOL_ACC and rel(d, o.data) < RTOL_ACC
    # finish on a reconstruction without the subtracted slice: with it, some
    # summed weights approach -1 and weight + 1 amplifies summation-order noise
    w[5] = 1.0
    r.setup()
    r.insert_slices_wiener(sl, rt, w, snr, undo)
    o = oracle.OracleVolume(N, "fp32")
    o.insert_wiener(sl, rt, w, snr, undo, mode, sym)
    out = r.finish(True).numpy()
    want, _ = o.finish(True, wiener=True)
    assert rel(out, want) < RTOL_FFT
    # the single-slice API and the missing-curve error
    r2 = Reconstructors.get("wiener_fourier", {"size": [N] * 3, "sym": sym, "mode": mode})
    r2.setup()
    img = EMData(sl[0], is_complex=True, attrs={"reconstruct_preproc": 1,
                                                "ctf_snr_total": snr[0].tolist()})
    from eman2_b200 import Transform
    assert r2.insert_slice(img, Transform(rt[0].reshape(-1)), 1.0) == 0
    o2 = oracle.OracleVolume(N, "fp32")
    o2.insert_wiener(sl[:1], rt[:1], np.ones(1, np.float32), snr[:1], None, mode, sym)
    d2, n2 = r2.get_accumulators()
    assert rel(n2, o2.norm) < RTOL_ACC and rel(d2, o2.data) < RTOL_ACC
    with pytest.raises(NotExistingObjectException):
        r2.insert_slice(EMData(sl[1], is_complex=True, attrs={"reconstruct_preproc": 1}),
                        Transform(rt[1].reshape(-1)), 1.0)


def test_iter_matches_oracle(gpu):
    """fourier_iter: first pass (resolution-dependent width), then with a
    complex reference volume (the update rule), then with a real seed map
    transformed on the device."""
    from eman2_b200 import Reconstructors
    N, n, sym = 24, 10, "d2"
    sl, rt = rand_slices(N, n, 111), rand_rots(n, 112)
    w = np.random.default_rng(113).uniform(0.5, 1.0, n).astype(np.float32)
    w[3] = -0.5                                          # any weight goes in as is
    r = Reconstructors.get("fourier_iter", {"size": [N] * 3, "sym": sym})
    r.setup()
    r.insert_slices(sl, rt, w, schedule="scatter")
    d, nrm = r.get_accumulators()
    o = oracle.OracleVolume(N, "fp32")
    o.insert_iter(sl, rt, w, sym)
    assert rel(nrm, o.norm) < RTOL_ACC and rel(d, o.data) < RTOL_ACC
    ref = np.random.default_rng(114).normal(size=(N, N, N + 2)).astype(np.float32)
    r.setup_seed(ref)
    r.insert_slices(sl, rt, w, schedule="scatter")
    d, nrm = r.get_accumulators()
    o = oracle.OracleVolume(N, "fp32")
    o.insert_iter(sl, rt, w, sym, ref=ref)
    assert rel(nrm, o.norm) < RTOL_ACC and rel(d, o.data) < RTOL_ACC
    out = r.finish(True).numpy()
    want, _ = o.finish(True)
    assert rel(out, want) < RTOL_FFT
    # a real seed: phase origin to corner, then r2c, on the device
    seed = np.random.default_rng(115).normal(size=(N, N, N)).astype(np.float32)
    spec = np.fft.rfftn(np.roll(seed.astype(np.float64), (N // 2,) * 3, axis=(0, 1, 2)))
    cref = np.ascontiguousarray(spec.astype(np.complex64)).view(np.float32).reshape(N, N, N + 2)
    r2 = Reconstructors.get("fourier_iter", {"size": [N] * 3, "sym": sym})
    r2.setup_seed(seed)
    r2.insert_slices(sl, rt, w, schedule="scatter")
    o = oracle.OracleVolume(N, "fp32")
    o.insert_iter(sl, rt, w, sym, ref=cref)
    d2, n2 = r2.get_accumulators()
    assert rel(n2, o.norm) < RTOL_ACC and rel(d2, o.data) < RTOL_FFT
    assert r2.determine_slice_agreement(None, None) == 0


def test_agreement_matches_oracle(gpu):
    N, n = 32, 30
    sl, rt = rand_slices(N, n, 71), rand_rots(n, 72)
    w = np.ones(n, np.float32)
    r = recon(N, "gauss_2", "d2")
    r.insert_slices(sl, rt, w)
    got = r.slice_agreement(sl[:5], rt[:5], w[:5], apix=1.0)
    o = oracle_insert(N, sl, rt, w, "gauss_2", "d2")
    for i in range(5):
        want = o.compare(sl[i], rt[i], 1.0, "d2", 1.0)
        np.testing.assert_allclose(got[i], want, rtol=1e-5, atol=1e-6)


def test_seed_setup_matches_reference_rule(gpu):
    """setup_seed: data = seed*w; weights w, halved on x=0 and x=N/2 planes
    except four cells (libEM/reconstructor.cpp:865-895)."""
    from eman2_b200 import Reconstructors
    N = 16
    seed = np.random.default_rng(81).normal(size=(N, N, N + 2)).astype(np.float32)
    r = Reconstructors.get("fourier", {"size": [N] * 3, "sym": "c1"})
    r.setup_seed(seed, 2.5)
    d, nm = r.get_accumulators()
    assert np.array_equal(d, seed * np.float32(2.5))
    want = np.full((N, N, N // 2 + 1), 2.5, np.float32)
    want[:, :, 0] = want[:, :, -1] = 1.25
    for x in (0, N // 2):
        want[0, N // 2, x] = 2.5
        want[N // 2, 0, x] = 2.5
    assert np.array_equal(nm, want)


def test_column_kernel_many_blocks_matches_oracle(gpu):
    """More slices than one slice block: several work items per tile, partial
    sums flushed with atomics.  1280 slices on a 40^3 volume put ~5e4 taps on
    the centre cells, where FP32 summation noise (of the FP32-faithful oracle
    as much as of the GPU) approaches 1e-5.  Against the same taps summed in
    FP64 the GPU's short FP32 chains (small slice blocks near the origin)
    stay within 2e-6."""
    N, n = 40, 160
    sl, rt = rand_slices(N, n, 91), rand_rots(n, 92)
    w = np.random.default_rng(93).uniform(0.5, 1.0, n).astype(np.float32)
    r = recon(N, "gauss_5", "d4")    # 160 x 8 = 1280 slices -> several blocks
    r.insert_slices(sl, rt, w, schedule="gather")
    d, nm = r.get_accumulators()
    o = oracle_insert(N, sl, rt, w, "gauss_5", "d4")
    oa = oracle_insert(N, sl, rt, w, "gauss_5", "d4", "fp32acc64")
    assert np.array_equal(nm != 0, o.norm != 0)
    for got, f32, acc in ((d, o.data, oa.data), (nm, o.norm, oa.norm)):
        assert rel(got, acc) < RTOL_ACC
        # no worse than the reference's own sequential FP32 sum, which on these
        # dense centre cells is itself ~2e-5 from the exact sum
        assert rel(got, acc) <= rel(f32, acc) + 1e-7
        assert rel(got, f32) <= 1.5 * rel(f32, acc) + RTOL_ACC


@pytest.mark.parametrize("sched", ["scatter", "gather"])
@pytest.mark.parametrize("mode", ["gauss_2", "gauss_5", "nearest_neighbor"])
@pytest.mark.parametrize("sym", ["tet", "oct", "icos"])
def test_platonic_symmetry_matches_oracle(gpu, sched, mode, sym):
    """The tetrahedral, octahedral and icosahedral groups (12, 24, 60 copies
    of every slice) through both schedules."""
    N, n = 24, 6
    sl, rt = rand_slices(N, n, 111), rand_rots(n, 112)
    w = np.random.default_rng(113).uniform(0.5, 1.0, n).astype(np.float32)
    r = recon(N, mode, sym)
    assert r.insert_slices(sl, rt, w, schedule=sched) == [0] * n
    d, nm = r.get_accumulators()
    o = oracle_insert(N, sl, rt, w, mode, sym)
    assert np.array_equal(nm != 0, o.norm != 0)
    # 60 copies of every slice into a 24^3 volume: the FP32 order noise of
    # the oracle's own sums grows past RTOL_ACC, so the GPU is held to the
    # same taps summed in FP64, within RTOL_ACC or the FP32 oracle's distance
    oa = oracle_insert(N, sl, rt, w, mode, sym, "fp32acc64")
    for got, want, own in ((nm, oa.norm, o.norm), (d, oa.data, o.data)):
        assert rel(got, want) < max(RTOL_ACC, 2 * rel(own, want))
    m = o.norm != 0
    assert np.max(np.abs(nm[m] - o.norm[m]) / o.norm[m]) < 1e-4


@pytest.mark.parametrize("sched", ["scatter", "gather_column3", "gather_column", "gather_v1"])
def test_gauss5_far_taps_every_cell(gpu, sched):
    """gauss_5 reaches 3.5 voxels on one side of a pixel and 2.5 on the other,
    so a pixel's conjugate taps reach a voxel tile from the other side than
    its direct taps: every cell's weight and normalised value at N = 96, d7,
    against the oracle, including the periphery where only far taps (weights
    down to 1e-9) land."""
    N, n = 96, 24
    sl, rt = rand_slices(N, n, 121), rand_rots(n, 122)
    w = np.random.default_rng(123).uniform(0.5, 1.0, n).astype(np.float32)
    r = recon(N, "gauss_5", "d7")
    if sched != "scatter":
        use_tile(N, "gauss_5", "d7", {"gather_v1": 0, "gather_column": 4, "gather_column3": 5}[sched])
    try:
        r.insert_slices(sl, rt, w, schedule="scatter" if sched == "scatter" else "gather")
    finally:
        use_tile(N, "gauss_5", "d7", -1)
    d, nm = r.get_accumulators()
    o = oracle_insert(N, sl, rt, w, "gauss_5", "d7")
    assert np.array_equal(nm != 0, o.norm != 0)
    m = o.norm != 0
    assert np.max(np.abs(nm[m] - o.norm[m]) / o.norm[m]) < 1e-4
    gd = r.finish(False).numpy()
    want, _ = o.finish(False)
    assert rel(gd, want) < 1e-5


def test_clear_zeroes_and_insertion_continues(gpu):
    """FourierReconstructor::clear (libEM/reconstructor.cpp:999-1020): both
    accumulators zeroed; the handle stays set up and later inserts match a
    fresh reconstruction of only those slices."""
    N, n = 24, 10
    sl, rt = rand_slices(N, n, 131), rand_rots(n, 132)
    w = np.ones(n, np.float32)
    r = recon(N, "gauss_5", "c2")
    r.insert_slices(sl[:5], rt[:5], w[:5])
    d, nm = r.get_accumulators()
    assert np.any(d != 0) and np.any(nm != 0)
    r.clear()
    d, nm = r.get_accumulators()
    assert not np.any(d) and not np.any(nm)
    r.insert_slices(sl[5:], rt[5:], w[5:])
    d, nm = r.get_accumulators()
    o = oracle_insert(N, sl[5:], rt[5:], w[5:], "gauss_5", "c2")
    assert rel(d, o.data) < RTOL_ACC and rel(nm, o.norm) < RTOL_ACC


@pytest.mark.parametrize("doift", [False, True])
def test_sqrtnorm_finish_matches_oracle(gpu, doift):
    """normalize_threed with sqrtnorm (libEM/reconstructor.cpp:377): every
    complex value divided by the square root of its summed weight."""
    N, n = 32, 30
    sl, rt = rand_slices(N, n, 141), rand_rots(n, 142)
    w = np.random.default_rng(143).uniform(0.5, 1.0, n).astype(np.float32)
    r = recon(N, "gauss_2", "d1", sqrtnorm=True)
    r.insert_slices(sl, rt, w)
    out = r.finish(doift).numpy()
    o = oracle_insert(N, sl, rt, w, "gauss_2", "d1")
    want, _ = o.finish(doift, sqrtnorm=True)
    assert rel(out, want) < (RTOL_FFT if doift else RTOL_ACC)
    # and it differs from the plain normalisation
    o2 = oracle_insert(N, sl, rt, w, "gauss_2", "d1")
    plain, _ = o2.finish(doift)
    assert rel(out, plain) > 1e-2


@pytest.mark.parametrize("ret_fourier", [1, 0])
@pytest.mark.parametrize("shift", [(0.0, 0.0), (2.5, -1.25)])
def test_projection_matches_oracle(gpu, ret_fourier, shift):
    """FourierReconstructor::projection (libEM/reconstructor.cpp:1383-1445):
    nearest-voxel slice of the current accumulators at the transform's
    rotation (x=0 and Nyquist columns written Hermitian as the 2-D
    set_complex_at writes them), shifted by its translation, and for
    ret_fourier=0 moved to the centre and inverse transformed."""
    from eman2_b200 import Transform
    N, n = 32, 40
    sl, rt = rand_slices(N, n, 151), rand_rots(n, 152)
    w = np.ones(n, np.float32)
    r = recon(N, "gauss_2", "c1")
    r.insert_slices(sl, rt, w)
    o = oracle_insert(N, sl, rt, w, "gauss_2", "c1")
    for k in range(3):
        rot = rand_rots(1, 160 + k)[0]
        m = np.zeros((3, 4), np.float32)
        m[:, :3] = rot
        m[0, 3], m[1, 3] = shift
        got = r.projection(Transform(m), ret_fourier).numpy()
        want = o.projection(rot, shift[0], shift[1], bool(ret_fourier))
        assert got.shape == ((N, N + 2) if ret_fourier else (N, N))
        assert rel(got, want) < 2e-6 if ret_fourier else rel(got, want) < RTOL_FFT
    # the x=0 column is Hermitian as the reference writes it
    if ret_fourier:
        c = got[:, 0] + 1j * got[:, 1]
        for y in range(1, N // 2):
            assert c[y] == np.conj(c[N - y])


@pytest.mark.parametrize("mode", ["gauss_2", "gauss_5", "nearest_neighbor", "trilinear"])
@pytest.mark.parametrize("NZ", [16, 48])
def test_noncubic_volume_matches_oracle(gpu, mode, NZ):
    """size=[N, N, NZ] (square slices, e.g. programs/e2tomogram.py:2024): the
    z coordinate scaled by NZ, windows clamped to +-NZ/2, the volume
    [NZ][N][N+2]; accumulators, finish(False) and finish(True) against the
    oracle, through the batched call and the plain insert_slice loop."""
    from eman2_b200 import EMData, Transform
    N, n = 32, 12
    sl, rt = rand_slices(N, n, 171), rand_rots(n, 172)
    w = np.random.default_rng(173).uniform(0.5, 1.0, n).astype(np.float32)
    o = oracle.OracleVolume(N, "fp32", NZ=NZ)
    o.insert(sl, rt, w, mode, "c2")
    for form in ("batched", "plain"):
        from eman2_b200 import Reconstructors
        r = Reconstructors.get("fourier", {"size": [N, N, NZ], "sym": "c2", "mode": mode})
        r.setup()
        if form == "batched":
            r.insert_slices(sl, rt, w)
        else:
            for i in range(n):
                img = EMData(sl[i], is_complex=True, attrs={"reconstruct_preproc": 1})
                assert r.insert_slice(img, Transform(rt[i]), float(w[i])) == 0
        d, nm = r.get_accumulators()
        assert d.shape == (NZ, N, N + 2) and nm.shape == (NZ, N, N // 2 + 1)
        assert rel(d, o.data) < RTOL_ACC and rel(nm, o.norm) < RTOL_ACC
        assert np.array_equal(nm != 0, o.norm != 0)
        real = r.finish(True).numpy()
        want, _ = o.copy().finish(True)
        assert real.shape == (NZ, N, N)
        assert rel(real, want) < RTOL_FFT
    r = Reconstructors.get("fourier", {"size": [N, N, NZ], "sym": "c2", "mode": mode})
    r.setup()
    r.insert_slices(sl, rt, w)
    got = r.finish(False).numpy()
    want, _ = o.copy().finish(False)
    assert rel(got, want) < RTOL_ACC


def test_noncubic_volume_refuses_cubic_only_paths(gpu):
    from eman2_b200 import Reconstructors, Transform
    from eman2_b200.batch import BatchReconstructor
    from eman2_b200.exceptions import UnsupportedParameterException
    from eman2_b200.particles import particle_meta
    N, NZ = 32, 16
    r = Reconstructors.get("fourier", {"size": [N, N, NZ], "sym": "c1"})
    r.setup()
    with pytest.raises(UnsupportedParameterException):
        r.projection(Transform(), 1)
    with pytest.raises(UnsupportedParameterException):
        r.slice_agreement(rand_slices(N, 1, 1), rand_rots(1, 2), np.ones(1, np.float32))
    b = BatchReconstructor([{"size": [N, N, NZ], "sym": "c1"}])
    with pytest.raises(UnsupportedParameterException):
        b.insert_particles([np.zeros((2, 24, 24), np.float32)], [particle_meta(rand_rots(2, 3))])
