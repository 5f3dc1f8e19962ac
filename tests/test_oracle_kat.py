"""Known-answer tests of the CPU oracle: exact taps of a
single pixel, Hermitian duplicates on the x=0 plane, insert-then-remove,
dihedral operators, reconstruction conventions (a blob lands where it was
projected; noiseless projections reproduce the phantom), agreement of a
slice with itself."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import oracle


def test_fast_exp_table_and_index_rule():
    lib = oracle._lib()
    for f, g in [(0.0, 0), (-0.0101, 1), (-0.0099, 0), (-0.01, 0), (-1.0, 50), (-19.98, 999)]:
        # -0.01f is 0.00999999977...: -f*50+0.5 stays below 1, entry 0
        assert lib.or_fast_exp_value(f) == np.float32(math.exp(-g / 50.0))
    # outside the table: exp()
    assert lib.or_fast_exp_value(-20.5) == np.float32(math.exp(-20.5))


def test_single_pixel_gauss2_taps_exact():
    """A pixel at an integer point (3,2,1): 8 taps, the centre tap with the
    table's exp(0) = 1 and the others with exp(-round(50*h*r^2)/50)."""
    N = 16
    v = oracle.OracleVolume(N, "fp32")
    v.insert_pixels("gauss_2", np.array([[3, 2, 1, 1.0, 0.5, 1.0]], np.float32))
    nz = np.argwhere(v.norm != 0)
    assert len(nz) == 8
    h = np.float32(1.0) / np.float32(4.0 / (math.pi * math.pi))
    for z, y, x in nz:
        r = (x - 3) ** 2 + (y - 2) ** 2 + (z - 1) ** 2
        f = np.float32(-np.float32(r) * h)
        g = int(-float(f) * 50.0 + 0.5)
        assert v.norm[z, y, x] == np.float32(math.exp(-g / 50.0))
        assert v.data[z, y, 2 * x] == v.norm[z, y, x]
        assert v.data[z, y, 2 * x + 1] == np.float32(0.5) * v.norm[z, y, x]


def test_x0_plane_hermitian_duplicates():
    """Nearest insert at (0,3,2): conjugate at (0,-3,-2), direct at (0,3,2),
    weight only at the direct cell (libEM/emdata_core.h:375-386)."""
    N = 16
    v = oracle.OracleVolume(N, "fp32")
    v.insert_pixels("nearest_neighbor", np.array([[0, 3, 2, 1.5, 0.25, 2.0]], np.float32))
    assert v.data[2, 3, 0] == 3.0 and v.data[2, 3, 1] == 0.5
    assert v.data[N - 2, N - 3, 0] == 3.0 and v.data[N - 2, N - 3, 1] == -0.5
    assert v.norm[2, 3, 0] == 2.0 and v.norm[N - 2, N - 3, 0] == 0.0
    # origin: real part only, imaginary part forced to 0
    v2 = oracle.OracleVolume(N, "fp32")
    v2.insert_pixels("nearest_neighbor", np.array([[0, 0, 0, 1.0, 7.0, 1.0]], np.float32))
    assert v2.data[0, 0, 0] == 1.0 and v2.data[0, 0, 1] == 0.0


def test_nyquist_minus_side_adds_conjugate_twice():
    """x = -(N/2): the conjugate lands twice on the same cell
    (libEM/emdata_core.h:387-403 then :397-403)."""
    N = 16
    v = oracle.OracleVolume(N, "fp32")
    v.insert_pixels("nearest_neighbor", np.array([[-8, 2, 1, 1.0, 1.0, 1.0]], np.float32))
    cell = v.data[N - 1, N - 2, 2 * 8: 2 * 8 + 2]
    assert cell[0] == 2.0 and cell[1] == -2.0
    assert v.norm[N - 1, N - 2, 8] == 1.0


def test_insert_then_remove_is_zero():
    """The intent of the reference's disabled notest_insert_remove
    (rt/pyem/test_reconstructor.py:48-90), through the inserter directly (a
    negative insert_slice weight selects the SSNR path instead): +w then -w
    leaves ~0."""
    N = 24
    rng = np.random.default_rng(3)
    px = np.empty((500, 6), np.float32)
    px[:, :3] = rng.uniform(-10, 10, (500, 3))
    px[:, 3:5] = rng.normal(size=(500, 2))
    px[:, 5] = 1.0
    neg = px.copy()
    neg[:, 5] = -1.0
    for mode in ("nearest_neighbor", "gauss_2", "gauss_5"):
        v = oracle.OracleVolume(N, "fp32")
        v.insert_pixels(mode, px)
        v.insert_pixels(mode, neg)
        assert np.abs(v.data).max() < 1e-5 and np.abs(v.norm).max() < 1e-5


def test_negative_weight_needs_class_ssnr():
    """do_insert_slice_work with weight < 0 reads class_ssnr; without it the
    oracle (like the reference) refuses."""
    N = 16
    v = oracle.OracleVolume(N, "fp32")
    with pytest.raises(RuntimeError):
        v.insert(np.zeros((1, N, N + 2), np.float32), np.eye(3, dtype=np.float32)[None],
                 -np.ones(1, np.float32))


def test_dihedral_operators():
    """DSym::get_sym (libEM/symmetry.cpp:1452-1470): d1 = {identity, alt 180}."""
    ops = oracle.sym_ops("d1")
    assert ops.shape == (2, 3, 3)
    np.testing.assert_allclose(ops[0], np.eye(3), atol=1e-7)
    np.testing.assert_allclose(ops[1], np.diag([1.0, -1.0, -1.0]), atol=1e-7)
    d7 = oracle.sym_ops("d7")
    assert d7.shape == (14, 3, 3)
    for m in d7:
        np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-6)
    # c4: rotations about z by multiples of 90 degrees
    c4 = oracle.sym_ops("c4")
    np.testing.assert_allclose(c4[1], [[0, 1, 0], [-1, 0, 0], [0, 0, 1]], atol=1e-7)


def _reconstruct(ps, N, mode="gauss_2", sym="c1"):
    sl = np.stack([oracle.particle_to_slice(ps.images[i], N, ps.shifts[i]) for i in range(len(ps.images))])
    v = oracle.OracleVolume(N, "fp32")
    v.insert(sl, ps.rots, ps.weights, mode, sym)
    return v


def test_blob_lands_where_it_was_projected():
    """One off-centre Gaussian: the map's peak is at its centre (index and
    orientation conventions of projection, slice and volume agree)."""
    from eman2_b200.synth import Phantom, make_particles
    box, N = 24, 36
    ph = Phantom(np.array([[4.0, -3.0, 2.0]]), np.array([2.0]), np.array([1.0]))
    ps = make_particles(box, 300, seed=5, snr=1e6, shift=2.0, phantom=ph)
    real, _ = _reconstruct(ps, N).finish(True)
    z, y, x = np.unravel_index(np.argmax(real), real.shape)
    assert (x - N // 2, y - N // 2, z - N // 2) == (4, -3, 2)


def test_noiseless_projections_reproduce_phantom():
    """FSC between the reconstruction and the phantom stays high up to 0.6
    Nyquist.  finish() applies no interpolation-kernel correction (the
    reference's callers apply math.gausskernelfix afterwards,
    programs/e2make3dpar.py:421-428), so the map is the phantom times the
    gauss_2 kernel's real-space profile: shells correlate at ~0.95-0.999."""
    from eman2_b200.synth import make_particles, phantom_volume
    box, N = 24, 36
    ps = make_particles(box, 1500, seed=9, snr=1e6, shift=1.0)
    v = _reconstruct(ps, N)
    real, _ = v.finish(True)
    ref = np.zeros((N, N, N), np.float32)
    o = (N - box) // 2
    ref[o:o + box, o:o + box, o:o + box] = phantom_volume(ps.phantom, box)
    fa = np.fft.rfftn(real.astype(np.float64)).astype(np.complex64)
    fb = np.fft.rfftn(ref.astype(np.float64)).astype(np.complex64)
    fsc = oracle.fsc(fa.view(np.float32).reshape(N, N, N + 2), fb.view(np.float32).reshape(N, N, N + 2))
    assert (fsc[1: int(0.6 * N / 2)] > 0.93).all(), fsc
    assert fsc[1] > 0.995


def test_agreement_of_slice_with_itself():
    """A volume built from one smooth slice agrees with that slice: absqual ~ 1
    (nearest-neighbour cells average the few pixels that land in them)."""
    N = 32
    ax = np.arange(N) - N // 2
    yy, xx = np.meshgrid(ax, ax, indexing="ij")
    img = (np.exp(-((xx - 3) ** 2 + (yy + 2) ** 2) / 18.0)
           + 0.5 * np.exp(-((xx + 5) ** 2 + (yy - 4) ** 2) / 8.0)).astype(np.float32)
    sl = oracle.preprocess_slice(img)
    rot = oracle.eman_matrix(20.0, 30.0, 40.0)
    v = oracle.OracleVolume(N, "fp32")
    v.insert(sl[None], rot[None], np.ones(1, np.float32), "nearest_neighbor", "c1")
    out = v.compare(sl, rot, 1.0, "c1", 1.0)
    assert out[1] > 0.9, out
    assert abs(out[0] - 1.0) < 0.1, out       # reconstruct_norm


def test_fp32_and_fp64_oracles_agree():
    N, n = 24, 10
    rng = np.random.default_rng(17)
    sl = rng.normal(size=(n, N, N + 2)).astype(np.float32)
    from eman2_b200.synth import quaternion_blocks, random_quaternions
    rt = quaternion_blocks(random_quaternions(n, rng))
    w = np.ones(n, np.float32)
    a, b, c = (oracle.OracleVolume(N, k) for k in ("fp32", "fp32acc64", "fp64"))
    for v in (a, b, c):
        v.insert(sl, rt, w, "gauss_5", "c2")
    assert oracle.rel_l2(a.data, b.data) < 2e-6      # summation order only
    assert oracle.rel_l2(b.data, c.data) < 1e-4      # FP32 vs FP64 tap arithmetic


def test_kernel_fix_known_values():
    """math.gausskernelfix (libEM/processor.h:4131-4176): the voxel at
    (floor(nx/2), floor(ny/2), floor(nz/2)) is unchanged; a voxel at squared
    distance d is multiplied by exp(d * gauss_width / ny^2), with ny (not nx
    or nz) in the width's scale."""
    v = np.ones((6, 8, 10), np.float32)          # nz, ny, nx
    out = oracle.kernel_fix(v, 4.0)
    assert out[3, 4, 5] == 1.0
    sv = np.float32(4.0) / np.float32(64)
    for (z, y, x) in [(3, 4, 6), (0, 0, 0), (5, 7, 9), (3, 1, 5)]:
        d = np.float32((x - 5) ** 2 + (y - 4) ** 2 + (z - 3) ** 2)
        assert out[z, y, x] == np.float32(1.0 / math.exp(float(np.float32(-d * sv))))
    c = oracle.clip_centre(np.arange(8 * 8 * 8, dtype=np.float32).reshape(8, 8, 8), (4, 6, 2))
    assert c.shape == (2, 6, 4) and c[0, 0, 0] == 3 * 64 + 1 * 8 + 2


def test_wiener_pixel_weight_and_disk():
    """WienerFourierReconstructor (libEM/reconstructor.cpp:1679-1731): each
    pixel of an identity-oriented slice adds, at its own voxel (nearest), the
    SNR curve interpolated at rn = |(x, y)|/N * 2*len as weight; pixels at
    rn >= .5 add nothing; the Wiener finish divides by weight + 1."""
    N = 16
    snr = np.linspace(4.0, 1.0, 8).astype(np.float32)          # 8 entries
    for (x, y) in [(3, 2), (0, 5), (6, -3), (7, 4)]:
        sl = np.zeros((N, N + 2), np.float32)
        sl[y % N, 2 * x] = 1.0
        v = oracle.OracleVolume(N, "fp32")
        v.insert_wiener(sl[None], np.eye(3, dtype=np.float32)[None], np.ones(1, np.float32),
                        snr[None], mode="nearest_neighbor")
        rx, ry = np.float32(x) / np.float32(N), np.float32(y) / np.float32(N)
        rn = np.float32(math.hypot(rx, ry))
        if rn >= 0.5:                      # every disk pixel adds its weight; this one is outside
            assert v.norm[0, y % N, x] == 0.0
            continue
        rn = np.float32(rn * np.float32(16.0))
        k = int(math.floor(rn))
        t = np.float32(rn - np.float32(k))
        want = np.float32((np.float32(1) - t) * snr[k] + t * snr[k + 1])
        got = v.norm[0, y % N, x]          # volumes are [z][y][x]; identity: voxel (x, y, 0)
        assert got == want
        d = v.data[0, y % N, 2 * x]
        v.normalize(wiener=True)
        if x:
            assert v.data[0, y % N, 2 * x] == np.float32(d / (want + np.float32(1)))


def test_iter_first_pass_width_and_x_clamp():
    """FourierIterReconstructor without a reference (libEM/reconstructor.cpp:609-628):
    taps weighted by fast_exp(-r * h), h = 1/(|p|^2/4000 + .15); the window is
    clamped to |x| <= N/2 - 1 but |y|, |z| <= N/2."""
    N = 16
    sl = np.zeros((N, N + 2), np.float32)
    sl[2, 2 * 3] = 1.0                                   # pixel (3, 2) -> point (3, 2, 0)
    v = oracle.OracleVolume(N, "fp32")
    v.insert_iter(sl[None], np.eye(3, dtype=np.float32)[None], np.ones(1, np.float32))
    hs = np.float32(9 + 4)
    h = np.float32(1.0 / (float(hs / np.float32(4000)) + 0.15))
    for (i, j, k) in [(3, 2, 0), (4, 2, 1), (3, 3, -1)]:      # taps inside the exp table
        r = np.float32((i - 3) ** 2 + (j - 2) ** 2 + k ** 2)
        g = int(-float(np.float32(-r * h)) * 50.0 + 0.5)
        want = np.float32(math.exp(-g / 50.0))
        assert v.data[k % N, j % N, 2 * i] == want                  # the pixel's value * gg
    # a pixel near x = N/2: no tap at x = N/2 (nx2 = N/2 - 1), taps at y = -N/2 kept
    sl2 = np.zeros((N, N + 2), np.float32)
    v2 = oracle.OracleVolume(N, "fp32")
    v2.insert_iter(sl2[None], np.eye(3, dtype=np.float32)[None], np.ones(1, np.float32))
    assert v2.norm[:, :, N // 2].max() == 0.0
    assert v2.norm[:, N // 2, :].max() > 0.0


def test_iter_reference_update_rule():
    """With a reference volume the value inserted is dt + ref(i,j,k) - ref(p)
    (ref(p) trilinear): a slice equal to the reference's section through a
    constant reference inserts dt (the update terms cancel), weights
    unchanged by the reference."""
    N = 16
    ref = np.zeros((N, N, N + 2), np.float32)
    ref[..., 0::2] = 2.0                                # constant real reference
    sl = np.zeros((N, N + 2), np.float32)
    sl[1, 2 * 2] = 1.0
    a = oracle.OracleVolume(N, "fp32")
    a.insert_iter(sl[None], np.eye(3, dtype=np.float32)[None], np.ones(1, np.float32), ref=ref)
    b = oracle.OracleVolume(N, "fp32")
    b.insert_iter(sl[None], np.eye(3, dtype=np.float32)[None], np.ones(1, np.float32), ref=ref * 0)
    # interior cells: the constant reference cancels; radius > N/2 cells are skipped in both
    np.testing.assert_allclose(a.data, b.data, atol=1e-6)
    np.testing.assert_array_equal(a.norm, b.norm)


@pytest.mark.parametrize("N", [16, 20])
def test_normalize_weights_conjugate_pairs(N):
    """normalize_threed sums conjugate-pair weights on the x=0 and x=N/2
    planes and doubles five cells (libEM/reconstructor.cpp:339-364)."""
    v = oracle.OracleVolume(N, "fp64")
    rng = np.random.default_rng(N)
    v.norm[:] = rng.uniform(1, 2, v.norm.shape)
    before = v.norm.copy()
    v.normalize()
    h = N // 2
    # (0, y, z) and (0, -y, -z) hold the same summed weight
    for (y, z) in [(1, 2), (3, -1), (h - 1, 1)]:
        a = v.norm[z % N, y % N, 0]
        b = v.norm[(-z) % N, (-y) % N, 0]
        assert a == b == before[z % N, y % N, 0] + before[(-z) % N, (-y) % N, 0]
    assert v.norm[h, 0, 0] == 2 * before[h, 0, 0]
    assert v.norm[0, h, h] == 2 * before[0, h, h]
