"""CPU checks of the accuracy harness's oracle side (oracle/accuracy.py): the
batched prologue equals the per-particle restatement, the task split with
one task is the sequential reconstructor, and the FSC follows the
reference's shell rule."""
from __future__ import annotations

import numpy as np

from oracle import accuracy, oracle


def test_batched_prologue_equals_per_particle():
    from eman2_b200.synth import make_particles
    box, N, n = 24, 36, 10
    ps = make_particles(box, n, seed=3, snr=0.5, shift=3.0, weights=(0.5, 1.0), ctf=True)
    ps.shifts[0] = 0.0                       # the identity-translation branch (copy)
    ps.defocus[1] = 0.0                      # no phase flip
    got = accuracy.slices_from_particles(ps.images, N, ps.shifts, ps.defocus, threads=3, chunk=4)
    for i in range(n):
        want = oracle.particle_to_slice(ps.images[i], N, ps.shifts[i],
                                        {"defocus": float(ps.defocus[i])})
        np.testing.assert_array_equal(got[i], want)


def test_batched_prologue_box_larger_than_pad():
    rng = np.random.default_rng(5)
    imgs = rng.normal(size=(3, 20, 20)).astype(np.float32)
    sh = np.zeros((3, 2), np.float32)
    got = accuracy.slices_from_particles(imgs, 16, sh, None)
    for i in range(3):
        np.testing.assert_array_equal(got[i], oracle.particle_to_slice(imgs[i], 16, sh[i], None))


def test_one_task_is_the_sequential_reconstructor():
    from eman2_b200.synth import quaternion_blocks, random_quaternions
    N, n = 16, 9
    rng = np.random.default_rng(7)
    sl = rng.normal(size=(n, N, N + 2)).astype(np.float32)
    rots = quaternion_blocks(random_quaternions(n, rng))
    w = rng.uniform(0.5, 1, n).astype(np.float32)
    v = oracle.OracleVolume(N, "fp32")
    v.insert(sl, rots, w, "gauss_5", "d2")
    t1 = accuracy.insert_tasks(N, sl, rots, w, "gauss_5", "d2", "fp32", tasks=1)
    np.testing.assert_array_equal(t1.data, v.data)
    np.testing.assert_array_equal(t1.norm, v.norm)
    # three tasks: the same sums in another order
    t3 = accuracy.insert_tasks(N, sl, rots, w, "gauss_5", "d2", "fp32", tasks=3)
    assert oracle.rel_l2(t3.data, v.data) < 1e-6
    manual = [oracle.OracleVolume(N, "fp32") for _ in range(3)]
    for t in range(3):
        idx = np.arange(t, n, 3)
        manual[t].insert(sl[idx], rots[idx], w[idx], "gauss_5", "d2")
    np.testing.assert_array_equal(t3.data, manual[0].data + manual[1].data + manual[2].data)


def _fsc_loop(d1, d2):
    """calc_fourier_shell_correlation (libEM/sparx/emdata_sparx.cpp:945-983) as
    loops, w = 1: float shell index, double sums, Friedel half skipped."""
    f32 = np.float32
    nz, ny, lsd2 = d1.shape
    nx = lsd2 - 2
    nx2, ny2, nz2 = nx // 2, ny // 2, nz // 2
    dx2 = f32(1.0) / f32(nx2) / f32(nx2)
    dy2 = f32(1.0) / f32(ny2) / f32(ny2)
    dz2 = f32(1.0) / f32(max(nz2, 1)) / f32(max(nz2, 1))
    inc = nx2
    ret, n1, n2 = np.zeros(inc + 1), np.zeros(inc + 1), np.zeros(inc + 1)
    for iz in range(nz):
        kz = iz - nz if iz > nz2 else iz
        argz = f32(kz * kz) * dz2
        for iy in range(ny):
            ky = iy - ny if iy > ny2 else iy
            argy = f32(argz + f32(ky * ky) * dy2)
            for ix in range(0, lsd2, 2):
                if ix > 0 or (kz >= 0 and (ky >= 0 or kz != 0)):
                    argx = f32(0.5) * np.sqrt(f32(argy + f32(f32(ix * ix) * f32(0.25)) * dx2))
                    t = f32(inc * 2) * f32(argx)
                    r = int(t + f32(0.5))
                    if r <= inc:
                        a, b = d1[iz, iy, ix:ix + 2].astype(float), d2[iz, iy, ix:ix + 2].astype(float)
                        ret[r] += a[0] * b[0] + a[1] * b[1]
                        n1[r] += a[0] * a[0] + a[1] * a[1]
                        n2[r] += b[0] * b[0] + b[1] * b[1]
    return ret / np.sqrt(n1 * n2)


def test_fsc_shell_rule():
    rng = np.random.default_rng(9)
    N = 20
    a = rng.normal(size=(N, N, N + 2)).astype(np.float32)
    f = accuracy.fsc(a, a)
    assert f.shape == (N // 2 + 1,)
    np.testing.assert_allclose(f, 1.0, rtol=1e-12)
    b = a + 0.1 * rng.normal(size=a.shape).astype(np.float32)
    np.testing.assert_allclose(accuracy.fsc(a, b), _fsc_loop(a, b), rtol=1e-12)
    # a volume against its negation: -1 everywhere but the empty shells
    assert np.all(accuracy.fsc(a, -a) < -0.999999)


def test_compare_and_report():
    rng = np.random.default_rng(11)
    N = 12
    d = rng.normal(size=(N, N, N + 2))
    n = rng.uniform(0.5, 1, size=(N, N, N // 2 + 1))
    rep = accuracy.report({"x": (d * (1 + 1e-7), n)}, (d, n), (d, n))
    assert rep["x"]["vs_fp32_oracle"]["rel_l2_complex"] < 2e-7
    assert rep["x"]["vs_fp64_oracle"]["rel_l2_weight"] == 0.0
    assert rep["fp32_oracle_vs_fp64"]["fsc_min"] == 1.0
