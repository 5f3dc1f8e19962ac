"""Accuracy at the configurations' own sizes: the plain and batched GPU forms
against the oracle fed the same seeded raw particles.

Bar: relative L2 <= 1e-5 on the normalised complex volume (finish(False)) and
on the weight volume (normout) against the FP32-faithful oracle, and FSC >=
0.9999 in every shell (the reference's shell rule).  Against the FP64 oracle
the GPU is required to be no further than the FP32 oracle itself is (times
two, plus 1e-6 for the cuFFT/pocketfft boundary): the error that remains is
FP32 arithmetic the reference shares.  Against the oracle that makes the
same FP32 taps and adds them in FP64 (summation order removed) the GPU is
within the same 1e-5.

The reports are printed as JSON (``pytest -s`` shows them).
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from tests import accuracy_harness as H

pytestmark = pytest.mark.gpu

RTOL = 1e-5
FSC_MIN = 0.9999


def _check(rep: dict, label: str):
    print(f"\naccuracy {label}: " + json.dumps(rep, default=float))
    own = rep["fp32_oracle_vs_fp64"]
    forms = [k for k, v in rep.items() if isinstance(v, dict) and "vs_fp32_oracle" in v]
    assert forms
    for k in forms:
        a, b = rep[k]["vs_fp32_oracle"], rep[k]["vs_fp64_oracle"]
        assert a["rel_l2_complex"] <= RTOL, (k, a)
        assert a["rel_l2_weight"] <= RTOL, (k, a)
        assert a["fsc_min"] >= FSC_MIN, (k, a)
        assert a["support_mismatch"] == 0, (k, a)
        assert b["fsc_min"] >= FSC_MIN, (k, b)
        assert b["rel_l2_complex"] <= 2 * own["rel_l2_complex"] + 1e-6, (k, b, own)
        assert b["rel_l2_weight"] <= 2 * own["rel_l2_weight"] + 1e-6, (k, b, own)
        e = rep[k]["vs_exact_sums"]
        assert e["rel_l2_complex"] <= RTOL and e["rel_l2_weight"] <= RTOL, (k, e)


def test_c1_full(gpu):
    """Box 64 padded to 96, 2,000 particles, gauss_2, c1 (every particle)."""
    rep = H.run_case("c1", gpu)
    assert rep["case"]["particles"] == 2000
    _check(rep, "c1")


def test_c2_full_with_agreement(gpu):
    """Box 128 padded to 192, 20,000 particles, gauss_2, c1, CTF, plus the
    agreement pass (sub=False) on 512 of the slices against the full volume."""
    rep = H.run_case("c2", gpu)
    assert rep["case"]["particles"] == 20000
    _check(rep, "c2")
    assert rep["agreement_max_rel_diff"] < 1e-4


def test_c4_subsample_with_agreement(gpu):
    """Box 256 padded to 384, gauss_5, d7, CTF: 64 particles (896 slices in
    one launch of the column kernel), agreement on 32 slices."""
    rep = H.run_case("c4", gpu)
    _check(rep, "c4 (64-particle subsample)")
    assert rep["agreement_max_rel_diff"] < 1e-4


def test_c4g2_two_buckets_both_gather_kernels(gpu):
    """Box 256 padded to 384, gauss_2, d7: 320 particles = 4,480 slices, so the
    work order spans two slice buckets; the pixel-major and the column kernel
    each against the oracle."""
    rep = H.run_case("c4g2", gpu, forms=("batched",))
    assert "batched_pixel" in rep and "batched_column" in rep
    _check(rep, "c4g2 (320 particles, two buckets)")


def test_batched_graph_pairs(gpu):
    """Even/odd half-map pairs of two phantoms (box 64 gauss_5 d7, box 160
    gauss_2 c1), four reconstructions inserted by one CUDA-graph replay."""
    out = H.graph_case(gpu)
    assert len(out["jobs"]) == 4
    for rep in out["jobs"]:
        _check(rep, f"graph job {rep['job']}")


def test_c4_full_launch_column_kernel_vs_fp64_partials(gpu):
    """The full 2,048-particle launch of the large job (box 256 padded to 384,
    gauss_5, d7: 28,672 slices over seven slice buckets) through the column
    kernel, against the same particles through the register-tile gather,
    which keeps every voxel's sum over all slices in FP64 (pinned to the
    oracle at small sizes): the column kernel's blocked FP32 sums within
    1e-5.  The scatter (plain form) is reported beside it: with ~10^6 FP32
    atomic adds on the cells near the origin its own order noise is ~1e-4,
    the level a sequential FP32 sum reaches too."""
    from eman2_b200.batch import set_tile
    from oracle import accuracy
    c = dict(H.CASES["c4"])
    ps, meta = H.render(c, gpu, 2048)
    res = {}
    for name, tile, sched in (("column", -1, "gather"), ("fp64_partials", 0, "gather"),
                              ("scatter", -1, "scatter")):
        r = H._recon(c)
        if tile != -1:
            set_tile(c["N"], c["mode"], 14, tile)
        try:
            r.insert_particles(ps.images, meta, schedule=sched)
            res[name] = H._finish(r)
        finally:
            if tile != -1:
                set_tile(c["N"], c["mode"], 14, -1)
            r.close()
    ref = res["fp64_partials"]
    col = accuracy.compare(*res["column"], *ref)
    sca = accuracy.compare(*res["scatter"], *ref)
    print("\naccuracy c4 2048 column vs fp64 partials: " + json.dumps(col))
    print("accuracy c4 2048 scatter vs fp64 partials: " + json.dumps(sca))
    assert col["rel_l2_complex"] <= RTOL and col["rel_l2_weight"] <= RTOL
    assert col["fsc_min"] >= FSC_MIN and col["support_mismatch"] == 0
    assert sca["fsc_min"] >= FSC_MIN and sca["support_mismatch"] == 0


def test_c4g2_full_launch_vs_exact_sums(gpu):
    """Box 256 padded to 384, gauss_2, d7: one 2,048-particle launch (28,672
    slices, seven buckets) through both gather kernels, against the oracle
    that makes the same FP32 taps and adds them in FP64."""
    rep = H.run_case("c4g2", gpu, n=2048, forms=("batched",), tasks=16)
    print("\naccuracy c4g2 2048: " + json.dumps(rep, default=float))
    for k in ("batched_pixel", "batched_column"):
        e = rep[k]["vs_exact_sums"]
        assert e["rel_l2_complex"] <= RTOL and e["rel_l2_weight"] <= RTOL, (k, e)
        assert e["fsc_min"] >= FSC_MIN and e["support_mismatch"] == 0, (k, e)
        assert rep[k]["vs_fp64_oracle"]["fsc_min"] >= FSC_MIN
