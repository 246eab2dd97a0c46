"""The Hogbom CLEAN oracle pinned against the reference (CPU only).

tconvolve_oracle_hogbom.c restates current/tHogbomCleanOMP/HogbomGolden.cc; these tests check its
model and residual bit for bit (sha256) against the reference's own outputs recorded in
tests/golden/hogbom.json (generator: tests/golden/make_golden_hogbom.py), and the edge cases the
reference's code defines (ties, all-zero images, the threshold stop, the PSF row quirk).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN_DIR, sha

sys.path.insert(0, GOLDEN_DIR)
from make_golden_hogbom import cases  # noqa: E402


@pytest.fixture(scope="module")
def hog_golden():
    with open(os.path.join(GOLDEN_DIR, "hogbom.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["w128", "w256", "w100", "w128_psf256", "stop"])
def test_hogbom_oracle_bit_exact(orc, hog_golden, name):
    dirty, psf = cases()[name]
    ref = hog_golden["cases"][name]
    assert sha(dirty) == ref["sha256"]["dirty"] and sha(psf) == ref["sha256"]["psf"], "input generator drifted"
    p = hog_golden["params"]
    r = orc.hogbom(dirty, psf, p["niters"], p["gain"], p["threshold"])
    assert sha(r["model"]) == ref["sha256"]["model"]
    assert sha(r["residual"]) == ref["sha256"]["residual"]
    assert r["skipped_rows"] == 0
    if name == "stop":
        assert 0 < r["stopped_at"] < p["niters"] and r["done"] == r["stopped_at"]
    else:
        assert r["done"] == p["niters"]


def test_find_peak_rules(orc):
    """Strict '>' on |value| in index order (HogbomGolden.cc:131-137): the first of equal
    magnitudes wins, a negative value keeps its sign, an all-zero image gives (0, 0)."""
    a = np.zeros(100, np.float32)
    assert orc.find_peak(a) == (0.0, 0)
    a[[7, 30, 60]] = [-2.0, 2.0, 1.5]
    assert orc.find_peak(a) == (-2.0, 7)
    a[3] = 2.0
    assert orc.find_peak(a) == (2.0, 3)


def test_psf_row_quirk(orc):
    """subtractPSF takes the PSF row as y - (ry - px) (HogbomGolden.cc:108).  With the PSF peak on
    the diagonal this is the plain shift; off it, the oracle skips the rows that fall outside the
    PSF (the reference reads out of bounds there) and counts them."""
    w = 32
    psf = np.zeros((w, w), np.float32)
    psf[16, 16] = 1.0
    psf[16, 17] = 0.5
    res = np.zeros(w * w, np.float32)
    res[10 * w + 12] = 4.0
    skipped = orc.lib().orc_subtract_psf(orc._p(psf.ravel()), w, orc._p(res), w, 10 * w + 12, 16 * w + 16,
                                         np.float32(4.0), np.float32(0.1))
    assert skipped == 0
    assert res[10 * w + 12] == np.float32(4.0) - np.float32(np.float32(0.1) * np.float32(4.0))
    assert res[10 * w + 13] == -np.float32(np.float32(0.1 * np.float32(4.0)) * np.float32(0.5))
    psf2 = np.zeros((w, w), np.float32)
    psf2[8, 20] = 1.0  # peak off the diagonal: px = 20, py = 8
    res2 = np.zeros(w * w, np.float32)
    skipped = orc.lib().orc_subtract_psf(orc._p(psf2.ravel()), w, orc._p(res2), w, 5 * w + 5, 8 * w + 20,
                                         np.float32(1.0), np.float32(0.1))
    # rows y = 0 .. 28 map to PSF rows y - (5 - 20) = y + 15: rows 17..28 fall outside the PSF
    assert skipped == 12
