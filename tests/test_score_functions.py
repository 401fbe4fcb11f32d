"""neurogpu_b200.score_functions against the reference's own
GUI/score_functions.py outputs (tests/golden/score_vectors.npz, made by
tests/golden/make_score_golden.py from the reference module on oracle traces
of the shipped TTPC model).  Bound: 1e-12 relative (the restatement keeps the
reference's operation order; numpy's vectorised forms may round the last bit
differently)."""
from pathlib import Path

import numpy as np
import pytest

from neurogpu_b200 import score_functions as sf

Z = np.load(Path(__file__).resolve().parent / "golden" / "score_vectors.npz")
NAMES = [str(n) for n in Z["names"]]


@pytest.mark.parametrize("name", NAMES)
def test_matches_reference_module(name):
    f = getattr(sf, name)
    want = Z["scores"][NAMES.index(name)]
    t = Z["target"]
    for j, d in enumerate(Z["data"]):
        if np.isnan(want[j]):
            with pytest.raises(Exception):
                f(list(t), list(d), 0.1)
            continue
        for args in ((list(t), list(d)), (t, d)):
            got = float(f(*args, 0.1))
            assert got == pytest.approx(want[j], rel=1e-12, abs=1e-12), (name, j, got, want[j])


@pytest.mark.parametrize("name", NAMES)
def test_batch_matches_single(name):
    want = Z["scores"][NAMES.index(name)]
    ok = ~np.isnan(want)
    got = sf.score_batch(name, Z["target"], Z["data"][ok], 0.1)
    np.testing.assert_allclose(got, want[ok], rtol=1e-12, atol=1e-12)


def test_dtw_matches_plain_recursion():
    """The anti-diagonal DTW against the textbook double loop on a small case."""
    rng = np.random.default_rng(4)
    a, b = rng.normal(size=17), rng.normal(size=13)
    D = np.full((18, 14), np.inf)
    D[0, 0] = 0
    for i in range(1, 18):
        for j in range(1, 14):
            D[i, j] = abs(a[i - 1] - b[j - 1]) + min(D[i - 1, j], D[i, j - 1], D[i - 1, j - 1])
    assert sf.DTWDistance(a, b) == D[16, 12] / 17
