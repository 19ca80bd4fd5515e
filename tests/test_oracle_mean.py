"""The reference's running statistics (D3Q27_MACRO_Mean::outputMacro,
macro.h:117-171) in the oracle harness: the moving-average mean and the
Welford-type co-moments equal the two-pass mean and sum of products."""
import numpy as np
import pytest

import oracle


def test_welford_update_matches_two_pass_statistics():
    if not oracle.reference_available(0):
        pytest.skip("reference harness not built")
    ref = oracle.Reference(0)
    rng = np.random.default_rng(0)
    n, K = 500, 40
    v = 0.05 + 0.01 * rng.standard_normal((K, 3, n))
    st = np.zeros((9, n))
    for k in range(K):
        ref.mean_update(np.vstack([np.ones((1, n)), v[k]]), st, k)
    d = v - v.mean(axis=0)
    S = np.einsum("kan,kbn->abn", d, d)
    np.testing.assert_allclose(st[:3], v.mean(axis=0), rtol=0, atol=1e-15)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    for j, (a, b) in enumerate(pairs):
        np.testing.assert_allclose(st[3 + j], S[a, b], rtol=0, atol=1e-15)
