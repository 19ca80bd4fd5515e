"""Running velocity statistics (lbm_set_statistics, D3Q27_MACRO_Mean) on the
GPU against the reference's own update (oracle Reference.mean_update) applied
to the macro field of every step."""
import numpy as np
import pytest

import oracle
from helpers import GEO, duct_map, rel_linf, seeded_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


@pytest.mark.parametrize("storage,dtype,tol", [("F64", np.float64, 1e-12), ("F32", np.float32, 1e-5)])
def test_statistics_match_the_reference_update(pl, port, storage, dtype, tol):
    if not oracle.reference_available(0):
        pytest.skip("reference harness not built")
    ref = oracle.Reference(0)
    X, Y, Z = 30, 10, 9
    rng = np.random.default_rng(3)
    lat = pl.LBM(X, Y, Z, viscosity=0.01, storage=getattr(pl, "STORE_" + storage))
    lat.set_map(duct_map(X, Y, Z))
    lat.set_inflow(0.03 * np.ones((Z, Y)), None, None)
    lat.set_populations(seeded_state(port, rng, X, Y, Z).astype(dtype))
    lat.set_statistics(True)
    n = X * Y * Z
    st = np.zeros((9, n), dtype)
    K = 12
    for k in range(K):
        lat.step(1)
        m = lat.macro().astype(dtype).reshape(4, n)
        ref.mean_update(m, st, k)
    mean, cov, count = lat.statistics()
    assert count == K
    assert rel_linf(mean.reshape(3, n), st[:3]) <= tol
    assert rel_linf(cov.reshape(6, n) * K, st[3:]) <= tol * 10
    lat.close()


def test_one_call_equals_single_steps(pl, port):
    X, Y, Z = 24, 10, 8
    out = []
    for split in (False, True):
        rng = np.random.default_rng(4)
        lat = pl.LBM(X, Y, Z, viscosity=0.01)
        lat.set_map(duct_map(X, Y, Z, GEO["INFLOW"], GEO["OUTFLOW_EQ"]))
        lat.set_inflow(0.03 * np.ones((Z, Y)), None, None)
        lat.set_populations(seeded_state(port, rng, X, Y, Z).astype(np.float32))
        lat.set_statistics(True)
        if split:
            for _ in range(9):
                lat.step(1)
        else:
            lat.step(9, sums=True)
        out.append(lat.statistics())
        lat.set_statistics(False)
        with pytest.raises(pl.LbmError):
            lat.statistics()
        lat.close()
    assert out[0][2] == out[1][2] == 9
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
