"""The numpy restatement of the D3Q7 scalar operators (oracle/ade.py) against
TNL-LBM's own D3Q7 headers compiled through the reference harness, on CPU."""
import numpy as np
import pytest

from oracle import ade, reference_available

pytestmark = pytest.mark.skipif(not reference_available(), reason="reference harness not built")


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    return Reference(0)


@pytest.mark.parametrize("coll", ["SRT", "MRT", "CLBM"])
def test_collision_matches_reference_headers(ref, coll):
    rng = np.random.default_rng(7)
    n = 500
    phi0 = rng.uniform(0.5, 2.0, n)
    v = rng.uniform(-0.08, 0.08, (n, 3))
    g = ade.feq(phi0, v) * (1 + rng.uniform(-0.05, 0.05, (n, 7)))
    D = 0.0123
    mine, phi = ade.collide(g, v, D, coll)
    theirs = np.ascontiguousarray(g)
    phi_ref = ref.ade_collide(theirs, v, D, coll)
    np.testing.assert_allclose(phi, phi_ref, rtol=1e-15, atol=0)
    np.testing.assert_allclose(mine, theirs, rtol=1e-13, atol=1e-16)
    # the collision conserves phi
    np.testing.assert_allclose(theirs.sum(axis=1), phi_ref, rtol=1e-13)


def test_srt_equilibrium_is_a_fixed_point(ref):
    # (the moment-space collisions relax the second moments towards
    # phi (u_a^2 + c_s^2), which the second-order feq does not carry)
    rng = np.random.default_rng(3)
    phi = rng.uniform(0.5, 2.0, 50)
    v = rng.uniform(-0.05, 0.05, (50, 3))
    g = np.ascontiguousarray(ade.feq(phi, v))
    h = g.copy()
    ref.ade_collide(h, v, 0.05, "SRT")
    np.testing.assert_allclose(h, g, rtol=1e-12, atol=1e-15)


def test_coupled_run_rejects_order_dependent_scalar_sites(ref):
    X, Y, Z = 6, 5, 4
    f = np.ones((27, Z + 2, Y + 2, X + 2)) / 27
    g = np.ones((7, Z + 2, Y + 2, X + 2)) / 7
    m = np.zeros((Z, Y, X), np.int16)
    am = np.zeros((Z, Y, X), np.int16)
    am[:, :, -1] = 8  # GEO_OUTFLOW_RIGHT of d3q7/bc.h
    with pytest.raises(RuntimeError):
        ref.aa_ade_run(f, m, g, am, coll="SRT", eq="EQ")
