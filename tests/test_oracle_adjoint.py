"""The per-site transpose used by the discrete adjoint, pinned on the CPU.

oracle/adjoint.py restates the transpose of the SRT update with a body force
that the GPU adjoint kernel applies (tnl-lbm_b200/csrc/adjoint.cuh).  Here it
is checked against
  * the reference's own adjoint collision, D3Q27_SRT_ADJOINT::collision
    (col_srt_adjoint.h:50-109), at rho = 1 and F = 0, where the two agree;
  * the reference's adjoint data term, D3Q27_EQ_ADJOINT::collisionWithData
    (eq_adjoint.h:30-33), which is the gradient of 1/2 [(rho - rho_m)^2 +
    |u - u_m|^2] with respect to the populations;
  * central finite differences of the forward SRT update (checked itself
    against the reference's D3Q27_SRT collision), at rho != 1 and F != 0.
"""
import numpy as np
import pytest

import oracle
from oracle import adjoint as adj

NU = 0.013


def reference():
    if not oracle.reference_available(0):
        pytest.skip("reference harness not built")
    return oracle.Reference(0)


def random_state(rng, n, rho0=1.0, du=0.05, noise=0.01):
    rho = rho0 * (1 + 0.02 * rng.standard_normal(n))
    u = du * rng.standard_normal((n, 3))
    f = adj.feq(rho, u) * (1 + noise * rng.standard_normal((n, 27)))
    return f


def test_forward_update_matches_the_reference_srt_collision():
    ref = reference()
    rng = np.random.default_rng(1)
    f = random_state(rng, 50)
    F = np.array([2e-4, -1e-4, 5e-5])
    out = adj.srt_collide(f, np.tile(F, (50, 1)), NU)
    g = np.ascontiguousarray(f.copy())
    ref.collide(g, coll="SRT", eq="EQ", nu=NU, force=tuple(F))
    np.testing.assert_allclose(out, g, rtol=1e-13, atol=1e-15)


def test_transpose_equals_reference_adjoint_collision_at_unit_density():
    ref = reference()
    rng = np.random.default_rng(2)
    n = 64
    u = 0.05 * rng.standard_normal((n, 3))
    # populations with density 1 and momentum u: equilibrium plus a
    # perturbation orthogonal to the conserved moments
    f = adj.feq(np.ones(n), u)
    p = 0.001 * rng.standard_normal((n, 27))
    M = np.vstack([np.ones(27), adj.CX, adj.CY, adj.CZ]).astype(float)
    p -= (p @ np.linalg.pinv(M)) @ M
    f = f + p
    rho, uu = adj.moments(f, np.zeros((n, 3)))
    np.testing.assert_allclose(rho, 1.0, atol=1e-14)
    lam = rng.standard_normal((n, 27))
    g, _ = adj.srt_vjp(f, np.zeros((n, 3)), NU, lam)
    r = ref.srt_adjoint_collision(lam, uu, NU)
    np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-12)


def test_objective_gradient_equals_reference_data_term():
    ref = reference()
    rng = np.random.default_rng(3)
    n = 40
    f = random_state(rng, n)
    rho, u = adj.moments(f, np.zeros((n, 3)))
    target = np.column_stack([rho + 0.01 * rng.standard_normal(n), u + 0.01 * rng.standard_normal((n, 3))])
    _, gf, _ = adj.objective_gradient(f, np.zeros((n, 3)), target, 1.0)
    macro = np.column_stack([rho, u, target])
    np.testing.assert_allclose(gf, ref.adjoint_data_term(macro), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("rho0,force", [(1.0, 0.0), (1.07, 3e-4), (0.93, -2e-4)])
def test_transpose_against_finite_differences(rho0, force):
    rng = np.random.default_rng(4)
    n = 6
    f = random_state(rng, n, rho0=rho0)
    F = force * rng.standard_normal((n, 3))
    lam = rng.standard_normal((n, 27))
    g, dF = adj.srt_vjp(f, F, NU, lam)
    h = 1e-6
    for j in range(27):
        e = np.zeros(27)
        e[j] = h
        fd = ((lam * adj.srt_collide(f + e, F, NU)).sum(axis=1) - (lam * adj.srt_collide(f - e, F, NU)).sum(axis=1)) / (2 * h)
        np.testing.assert_allclose(g[:, j], fd, rtol=1e-7, atol=1e-9)
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        fd = ((lam * adj.srt_collide(f, F + e, NU)).sum(axis=1) - (lam * adj.srt_collide(f, F - e, NU)).sum(axis=1)) / (2 * h)
        np.testing.assert_allclose(dF[:, a], fd, rtol=1e-7, atol=1e-9)
