"""The discrete adjoint (lbm_adjoint_* of the C-ABI) on the GPU.

The adjoint transposes every A-A step exactly, so in FP64 its gradients must
equal central finite differences of the objective to the differencing error
(relative 1e-6 here).  With FP32 storage the adjoint populations stay FP64,
and the gradient agrees with the FP64 run's to 1e-4.  Checked for the force control and for the initial
populations, on a duct with walls, a velocity inlet (GEO_INFLOW) and a
fixed-density outlet (GEO_OUTFLOW_EQ), on symmetry planes and on a periodic
box; the checkpoint interval must not change the result; the forward pass
with a uniform force is the production SRT step.  The per-site transpose
itself is pinned on the CPU to the reference's adjoint collision
(tests/test_oracle_adjoint.py).
"""
import numpy as np
import pytest

from helpers import GEO, duct_map, rel_linf, seeded_state

pytestmark = pytest.mark.gpu

NU = 0.04
X, Y, Z = 20, 10, 9


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def channel(pl, port, storage, kind="duct", seed=7):
    rng = np.random.default_rng(seed)
    periodic = kind == "periodic"
    lat = pl.LBM(X, Y, Z, viscosity=NU, collision=pl.COLL_SRT, equilibrium=pl.EQ_SECOND_ORDER, storage=storage,
                 periodic=periodic)
    if kind == "duct":
        m = duct_map(X, Y, Z, GEO["INFLOW"], GEO["OUTFLOW_EQ"])
    elif kind == "sym":
        m = duct_map(X, Y, Z, GEO["INFLOW"], GEO["OUTFLOW_EQ"])
        m[0], m[-1] = GEO["SYM_BOTTOM"], GEO["SYM_TOP"]
        m[:, 0], m[:, -1] = GEO["SYM_BACK"], GEO["SYM_FRONT"]
        m[1:-1, 1:-1, 0], m[1:-1, 1:-1, -1] = GEO["INFLOW"], GEO["OUTFLOW_EQ"]
        m[1:-1, 1:-1, 1:-1] = GEO["FLUID"]
    else:
        m = np.full((Z, Y, X), GEO["PERIODIC"], np.uint8)
    if not periodic:
        lat.set_map(m)
        lat.set_inflow(0.02 + 0.005 * rng.random((Z, Y)), 0.002 * rng.random((Z, Y)), None)
    f0 = seeded_state(port, rng, X, Y, Z, eq="EQ")
    force = 1e-4 * rng.standard_normal((3, Z, Y, X))
    fluid = np.flatnonzero((m == GEO["FLUID"]) | (m == GEO["PERIODIC"]))
    samples = rng.choice(fluid, size=16, replace=False)
    target = np.column_stack([1 + 0.01 * rng.standard_normal(16), 0.02 * rng.standard_normal((16, 3))])
    return lat, m, f0, force, samples, target, rng


def run(lat, f0, force, samples, target, nsteps, every=0, w_rho=0.7):
    lat.set_populations(f0)
    lat.iteration = 0
    return lat.adjoint_forward(force, nsteps, samples, target, checkpoint_every=every, rho_weight=w_rho)


@pytest.mark.parametrize("kind", ["duct", "sym", "periodic"])
def test_force_gradient_matches_finite_differences(pl, port, kind):
    lat, m, f0, force, samples, target, rng = channel(pl, port, pl.STORE_F64, kind)
    N = 24
    run(lat, f0, force, samples, target, N, every=5)
    g = lat.adjoint_backward()
    active = np.flatnonzero((m != GEO["NOTHING"]).ravel())
    h = 1e-7
    scale = np.max(np.abs(g))
    assert scale > 0
    for _ in range(12):
        k, s = int(rng.integers(3)), int(rng.choice(active))
        idx = np.unravel_index(s, m.shape)
        fp, fm = force.copy(), force.copy()
        fp[(k,) + idx] += h
        fm[(k,) + idx] -= h
        fd = (run(lat, f0, fp, samples, target, N) - run(lat, f0, fm, samples, target, N)) / (2 * h)
        assert abs(fd - g[(k,) + idx]) <= 1e-6 * scale, (k, idx, fd, g[(k,) + idx])
    lat.close()


def test_initial_population_gradient_matches_finite_differences(pl, port):
    lat, m, f0, force, samples, target, rng = channel(pl, port, pl.STORE_F64, "duct", seed=8)
    N = 17  # odd: the final state is read with the odd-step pattern
    run(lat, f0, force, samples, target, N, every=4)
    _, gp = lat.adjoint_backward(populations=True)
    h = 1e-7
    scale = np.max(np.abs(gp))
    # entries with large gradients and random ones (ghost layer included)
    picks = list(np.argsort(np.abs(gp).ravel())[-6:]) + list(rng.integers(0, gp.size, 6))
    for flat in picks:
        idx = np.unravel_index(int(flat), gp.shape)
        fp, fm = f0.copy(), f0.copy()
        fp[idx] += h
        fm[idx] -= h
        fd = (run(lat, fp, force, samples, target, N) - run(lat, fm, force, samples, target, N)) / (2 * h)
        assert abs(fd - gp[idx]) <= 1e-6 * scale, (idx, fd, gp[idx])
    lat.close()


def test_checkpoint_interval_does_not_change_the_gradient(pl, port):
    lat, m, f0, force, samples, target, _ = channel(pl, port, pl.STORE_F64, "duct", seed=9)
    N = 21
    out = []
    for every in (1, 4, 0, N):
        loss = run(lat, f0, force, samples, target, N, every=every)
        out.append((loss, lat.adjoint_backward(populations=True)))
    for loss, (g, gp) in out[1:]:
        assert loss == out[0][0]
        assert np.array_equal(g, out[0][1][0])
        assert np.array_equal(gp, out[0][1][1])
    lat.close()


@pytest.mark.parametrize("storage", ["F64", "F32"])
def test_forward_with_uniform_force_is_the_production_step(pl, port, storage):
    lat, m, f0, force, samples, target, _ = channel(pl, port, getattr(pl, "STORE_" + storage), "duct", seed=10)
    dtype = np.float64 if storage == "F64" else np.float32
    f0 = f0.astype(dtype)
    run(lat, f0, None, samples, target, 15)
    fa = lat.get_populations()
    assert lat.iteration == 15
    lat.set_populations(f0)
    lat.iteration = 0
    lat.step(15)
    assert rel_linf(fa, lat.get_populations()) <= (1e-12 if storage == "F64" else 1e-6)
    lat.close()


def test_fp32_gradient_agrees_with_fp64(pl, port):
    """FP32 storage with the adjoint evaluated and accumulated in FP64: the
    gradient differs from the FP64 run's only through the FP32 primal."""
    res = []
    for storage in ("F64", "F32"):
        lat, m, f0, force, samples, target, _ = channel(pl, port, getattr(pl, "STORE_" + storage), "duct", seed=11)
        run(lat, f0.astype(np.float64 if storage == "F64" else np.float32), force, samples, target, 30, every=6)
        res.append(lat.adjoint_backward())
        lat.close()
    assert rel_linf(res[1], res[0]) <= 1e-4


def test_autograd_function_keeps_a_cuda_control_on_the_device(pl, port):
    """A CUDA force tensor is read in place and its gradient written on the
    device; the values equal those of the host path bit for bit."""
    import torch
    from pytnl_lbm.adjoint import objective
    lat, m, f0, force, samples, target, _ = channel(pl, port, pl.STORE_F32, "duct", seed=13)
    f0 = f0.astype(np.float32)
    ft = torch.tensor(force, dtype=torch.float64, device="cuda", requires_grad=True)
    J = objective(ft, lat, f0, 14, samples, target, checkpoint_every=4, rho_weight=0.5)
    J.backward()
    assert ft.grad.is_cuda
    J_host = run(lat, f0, force, samples, target, 14, every=4, w_rho=0.5)
    g_host = lat.adjoint_backward()
    assert float(J.detach()) == J_host
    np.testing.assert_array_equal(ft.grad.cpu().numpy(), g_host)
    lat.close()


def test_autograd_function(pl, port):
    import torch
    from pytnl_lbm.adjoint import objective
    lat, m, f0, force, samples, target, _ = channel(pl, port, pl.STORE_F64, "duct", seed=12)
    ft = torch.tensor(force, dtype=torch.float64, requires_grad=True)
    J = objective(ft, lat, f0, 12, samples, target, checkpoint_every=3, rho_weight=0.7)
    (2.5 * J).backward()
    run(lat, f0, force, samples, target, 12, every=3)
    g = lat.adjoint_backward(seed=2.5)
    assert float(J.detach()) == pytest.approx(run(lat, f0, force, samples, target, 12), rel=0, abs=0)
    np.testing.assert_array_equal(ft.grad.numpy(), g)
    lat.close()


def test_unsupported_configurations_are_rejected(pl, port):
    lat = pl.LBM(8, 6, 5, viscosity=0.01, periodic=True)  # cumulant
    with pytest.raises(pl.LbmError) as e:
        lat.adjoint_forward(None, 3, [1], [[1, 0, 0, 0]])
    assert e.value.code == 2
    lat.close()
    lat = pl.LBM(8, 6, 5, viscosity=0.01, collision=pl.COLL_SRT, equilibrium=pl.EQ_SECOND_ORDER)
    lat.set_map(duct_map(8, 6, 5, GEO["INFLOW_LEFT"], GEO["OUTFLOW_EQ"]))
    with pytest.raises(pl.LbmError) as e:
        lat.adjoint_forward(None, 3, [60], [[1, 0, 0, 0]])
    assert e.value.code == 2
    lat.set_map(duct_map(8, 6, 5, GEO["INFLOW"], GEO["OUTFLOW_EQ"]))
    with pytest.raises(pl.LbmError):
        lat.adjoint_forward(None, 3, [0], [[1, 0, 0, 0]])  # a GEO_NOTHING site
    with pytest.raises(pl.LbmError):
        lat.adjoint_forward(None, 3, [115, 115], [[1, 0, 0, 0]] * 2)  # listed twice
    with pytest.raises(pl.LbmError):
        lat.adjoint_backward()  # no forward pass
    lat.close()


def test_channel_configuration_gradient_matches_finite_differences(pl):
    """The differentiation configuration at its full size: a 256 x 64 x 64
    channel with bounce-back walls, a velocity inlet at u_max = 0.03 and a
    per-cell x-force control of seeded Gaussian bumps (amplitude 1e-3), the L2
    velocity mismatch on 8 cross-sections against the flow of another seeded
    control, 4000 steps with sqrt(N) checkpoints.  On 32 random fluid cells
    the FP64 gradient agrees with central finite differences of the FP64
    objective to 1e-4 relative per cell (differences below 1e-3 of the
    largest gradient taken relative to that floor).  The gradient of the FP32
    run (FP32 primal, FP64 adjoint) is the exact gradient of the FP32
    trajectory, which parts from the FP64 one under this strong forcing: it
    agrees with the FP64 differences to 2e-4 of the largest gradient
    (measured 1.35e-4 on a B200)."""
    import json
    from pytnl_lbm import adjoint_check
    res = adjoint_check.check(steps=4000, fd_cells=32)
    msg = json.dumps(res)
    assert res["fd_max_rel_err"] <= 1e-4, msg
    assert res["fd_f32_max_normwise_err"] <= 2e-4, msg
    assert res["f32_vs_f64_grad_rel_linf"] <= 2e-4, msg
