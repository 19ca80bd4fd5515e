"""Coupled D3Q7 advection-diffusion scalar (lbm_ade_*) against the reference.

The checker is TNL-LBM's own coupled update (cudaLBMKernel<NSE, ADE> of
include/lbm3d/kernels.h:114-196 with the d3q7 operator headers), compiled
from the reference tree through oracle/ref_harness.cpp.  Both the flow and
the scalar populations, the macro field and phi are compared after several
steps of either parity, for every scalar collision, with a periodic lattice
and with a duct map plus scalar inlet, symmetry outlet, walls and solids.
"""
import numpy as np
import pytest

from helpers import GEO, duct_map, rel_linf, seeded_state

pytestmark = pytest.mark.gpu

ADE_GEO = dict(FLUID=0, WALL=1, WALL_BODY=2, SOLID=3, INFLOW=7, PERIODIC=9, NOTHING=10, SYM_TOP=12, SYM_BOTTOM=13,
               SYM_LEFT=14, SYM_RIGHT=15, SYM_BACK=16, SYM_FRONT=17)


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference, reference_available
    if not reference_available(0):
        pytest.skip("reference harness not built")
    return Reference(0)


def scalar_state(rng, X, Y, Z, dtype):
    """Equilibrium of a random phi field (zero velocity) with a small noise, ghosts included."""
    from oracle import ade
    phi = 1.0 + 0.2 * rng.standard_normal((Z + 2) * (Y + 2) * (X + 2))
    v = 0.02 * rng.standard_normal((phi.size, 3))
    g = ade.feq(phi, v).T.reshape(7, Z + 2, Y + 2, X + 2)
    g *= 1 + 0.01 * rng.standard_normal(g.shape)
    return np.ascontiguousarray(g.astype(dtype))


def scalar_duct_map(X, Y, Z):
    m = np.full((Z, Y, X), ADE_GEO["FLUID"], np.uint8)
    m[:, :, 0] = ADE_GEO["INFLOW"]
    m[:, :, -1] = ADE_GEO["SYM_RIGHT"]
    m[:, 1, :] = ADE_GEO["WALL"]
    m[:, -2, :] = ADE_GEO["WALL"]
    m[1, :, :] = ADE_GEO["WALL_BODY"]
    m[-2, :, :] = ADE_GEO["WALL"]
    m[:, 0, :] = ADE_GEO["NOTHING"]
    m[:, -1, :] = ADE_GEO["NOTHING"]
    m[0, :, :] = ADE_GEO["NOTHING"]
    m[-1, :, :] = ADE_GEO["NOTHING"]
    m[Z // 2, Y // 2, X // 3] = ADE_GEO["SOLID"]
    m[Z // 2, 2, X // 2] = ADE_GEO["SYM_BACK"]
    return m


CASES = [
    # (storage, coll, eq, cum_flags, periodic, ade_coll, start_iter, per-site diffusion)
    ("F64", "CUM", "INV_CUM", 0, False, "SRT", 0, False),
    ("F64", "CUM", "INV_CUM", 0, False, "MRT", 1, True),
    ("F64", "CUM", "INV_CUM", 0, True, "CLBM", 0, False),
    ("F64", "SRT", "EQ", 0, False, "CLBM", 1, False),
    ("F64", "MRT", "INV_CUM", 0, True, "SRT", 1, True),
    ("F32", "CUM", "INV_CUM", 0, False, "CLBM", 0, False),
    ("F32", "CUM", "INV_CUM", 0, True, "MRT", 1, True),
    ("F32S", "CUM", "INV_CUM", 0, False, "SRT", 1, False),
]


@pytest.mark.parametrize("storage,coll,eq,flags,periodic,ade_coll,start,field", CASES)
def test_coupled_step_matches_reference(pl, ref, port, storage, coll, eq, flags, periodic, ade_coll, start, field):
    X, Y, Z = 37, 11, 9
    rng = np.random.default_rng(X + 100 * start + (7 if periodic else 0))
    dtype = np.float64 if storage == "F64" else np.float32
    f0 = seeded_state(port, rng, X, Y, Z, eq=eq)
    g0 = scalar_state(rng, X, Y, Z, np.float64)
    nu, D, phi_in = 0.02, 0.013, 1.7
    dfield = (0.005 + 0.02 * rng.random((Z, Y, X))) if field else None
    if periodic:
        m = np.full((Z, Y, X), GEO["PERIODIC"], np.uint8)
        am = np.full((Z, Y, X), ADE_GEO["FLUID"], np.uint8)
        am[Z // 2, Y // 2, X // 2] = ADE_GEO["SOLID"]
        inflow = None
    else:
        m = duct_map(X, Y, Z, GEO["INFLOW_LEFT"], GEO["OUTFLOW_EQ"])
        am = scalar_duct_map(X, Y, Z)
        inflow = (0.03 * np.ones((Z, Y)), 0.002 * np.ones((Z, Y)), None)
    steps = 6

    lat = pl.LBM(X, Y, Z, viscosity=nu, collision=getattr(pl, "COLL_" + coll), cum_flags=flags,
                 equilibrium={"EQ": pl.EQ_SECOND_ORDER, "INV_CUM": pl.EQ_INV_CUM}[eq], storage=getattr(pl, "STORE_" + storage), periodic=periodic)
    if not periodic:
        lat.set_map(m)
        lat.set_inflow(*inflow)
    lat.ade_enable(D, collision=getattr(pl, "ADE_" + ade_coll), inflow_phi=phi_in)
    lat.ade_set_map(am)
    if field:
        lat.ade_set_diffusion(dfield)
    lat.set_populations(f0.astype(dtype))
    lat.ade_set_populations(g0.astype(dtype))
    lat.iteration = start
    lat.step(steps, macro=True)
    fg, gg = lat.get_populations(), lat.ade_get_populations()
    mg, pg = lat.macro(), lat.ade_phi()
    assert lat.status() == 0
    lat.close()

    fo, go = np.ascontiguousarray(f0.astype(dtype)), np.ascontiguousarray(g0.astype(dtype))
    mo = np.zeros((4, Z, Y, X), dtype)
    po = np.zeros((Z, Y, X), dtype)
    ref.aa_ade_run(fo, m, go, am, coll=coll, eq=eq, ade_coll=ade_coll, nu=nu, D=D, inflow=inflow, dfield=dfield,
                   inflow_phi=phi_in, start_iter=start, nsteps=steps - 1)
    ref.aa_ade_run(fo, m, go, am, coll=coll, eq=eq, ade_coll=ade_coll, nu=nu, D=D, inflow=inflow, dfield=dfield,
                   inflow_phi=phi_in, macro=mo, phi=po, start_iter=start + steps - 1, nsteps=1)
    tol = 1e-12 if storage == "F64" else 1e-5
    assert rel_linf(fg, fo) < tol
    assert rel_linf(gg, go) < tol
    assert rel_linf(mg[0], mo[0]) < tol
    assert rel_linf(pg, po) < tol
    # inlet sites carry the imposed phi, NOTHING sites zero
    if not periodic:
        inlet = am == ADE_GEO["INFLOW"]
        np.testing.assert_allclose(pg[inlet], phi_in, rtol=1e-6)
        assert np.all(pg[am == ADE_GEO["NOTHING"]] == 0)


def test_scalar_does_not_change_the_flow(pl, port):
    X, Y, Z = 40, 12, 10
    rng = np.random.default_rng(5)
    f0 = seeded_state(port, rng, X, Y, Z)
    out = []
    for with_scalar in (False, True):
        lat = pl.LBM(X, Y, Z, viscosity=0.02, storage=pl.STORE_F64)
        lat.set_map(duct_map(X, Y, Z))
        lat.set_inflow(0.03 * np.ones((Z, Y)), None, None)
        if with_scalar:
            lat.ade_enable(0.01, collision=pl.ADE_CLBM)
            lat.ade_init_equilibrium(uniform_phi=1.0)
        lat.set_populations(f0)
        lat.step(9, macro=True, sums=True)
        out.append((lat.get_populations(), lat.sums()))
        lat.close()
    assert rel_linf(out[1][0], out[0][0]) < 1e-13
    np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-12)


def test_uniform_scalar_at_rest_stays_uniform_and_is_conserved(pl):
    X, Y, Z = 32, 8, 8
    lat = pl.LBM(X, Y, Z, viscosity=0.02, storage=pl.STORE_F64, periodic=True)
    lat.init_equilibrium()
    lat.ade_enable(0.02, collision=pl.ADE_MRT)
    phi = 1.0 + 0.1 * np.sin(2 * np.pi * np.arange(X) / X)[None, None, :] * np.ones((Z, Y, X))
    lat.ade_init_equilibrium(phi=phi)
    lat.step(50, macro=True)
    p = lat.ade_phi()
    # periodic diffusion of a sine: total conserved, amplitude decays
    np.testing.assert_allclose(p.sum(), phi.sum(), rtol=1e-12)
    assert np.ptp(p) < np.ptp(phi)
    lat.close()


def test_refusals(pl):
    lat = pl.LBM(8, 8, 8, viscosity=0.02, storage=pl.STORE_F16S, periodic=True)
    with pytest.raises(pl.LbmError):
        lat.ade_enable(0.01)
    lat.close()
    lat = pl.LBM(8, 8, 8, viscosity=0.02, storage=pl.STORE_F32, periodic=True)
    lat.ade_enable(0.01)
    bad = np.zeros((8, 8, 8), np.uint8)
    bad[0, 0, 0] = 8  # GEO_OUTFLOW_RIGHT depends on the site order
    with pytest.raises(pl.LbmError):
        lat.ade_set_map(bad)
    with pytest.raises(pl.LbmError):
        lat.set_streaming(pl.STREAMING_AB)
    with pytest.raises(pl.LbmError):
        lat.ade_phi()  # no observation step yet
    lat.ade_disable()
    lat.set_streaming(pl.STREAMING_AB)
    lat.close()


@pytest.mark.parametrize("X", [37, 40])
@pytest.mark.parametrize("flags", [0, 3])
@pytest.mark.parametrize("ade_coll", ["SRT", "MRT", "CLBM"])
@pytest.mark.parametrize("start,field", [(0, False), (1, True)])
def test_two_site_coupled_step_matches_reference(pl, port, X, flags, ade_coll, start, field):
    """The two-site coupled step (LBM_KERNEL_PAIR on FP32 storage): its plain
    steps against the reference's coupled update, at the FP32 tolerance of the
    one-site kernel.  The duct's inlet, outlet, wall and rim sites and the
    scalar's boundary sites take the one-site update inside the same launch."""
    from oracle import Reference, reference_available
    if not reference_available(flags):
        pytest.skip("reference harness not built")
    ref = Reference(flags)
    Y, Z = 11, 9
    rng = np.random.default_rng(X + 100 * start + flags)
    f0 = seeded_state(port, rng, X, Y, Z, eq="INV_CUM")
    g0 = scalar_state(rng, X, Y, Z, np.float64)
    nu, D, phi_in = 0.02, 0.013, 1.7
    dfield = (0.005 + 0.02 * rng.random((Z, Y, X))) if field else None
    m = duct_map(X, Y, Z, GEO["INFLOW_LEFT"], GEO["OUTFLOW_EQ"])
    am = scalar_duct_map(X, Y, Z)
    inflow = (0.03 * np.ones((Z, Y)), 0.002 * np.ones((Z, Y)), None)
    steps = 7
    lat = pl.LBM(X, Y, Z, viscosity=nu, cum_flags=flags, equilibrium=pl.EQ_INV_CUM, storage=pl.STORE_F32)
    lat.set_map(m)
    lat.set_inflow(*inflow)
    lat.ade_enable(D, collision=getattr(pl, "ADE_" + ade_coll), inflow_phi=phi_in)
    lat.ade_set_map(am)
    if field:
        lat.ade_set_diffusion(dfield)
    lat.set_kernel(pl.KERNEL_PAIR)
    lat.set_populations(f0.astype(np.float32))
    lat.ade_set_populations(g0.astype(np.float32))
    lat.iteration = start
    lat.step(steps)
    fg, gg = lat.get_populations(), lat.ade_get_populations()
    assert lat.status() == 0
    lat.close()
    fo, go = np.ascontiguousarray(f0.astype(np.float32)), np.ascontiguousarray(g0.astype(np.float32))
    ref.aa_ade_run(fo, m, go, am, coll="CUM", eq="INV_CUM", ade_coll=ade_coll, nu=nu, D=D, inflow=inflow, dfield=dfield,
                   inflow_phi=phi_in, start_iter=start, nsteps=steps)
    assert rel_linf(fg, fo) < 1e-5
    assert rel_linf(gg, go) < 1e-5
