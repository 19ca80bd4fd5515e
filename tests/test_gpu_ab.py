"""GPU parity of the A-B pull step (LBM_STREAMING_AB) against the reference's
own A-B code (oracle/_ref/libref_ab_*, pinned to the A-A harness by
tests/test_oracle_ab.py), through the C-ABI.

Covers every site type of D3Q27_BC_All, including the three the in-place A-A
step cannot run (GEO_INFLOW_BB_LEFT, GEO_OUTFLOW_RIGHT,
GEO_OUTFLOW_RIGHT_INTERP), with the tolerances of the A-A parity tests.
"""
import zlib

import numpy as np
import pytest

import oracle
from helpers import COLL_IDS, EQ_IDS, GEO, duct_map, rel_linf, rel_linf_fields, seeded_state, tgv_fields

pytestmark = pytest.mark.gpu


def ke_of(macro):
    m = macro.astype(np.float64)
    return float((m[0] * (m[1] ** 2 + m[2] ** 2 + m[3] ** 2)).sum())


TOL = {np.float64: 1e-12, np.float32: 1e-5}
# the velocity is a quotient of differences of populations, which amplifies
# their FP32 rounding; the FP32 parity bar is on the populations (TOL) and
# the kinetic energy (KE_TOL)
FIELD_TOL = {np.float64: 1e-12, np.float32: 3e-5}
KE_TOL = {np.float64: 1e-12, np.float32: 1e-6}


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def reference_ab(flags):
    if not oracle.reference_ab_available(flags):
        pytest.skip("reference A-B harness not built")
    return oracle.ReferenceAB(flags)


def run_both(pl, f0, geo_map, *, coll="CUM", flags=0, eq="INV_CUM", nu=0.01, force=(0.0, 0.0, 0.0), inflow=None,
             steps=5, dtype=np.float64, periodic=False, use_graphs=True):
    Z, Y, X = geo_map.shape
    lat = pl.LBM(X, Y, Z, viscosity=nu, collision=COLL_IDS[coll], cum_flags=flags, equilibrium=EQ_IDS[eq],
                 storage=pl.STORE_F64 if dtype == np.float64 else pl.STORE_F32, periodic=periodic, force=force,
                 use_graphs=use_graphs)
    lat.set_streaming(pl.STREAMING_AB)
    if not periodic:
        lat.set_map(geo_map)
    if inflow is not None:
        lat.set_inflow(*inflow)
    lat.set_populations(f0.astype(dtype))
    lat.step(steps, macro=True, sums=True)
    fg, mg = lat.get_populations(dtype=np.float64), lat.macro()
    assert lat.status() == 0
    lat.close()
    fo = np.ascontiguousarray(f0.astype(dtype))
    mo = np.zeros((4, Z, Y, X), dtype)
    reference_ab(flags if coll == "CUM" else 0).ab_run(fo, geo_map.astype(np.int16), coll=coll, eq=eq, nu=nu, force=force,
                                                       inflow=inflow, macro=mo, nsteps=steps)
    return fg, fo, mg, mo


@pytest.mark.parametrize("coll,flags,eq", [("CUM", 0, "INV_CUM"), ("CUM", 3, "INV_CUM"), ("SRT", 0, "EQ"),
                                           ("BGK", 0, "EQ"), ("MRT", 0, "EQ")])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_periodic_taylor_green(pl, port, coll, flags, eq, dtype):
    X, Y, Z = 24, 16, 12
    f0 = port.allocate(X, Y, Z)
    port.init_equilibrium(f0, X, Y, Z, eq=eq, fields=tgv_fields(X, Y, Z, u0=0.05))
    m = np.full((Z, Y, X), GEO["PERIODIC"], np.uint8)
    force = (1e-6, -2e-6, 0.0) if coll != "CUM" else (0.0, 0.0, 0.0)
    fg, fo, mg, mo = run_both(pl, f0, m, coll=coll, flags=flags, eq=eq, nu=0.004, force=force, steps=11, dtype=dtype,
                              periodic=True)
    assert rel_linf(fg, fo) <= TOL[dtype]
    assert rel_linf_fields(mg, mo) <= FIELD_TOL[dtype]
    assert abs(ke_of(mg) - ke_of(mo)) <= KE_TOL[dtype] * ke_of(mo)


def ab_map(kind, rng, X, Y, Z):
    if kind in ("bb_left", "outflow_right", "outflow_interp"):
        inlet = GEO["INFLOW_BB_LEFT"] if kind == "bb_left" else GEO["INFLOW_LEFT"]
        outlet = {"bb_left": GEO["OUTFLOW_EQ"], "outflow_right": GEO["OUTFLOW_RIGHT"],
                  "outflow_interp": GEO["OUTFLOW_RIGHT_INTERP"]}[kind]
        return duct_map(X, Y, Z, inlet, outlet)
    if kind == "eq_left":
        return duct_map(X, Y, Z, GEO["INFLOW_EQ_LEFT"], GEO["OUTFLOW_RIGHT"])
    # every site type of D3Q27_BC_All at random
    return rng.integers(0, 17, size=(Z, Y, X)).astype(np.uint8)


@pytest.mark.parametrize("kind", ["bb_left", "outflow_right", "outflow_interp", "eq_left", "random"])
@pytest.mark.parametrize("coll,flags,eq", [("CUM", 0, "INV_CUM"), ("CUM", 3, "INV_CUM"), ("SRT", 0, "EQ"),
                                           ("MRT", 0, "EQ")])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_boundary_conditions(pl, port, kind, coll, flags, eq, dtype):
    rng = np.random.default_rng(zlib.crc32(f"{kind}-{coll}-{flags}".encode()))
    X, Y, Z = 33, 11, 9
    m = ab_map(kind, rng, X, Y, Z)
    f0 = seeded_state(port, rng, X, Y, Z, eq=eq)
    prof = (0.02 * rng.random((Z, Y)), 0.004 * rng.random((Z, Y)), -0.003 * rng.random((Z, Y)))
    fg, fo, mg, mo = run_both(pl, f0, m, coll=coll, flags=flags, eq=eq, nu=0.02, force=(1e-5, 0.0, 2e-6),
                              inflow=prof, steps=7, dtype=dtype)
    assert rel_linf(fg, fo) <= TOL[dtype]
    assert rel_linf_fields(mg, mo) <= FIELD_TOL[dtype]
    assert abs(ke_of(mg) - ke_of(mo)) <= KE_TOL[dtype] * ke_of(mo)


@pytest.mark.parametrize("steps", [16, 17, 40])
def test_graphs_and_buffer_rotation(pl, port, steps):
    """Graph replay with the two buffers rotating (even and odd step counts)."""
    rng = np.random.default_rng(steps)
    X, Y, Z = 40, 12, 10
    m = ab_map("outflow_interp", rng, X, Y, Z)
    f0 = seeded_state(port, rng, X, Y, Z)
    prof = (0.03 * np.ones((Z, Y)), None, None)
    out = [run_both(pl, f0, m, inflow=prof, steps=steps, use_graphs=g)[0] for g in (True, False)]
    assert np.array_equal(out[0], out[1])


def test_switching_patterns(pl, port):
    X, Y, Z = 12, 8, 7
    lat = pl.LBM(X, Y, Z, viscosity=0.01)
    m = duct_map(X, Y, Z, GEO["INFLOW_BB_LEFT"], GEO["OUTFLOW_RIGHT"])
    with pytest.raises(pl.LbmError) as e:
        lat.set_map(m)
    assert e.value.code == 2
    lat.set_streaming(pl.STREAMING_AB)
    assert lat.streaming == pl.STREAMING_AB
    lat.set_map(m)
    with pytest.raises(pl.LbmError):
        lat.set_streaming(pl.STREAMING_AA)  # the map holds A-B-only types
    lat.set_map(duct_map(X, Y, Z))
    lat.set_streaming(pl.STREAMING_AA)
    assert lat.streaming == pl.STREAMING_AA
    lat.close()
