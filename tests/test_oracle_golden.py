"""The oracle port against the reference's golden vectors (CPU only).

The fixtures in tests/golden were produced by TNL-LBM's own per-site code
(tests/golden/make_golden.py); these tests pin the C restatement in
oracle/lbm_oracle.c to them, bit for bit in FP64.
"""
import numpy as np
import pytest

import oracle
from helpers import COLL_IDS, duct_map, random_map, rel_linf, seeded_state

COLLS = ["CUM", "SRT", "BGK", "MRT"]


@pytest.mark.parametrize("key,coll,flags", [("site_CUM_0", "CUM", 0), ("site_CUM_2", "CUM", 2), ("site_CUM_3", "CUM", 3),
                                            ("site_SRT", "SRT", 0), ("site_BGK", "BGK", 0), ("site_MRT", "MRT", 0)])
def test_site_collision_matches_golden(port, golden, key, coll, flags):
    f = golden[key + "_in"].copy()
    macro = port.collide(f, coll=coll, eq="INV_CUM", cum_flags=flags, nu=float(golden["site_nu"]),
                         force=tuple(golden["site_force"]))
    assert np.array_equal(f, golden[key + "_out"]), rel_linf(f, golden[key + "_out"])
    assert np.array_equal(macro, golden[key + "_macro"])


LATTICES = ["tgv_cum2017", "duct_cum", "duct_eq_cumaa", "sym_srt", "mix_bgk", "periodic_mrt"]


@pytest.mark.parametrize("name", LATTICES)
def test_lattice_run_matches_golden(port, golden, name):
    p = "lat_" + name
    flags, coll, eq, nu, fx, fy, fz, steps = golden[p + "_params"]
    f = golden[p + "_in"].copy()
    m = golden[p + "_map"]
    prof = golden[p + "_inflow"]
    macro = np.zeros_like(golden[p + "_macro"])
    port.aa_run(f, m, coll=COLLS[int(coll)], eq=["EQ", "INV_CUM"][int(eq)], cum_flags=int(flags), nu=nu,
                force=(fx, fy, fz), inflow=(prof[0], prof[1], None), macro=macro, nsteps=int(steps))
    assert np.array_equal(f, golden[p + "_out"]), rel_linf(f, golden[p + "_out"])
    assert np.array_equal(macro, golden[p + "_macro"])


def test_tgv16_kinetic_energy_matches_golden(port, golden):
    from helpers import tgv_fields
    N = 16
    f = port.allocate(N, N, N)
    port.init_equilibrium(f, N, N, N, eq="INV_CUM", fields=tgv_fields(N, N, N))
    m = np.full((N, N, N), 9, np.int16)
    macro = np.zeros((4, N, N, N))
    ke = []
    for s in range(10):
        port.aa_run(f, m, coll="CUM", eq="INV_CUM", cum_flags=3, nu=float(golden["tgv16_nu"]), macro=macro,
                    start_iter=2 * s, nsteps=2)
        ke.append((macro[0] * (macro[1] ** 2 + macro[2] ** 2 + macro[3] ** 2)).sum() / 2.0 / N ** 3)
    # the fields are bitwise equal; only numpy's summation of them could differ
    np.testing.assert_allclose(ke, golden["tgv16_ke"], rtol=1e-14, atol=0)
    # probes after odd steps, as the reference's probe on even iterations
    # (sim_4.cu:369-372); the energy stays near u0^2/8 over these 20 steps
    assert np.all(np.abs(np.array(ke) / (0.05 ** 2 / 8) - 1) < 0.2)


@pytest.mark.parametrize("coll", COLLS)
def test_collision_conserves_mass_and_momentum(port, coll):
    rng = np.random.default_rng(7)
    rho = 1 + 0.05 * rng.standard_normal(128)
    u = 0.05 * rng.standard_normal((3, 128))
    f = port.equilibrium(rho, *u, eq="EQ") * (1 + 0.05 * rng.standard_normal((128, 27)))
    f = np.ascontiguousarray(f)
    cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
    cy = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1])
    cz = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])
    before = np.stack([f.sum(1), f @ cx, f @ cy, f @ cz])
    g = f.copy()
    port.collide(g, coll=coll, eq="INV_CUM", cum_flags=3 if coll == "CUM" else 0, nu=0.01)
    after = np.stack([g.sum(1), g @ cx, g @ cy, g @ cz])
    np.testing.assert_allclose(after, before, rtol=0, atol=1e-14)


def test_cumulant_keeps_its_equilibrium(port):
    """The equilibrium of the equilibrium cumulants is a fixed point of the
    default cumulant collision (col_cum.h with eq_inv_cum.h).  With the
    anti-aliasing terms it is not: col_cum.h:237-239 subtracts (rho - 1), the
    deviation-variable form of k_000, so Dxu = -1/(2 rho) at equilibrium; the
    oracle and the kernels reproduce that behaviour."""
    rng = np.random.default_rng(3)
    rho = 1 + 0.02 * rng.standard_normal(64)
    u = 0.04 * rng.standard_normal((3, 64))
    f = port.equilibrium(rho, *u, eq="INV_CUM")
    g = f.copy()
    port.collide(g, coll="CUM", eq="INV_CUM", cum_flags=0, nu=0.02)
    np.testing.assert_allclose(g, f, rtol=1e-12, atol=1e-15)
    h = f.copy()
    port.collide(h, coll="CUM", eq="INV_CUM", cum_flags=2, nu=0.02)
    assert np.abs(h - f).max() > 1e-4


@pytest.mark.skipif(not oracle.reference_available(0), reason="reference harness not built")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("kind", ["duct", "random", "ordered"])
def test_port_matches_reference_on_lattices(port, dtype, kind):
    """Independent check of the restatement against the reference's own code on
    fresh random inputs (needs oracle/_ref)."""
    rng = np.random.default_rng(11)
    X, Y, Z = 9, 7, 6
    if kind == "duct":
        m = duct_map(X, Y, Z).astype(np.int16)
    elif kind == "random":
        m = random_map(rng, X, Y, Z).astype(np.int16)
    else:  # order-dependent site types, run sequentially by both
        m = duct_map(X, Y, Z, inlet=4, outlet=7).astype(np.int16)
    for flags in (0, 3):
        ref = oracle.Reference(flags)
        for coll in COLLS:
            f = seeded_state(port, rng, X, Y, Z, dtype=dtype)
            prof = (0.02 * rng.random((Z, Y)), 0.004 * rng.random((Z, Y)), None)
            a, b = f.copy(), f.copy()
            ma = np.zeros((4, Z, Y, X), dtype)
            mb = ma.copy()
            port.aa_run(a, m, coll=coll, cum_flags=flags, nu=0.02, force=(1e-5, 0, 0), inflow=prof, macro=ma, nsteps=5)
            ref.aa_run(b, m, coll=coll, nu=0.02, force=(1e-5, 0, 0), inflow=prof, macro=mb, nsteps=5)
            assert np.array_equal(a, b), (coll, flags, rel_linf(a, b))
            assert np.array_equal(ma, mb)
