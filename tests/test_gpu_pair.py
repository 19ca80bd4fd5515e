"""The two-site step kernel (LBM_KERNEL_PAIR) against the direct kernel.

Both kernels compute the same update; they differ only in how the multiply-adds
of the collision (the cumulant, SRT, BGK or MRT-LES) are fused (the packed f32x2 instructions take the
products and sums as written, the scalar kernel lets the compiler contract
them), so the states agree to FP32 rounding.  After 7 steps:
  FP32 / shifted FP32 storage   |f_pair - f_direct| <= 2e-6
  FP16 storage                  <= 4e-5 (a 1-ulp difference before the store
                                 can move a value by one FP16 step of the
                                 scaled deviation)
  BF16 storage                  <= 4e-4 (one BF16 step)
  16-bit fixed point            <= 4e-5 (a few quanta of at most 3.8e-6)
  stochastically rounded        4 times the bound of the format: a different
  FP16 / BF16                   value before the store draws an independent
                                rounding, and the draws of 7 steps add up
on the populations, 8 times those bounds on the macro fields (the density sums
27 populations, whose roundings are independent under stochastic rounding), and
on the FP64 sums 1e-6 relative or 8 times the population bound per site.
Widths that are odd, smaller than a block and not a multiple of one, periodic
lattices, the duct's boundary map and random maps with every race-free site
type (which puts periodic sites next to non-periodic ones on the lattice edges,
the pairs that move their populations one site at a time) are covered.  The
oracle parity of the pair kernel is part of test_gpu_parity.py
(its KERNELS list).
"""
import numpy as np
import pytest

from helpers import duct_map, random_map, seeded_state

pytestmark = pytest.mark.gpu

STORAGES = {"F32": 2e-6, "F32S": 2e-6, "F16S": 4e-5, "F16SR": 1.6e-4, "BF16S": 4e-4, "BF16SR": 1.6e-3,
            "I16S": 4e-5}


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def run(pl, kernel, f0, X, Y, Z, storage, flags, kind, rng_seed, steps=7):
    lat = pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=flags, storage=getattr(pl, "STORE_" + storage),
                 periodic=(kind == "periodic"), force=(1e-5, 0.0, 2e-6))
    try:
        if kind == "duct":
            lat.set_map(duct_map(X, Y, Z))
            lat.set_inflow(0.02 * np.ones((Z, Y)), 0.003 * np.ones((Z, Y)), None)
        elif kind == "random":
            lat.set_map(random_map(np.random.default_rng(rng_seed), X, Y, Z))
            lat.set_inflow(0.02 * np.ones((Z, Y)), None, None)
        lat.set_kernel(kernel)
        lat.set_populations(f0.astype(np.float32))
        lat.step(steps, macro=True, sums=True)
        assert lat.status() == 0
        return lat.get_populations(), lat.macro(), lat.sums()
    finally:
        lat.close()


@pytest.mark.parametrize("storage", list(STORAGES))
@pytest.mark.parametrize("kind", ["periodic", "duct", "random"])
@pytest.mark.parametrize("shape", [(128, 16, 8), (37, 9, 7), (5, 4, 3), (300, 10, 8)])
def test_pair_kernel_matches_direct_kernel(pl, port, storage, kind, shape):
    X, Y, Z = shape
    rng = np.random.default_rng(X * 31 + Y * 7 + Z)
    f0 = seeded_state(port, rng, X, Y, Z)
    tol = STORAGES[storage]
    for flags in (0, 3):
        fd, md, sd = run(pl, pl.KERNEL_DIRECT, f0, X, Y, Z, storage, flags, kind, X + Y)
        fp, mp, sp = run(pl, pl.KERNEL_PAIR, f0, X, Y, Z, storage, flags, kind, X + Y)
        assert np.isfinite(fp).all()
        assert np.max(np.abs(fp.astype(np.float64) - fd)) <= tol
        assert np.max(np.abs(mp.astype(np.float64) - md)) <= 8 * tol
        np.testing.assert_allclose(sp, sd, rtol=1e-6, atol=8 * tol * X * Y * Z)


def test_pair_kernel_long_run_tracks_direct_kernel(pl, port):
    """A periodic Taylor-Green run of 200 steps at high Reynolds number: the
    pair kernel's FP32 kinetic energy is as close to that of an FP64 run as the
    direct kernel's FP32 kinetic energy is (two FP32 runs with different
    rounding drift apart at this Reynolds number by a few 1e-6)."""
    X, Y, Z = 64, 32, 32
    out = []
    for kernel, storage in ((pl.KERNEL_DIRECT, pl.STORE_F64), (pl.KERNEL_DIRECT, pl.STORE_F32),
                            (pl.KERNEL_PAIR, pl.STORE_F32)):
        lat = pl.LBM(X, Y, Z, viscosity=0.002, cum_flags=3, storage=storage, periodic=True)
        lat.set_kernel(kernel)
        lat.init_taylor_green(0.05, 1.0)
        lat.step(200, sums=True)
        out.append(lat.sums())
        lat.close()
    ref = out[0]
    err_direct = abs(out[1][4] - ref[4]) / ref[4]
    err_pair = abs(out[2][4] - ref[4]) / ref[4]
    assert err_pair <= max(2 * err_direct, 2e-5)
    assert abs(out[2][0] - ref[0]) <= 1e-6 * ref[0]


def test_pair_kernel_falls_back_for_fp64(pl, port):
    """FP64 arithmetic has no two-site kernel: LBM_KERNEL_PAIR runs the direct
    kernel, bit for bit."""
    X, Y, Z = 40, 9, 7
    rng = np.random.default_rng(11)
    f0 = seeded_state(port, rng, X, Y, Z, eq="EQ")
    res = []
    for kernel in (pl.KERNEL_DIRECT, pl.KERNEL_PAIR):
        lat = pl.LBM(X, Y, Z, viscosity=0.01, collision=pl.COLL_MRT, equilibrium=pl.EQ_SECOND_ORDER,
                     storage=pl.STORE_F64, periodic=True)
        lat.set_kernel(kernel)
        lat.set_populations(f0)
        lat.step(5)
        res.append(lat.get_populations())
        lat.close()
    assert np.array_equal(res[0], res[1])


def run_collision(pl, kernel, f0, X, Y, Z, storage, coll, eq, kind, steps=7):
    lat = pl.LBM(X, Y, Z, viscosity=0.01, collision=coll, equilibrium=eq, storage=getattr(pl, "STORE_" + storage),
                 periodic=(kind == "periodic"), force=(1e-5, 0.0, 2e-6))
    try:
        if kind == "duct":
            lat.set_map(duct_map(X, Y, Z))
            lat.set_inflow(0.02 * np.ones((Z, Y)), 0.003 * np.ones((Z, Y)), None)
        elif kind == "random":
            lat.set_map(random_map(np.random.default_rng(X + Y), X, Y, Z))
            lat.set_inflow(0.02 * np.ones((Z, Y)), None, None)
        lat.set_kernel(kernel)
        lat.set_populations(f0.astype(np.float32))
        lat.step(steps, macro=True, sums=True)
        assert lat.status() == 0
        return lat.get_populations(), lat.macro(), lat.sums()
    finally:
        lat.close()


@pytest.mark.parametrize("coll", ["SRT", "BGK", "MRT"])
@pytest.mark.parametrize("storage", ["F32", "F32S", "F16S", "BF16SR"])
@pytest.mark.parametrize("kind", ["periodic", "duct", "random"])
@pytest.mark.parametrize("shape", [(128, 16, 8), (37, 9, 7)])
def test_pair_kernel_other_collisions_match_direct_kernel(pl, port, coll, storage, kind, shape):
    """SRT (both equilibria), BGK and MRT-LES on the two-site kernel: the same
    update as the direct kernel to the bounds of the cumulant above."""
    X, Y, Z = shape
    rng = np.random.default_rng(X * 13 + Y)
    f0 = seeded_state(port, rng, X, Y, Z, eq="EQ")
    tol = STORAGES[storage]
    eqs = (pl.EQ_SECOND_ORDER, pl.EQ_INV_CUM) if coll == "SRT" else (pl.EQ_SECOND_ORDER,)
    for eq in eqs:
        c = getattr(pl, "COLL_" + coll)
        fd, md, sd = run_collision(pl, pl.KERNEL_DIRECT, f0, X, Y, Z, storage, c, eq, kind)
        fp, mp, sp = run_collision(pl, pl.KERNEL_PAIR, f0, X, Y, Z, storage, c, eq, kind)
        assert np.isfinite(fp).all()
        assert np.max(np.abs(fp.astype(np.float64) - fd)) <= tol, (eq, np.max(np.abs(fp - fd)))
        assert np.max(np.abs(mp.astype(np.float64) - md)) <= 8 * tol
        np.testing.assert_allclose(sp, sd, rtol=1e-6, atol=8 * tol * X * Y * Z)


def test_autotune_may_choose_the_pair_kernel(pl):
    lat = pl.LBM(256, 32, 16, viscosity=0.01, storage=pl.STORE_F16S, periodic=True)
    lat.init_equilibrium()
    lat.autotune(4)
    assert lat.kernel in (pl.KERNEL_DIRECT, pl.KERNEL_PAIR, pl.KERNEL_TILE)
    lat.step(4, sums=True)
    assert abs(lat.sums()[0] - 256 * 32 * 16) < 1e-3
    lat.close()

