"""The bounded waits of the tile kernel (LBM_KERNEL_TILE) and the status word.

Every mbarrier wait of the tile kernel gives up after a bounded number of
tries, sets LBM_STATUS_TIMEOUT in the handle's device status word and lets
the kernel return; the CTA still waits for the bulk copies it issued before
it exits.  lbm_set_wait_limit(h, 0) makes the tile loop's waits give up at
once while the copies are in flight, so the path runs here without a fault
and without a wait that never ends: the status reports the timeout, reading
it clears it, and after the limit is restored the lattice steps normally,
equal bit for bit to the direct kernel.
"""
import numpy as np
import pytest

from helpers import duct_map, seeded_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


@pytest.mark.parametrize("kind", ["periodic", "duct"])
def test_tile_kernel_timeout_is_reported_and_the_next_steps_run(pl, port, kind):
    X, Y, Z = 200, 12, 10
    rng = np.random.default_rng(5)
    f0 = seeded_state(port, rng, X, Y, Z).astype(np.float32)

    def lattice(kernel):
        lat = pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=0, storage=pl.STORE_F32, periodic=kind == "periodic",
                     use_graphs=False)
        if kind == "duct":
            lat.set_map(duct_map(X, Y, Z))
            lat.set_inflow(0.02 * np.ones((Z, Y)), None, None)
        lat.set_kernel(kernel)
        lat.set_populations(f0)
        return lat

    lat = lattice(pl.KERNEL_TILE)
    assert lat.status() == 0
    lat.set_wait_limit(0)
    lat.step(1)
    assert lat.status() & pl.STATUS_TIMEOUT
    assert lat.status() == 0  # reading the status cleared it
    # the limit restored, the same start runs through
    lat.set_wait_limit(-1)
    lat.set_populations(f0)
    lat.iteration = 0
    lat.step(3)
    assert lat.status() == 0
    got = lat.get_populations()
    lat.close()
    ref = lattice(pl.KERNEL_DIRECT)
    ref.step(3)
    expected = ref.get_populations()
    ref.close()
    assert np.array_equal(got, expected)
