"""z-slab decomposition on the GPU: slabs with halo exchange must reproduce the
single lattice bit for bit (same per-site code, same inputs to every site), with
the direct kernel and with the two-site kernel (whose slabs leave the z wrap to
the halo exchange).

All slabs run on device 0 here; across GPUs the exchange kernel reads the
sender's memory with peer loads, the same copies over NVLink.
"""
import numpy as np
import pytest

from helpers import GEO, duct_map, seeded_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


@pytest.mark.parametrize("storage", ["F64", "F32", "F16S"])
@pytest.mark.parametrize("nslabs", [1, 2, 3])
@pytest.mark.parametrize("start", [0, 1])
@pytest.mark.parametrize("kind", ["periodic", "duct"])
@pytest.mark.parametrize("kernel", ["DIRECT", "PAIR"])
def test_slabs_match_the_single_lattice(pl, port, storage, nslabs, start, kind, kernel):
    from pytnl_lbm.slabs import SlabLattice
    X, Y, Z = 40, 10, 21
    rng = np.random.default_rng(nslabs + 10 * start)
    f0 = seeded_state(port, rng, X, Y, Z)
    st = getattr(pl, "STORE_" + storage)
    dtype = np.float64 if storage == "F64" else np.float32
    periodic = kind == "periodic"
    kw = dict(viscosity=0.01, cum_flags=3, storage=st)
    if not periodic:
        # the duct: inlet and outlet in x, walls and rims in y and z; the slab
        # faces cut through the fluid
        m = duct_map(X, Y, Z)
        inflow = (0.02 * np.ones((Z, Y)), None, None)

    single = pl.LBM(X, Y, Z, periodic=periodic, **kw)
    slabs = SlabLattice(X, Y, Z, nslabs, periodic=periodic, periodic_z=periodic, **kw)
    for lat in (single, slabs):
        lat.set_kernel(getattr(pl, "KERNEL_" + kernel))
        if not periodic:
            lat.set_map(m)
            lat.set_inflow(*inflow)
        lat.set_populations(f0.astype(dtype))
        lat.iteration = start
    single.step(9, macro=True)
    slabs.step(9, macro=True)
    a = single.get_populations()
    b = slabs.get_populations()
    # interior and the slab faces: bit for bit
    np.testing.assert_array_equal(a[:, 1:-1], b[:, 1:-1])
    np.testing.assert_array_equal(single.macro(), slabs.macro())
    single.close()
    slabs.close()


def test_slab_flag_refuses_ab_and_scalar(pl):
    lat = pl.LBM(8, 8, 8, viscosity=0.02, periodic=True)
    lat.set_streaming(pl.STREAMING_AB)
    with pytest.raises(pl.LbmError):
        pl._abi.check(lat.lib.lbm_set_distributed_z(lat.h, 1))
    lat.close()
