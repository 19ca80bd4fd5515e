"""The allocation-free sums entry point against the regular sums, through the C-ABI.

Some callers of this library cannot allocate device memory at the point where
they want a reduction: an application whose own pool allocator owns the
device, or a real-time loop that must not stall on an allocation.  lbm_macro_sums_noalloc serves them: it reduces a macro field with
partial sums kept in a fixed file-scope device array, and the caller passes
the already-allocated input and output.  This test checks it against the
regular path (lbm_step with LBM_STEP_SUMS, then lbm_get_sums) on two calls in
a row, which share and reuse that array.

The file is named to be collected last, so that a failure here comes after
every other test has run; it builds its own lattices and also passes when run
alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from helpers import duct_map

pytestmark = pytest.mark.gpu

# the sums tests' tolerance for FP64 sums of the same values in another order
RTOL = 1e-12


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def noalloc_fn(pl):
    fn = pl.library().lbm_macro_sums_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    return fn


# 2048 blocks of 256 threads cover 524,288 sites in one pass; the larger
# lattice makes every block walk its grid-stride loop more than once
@pytest.mark.parametrize("shape", [(150, 40, 30), (128, 96, 72)], ids=["one_pass", "grid_stride"])
@pytest.mark.parametrize("storage,dtype_code", [("F32", 1), ("F64", 0)])
def test_noalloc_sums_match_regular_sums_on_two_calls(pl, storage, dtype_code, shape):
    import torch
    fn = noalloc_fn(pl)
    X, Y, Z = shape
    rng = np.random.default_rng(42)
    lat = pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=0, storage=getattr(pl, "STORE_" + storage))
    lat.set_map(duct_map(X, Y, Z))
    lat.set_inflow(0.03 * np.ones((Z, Y)), None, None)
    rho = 1 + 0.01 * rng.standard_normal((Z, Y, X))
    u = 0.02 * rng.standard_normal((3, Z, Y, X))
    lat.init_equilibrium(rho, *u)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")  # the caller's output buffer
    for call in range(2):
        lat.step(3, macro=True, sums=True)
        expected = lat.sums()
        view = lat.device_view()
        rc = fn(view.macro, dtype_code, X * Y * Z, out.data_ptr(), view.stream)
        assert rc == 0, pl.library().lbm_last_error().decode()
        lat.synchronize()
        got = out.cpu().numpy()
        scale = abs(expected[0])
        np.testing.assert_allclose(got[:5], expected[:5], rtol=RTOL, atol=RTOL * scale, err_msg=f"call {call}")
        assert got[5] == expected[5] == 0
    lat.close()


def test_noalloc_rejects_sizes_beyond_its_maximum(pl):
    import torch
    fn = noalloc_fn(pl)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    too_many = (1 << 40) + 1
    # the size is checked before anything is launched
    assert fn(out.data_ptr(), 0, too_many, out.data_ptr(), None) == 5
    assert b"exceed the maximum" in pl.library().lbm_last_error()
    assert fn(out.data_ptr(), 0, 0, out.data_ptr(), None) == 1
    assert fn(out.data_ptr(), 7, 16, out.data_ptr(), None) == 1


def test_noalloc_calls_allocate_no_device_memory(pl):
    """After the set-up call, further calls leave the device's free memory
    unchanged (cudaMemGetInfo)."""
    import torch
    fn = noalloc_fn(pl)
    X, Y, Z = 96, 40, 30
    lat = pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=0, storage=pl.STORE_F32, periodic=True)
    lat.init_equilibrium()
    lat.step(2, macro=True)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    view = lat.device_view()
    assert fn(view.macro, 1, X * Y * Z, out.data_ptr(), view.stream) == 0
    lat.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert fn(view.macro, 1, X * Y * Z, out.data_ptr(), view.stream) == 0
    lat.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    lat.close()


def test_noalloc_counts_a_nonfinite_density(pl):
    """A NaN population spreads to a few sites' densities: the regular path
    reports them (LBM_ERR_NONFINITE) and the allocation-free sums count
    exactly the non-finite densities of the macro field."""
    import torch
    fn = noalloc_fn(pl)
    X, Y, Z = 32, 16, 12
    lat = pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=0, storage=pl.STORE_F64, periodic=True)
    lat.init_equilibrium()
    f = lat.get_populations()
    f[0, 5, 6, 7] = np.nan
    lat.set_populations(f)
    lat.step(2, macro=True, sums=True)
    with pytest.raises(pl.LbmError) as e:
        lat.sums()
    assert e.value.code == 4
    bad = int(np.count_nonzero(~np.isfinite(lat.macro()[0])))
    assert bad >= 1
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    for call in range(2):
        view = lat.device_view()
        assert fn(view.macro, 0, X * Y * Z, out.data_ptr(), view.stream) == 0
        lat.synchronize()
        assert out.cpu().numpy()[5] == bad, f"call {call}"
    lat.close()
