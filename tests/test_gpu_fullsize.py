"""The benchmark workloads at their full sizes, through properties that do
not depend on an oracle run (the CPU reference at these sizes would take
hours; the parity at the configurations' own small sizes is in
test_gpu_baseline_configs.py).

* The duct 512 x 128 x 128 (the bench's FP32 workload): the two-site step the
  autotuner picks and the one-site step compute the same update; after 20
  steps their populations agree to the two-site kernel's FP32 bound (2e-6,
  tests/test_gpu_pair.py) and their FP64 sums to 1e-6.
* The Taylor-Green vortex 512^3 (the largest single-GPU configuration) in
  FP32 and in FP16 shifted storage on the two-site kernel: mass is conserved,
  the total momentum stays zero (the initial field is antisymmetric in every
  velocity component), the kinetic energy decays, and no density is
  non-finite.
"""
import importlib.util
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_fullsize", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def interior(lat):
    """Device view of the interior populations [27, Z, Y, X] (no copy)."""
    t = lat.populations_tensor()
    x0 = lat.device_view().x0
    return t[:, 1:-1, 1:-1, x0:x0 + lat.X]


def test_duct_full_size_two_site_step_tracks_one_site_step(pl):
    import torch
    bench = load_bench()
    spec = bench.workload_spec("duct")
    lats = []
    for kernel in ("direct", "pair"):
        lat, _ = bench.make_lattice(pl, spec, "f32", 0, kernel)
        lat.step(20, sums=True)
        lats.append(lat)
    sums = [lat.sums() for lat in lats]
    a, b = interior(lats[0]), interior(lats[1])
    worst = 0.0
    for q in range(27):  # one slot at a time: no full-size temporaries
        worst = max(worst, float(torch.max(torch.abs(a[q] - b[q]))))
    for lat in lats:
        lat.close()
    assert worst <= 2e-6, worst
    np.testing.assert_allclose(sums[1][:5], sums[0][:5], rtol=1e-6, atol=1e-6 * sums[0][0])
    assert sums[0][5] == sums[1][5] == 0


def test_taylor_green_512_invariants(pl):
    N = 512
    nu = 0.05 * (N / (2 * math.pi)) / 1600.0
    sums = {}
    for storage in ("F32", "F16S"):
        lat = pl.LBM(N, N, N, viscosity=nu, cum_flags=pl.CUM_GEIER_2017 | pl.CUM_ANTIALIAS,
                     equilibrium=pl.EQ_INV_CUM, storage=getattr(pl, "STORE_" + storage), periodic=True)
        lat.set_kernel(pl.KERNEL_PAIR)
        lat.init_taylor_green(0.05, 1.0)
        lat.step(2, sums=True)
        s0 = lat.sums()
        lat.step(18, sums=True)
        sums[storage] = (s0, lat.sums())
        lat.close()
    sites = float(N) ** 3
    scale = sites * 0.05 / 4  # sum rho |u| ~ sites U0 / 4
    for storage, (s0, s1) in sums.items():
        # mass: FP32 arithmetic and FP64 sums; the 16-bit storage drifts by
        # about 1e-8 per site and step
        assert abs(s1[0] / s0[0] - 1) <= (1e-7 if storage == "F32" else 1e-6), storage
        # momentum: zero by symmetry of the initial field
        assert np.max(np.abs(s1[1:4])) <= 1e-6 * scale, (storage, s1[1:4])
        assert s1[5] == 0
    # FP32: the vortex decays; FP16 storage follows FP32 (its storage steps
    # stir acoustic noise of ~1e-5 of the kinetic energy in these 20 steps)
    assert sums["F32"][1][4] < sums["F32"][0][4]
    assert abs(sums["F16S"][1][4] / sums["F32"][1][4] - 1) <= 1e-4
