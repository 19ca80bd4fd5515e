"""pytnl_lbm.State / execute over a real lattice on the GPU.

The driver steps in CUDA-graph batches between actions; the probes must see
the same sums as a hand-written loop that steps one observation at a time,
and a run stopped by the wall-time limit and resumed from its checkpoint
must end bit for bit where an uninterrupted run ends.
"""
import numpy as np
import pytest

from helpers import GEO, duct_map

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def tgv(pl, n=24):
    lat = pl.LBM(n, n, n, viscosity=0.02, cum_flags=3, storage=pl.STORE_F64, periodic=True)
    return lat


def test_probes_see_the_sums_of_a_plain_loop(pl, tmp_path):
    class KE(pl.State):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            self.seen = []

        def resetDFs(self):
            self.nse.lattice.init_taylor_green(0.05, 1.0)

        def probe1(self):
            if self.sums is not None and self.nse.iterations > 0:
                self.seen.append((self.nse.iterations, self.sums.copy()))

    lat = tgv(pl)
    st = KE("tgv", lat, phys_final_time=99, results_root=str(tmp_path))
    st.cnt[pl.Actions.PROBE1].period = 25
    pl.execute(st)
    assert [it for it, _ in st.seen] == [25, 50, 75, 100]  # the last batch ends on a probe
    assert lat.iteration == 100
    ref = tgv(pl)
    ref.init_taylor_green(0.05, 1.0)
    for it, s in st.seen:
        ref.step(it - ref.iteration - 1)
        ref.step(1, macro=True, sums=True)
        np.testing.assert_array_equal(ref.sums(), s)
    assert ref.iteration == 100
    np.testing.assert_array_equal(ref.get_populations(), lat.get_populations())
    lat.close()
    ref.close()


def test_wall_time_checkpoint_resumes_bit_for_bit(pl, tmp_path):
    X, Y, Z = 40, 12, 10

    class Duct(pl.State):
        def setupBoundaries(self):
            self.map[...] = duct_map(X, Y, Z, GEO["INFLOW_LEFT"], GEO["OUTFLOW_EQ"])

        def resetDFs(self):
            lat = self.nse.lattice
            lat.set_inflow(0.02 * np.ones((Z, Y)), None, None)
            lat.init_equilibrium()

    def lattice():
        return pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=0, storage=pl.STORE_F32)

    full = lattice()
    st = Duct("full", full, phys_final_time=60, results_root=str(tmp_path))
    st.cnt[pl.Actions.PROBE1].period = 20
    pl.execute(st)
    assert full.iteration == 61 and st.flagExists("finished")

    first = lattice()
    st1 = Duct("cut", first, phys_final_time=60, wall_time=1e-9, max_batch=13, results_root=str(tmp_path))
    st1.cnt[pl.Actions.PROBE1].period = 20
    pl.execute(st1)
    assert first.iteration == 13 and st1.flagExists("loadstate")
    second = lattice()
    st2 = Duct("cut", second, results_root=str(tmp_path))
    pl.execute(st2)
    assert second.iteration == 61 and st2.flagExists("finished")
    np.testing.assert_array_equal(st2.map, duct_map(X, Y, Z, GEO["INFLOW_LEFT"], GEO["OUTFLOW_EQ"]))
    np.testing.assert_array_equal(full.get_populations(), second.get_populations())
    for lat in (full, first, second):
        lat.close()
