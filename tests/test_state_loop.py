"""Host logic of pytnl_lbm.State / execute on CPU, against a fake lattice.

The driver mirrors include/lbm3d/core.h:47-112 and the counters, flags and
checkpoint handling of include/lbm3d/state.hpp; these tests check the
iterations at which hooks and actions run, the batching of steps between
actions, the output cuts, the wall-time checkpoint and resume, and the
termination on a non-finite density.  No GPU is used.
"""
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tnl-lbm_b200"))

import pytnl_lbm as pl  # noqa: E402
from pytnl_lbm import Actions, State, execute  # noqa: E402


class FakeLattice:
    """Records step calls; macro field = iteration-dependent ramps."""

    def __init__(self, X=6, Y=5, Z=4, periodic=False, nan_at=None):
        self.X, self.Y, self.Z = X, Y, Z
        self.desc = types.SimpleNamespace(periodic=1 if periodic else 0)
        self.iteration = 0
        self.steps = []  # (start iteration, n, observed)
        self.map = None
        self.nan_at = nan_at
        self.macro_valid = False
        self.saved = {}

    def init_equilibrium(self):
        self.inited = True

    def set_map(self, m):
        self.map = np.array(m, copy=True)

    def step(self, n, macro=False, sums=False):
        self.steps.append((self.iteration, n, bool(macro or sums)))
        self.iteration += n
        self.macro_valid = macro

    def sums(self):
        if self.nan_at is not None and self.iteration >= self.nan_at:
            raise pl.LbmError(4, "non-finite density")
        return np.array([self.X * self.Y * self.Z, 0, 0, 0, 0, 0], float)

    def macro(self):
        assert self.macro_valid, "macro requested without a macro step"
        z, y, x = np.meshgrid(np.arange(self.Z), np.arange(self.Y), np.arange(self.X), indexing="ij")
        return np.stack([1.0 + 0 * x, x + 100 * self.iteration, y, z]).astype(float)

    def get_populations(self, layout=0):
        f = np.zeros((27, self.Z, self.Y, self.X))
        f[0] = 1.0
        return f

    def get_map(self):
        return np.array(self.map, copy=True)

    def save_checkpoint(self, path):
        with open(path, "wb") as fh:
            np.savez(fh, iteration=self.iteration, map=self.map)

    def load_checkpoint(self, path):
        with open(path, "rb") as fh:
            d = np.load(fh)
            self.iteration = int(d["iteration"])
            self.map = d["map"]

    def synchronize(self):
        pass


class Probing(State):
    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.probes = []

    def probe1(self):
        self.probes.append(self.nse.iterations)


def test_counters_fire_on_the_reference_iterations_and_steps_are_batched(tmp_path):
    lat = FakeLattice()
    st = Probing("a", lat, phys_dt=1.0, phys_final_time=35, results_root=str(tmp_path))
    st.cnt[Actions.PROBE1].period = 10
    execute(st)
    # probe at t = 0 (initial snapshot) and every 10 iterations; the loop ends
    # at the first iteration with physTime > physFinalTime
    assert st.probes == [0, 10, 20, 30]
    assert lat.iteration == 36
    assert lat.steps == [(0, 10, True), (10, 10, True), (20, 10, True), (30, 6, False)]
    assert st.flagExists("finished") and not st.flagExists("loadstate")


def test_physical_time_step_sets_the_action_iterations(tmp_path):
    lat = FakeLattice()
    st = Probing("dt", lat, phys_dt=0.3, phys_final_time=3.0, results_root=str(tmp_path))
    st.cnt[Actions.PROBE1].period = 1.0
    execute(st)
    # first iterations with 0.3 * it >= k: 0, 4 (1.2), 7 (2.1), 10 (3.0 up to rounding)
    expect = [0]
    for k in (1, 2, 3):
        it = 0
        while 0.3 * it < k:
            it += 1
        expect.append(it)
    assert st.probes == [e for e in expect if 0.3 * e <= 3.0 + 0.3]
    assert 0.3 * lat.iteration > 3.0 and 0.3 * (lat.iteration - 1) <= 3.0


def test_per_step_hooks_force_single_steps(tmp_path):
    class Inflow(State):
        calls = 0

        def updateKernelVelocities(self):
            Inflow.calls += 1

    lat = FakeLattice()
    st = Inflow("b", lat, phys_final_time=7, results_root=str(tmp_path))
    execute(st)
    assert Inflow.calls == 8
    assert all(n == 1 for _, n, _ in lat.steps) and lat.iteration == 8


def test_cuts_are_written_from_the_observed_macro_field(tmp_path):
    lat = FakeLattice()
    st = State("c", lat, phys_final_time=20, results_root=str(tmp_path))
    st.cnt[Actions.OUT2D].period = 10
    st.add2Dcut_X(2, "cutx")
    st.add2Dcut_Z(1, "cutz")
    st.add3Dcut(1, 1, 1, 3, 2, 2, "box")
    st.cnt[Actions.OUT3DCUT].period = 10
    execute(st)
    d = st.results_dir
    c0 = np.load(os.path.join(d, "cutx_000000.npy"))  # initial condition: rho 1, zero velocity
    assert c0.shape == (4, lat.Z, lat.Y) and np.all(c0[0] == 1) and np.all(c0[1:] == 0)
    c1 = np.load(os.path.join(d, "cutx_000001.npy"))  # after 10 iterations
    assert np.all(c1[1] == 2 + 100 * 10)
    cz = np.load(os.path.join(d, "cutz_000002.npy"))
    assert cz.shape == (4, lat.Y, lat.X) and np.all(cz[3] == 1)
    box = np.load(os.path.join(d, "box_000001.npy"))
    assert box.shape == (4, 2, 2, 3) and np.all(box[1][:, :, 0] == 1 + 1000)


def test_wall_time_saves_a_checkpoint_and_the_next_run_resumes(tmp_path):
    lat = FakeLattice()
    st = Probing("d", lat, phys_final_time=20, wall_time=1e-9, results_root=str(tmp_path), max_batch=7)
    st.cnt[Actions.PROBE1].period = 5
    execute(st)
    # the wall-time check after the first batch (up to the probe at 5) saves and stops
    assert lat.iteration == 5 and st.probes == [0, 5]
    assert st.flagExists("loadstate")
    assert os.path.exists(os.path.join(st.results_dir, "checkpoint"))
    assert not os.path.exists(os.path.join(st.results_dir, "checkpoint_tmp"))
    lat2 = FakeLattice()
    st2 = Probing("d", lat2, phys_final_time=1e10, results_root=str(tmp_path))
    assert st2.canCompute()
    execute(st2)
    assert lat2.steps[0][0] == 5  # resumed at the saved iteration
    # counters, periods and the final time come from the checkpoint
    assert st2.probes == [10, 15, 20] and st2.nse.physFinalTime == 20
    assert lat2.iteration == 21
    assert st2.flagExists("finished") and not st2.flagExists("loadstate")
    assert not st2.canCompute()


def test_non_finite_density_terminates(tmp_path):
    lat = FakeLattice(nan_at=20)
    st = State("e", lat, phys_final_time=100, results_root=str(tmp_path))
    st.cnt[Actions.PROBE2].period = 10
    execute(st)
    assert lat.iteration == 20
    assert st.nse.terminate and st.flagExists("terminated")


def test_project_png_marks_walls(tmp_path):
    from PIL import Image
    img = np.zeros((8, 8, 3), np.uint8)
    img[:, :4] = 255  # left half lit
    path = str(tmp_path / "wall.png")
    Image.fromarray(img).save(path)
    lat = FakeLattice(X=6, Y=5, Z=4)
    st = State("f", lat, results_root=str(tmp_path))
    assert st.projectPNG_X(path, 3)
    plane = st.map[:, :, 3]  # [z, y]; a = z selects the pixel column
    wall = plane == pl.GEO["WALL"]
    for z in range(lat.Z):
        col = int(np.trunc(z / (lat.Z - 1) * 7))
        assert np.all(wall[z, :] == (col < 4))
    assert not st.projectPNG_X(str(tmp_path / "missing.png"), 0)
