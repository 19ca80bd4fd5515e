"""State / execute: the Python-side simulation driver of the binding.

Mirrors the reference's user surface for Python solvers: ``State`` carries
the hooks that ``PyState`` lets Python override (include/lbm3d/py_state.h:
40-157, exported at :159-302), the action counters of include/lbm3d/state.h:
48-71, the result-directory flags, wall-time limit and checkpoint/resume of
include/lbm3d/state.hpp:149-211, 945-1049, and ``execute(state)`` runs the
time loop of include/lbm3d/core.h:47-112.

Differences, all on the host side of the hot path:

* ``nse`` wraps one ``LBM`` lattice on one GPU (no MPI blocks); ``physTime()``
  is ``physDt * iterations`` as in include/lbm3d/lbm.h:61-64.
* Checkpoints are the binary files of ``lbm_checkpoint_save`` (ADIOS2 is not
  part of this build), written to ``results_<id>/checkpoint_tmp`` and renamed
  over ``results_<id>/checkpoint``.
* 2D cuts and 3D boxes registered with ``add2Dcut_*`` / ``add3Dcut`` are
  written as ``.npy`` arrays of the macro fields (rho, vx, vy, vz) under
  ``results_<id>/`` instead of ADIOS2 files.
* The loop steps in CUDA-graph batches: when no per-step hook
  (``updateKernelData``, ``updateKernelVelocities``, ``computeBeforeLBMKernel``,
  ``computeAfterLBMKernel``) is overridden, the steps up to the next counter
  action, the final time or the wall-time check run as one ``lbm_step`` call;
  the iterations at which hooks and actions run are those of the reference.
  Only the step before an action outputs the macro field and the FP64 sums.
"""
from __future__ import annotations

import enum
import math
import os
import time

import numpy as np


class Actions(enum.IntEnum):
    """Counter slots of include/lbm3d/state.h:58-71."""
    STAT_RESET = 0
    STAT2_RESET = 1
    PRINT = 2
    OUT2D = 3
    OUT3D = 4
    OUT3DCUT = 5
    PROBE1 = 6
    PROBE2 = 7
    PROBE3 = 8
    SAVESTATE = 9


MAX_COUNTER = len(Actions)
STAT_RESET, STAT2_RESET, PRINT, OUT2D, OUT3D, OUT3DCUT, PROBE1, PROBE2, PROBE3, SAVESTATE = tuple(Actions)


class Counter:
    """``counter`` of include/lbm3d/state.h:48-56: an action is due at time t
    when its period is positive and t >= count * period."""

    def __init__(self, period: float = -1.0):
        self.count = 0
        self.period = float(period)

    def action(self, t: float) -> bool:
        return self.period > 0 and t >= self.count * self.period

    def next_time(self) -> float:
        return self.count * self.period if self.period > 0 else math.inf


class NSE:
    """The ``nse`` member of State: one lattice plus the reference's time
    bookkeeping (include/lbm3d/lbm.h:40-64)."""

    def __init__(self, lattice, phys_dt: float = 1.0, phys_final_time: float = 1e10):
        self.lattice = lattice
        self.physDt = float(phys_dt)
        self.physFinalTime = float(phys_final_time)
        self.physStartTime = 0.0
        self.startIterations = 0
        self.terminate = False

    @property
    def iterations(self) -> int:
        return self.lattice.iteration

    @iterations.setter
    def iterations(self, it: int):
        self.lattice.iteration = int(it)

    def physTime(self) -> float:
        return self.physDt * self.iterations

    def sites(self) -> int:
        return self.lattice.X * self.lattice.Y * self.lattice.Z


# D3Q27 velocity components in the lattice's direction order
_CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
_CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1])
_CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])


def macro_from_populations(f):
    """rho, vx, vy, vz [4, Z, Y, X] of populations [27, Z, Y, X] (the initial
    macro field of State::reset, state.hpp:1138-1140; no force shift)."""
    f = np.asarray(f, np.float64)
    rho = f.sum(axis=0)
    out = np.empty((4,) + rho.shape)
    out[0] = rho
    out[1] = np.tensordot(_CX, f, axes=1) / rho
    out[2] = np.tensordot(_CY, f, axes=1) / rho
    out[3] = np.tensordot(_CZ, f, axes=1) / rho
    return out


_PER_STEP_HOOKS = ("updateKernelData", "updateKernelVelocities", "computeBeforeLBMKernel", "computeAfterLBMKernel")


def _log(msg: str):
    import logging
    logging.getLogger("pytnl_lbm").info(msg)


class _NpyWriter:
    """Stand-in for the reference's output writer: named arrays as .npy files."""

    def __init__(self, directory: str, tag: str):
        self.directory = directory
        self.tag = tag

    def write(self, name: str, array):
        np.save(os.path.join(self.directory, f"{self.tag}_{name}.npy"), np.asarray(array))


class State:
    """Simulation state around one lattice (State<NSE> of include/lbm3d/state.h).

    Subclass and override the hooks.  ``lattice`` is a ``pytnl_lbm.LBM``;
    ``phys_dt`` converts iterations to the physical time that the counters,
    ``physFinalTime`` and the output cycles use.  ``wall_time`` (seconds, <= 0
    for none) ends the run with a checkpoint, as ``wallTime`` does.
    """

    def __init__(self, id: str, lattice, *, phys_dt: float = 1.0, phys_final_time: float = 1e10,
                 wall_time: float = -1.0, results_root: str = ".", max_batch: int = 1000):
        self.id = str(id)
        self.nse = NSE(lattice, phys_dt, phys_final_time)
        self.cnt = [Counter() for _ in range(MAX_COUNTER)]
        self.wallTime = float(wall_time)
        self.max_batch = max(1, int(max_batch))
        self.probe_needs_macro_on_host = False
        self.results_dir = os.path.join(results_root, f"results_{self.id}")
        os.makedirs(self.results_dir, exist_ok=True)
        self.probe2Dvec = []  # (axis, position, name)
        self.probe3Dvec = []  # (origin, extent, name)
        self.macro = None	  # host copy of the macro field [4, Z, Y, X] after an observed step
        self.sums = None	  # FP64 sums of the last observed step
        self.map = None
        if not lattice.desc.periodic:
            from . import GEO
            self.map = np.full((lattice.Z, lattice.Y, lattice.X), GEO["FLUID"], np.uint8)
        self._t0 = time.perf_counter()
        self._glups_prev = (0.0, 0)
        self._observed = False

    # ---- hooks that solvers override (py_state.h:40-157) --------------------------
    def probe1(self):
        pass

    def probe2(self):
        pass

    def probe3(self):
        pass

    def statReset(self):
        pass

    def stat2Reset(self):
        pass

    def outputData(self, writer, time: float, cycle: int):
        """Extra 3D output next to the macro field (writer.write(name, array))."""

    def setupBoundaries(self):
        """Set ``self.map`` (GEO types, [Z][Y][X]) for a non-periodic lattice."""

    def estimateMemoryDemands(self) -> bool:
        return True	 # the lattice was allocated by its constructor

    def resetDFs(self):
        """Initial populations: rest equilibrium (state.hpp:1143-1149)."""
        self.nse.lattice.init_equilibrium()

    def reset(self):
        """state.hpp:1124-1141: populations, then the map (all fluid, then the
        solver's boundaries), then the map on the device."""
        self.resetDFs()
        if self.map is not None:
            from . import GEO
            self.map[...] = GEO["FLUID"]
            self.setupBoundaries()
            self.nse.lattice.set_map(self.map)

    def updateKernelData(self):
        pass

    def updateKernelVelocities(self):
        pass

    def computeBeforeLBMKernel(self):
        pass

    def computeAfterLBMKernel(self):
        pass

    def copyAllToDevice(self):
        if self.map is not None:
            self.nse.lattice.set_map(self.map)

    def copyAllToHost(self):
        self.nse.lattice.synchronize()

    # ---- configuration ------------------------------------------------------------
    def add2Dcut_X(self, x: int, name: str):
        self.probe2Dvec.append(("X", int(x), str(name)))

    def add2Dcut_Y(self, y: int, name: str):
        self.probe2Dvec.append(("Y", int(y), str(name)))

    def add2Dcut_Z(self, z: int, name: str):
        self.probe2Dvec.append(("Z", int(z), str(name)))

    def add3Dcut(self, ox: int, oy: int, oz: int, lx: int, ly: int, lz: int, name: str):
        self.probe3Dvec.append(((int(ox), int(oy), int(oz)), (int(lx), int(ly), int(lz)), str(name)))

    def _projectPNG(self, filename, plane, pos, rotate, mirror, flip, amin, amax, bmin, bmax):
        """Wall sites from the non-black pixels of a PNG (state.hpp:766-889)."""
        if not os.path.exists(filename):
            return False
        if self.map is None:
            raise ValueError("projectPNG needs a lattice with a map (periodic=False)")
        from PIL import Image
        from . import GEO
        img = np.asarray(Image.open(filename).convert("RGB"))
        h, w = img.shape[:2]
        lit = img.astype(np.int64)
        lit = (lit[..., 0] << 16) + (lit[..., 1] << 8) + lit[..., 2]
        lat = self.nse.lattice
        n = {"x": lat.X, "y": lat.Y, "z": lat.Z}
        # (a axis, b axis) of each plane
        a_ax, b_ax = {"X": ("z", "y"), "Y": ("z", "x"), "Z": ("x", "y")}[plane]
        a = np.arange(n[a_ax], dtype=np.float64) / (n[a_ax] - 1)
        a = amin + a * (amax - amin)
        if mirror:
            a = 1.0 - a
        b = np.arange(n[b_ax], dtype=np.float64) / (n[b_ax] - 1)
        b = bmin + b * (bmax - bmin)
        if flip:
            b = 1.0 - b
        A, B = np.meshgrid(a, b, indexing="ij")	 # [na, nb]
        ia, ib = (B, A) if rotate else (A, B)
        px = np.clip(np.trunc(ia * (w - 1)).astype(np.int64), 0, w - 1)
        py = np.clip(np.trunc(ib * (h - 1)).astype(np.int64), 0, h - 1)
        wall = lit[py, px] > 0	# [na, nb]
        view = {"X": self.map[:, :, pos], "Y": self.map[:, pos, :], "Z": self.map[pos, :, :]}[plane]
        # view axes: X -> (z, y), Y -> (z, x), Z -> (y, x)
        if plane == "Z":
            wall = wall.T
        view[wall] = GEO["WALL"]
        return True

    def projectPNG_X(self, filename, x0, rotate=False, mirror=False, flip=False, amin=0.0, amax=1.0, bmin=0.0, bmax=1.0):
        return self._projectPNG(filename, "X", int(x0), rotate, mirror, flip, amin, amax, bmin, bmax)

    def projectPNG_Y(self, filename, y0, rotate=False, mirror=False, flip=False, amin=0.0, amax=1.0, bmin=0.0, bmax=1.0):
        return self._projectPNG(filename, "Y", int(y0), rotate, mirror, flip, amin, amax, bmin, bmax)

    def projectPNG_Z(self, filename, z0, rotate=False, mirror=False, flip=False, amin=0.0, amax=1.0, bmin=0.0, bmax=1.0):
        return self._projectPNG(filename, "Z", int(z0), rotate, mirror, flip, amin, amax, bmin, bmax)

    # ---- flags and wall time (state.hpp:149-211, 1015-1049) -------------------------
    def _flag(self, name):
        return os.path.join(self.results_dir, f"flag.{name}")

    def flagCreate(self, name: str):
        open(self._flag(name), "a").close()

    def flagDelete(self, name: str):
        if os.path.exists(self._flag(name)):
            os.remove(self._flag(name))

    def flagExists(self, name: str) -> bool:
        return os.path.exists(self._flag(name))

    def canCompute(self) -> bool:
        if self.flagExists("loadstate"):
            return True
        return not (self.flagExists("finished") or self.flagExists("terminated"))

    def getWallTime(self, collective: bool = False) -> float:
        return time.perf_counter() - self._t0

    def wallTimeReached(self) -> bool:
        return self.wallTime > 0 and self.getWallTime() >= self.wallTime

    # ---- checkpoint (state.hpp:891-1012) ---------------------------------------------
    def checkpointState(self, mode: str, path: str):
        """mode "w": write the lattice (populations, map, inflow, iteration) to
        ``path`` and the driver's state (physFinalTime, counters, as
        state.hpp:891-914) to ``path + ".state.json"``; "r": read both back."""
        import json
        meta = path + ".state.json"
        if mode == "w":
            self.nse.lattice.save_checkpoint(path)
            with open(meta, "w") as fh:
                json.dump({"physFinalTime": self.nse.physFinalTime, "iterations": self.nse.iterations,
                           "counters": [[c.count, c.period] for c in self.cnt]}, fh)
        else:
            self.nse.lattice.load_checkpoint(path)
            with open(meta) as fh:
                d = json.load(fh)
            self.nse.physFinalTime = float(d["physFinalTime"])
            for c, (count, period) in zip(self.cnt, d["counters"]):
                c.count, c.period = int(count), float(period)

    def saveState(self):
        """Checkpoint into a staging file, then rename it over the previous
        checkpoint, so that a failed save leaves the old one intact."""
        tmp = os.path.join(self.results_dir, "checkpoint_tmp")
        dst = os.path.join(self.results_dir, "checkpoint")
        self.checkpointState("w", tmp)
        os.replace(tmp + ".state.json", dst + ".state.json")
        os.replace(tmp, dst)
        self.flagCreate("loadstate")

    def loadState(self):
        self.checkpointState("r", os.path.join(self.results_dir, "checkpoint"))
        if self.map is not None:
            self.map = self.nse.lattice.get_map()  # the checkpoint's map (copyMapToHost)
        self.nse.physStartTime = self.nse.physTime()
        self.nse.startIterations = self.nse.iterations
        self._glups_prev = (self.getWallTime(), self.nse.iterations)

    # ---- time loop pieces (state.hpp:1151-1600) ---------------------------------------
    def SimInit(self):
        if not self.estimateMemoryDemands():
            raise RuntimeError("Not enough memory available (CPU or GPU).")
        for c in self.cnt:
            c.count = 0
        self.cnt[SAVESTATE].count = 1  # skip the initial save of state
        self.nse.iterations = 0
        if self.flagExists("loadstate"):
            self.loadState()
            self.copyAllToDevice()
        else:
            self.reset()

    def _per_step_hooks(self) -> bool:
        cls = type(self)
        return any(getattr(cls, h) is not getattr(State, h) for h in _PER_STEP_HOOKS)

    def _due_iteration(self, counter: Counter) -> int:
        """First iteration whose physical time makes the counter's action due."""
        if counter.period <= 0:
            return 1 << 62
        t = counter.next_time()
        it = max(0, int(math.floor(t / self.nse.physDt)) - 1)
        while self.nse.physDt * it < t:
            it += 1
        return it

    def batch_length(self) -> int:
        """Steps until the next iteration at which an action, the final time
        or a per-step hook is due (1 when per-step hooks are overridden)."""
        if self._per_step_hooks():
            return 1
        it = self.nse.iterations
        end = it + self.max_batch
        for c, counter in enumerate(self.cnt):
            if c != SAVESTATE:	# SAVESTATE runs on wall time, checked after every batch
                end = min(end, max(it + 1, self._due_iteration(counter)))
        final = int(math.floor(self.nse.physFinalTime / self.nse.physDt))
        while self.nse.physDt * final <= self.nse.physFinalTime:
            final += 1
        return max(1, min(end, final) - it)

    def SimUpdate(self, nsteps: int = 1):
        """nsteps lattice updates; the last one outputs the macro field and the
        sums when an action other than PRINT or SAVESTATE is then due
        (state.hpp:1270-1280)."""
        lat = self.nse.lattice
        if nsteps == 1:
            self.computeBeforeLBMKernel()
        t_end = self.nse.physDt * (self.nse.iterations + nsteps)
        observe = any(self.cnt[c].action(t_end) for c in range(MAX_COUNTER) if c not in (PRINT, SAVESTATE))
        lat.step(nsteps, macro=observe, sums=observe)
        self._observed = observe

    def AfterSimUpdate(self):
        t = self.nse.physTime()
        skip = (PRINT, SAVESTATE) if self.probe_needs_macro_on_host else (PRINT, SAVESTATE, PROBE1)
        copy_macro = self._observed and any(self.cnt[c].action(t) for c in range(MAX_COUNTER) if c not in skip)
        nan_detected = False
        if self._observed:
            from . import LbmError
            try:
                self.sums = self.nse.lattice.sums()
            except LbmError:
                nan_detected = True	 # lbm_get_sums reports non-finite densities
        self.macro = self.nse.lattice.macro() if copy_macro else None
        if self._per_step_hooks():
            self.computeAfterLBMKernel()
        write_info = any(self.cnt[c].action(t) for c in (PRINT, OUT2D, OUT3D, OUT3DCUT, PROBE1, PROBE2, PROBE3))
        if write_info:
            self.cnt[PRINT].count += 1
        if nan_detected and self.nse.iterations > 1:
            _log("Detected NaN, terminating the simulation.")
            self.nse.terminate = True
        do = {c: self.cnt[c].action(t) for c in (PROBE1, PROBE2, PROBE3, OUT3D, OUT3DCUT, OUT2D)}
        if do[PROBE1]:
            self.probe1()
            self.cnt[PROBE1].count += 1
        if do[PROBE2]:
            self.probe2()
            self.cnt[PROBE2].count += 1
        if do[PROBE3]:
            self.probe3()
            self.cnt[PROBE3].count += 1
        if do[OUT3DCUT]:
            self.write3Dcut(t, self.cnt[OUT3DCUT].count)
            self.cnt[OUT3DCUT].count += 1
        if do[OUT2D]:
            self.write2D(t, self.cnt[OUT2D].count)
            self.cnt[OUT2D].count += 1
        if do[OUT3D]:
            self.write3D(t, self.cnt[OUT3D].count)
            self.cnt[OUT3D].count += 1
        if self.cnt[STAT_RESET].action(t):
            self.statReset()
            self.cnt[STAT_RESET].count += 1
        if self.cnt[STAT2_RESET].action(t):
            self.stat2Reset()
            self.cnt[STAT2_RESET].count += 1
        if write_info and self.nse.iterations > 1:
            now = self.getWallTime()
            t0, it0 = self._glups_prev
            lups = (self.nse.iterations - it0) * self.nse.sites() / max(1e-6, now - t0)
            self._glups_prev = (now, self.nse.iterations)
            _log(f"GLUPS={lups * 1e-9:.3f} iter={self.nse.iterations} t={t:1.3f}s dt={self.nse.physDt:1.2e} WT={now:.0f}s")

    def AfterSimFinished(self):
        its = self.nse.iterations - self.nse.startIterations
        if its > 1:
            _log(f"total walltime: {self.getWallTime():.1f} s, iterations: {its}")

    # ---- output (ADIOS2 replaced by .npy arrays of the macro field) ---------------------
    def _macro_or_fetch(self):
        if self.macro is None:
            if self.nse.iterations == self.nse.startIterations:
                from . import LAYOUT_INTERIOR
                self.macro = macro_from_populations(self.nse.lattice.get_populations(layout=LAYOUT_INTERIOR))
            else:
                self.macro = self.nse.lattice.macro()
        return self.macro

    def write2D(self, time: float, cycle: int):
        m = self._macro_or_fetch()
        for axis, pos, name in self.probe2Dvec:
            cut = {"X": m[:, :, :, pos], "Y": m[:, :, pos, :], "Z": m[:, pos, :, :]}[axis]
            np.save(os.path.join(self.results_dir, f"{name}_{cycle:06d}.npy"), cut)

    def write3Dcut(self, time: float, cycle: int):
        m = self._macro_or_fetch()
        for (ox, oy, oz), (lx, ly, lz), name in self.probe3Dvec:
            np.save(os.path.join(self.results_dir, f"{name}_{cycle:06d}.npy"),
                    m[:, oz:oz + lz, oy:oy + ly, ox:ox + lx])

    def write3D(self, time: float, cycle: int):
        m = self._macro_or_fetch()
        w = _NpyWriter(self.results_dir, f"output_3D_{cycle:06d}")
        for k, name in enumerate(("rho", "vx", "vy", "vz")):
            w.write(name, m[k])
        self.outputData(w, time, cycle)


def execute(state: State):
    """The time loop of include/lbm3d/core.h:47-112."""
    state.SimInit()
    state.AfterSimUpdate()	# snapshot of the initial condition
    per_step = state._per_step_hooks()
    quit = False
    while not quit:
        n = state.batch_length()
        if per_step:
            state.updateKernelData()
            state.updateKernelVelocities()
        state.SimUpdate(n)
        state.AfterSimUpdate()
        if state.wallTimeReached():
            state.copyAllToHost()
            _log("maximum wall time reached")
            state.saveState()
            quit = True
        elif state.cnt[SAVESTATE].action(state.getWallTime(True)):
            state.copyAllToHost()
            state.saveState()
            state.cnt[SAVESTATE].count += 1
        if state.nse.physTime() > state.nse.physFinalTime:
            _log("physFinalTime reached")
            quit = True
            state.flagCreate("finished")
            state.flagDelete("loadstate")
        if state.nse.terminate:
            _log("terminate flag triggered")
            quit = True
            state.flagCreate("terminated")
            state.flagDelete("loadstate")
    state.AfterSimFinished()
    state.nse.lattice.synchronize()
