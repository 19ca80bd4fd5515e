"""State / execute: the Python-side time loop of the binding.

Mirrors the reference's user surface: subclasses of ``State`` override the
virtual hooks that sim_NSE/sim_1.py overrides through PyState
(include/lbm3d/py_state.h:40-157) and ``execute(state)`` runs the loop of
include/lbm3d/core.h:47-112.  Output writers, checkpoint files and MPI are not
part of this hot-path binding.
"""
from __future__ import annotations

import math


class State:
    """Owns one ``LBM`` lattice; override the hooks to set up a simulation."""

    def __init__(self, lbm, final_iteration: int, probe_period: int = 0):
        self.lbm = lbm
        self.final_iteration = int(final_iteration)
        self.probe_period = int(probe_period)
        self.terminate = False

    # hooks (State virtuals, include/lbm3d/state.h:136-226)
    def setupBoundaries(self):
        """Set the GEO map (default: nothing for a periodic lattice)."""

    def resetDFs(self):
        """Initial populations (default: rest equilibrium incl. ghost layer)."""
        self.lbm.init_equilibrium()

    def updateKernelVelocities(self):
        """Per-step inflow update (State::updateKernelVelocities)."""

    def probe1(self):
        """Called every probe_period iterations after a step that produced
        macro fields and sums."""

    def SimInit(self):
        self.setupBoundaries()
        self.resetDFs()

    def SimUpdate(self, nsteps: int, observe: bool):
        self.lbm.step(nsteps, macro=observe, sums=observe)

    def AfterSimUpdate(self, observed: bool):
        if observed:
            s = self.lbm.sums()  # raises LbmError on a non-finite density
            if not math.isfinite(s[0]):
                self.terminate = True
            self.probe1()


def execute(state: State):
    """Time loop: init, then steps in chunks up to the next probe or the end."""
    state.SimInit()
    lbm = state.lbm
    while not state.terminate and lbm.iteration < state.final_iteration:
        state.updateKernelVelocities()
        remaining = state.final_iteration - lbm.iteration
        if state.probe_period > 0:
            to_probe = state.probe_period - (lbm.iteration % state.probe_period)
            n = min(remaining, to_probe)
            observe = (lbm.iteration + n) % state.probe_period == 0
        else:
            n, observe = remaining, False
        state.SimUpdate(n, observe)
        state.AfterSimUpdate(observe)
    lbm.synchronize()
