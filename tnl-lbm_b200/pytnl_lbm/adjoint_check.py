"""Gradient check of the discrete adjoint on a channel with a forcing control.

Case: a 256 x 64 x 64 D3Q27 channel (GEO_NOTHING rims, bounce-back walls one
site inside, a velocity inlet GEO_INFLOW at x = 0 with a parabolic profile of
u_max = 0.03, a fixed-density outlet GEO_OUTFLOW_EQ), SRT collision with the
second-order equilibrium.  The control is a per-cell body force along x made
of seeded Gaussian bumps of amplitude 1e-3; the objective is the L2 mismatch
J = 1/2 sum |u - u*|^2 of the velocity on 8 cross-sections after N steps,
against a target flow generated with a different seeded control.

Reports the time of the forward pass (with sqrt(N) checkpoints) and of the
backward pass, the device memory of the checkpoints, the agreement of the FP64
gradient and of the FP32 one (FP32 primal, FP64 adjoint) with central finite
differences of the FP64 objective on random cells, and of the two gradients
with each other.

    python -m pytnl_lbm.adjoint_check --steps 4000 --fd-cells 32
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import COLL_SRT, EQ_SECOND_ORDER, GEO, LBM, STORE_F32, STORE_F64

X, Y, Z = 256, 64, 64
U_MAX = 0.03
NU = 0.02


def channel_map():
    m = np.zeros((Z, Y, X), np.uint8)
    m[:, :, 0] = GEO["INFLOW"]
    m[:, :, -1] = GEO["OUTFLOW_EQ"]
    m[:, 1, :] = m[:, -2, :] = GEO["WALL"]
    m[1, :, :] = m[-2, :, :] = GEO["WALL"]
    m[:, 0, :] = m[:, -1, :] = GEO["NOTHING"]
    m[0, :, :] = m[-1, :, :] = GEO["NOTHING"]
    return m


def inlet_profile():
    """Product parabola between the wall sites y, z = 1 and N - 2."""
    y = (np.arange(Y) - 1) / (Y - 3)
    z = (np.arange(Z) - 1) / (Z - 3)
    py = np.clip(4 * y * (1 - y), 0, None)
    pz = np.clip(4 * z * (1 - z), 0, None)
    return U_MAX * np.outer(pz, py)


def bumps(seed, n=12, amplitude=1e-3, width=6.0):
    """Force field [3, Z, Y, X]: Gaussian bumps along x of the given amplitude."""
    rng = np.random.default_rng(seed)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    fx = np.zeros((Z, Y, X))
    for _ in range(n):
        cx, cy, cz = rng.uniform(20, X - 20), rng.uniform(8, Y - 8), rng.uniform(8, Z - 8)
        s = rng.choice([-1.0, 1.0])
        fx += s * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2) / (2 * width * width))
    fx *= amplitude / max(np.max(np.abs(fx)), 1e-30)
    F = np.zeros((3, Z, Y, X))
    F[0] = fx
    return F


def sample_sites(m):
    planes = [int(X * (k + 1) / 9) for k in range(8)]
    idx = []
    for x in planes:
        zz, yy = np.nonzero(m[:, :, x] == GEO["FLUID"])
        idx.append((zz * Y + yy) * X + x)
    return np.concatenate(idx).astype(np.int64)


def make(storage):
    lat = LBM(X, Y, Z, viscosity=NU, collision=COLL_SRT, equilibrium=EQ_SECOND_ORDER, storage=storage)
    m = channel_map()
    lat.set_map(m)
    lat.set_inflow(inlet_profile(), None, None)
    return lat, m


def run(lat, F, steps, samples, target, every=0):
    lat.init_equilibrium()
    return lat.adjoint_forward(F, steps, samples, target, checkpoint_every=every)


def target_velocities(steps, samples):
    """u* on the sample sites from the flow under a different control: the
    moments (sum c f + F*/2) / rho of the state after an even number of steps,
    whose A-A slots then hold the populations of their own sites."""
    assert steps % 2 == 0
    lat, m = make(STORE_F64)
    F = bumps(seed=99)
    lat.init_equilibrium()
    lat.adjoint_forward(F, steps, samples, np.zeros((len(samples), 4)), checkpoint_every=steps)
    lat.adjoint_release()
    f = lat.get_populations()[:, 1:-1, 1:-1, 1:-1].reshape(27, -1)[:, samples]
    lat.close()
    c = np.array([[0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1],
                  [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1],
                  [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1]], float)
    rho = f.sum(axis=0)
    u = (c @ f + 0.5 * F.reshape(3, -1)[:, samples]) / rho
    t = np.zeros((len(samples), 4))
    t[:, 0] = 1.0
    t[:, 1:] = u.T
    return t


def check(steps=4000, fd_cells=32, h=1e-6, seed=7):
    lat, m = make(STORE_F64)
    samples = sample_sites(m)
    target = target_velocities(steps, samples)
    F = bumps(seed=seed)
    every = int(math.ceil(math.sqrt(steps)))
    t0 = time.perf_counter()
    J = run(lat, F, steps, samples, target, every)
    t1 = time.perf_counter()
    g = lat.adjoint_backward()
    t2 = time.perf_counter()
    rng = np.random.default_rng(seed)
    fluid = np.flatnonzero((m == GEO["FLUID"]).ravel())
    cells = rng.choice(fluid, size=fd_cells, replace=False)
    scale = np.max(np.abs(g[0]))
    fds = []
    for c in cells:
        idx = np.unravel_index(int(c), m.shape)
        Fp, Fm = F.copy(), F.copy()
        Fp[(0,) + idx] += h
        Fm[(0,) + idx] -= h
        fds.append((run(lat, Fp, steps, samples, target, steps) - run(lat, Fm, steps, samples, target, steps)) / (2 * h))
    sy = (16 + X + 4 + 15) // 16 * 16  # row pitch of the FP64 layout
    pop_bytes = 27 * sy * (Y + 2) * (Z + 2) * 8
    lat.close()
    lat32, _ = make(STORE_F32)
    t3 = time.perf_counter()
    run(lat32, F, steps, samples, target, every)
    g32 = lat32.adjoint_backward()
    t4 = time.perf_counter()
    lat32.close()

    def rel_errs(grad):
        return [abs(fd - grad[(0,) + np.unravel_index(int(c), m.shape)]) / max(abs(fd), 1e-3 * scale)
                for c, fd in zip(cells, fds)]
    errs, errs32 = rel_errs(g), rel_errs(g32)
    normwise32 = [abs(fd - g32[(0,) + np.unravel_index(int(c), m.shape)]) / scale for c, fd in zip(cells, fds)]
    return {
        "case": f"channel {X}x{Y}x{Z}, SRT, inlet u_max {U_MAX}, nu {NU}, {steps} steps, {len(samples)} samples on 8 planes",
        "objective": J, "checkpoint_every": every,
        "f64_forward_s": t1 - t0, "f64_backward_s": t2 - t1, "f32_forward_backward_s": t4 - t3,
        "checkpoint_memory_gb_f64": (math.ceil(steps / every) + every + 2) * pop_bytes / 1e9,
        "fd_cells": fd_cells, "fd_step": h, "fd_max_rel_err": float(np.max(errs)), "fd_median_rel_err": float(np.median(errs)),
        "fd_f32_max_rel_err": float(np.max(errs32)), "fd_f32_max_normwise_err": float(np.max(normwise32)),
        "f32_vs_f64_grad_rel_linf": float(np.max(np.abs(g32[0] - g[0])) / scale),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--fd-cells", type=int, default=32)
    args = ap.parse_args(argv)
    print(json.dumps(check(args.steps, args.fd_cells)))


if __name__ == "__main__":
    main()
