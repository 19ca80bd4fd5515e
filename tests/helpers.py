"""Shared helpers of the test-suite: maps, seeded states, error measures."""
from __future__ import annotations

import numpy as np

GEO = dict(FLUID=0, WALL=1, INFLOW=2, INFLOW_LEFT=3, INFLOW_BB_LEFT=4, INFLOW_EQ_LEFT=5, OUTFLOW_EQ=6,
           OUTFLOW_RIGHT=7, OUTFLOW_RIGHT_INTERP=8, PERIODIC=9, NOTHING=10, SYM_TOP=11, SYM_BOTTOM=12,
           SYM_LEFT=13, SYM_RIGHT=14, SYM_BACK=15, SYM_FRONT=16)
COLL_IDS = {"CUM": 0, "SRT": 1, "BGK": 2, "MRT": 3}
EQ_IDS = {"EQ": 0, "INV_CUM": 1}
RACE_FREE_TYPES = np.array([0, 1, 2, 3, 5, 6, 9, 10, 11, 12, 13, 14, 15, 16], np.uint8)


def duct_map(X, Y, Z, inlet=GEO["INFLOW_LEFT"], outlet=GEO["OUTFLOW_EQ"]):
    """Rectangular duct of sim_NSE/sim_2.cu:140-157: walls one site inside the
    y/z rims, GEO_NOTHING rims, inlet at x = 0, outlet at x = X-1."""
    m = np.zeros((Z, Y, X), np.uint8)
    m[:, :, 0] = inlet
    m[:, :, -1] = outlet
    m[:, 1, :] = GEO["WALL"]
    m[:, -2, :] = GEO["WALL"]
    m[1, :, :] = GEO["WALL"]
    m[-2, :, :] = GEO["WALL"]
    m[:, 0, :] = GEO["NOTHING"]
    m[:, -1, :] = GEO["NOTHING"]
    m[0, :, :] = GEO["NOTHING"]
    m[-1, :, :] = GEO["NOTHING"]
    return m


def sym_box_map(X, Y, Z):
    m = np.zeros((Z, Y, X), np.uint8)
    m[0], m[-1] = GEO["SYM_BOTTOM"], GEO["SYM_TOP"]
    m[:, 0], m[:, -1] = GEO["SYM_BACK"], GEO["SYM_FRONT"]
    m[:, :, 0], m[:, :, -1] = GEO["SYM_LEFT"], GEO["SYM_RIGHT"]
    return m


def random_map(rng, X, Y, Z):
    return rng.choice(RACE_FREE_TYPES, size=(Z, Y, X)).astype(np.uint8)


def tgv_fields(X, Y, Z, u0=0.05, rho0=1.0):
    """Taylor-Green vortex of sim_NSE/sim_4.cu:152-160 at cell centres."""
    kx, ky, kz = 2 * np.pi / X, 2 * np.pi / Y, 2 * np.pi / Z
    z, y, x = np.meshgrid((np.arange(Z) + 0.5 - Z / 2) * kz, (np.arange(Y) + 0.5 - Y / 2) * ky,
                          (np.arange(X) + 0.5 - X / 2) * kx, indexing="ij")
    u = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -u0 * (kx / ky) * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(u)
    rho = rho0 + 3 * (u0 * u0 / 16) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    return rho, u, v, w


def seeded_state(port, rng, X, Y, Z, eq="INV_CUM", dtype=np.float64, noise=0.01, uniform=(1.0, 0.01, 0.0, 0.0)):
    """Equilibrium of a random (rho, u) field times a small multiplicative noise,
    ghost layer included."""
    f = port.allocate(X, Y, Z, np.float64)
    rho = 1 + 0.01 * rng.standard_normal((Z, Y, X))
    u = 0.03 * rng.standard_normal((3, Z, Y, X))
    port.init_equilibrium(f, X, Y, Z, eq=eq, fields=(rho, *u), uniform=uniform)
    f *= 1 + noise * rng.standard_normal(f.shape)
    return np.ascontiguousarray(f.astype(dtype))


def rel_linf(a, b):
    """Relative L-infinity error ||a - b||_inf / ||b||_inf (norm-wise)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_linf_fields(a, b):
    """Norm-wise relative L-infinity error of a macro field [rho, vx, vy, vz]:
    the density against its own scale, the velocity vector against max |u|
    over all three components (a component that is zero in the flow carries
    only rounding noise and has no scale of its own)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    vel_scale = max(np.max(np.abs(b[1:4])), 1e-300)
    return max(rel_linf(a[0], b[0]), float(np.max(np.abs(a[1:4] - b[1:4])) / vel_scale))


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))
