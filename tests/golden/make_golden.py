"""Generate the golden vectors of the D3Q27 A-A hot path from TNL-LBM's own code.

    python tests/golden/make_golden.py

Runs the reference's per-site operator headers (compiled unmodified from the
reference tree by oracle/Makefile into oracle/_ref/*.so, see
oracle/ref_harness.cpp) on small seeded inputs and stores inputs and outputs
in tests/golden/golden_d3q27.npz.  The reference has no golden data of its own
for this path (its only regression test covers the IBM matrices), so these
fixtures are the pinned record of its behaviour; the test-suite checks the
oracle port and the GPU kernels against them without needing the reference.

Cases (FP64 unless noted):
  site_<coll>[_<flags>]   64 random near-equilibrium sites through one
                          computeDensityAndVelocity + collision (with body force)
  lat_<name>              6x5x4 lattice, several A-A steps, populations incl. the
                          ghost layer and the final macro field
  tgv16_ke                16^3 Taylor-Green vortex (cumulant 2017 + anti-aliasing),
                          kinetic energy every 2 steps for 20 steps
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

SEED = 20260101


def near_eq_sites(rng, n, oracle_impl):
    rho = 1.0 + 0.05 * rng.standard_normal(n)
    u = 0.05 * rng.standard_normal((3, n))
    f = oracle_impl.equilibrium(rho, *u, eq="EQ")
    return np.ascontiguousarray(f * (1.0 + 0.05 * rng.standard_normal(f.shape)))


def duct_map(X, Y, Z, inlet, outlet):
    m = np.zeros((Z, Y, X), np.int16)
    m[:, :, 0] = inlet
    m[:, :, -1] = outlet
    m[:, 1, :] = 1
    m[:, -2, :] = 1
    m[1, :, :] = 1
    m[-2, :, :] = 1
    m[:, 0, :] = 10
    m[:, -1, :] = 10
    m[0, :, :] = 10
    m[-1, :, :] = 10
    return m


LATTICE_CASES = [
    # name, cum_flags, coll, eq, map kind, nu, force, steps
    ("tgv_cum2017", 3, "CUM", "INV_CUM", "periodic", 0.004, (0.0, 0.0, 0.0), 6),
    ("duct_cum", 0, "CUM", "INV_CUM", "duct_left", 0.01, (0.0, 0.0, 0.0), 6),
    ("duct_eq_cumaa", 2, "CUM", "INV_CUM", "duct_eqleft", 0.02, (1e-5, 0.0, 0.0), 5),
    ("sym_srt", 0, "SRT", "EQ", "sym", 0.05, (2e-5, -1e-5, 3e-6), 6),
    ("mix_bgk", 0, "BGK", "EQ", "mix", 0.03, (0.0, 1e-5, 0.0), 4),
    ("periodic_mrt", 0, "MRT", "EQ", "periodic", 0.002, (0.0, 0.0, 0.0), 6),
]


def lattice_map(kind, X, Y, Z, rng):
    if kind == "periodic":
        return np.full((Z, Y, X), 9, np.int16)
    if kind == "duct_left":
        return duct_map(X, Y, Z, 3, 6)
    if kind == "duct_eqleft":
        return duct_map(X, Y, Z, 5, 6)
    if kind == "sym":
        m = np.zeros((Z, Y, X), np.int16)
        m[0], m[-1] = 12, 11
        m[:, 0], m[:, -1] = 15, 16
        m[:, :, 0], m[:, :, -1] = 13, 14
        return m
    choices = np.array([0, 1, 2, 3, 5, 6, 9, 10, 11, 12, 13, 14, 15, 16], np.int16)
    return rng.choice(choices, size=(Z, Y, X)).astype(np.int16)


def main():
    oracle.build()
    port = oracle.Port()
    rng = np.random.default_rng(SEED)
    out = {}
    force = (1e-4, -2e-4, 3e-5)
    nu = 0.003
    # per-site collisions
    for coll, flags_list in (("CUM", (0, 2, 3)), ("SRT", (0,)), ("BGK", (0,)), ("MRT", (0,))):
        for flags in flags_list:
            ref = oracle.Reference(flags)
            f0 = near_eq_sites(rng, 64, port)
            f1 = f0.copy()
            macro = ref.collide(f1, coll=coll, eq="INV_CUM", nu=nu, force=force)
            key = f"site_{coll}" + (f"_{flags}" if coll == "CUM" else "")
            out[key + "_in"] = f0
            out[key + "_out"] = f1
            out[key + "_macro"] = macro
    out["site_nu"] = np.array(nu)
    out["site_force"] = np.array(force)
    # lattices
    X, Y, Z = 6, 5, 4
    for name, flags, coll, eq, kind, lnu, lforce, steps in LATTICE_CASES:
        ref = oracle.Reference(flags)
        m = lattice_map(kind, X, Y, Z, rng)
        f = ref.allocate(X, Y, Z)
        rho = 1 + 0.01 * rng.standard_normal((Z, Y, X))
        u = 0.03 * rng.standard_normal((3, Z, Y, X))
        ref.init_equilibrium(f, X, Y, Z, eq=eq, fields=(rho, *u), uniform=(1.0, 0.01, 0.0, 0.0))
        f *= 1 + 0.01 * rng.standard_normal(f.shape)
        prof = np.ascontiguousarray(0.02 * rng.random((Z, Y))), np.ascontiguousarray(0.005 * rng.random((Z, Y)))
        f_in = f.copy()
        macro = np.zeros((4, Z, Y, X))
        ref.aa_run(f, m, coll=coll, eq=eq, nu=lnu, force=lforce, inflow=(prof[0], prof[1], None), macro=macro,
                   nsteps=steps)
        p = "lat_" + name
        out[p + "_map"] = m
        out[p + "_in"] = f_in
        out[p + "_out"] = f
        out[p + "_macro"] = macro
        out[p + "_inflow"] = np.stack(prof)
        out[p + "_params"] = np.array([flags, ["CUM", "SRT", "BGK", "MRT"].index(coll), ["EQ", "INV_CUM"].index(eq),
                                       lnu, *lforce, steps])
    # Taylor-Green kinetic energy series
    N = 16
    ref = oracle.Reference(3)
    f = ref.allocate(N, N, N)
    k = 2 * np.pi / N
    c = (np.arange(N) + 0.5 - N / 2) * k
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    U0 = 0.05
    u = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(u)
    rho = 1 + 3 * (U0 * U0 / 16) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    ref.init_equilibrium(f, N, N, N, eq="INV_CUM", fields=(rho, u, v, w))
    m = np.full((N, N, N), 9, np.int16)
    nu_tgv = U0 * (N / (2 * np.pi)) / 1600.0
    ke = []
    macro = np.zeros((4, N, N, N))
    for s in range(10):
        ref.aa_run(f, m, coll="CUM", eq="INV_CUM", nu=nu_tgv, macro=macro, start_iter=2 * s, nsteps=2)
        ke.append((macro[0] * (macro[1] ** 2 + macro[2] ** 2 + macro[3] ** 2)).sum() / 2.0 / N ** 3)
    out["tgv16_ke"] = np.array(ke)
    out["tgv16_nu"] = np.array(nu_tgv)
    path = os.path.join(HERE, "golden_d3q27.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB, {len(out)} arrays)")


if __name__ == "__main__":
    main()
