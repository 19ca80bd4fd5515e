"""Precision of the shifted storage formats on the periodic Taylor-Green vortex.

The lattice is the 3D Taylor-Green vortex of sim_NSE/sim_4.cu (u0 = 0.05,
Re = 1600 on the 2 pi box, nu = u0 (N / 2 pi) / Re, D3Q27 cumulant with the
Geier-2017 and anti-aliasing variants, equilibrium initialisation through
D3Q27_EQ_INV_CUM).  Every storage format runs the same case; the series of

    E(t)   = sum rho |u|^2 / (2 rho0 V)                   (sim_4.cu:257-275)
    eps(t) = 2 nu sum rho |grad u|^2 / (2 rho0 V)         (sim_4.cu:279-301)

is compared with the FP64-storage run:

    ke_rel_err  = max_t |E_s(t) - E_f64(t)| / E_f64(t)
    eps_rel_err = max_t |eps_s(t) - eps_f64(t)| / eps_f64(t)

All runs compute in FP32 except the FP64 reference (FP64 arithmetic); the sums
are FP64 in every run.

    python -m pytnl_lbm.precision --n 256 --steps 20000 --every 200
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import COLL_CUM, CUM_ANTIALIAS, CUM_GEIER_2017, EQ_INV_CUM, KERNEL_DIRECT, KERNEL_PAIR, LBM, STORE_BF16S, \
    STORE_BF16SR, STORE_F16S, STORE_F16SR, STORE_F32, STORE_F32S, STORE_F64, STORE_I16S

STORAGES = {"f64": STORE_F64, "f32": STORE_F32, "f32s": STORE_F32S, "f16s": STORE_F16S, "bf16s": STORE_BF16S,
            "f16sr": STORE_F16SR, "bf16sr": STORE_BF16SR, "i16s": STORE_I16S}

U0 = 0.05
RE = 1600.0


def viscosity(n: int) -> float:
    return U0 * (n / (2 * math.pi)) / RE


def tgv_series(n: int, steps: int, every: int, storage: str, device: int = 0, kernel: int | None = None) -> dict:
    """E(t) and eps(t) every `every` steps (an even number: the A-A state is
    read after even steps, as the reference's probes are).  kernel: the step
    kernel (LBM_KERNEL_*); by default the two-site kernel for the formats
    with FP32 arithmetic, the one the throughput runs use."""
    if every % 2:
        raise ValueError("every must be even")
    nu = viscosity(n)
    lat = LBM(n, n, n, viscosity=nu, collision=COLL_CUM, cum_flags=CUM_GEIER_2017 | CUM_ANTIALIAS,
              equilibrium=EQ_INV_CUM, storage=STORAGES[storage], periodic=True, device=device)
    try:
        if kernel is None:
            kernel = KERNEL_DIRECT if storage == "f64" else KERNEL_PAIR
        lat.set_kernel(kernel)
        lat.init_taylor_green(U0, 1.0)
        vol = float(n) ** 3
        t, ke, eps = [], [], []
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            k = min(every, steps - done)
            lat.step(k, macro=True, sums=True)
            done += k
            s = lat.sums()
            t.append(done)
            ke.append(s[4] / 2.0 / vol)
            eps.append(2.0 * nu * lat.enstrophy_sum() / 2.0 / vol)
            if s[5] != 0:
                raise FloatingPointError(f"{storage}: non-finite density after {done} steps")
        lat.synchronize()
        secs = time.perf_counter() - t0
    finally:
        lat.close()
    return {"storage": storage, "n": n, "steps": steps, "t": t, "ke": ke, "eps": eps, "seconds": secs}


def compare(ref: dict, run: dict) -> dict:
    """Errors against the FP64 run: over the whole run, and up to the peak of
    the FP64 dissipation rate (after the peak the flow is turbulent and the
    rounding differences of any two runs grow exponentially)."""
    ke_r, ke = np.asarray(ref["ke"]), np.asarray(run["ke"])
    ep_r, ep = np.asarray(ref["eps"]), np.asarray(run["eps"])
    peak = int(np.argmax(ep_r)) + 1
    ke_e, ep_e = np.abs(ke - ke_r) / ke_r, np.abs(ep - ep_r) / ep_r
    return {"ke_rel_err": float(np.max(ke_e)), "eps_rel_err": float(np.max(ep_e)),
            "ke_final_rel_err": float(ke_e[-1]),
            "to_dissipation_peak": {"steps": int(ref["t"][peak - 1]), "ke_rel_err": float(np.max(ke_e[:peak])),
                                    "eps_rel_err": float(np.max(ep_e[:peak]))}}


def study(n: int, steps: int, every: int, storages=("f32", "f32s", "f16s", "bf16s"), device: int = 0) -> dict:
    ref = tgv_series(n, steps, every, "f64", device)
    out = {"workload": f"Taylor-Green {n}^3, Re {RE:g}, u0 {U0}, cumulant 2017+antialias, {steps} steps",
           "f64_seconds": ref["seconds"], "formats": {}}
    series = {"f64": {"t": ref["t"], "ke": ref["ke"], "eps": ref["eps"]}}
    for st in storages:
        run = tgv_series(n, steps, every, st, device)
        out["formats"][st] = dict(compare(ref, run), seconds=run["seconds"])
        series[st] = {"ke": run["ke"], "eps": run["eps"]}
    out["series"] = series
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--every", type=int, default=200)
    ap.add_argument("--storages", default="f32,f32s,f16s,bf16s")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="write the full result (with the FP64 series) as JSON")
    args = ap.parse_args(argv)
    res = study(args.n, args.steps, args.every, tuple(args.storages.split(",")), args.device)
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(res, fh)
    brief = {k: v for k, v in res.items() if k != "series"}
    print(json.dumps(brief))


if __name__ == "__main__":
    main()
