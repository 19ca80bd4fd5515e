"""Benchmark of the D3Q27 cumulant A-A hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload duct|tgv512|tgv64] [--storage f32|f64|f32s|f16s|bf16s|i16s]

Default workload: rectangular duct 512x128x128, FP32 storage, default cumulant
(the duct solver's configuration, sim_NSE/sim_2.cu:475), walls (GEO_WALL) one
site inside GEO_NOTHING rims, a velocity inlet with a parabolic profile at
u_max = 0.04 (GEO_INFLOW_LEFT), a fixed-density outlet (GEO_OUTFLOW_EQ),
nu = u_max * 126 / 2000 (Re = 2000) and a seeded uniform +-1% u_max velocity
perturbation.  A step is one A-A update of all 8,388,608 sites; the 1.8 GB
population array is far larger than the 126 MB L2, so no flush is needed.

N > 1 (torchrun): every rank runs an independent replica of the workload on
its own GPU ("replicas only": the path is one lattice per GPU; no collective
on the data path).  value = sites x steps of all ranks / max-over-ranks time.

The reference arm (--impl reference) times TNL-LBM's own per-site code, built
from the reference tree into oracle/_ref (oracle/ref_harness.cpp) with the
reference's OpenMP loop, on the host cores, for the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tnl-lbm_b200"))

METRIC = "D3Q27 cumulant A-A MLUPS, % HBM roofline; FP16-store vs FP32 at stated error"
BYTES_PER_ELEM = {"f64": 8, "f32": 4, "f32s": 4, "f16s": 2, "bf16s": 2, "f16sr": 2, "bf16sr": 2, "i16s": 2}
# the type the populations are stored in / the type the update computes in
DTYPE_LABEL = {"f64": "f64", "f32": "f32", "f32s": "f32", "f16s": "f16-store/f32", "bf16s": "bf16-store/f32",
               "f16sr": "f16-store/f32", "bf16sr": "bf16-store/f32", "i16s": "i16-store/f32"}


def workload_spec(name):
    if name == "duct":
        return dict(workload="duct 512x128x128, walls + parabolic inlet u_max=0.04 + fixed-density outlet, Re=2000",
                    X=512, Y=128, Z=128, kind="duct", cum_flags=0)
    if name == "duct_ade":
        return dict(workload="duct 512x128x128 as 'duct' with a coupled D3Q7 scalar (central-moment collision, D = nu, "
                             "phi = 1 at the inlet, symmetry outlet, bounce-back walls)",
                    X=512, Y=128, Z=128, kind="duct", cum_flags=0, ade=True)
    if name == "tgv512":
        return dict(workload="periodic Taylor-Green vortex 512^3, U0=0.05, Re=1600", X=512, Y=512, Z=512, kind="tgv",
                    cum_flags=3)
    if name == "ensemble64":
        return dict(workload="ensemble of 64 periodic Taylor-Green lattices, edges U{32,48,64,96,128} (seeded, "
                             "anisotropic), Re log-uniform in [100, 3200], U0=0.05, cumulant 2017+antialias",
                    X=0, Y=0, Z=0, kind="ensemble", cum_flags=3, count=64, edges=(32, 48, 64, 96, 128))
    if name == "ensemble_small":
        return dict(workload="ensemble of 512 small periodic Taylor-Green lattices, edges U{16,24,32} (seeded, "
                             "anisotropic), Re log-uniform in [100, 3200], U0=0.05, cumulant 2017+antialias",
                    X=0, Y=0, Z=0, kind="ensemble", cum_flags=3, count=512, edges=(16, 24, 32))
    if name == "adjoint":
        return dict(workload="discrete adjoint: channel 256x64x64, SRT, velocity inlet u_max=0.03, per-cell x-force control "
                             "(Gaussian bumps, amplitude 1e-3), L2 velocity mismatch on 8 cross-sections, 4000 steps, "
                             "sqrt(N) checkpoints, FP32 storage, FP64 gradient accumulation",
                    X=256, Y=64, Z=64, kind="adjoint", cum_flags=0)
    if name == "tgv256":
        return dict(workload="periodic Taylor-Green vortex 256^3, U0=0.05, Re=1600", X=256, Y=256, Z=256, kind="tgv",
                    cum_flags=3)
    if name == "tgv64":
        return dict(workload="periodic Taylor-Green vortex 64^3, U0=0.05, Re=1600", X=64, Y=64, Z=64, kind="tgv",
                    cum_flags=3)
    raise SystemExit(f"unknown workload {name}")


def ensemble_setup(count=64, seed=4321, u0=0.05, edges=(32, 48, 64, 96, 128)):
    """Member sizes and viscosities of an ensemble workload: each edge drawn
    from `edges`, Re log-uniform in [100, 3200] on the x box length,
    nu = u0 (X / 2 pi) / Re."""
    rng = np.random.default_rng(seed)
    edges = np.array(edges)
    sizes = [tuple(int(v) for v in rng.choice(edges, 3)) for _ in range(count)]
    re = np.exp(rng.uniform(math.log(100.0), math.log(3200.0), count))
    nus = [u0 * (sz[0] / (2 * math.pi)) / r for sz, r in zip(sizes, re)]
    return sizes, nus


def measure_ensemble(pl, local, spec, storage, steps, warmup, dist=None, world=1):
    """The ensemble workload: every launch shape timed over 256 steps, the
    autotuner's choice timed over `steps` steps, an e2e leg with the
    per-member sums read every step, and the same members run one after the
    other as single lattices on the two-site kernel (the single-lattice
    step's best kernel for these widths)."""
    import torch
    device = torch.device("cuda", local)
    sizes, nus = ensemble_setup(spec["count"], edges=spec["edges"])
    sites = sum(x * y * z for x, y, z in sizes)
    st = {"f64": pl.STORE_F64, "f32": pl.STORE_F32, "f32s": pl.STORE_F32S, "f16s": pl.STORE_F16S,
          "bf16s": pl.STORE_BF16S, "f16sr": pl.STORE_F16SR, "bf16sr": pl.STORE_BF16SR, "i16s": pl.STORE_I16S}[storage]
    ens = pl.Ensemble(sizes, nus, cum_flags=3, storage=st, device=local)
    ens.init_taylor_green(0.05)
    shapes = {}
    cands = ((128, 0), (256, 0), (128, 1), (128, 2)) + (((256, 3),) if storage != "f64" else ())
    for tile, gp in cands:
        ens.set_shape(tile, gp)
        ens.step(16)
        ens.synchronize()
        s0 = time.perf_counter()
        ens.step(256)
        ens.synchronize()
        shapes[f"{tile}/{gp}"] = round(sites * 256 / (time.perf_counter() - s0) / 1e6, 1)
    ens.init_taylor_green(0.05)
    shape = ens.autotune(3)
    ens.init_taylor_green(0.05)
    stream = torch.cuda.ExternalStream(ens.stream, device=device)
    warm = max(warmup, 16) + (max(warmup, 16) % 2)
    ens.step(warm)
    ens.synchronize()
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(steps)
        e1.record(stream)
        e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    secs_max = max_over_ranks(dist, secs, device)
    value = sites * steps * world / secs_max / 1e6
    ens.step(2, sums=True)
    ke_ens = ens.kinetic_energy()
    e2e_steps = max(10, min(steps // 4, 200))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ens.step(1, sums=True)
        ens.sums()
    e2e_secs = max_over_ranks(dist, time.perf_counter() - t0, device)
    ens.close()
    seq_secs = 0.0
    ke_seq = []
    for (X, Y, Z), nu in zip(sizes, nus):
        lat = pl.LBM(X, Y, Z, viscosity=nu, cum_flags=3, storage=st, periodic=True, device=local)
        lat.set_kernel(pl.KERNEL_PAIR)
        lat.init_taylor_green(0.05)
        lat.step(warm)
        lat.synchronize()
        ls = torch.cuda.ExternalStream(lat.device_view().stream, device=device)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(ls)
        lat.step(steps)
        a1.record(ls)
        a1.synchronize()
        seq_secs += a0.elapsed_time(a1) / 1e3
        lat.step(2, sums=True)
        ke_seq.append(pl.kinetic_energy(lat))
        lat.close()
    seq_value = sites * steps / seq_secs / 1e6
    ke_diff = float(np.max(np.abs(np.asarray(ke_seq) - ke_ens) / np.abs(np.asarray(ke_seq))))
    return {"sizes": sizes, "sites": sites, "value": value, "secs": secs, "secs_max": secs_max, "shapes": shapes,
            "shape": shape, "e2e_value": sites * e2e_steps * world / e2e_secs / 1e6, "e2e_steps": e2e_steps,
            "seq_value": seq_value, "ke_diff": ke_diff, "clocks": clk.summary()}


GRID_POLICIES = ["persistent", "one block per tile", "per-member launches in concurrent graph branches",
                 "persistent, two sites per thread (packed FP32)"]


def run_ensemble(args):
    """The ensemble workload's line: the autotuned batched step against the
    same members run one after the other as single lattices."""
    import torch
    import pytnl_lbm as pl
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(world, local, "nccl")
    spec = workload_spec(args.workload)
    r = measure_ensemble(pl, local, spec, args.storage, args.steps, args.warmup, dist, world)
    sizes, sites, shape = r["sizes"], r["sites"], r["shape"]
    bpe = BYTES_PER_ELEM[args.storage]
    achieved = 2 * 27 * bpe * sites / (r["secs"] / args.steps) / 1e9
    peak, peak_kind = read_peaks()
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(r["value"], 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(r["secs_max"] / args.steps * 1e3, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE_LABEL[args.storage],
            "data": "synthetic (seeded member sizes, viscosities and Taylor-Green initial states)",
            "config": {"workload": spec["workload"], "members": len(sizes), "sites": sites,
                       "storage": args.storage, "parallelism": f"replicas x{world}",
                       "l2": "populations (%.2f GB) larger than L2; no flush" % (27 * bpe * sites / 1e9)},
            "launch": {"tile_sites": shape[0], "grid": GRID_POLICIES[shape[1]], "autotuned": True},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s",
                         "algorithmic_bytes_per_site_update": 2 * 27 * bpe},
            "e2e": {"value": round(r["e2e_value"], 2), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 6 * 8 * len(sizes), "steps": r["e2e_steps"],
                    "per_step": "lbm_ensemble_step(1, LBM_STEP_SUMS) + lbm_ensemble_get_sums"},
            "shapes_mlups": r["shapes"],
            "sequential": {"value": round(r["seq_value"], 2), "unit": "MLUPS",
                           "speedup": round(r["value"] / r["seq_value"], 3),
                           "kinetic_energy_max_rel_diff": r["ke_diff"],
                           "how": f"the same {len(sizes)} members as single periodic lattices (lbm_create) on the "
                                  "two-site kernel, one after the other, each replayed from its CUDA graphs; summed "
                                  "device time"},
            "clocks": r["clocks"],
        }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


def run_reference_ensemble(args, spec, oracle, cores):
    """The reference's per-site code on each ensemble member in turn (the
    reference runs one lattice per solver instance), on all host cores."""
    sizes, nus = ensemble_setup(spec["count"], edges=spec["edges"])
    prec = np.float64 if args.storage == "f64" else np.float32
    impl = oracle.Reference(3, fast=True)
    total_sites = sum(x * y * z for x, y, z in sizes)
    # calibrate on the first member, then size the per-member step count so
    # that the whole sample takes about 20 s
    X, Y, Z = sizes[0]
    f = impl.allocate(X, Y, Z, prec)
    impl.init_equilibrium(f, X, Y, Z, eq="INV_CUM", fields=None)
    _, el = impl.aa_run(f, np.full((Z, Y, X), 9, np.int16), coll="CUM", nu=nus[0], nsteps=2, nthreads=cores,
                        return_time=True)
    rate = X * Y * Z * 2 / max(el, 1e-6)
    steps = int(max(2, min(args.steps, 20.0 * rate / total_sites)))
    steps += steps % 2
    elapsed = 0.0
    for (X, Y, Z), nu in zip(sizes, nus):
        f = impl.allocate(X, Y, Z, prec)
        impl.init_equilibrium(f, X, Y, Z, eq="INV_CUM", fields=None)
        _, el = impl.aa_run(f, np.full((Z, Y, X), 9, np.int16), coll="CUM", nu=nu, nsteps=steps, nthreads=cores,
                            return_time=True)
        elapsed += el
    value = total_sites * steps / elapsed / 1e6
    sample = (f"{steps} A-A steps of each of the {len(sizes)} members ({prec.__name__}), one after the other, "
              f"OpenMP on {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "MLUPS", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(elapsed / steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == np.float64 else "f32",
        "data": "synthetic (seeded member sizes and viscosities)",
        "config": {"workload": spec["workload"], "members": len(sizes), "sites": total_sites, "storage": args.storage,
                   "implementation": "TNL-LBM per-site headers (oracle/_ref) + reference OpenMP loop"},
        "cpu_baseline": {"value": round(value, 3), "unit": "MLUPS", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def duct_setup(X, Y, Z, seed=1234):
    """Map, inlet profile, viscosity and initial velocity field of the duct."""
    m = np.zeros((Z, Y, X), np.uint8)
    m[:, :, 0] = 3     # GEO_INFLOW_LEFT
    m[:, :, -1] = 6    # GEO_OUTFLOW_EQ
    m[:, 1, :] = 1
    m[:, -2, :] = 1
    m[1, :, :] = 1
    m[-2, :, :] = 1
    m[:, 0, :] = 10
    m[:, -1, :] = 10
    m[0, :, :] = 10
    m[-1, :, :] = 10
    u_max = 0.04
    # product parabola between the wall nodes y = 1 .. Y-2, z = 1 .. Z-2
    yy = (np.arange(Y) - 1.0) / (Y - 3.0)
    zz = (np.arange(Z) - 1.0) / (Z - 3.0)
    py = np.clip(4 * yy * (1 - yy), 0, None)
    pz = np.clip(4 * zz * (1 - zz), 0, None)
    prof = u_max * np.outer(pz, py)
    nu = u_max * 126.0 / 2000.0
    rng = np.random.default_rng(seed)
    pert = 0.01 * u_max * (2 * rng.random((3, Z, Y, X)) - 1)
    ux = prof[:, :, None] * np.ones((1, 1, X)) + pert[0]
    fluid = (m == 0)
    rho = np.ones((Z, Y, X))
    vx = np.where(fluid, ux, 0.0)
    vy = np.where(fluid, pert[1], 0.0)
    vz = np.where(fluid, pert[2], 0.0)
    return m, prof, nu, (rho, vx, vy, vz)


def workload_config(spec, storage, world):
    """The workload description both arms print as `config` (same keys and
    values for the same workload, so that the arms compare like for like)."""
    X, Y, Z = spec["X"], spec["Y"], spec["Z"]
    bpe = BYTES_PER_ELEM[storage]
    return {"workload": spec["workload"], "lattice": [X, Y, Z], "storage": storage,
            "collision": "cumulant" + (" Geier-2017+antialias" if spec["cum_flags"] == 3 else " default"),
            "streaming": "A-A in place", "parallelism": f"replicas x{world}",
            "l2": "populations (%.2f GB) larger than L2; no flush" % (27 * bpe * X * Y * Z / 1e9)}


def cpu_description():
    """Model name, logical CPUs and the vector ISA level of the timed CPU build."""
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    sys.path.insert(0, ROOT)
    import oracle
    return {"model": model, "logical_cpus": os.cpu_count(), "isa": oracle.host_isa_level()}


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(key):
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        d = json.load(fh)
    v = d.get(key)
    return None if v is None else float(v)


class ClockSampler:
    """SM clocks and clock-event reasons sampled in-process through NVML
    during a region: one sample on entry, one every `period_s` from a
    background thread, one on exit, so that a region of a few milliseconds
    still carries samples.  Without NVML it falls back to `nvidia-smi -lms`."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device_index, period_s=0.001):
        self.dev = device_index
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.samples = []
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _nvml_sample(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        power = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
        self.samples.append((float(sm), float(mx), int(reasons), power))

    def _loop(self):
        while not self._stop.wait(self.period):
            try:
                self._nvml_sample()
            except Exception:
                return

    def __enter__(self):
        import threading
        try:
            self.nvml = self._nvml_handle()
            self._nvml_sample()
            self.source = "nvml"
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.nvml is not None:
            self._stop.set()
            self._thread.join(timeout=5)
            try:
                self._nvml_sample()
            except Exception:
                pass
            return
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                bits = 0
                for (name, bit), field in zip(self.REASONS, parts[5:9]):
                    bits |= bit if field.lower() == "active" else 0
                self.samples.append((float(parts[1]), float(parts[2]), bits, None))

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [s[0] for s in self.samples]
        reasons = sorted({name for s in self.samples for name, bit in self.REASONS if s[2] & bit})
        out = {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm), "sm_max_mhz": max(s[1] for s in self.samples),
               "reasons": reasons, "samples": len(self.samples), "source": self.source}
        power = [s[3] for s in self.samples if s[3] is not None]
        if power:
            out["power_w_max"] = round(max(power), 1)
        return out


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, local, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, value, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def trt_plugin_id(pl):
    """Register the example two-relaxation-time collision plugin
    (tnl-lbm_b200/plugins/example_collisions.cu) in the open COLL slot."""
    cid = pl.COLL_PLUGIN_FIRST
    if pl.collision_name(cid) != "TRT":
        pl.register_collision(cid, pl.plugin_path("example_collisions"), "lbm_example_trt", name="TRT")
    return cid


def make_lattice(pl, spec, storage, device, kernel="direct", collision="cum"):
    st = {"f64": pl.STORE_F64, "f32": pl.STORE_F32, "f32s": pl.STORE_F32S, "f16s": pl.STORE_F16S,
          "bf16s": pl.STORE_BF16S, "f16sr": pl.STORE_F16SR, "bf16sr": pl.STORE_BF16SR, "i16s": pl.STORE_I16S}[storage]
    X, Y, Z = spec["X"], spec["Y"], spec["Z"]
    if spec["kind"] == "duct":
        m, prof, nu, fields = duct_setup(X, Y, Z)
        if collision == "plugin_trt":
            coll = trt_plugin_id(pl)
        else:
            coll = {"cum": pl.COLL_CUM, "srt": pl.COLL_SRT, "bgk": pl.COLL_BGK, "mrt": pl.COLL_MRT}[collision]
        lat = pl.LBM(X, Y, Z, viscosity=nu, collision=coll, cum_flags=spec["cum_flags"],
                     equilibrium=pl.EQ_INV_CUM if collision == "cum" else pl.EQ_SECOND_ORDER, storage=st,
                     device=device)
        lat.set_kernel({"tile": pl.KERNEL_TILE, "split": pl.KERNEL_SPLIT, "pair": pl.KERNEL_PAIR}.get(kernel, pl.KERNEL_DIRECT))
        lat.set_map(m)
        lat.set_inflow(prof, None, None)
        lat.init_equilibrium(*fields)
        if spec.get("ade"):
            # scalar types from the flow map: inlet -> INFLOW, outlet -> SYM_RIGHT, walls and rims alike
            am = np.choose(m, [0, 1, 0, 7, 0, 0, 15, 0, 0, 9, 10]).astype(np.uint8)
            lat.ade_enable(nu, collision=pl.ADE_CLBM, inflow_phi=1.0)
            lat.ade_set_map(am)
            lat.ade_init_equilibrium(uniform_phi=0.0)
        return lat, prof
    nu = 0.05 * (X / (2 * math.pi)) / 1600.0
    lat = pl.LBM(X, Y, Z, viscosity=nu, collision=pl.COLL_CUM, cum_flags=spec["cum_flags"],
                 equilibrium=pl.EQ_INV_CUM, storage=st, periodic=True, device=device)
    lat.set_kernel({"tile": pl.KERNEL_TILE, "split": pl.KERNEL_SPLIT, "pair": pl.KERNEL_PAIR}.get(kernel, pl.KERNEL_DIRECT))
    lat.init_taylor_green(0.05, 1.0)
    return lat, None


def time_steps(pl, lat, steps, warmup, stream):
    import torch
    # at least one full graph of steps in the warm-up, so that the graph is
    # captured and instantiated before the timed region; even parity at start
    lat.step(max(warmup, 16) + (max(warmup, 16) % 2))
    lat.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lat.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def duct_fp32_vs_fp64(pl, device, steps=5000, every=500):
    """The comparison of the duct configuration: the FP32 duct (two-site
    kernel, as timed) against an FP64 run of the same duct from the same
    initial state, kinetic energy every `every` steps and the velocity field
    after `steps` steps."""
    spec = workload_spec("duct")
    runs = {}
    for st, kernel in (("f64", "direct"), ("f32", "pair")):
        lat, _ = make_lattice(pl, spec, st, device, kernel)
        ke, mass = [], []
        t0 = time.perf_counter()
        for c in range(steps // every):
            lat.step(every, macro=(c == steps // every - 1), sums=True)
            s = lat.sums()
            ke.append(s[4])
            mass.append(s[0])
        runs[st] = (np.array(ke), np.array(mass), lat.macro(), time.perf_counter() - t0)
        lat.close()
    ke64, m64, mac64, t64 = runs["f64"]
    ke32, m32, mac32, t32 = runs["f32"]
    u_max = 0.04
    ke_rel = np.abs(ke32 / ke64 - 1)
    return {"workload": spec["workload"] + f", {steps} steps", "steps": steps,
            "ke_rel_err_max": float(np.max(ke_rel)), "ke_rel_err_final": float(ke_rel[-1]),
            "max_abs_du_over_umax": float(np.max(np.abs(mac32[1:] - mac64[1:])) / u_max),
            "max_abs_drho": float(np.max(np.abs(mac32[0] - mac64[0]))),
            "mass_rel_diff_final": float(abs(m32[-1] / m64[-1] - 1)),
            "how": f"kinetic energy sum rho |u|^2 every {every} steps, velocity and density after the last step; "
                   "FP64 storage on the one-site kernel, FP32 on the two-site kernel",
            "seconds": {"f64": round(t64, 2), "f32": round(t32, 2)}}


def tgv512_throughput(pl, device, steps, warmup, kernel16="pair"):
    """Throughput of the largest single-GPU configuration, the 512^3
    Taylor-Green vortex, in FP32, in FP16 shifted storage and in 16-bit
    fixed-point deviations."""
    import torch
    spec = workload_spec("tgv512")
    sites = spec["X"] * spec["Y"] * spec["Z"]
    peak, _ = read_peaks()
    out = {"workload": spec["workload"]}
    for st, kernel in (("f32", "pair"), ("f16s", kernel16), ("i16s", kernel16)):
        lat, _ = make_lattice(pl, spec, st, device, kernel)
        stream = torch.cuda.ExternalStream(lat.device_view().stream, device=torch.device("cuda", device))
        secs = time_steps(pl, lat, steps, warmup, stream)
        lat.close()
        mlups = sites * steps / secs / 1e6
        gbs = mlups * 1e6 * 2 * 27 * BYTES_PER_ELEM[st] / 1e9
        out[st] = {"mlups": round(mlups, 1), "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4),
                   "step_kernel": kernel}
    out["f16s_speedup_vs_f32"] = round(out["f16s"]["mlups"] / out["f32"]["mlups"], 3)
    out["i16s_speedup_vs_f32"] = round(out["i16s"]["mlups"] / out["f32"]["mlups"], 3)
    return out


def run_adjoint(args):
    """Forward pass with checkpoints plus backward pass of the discrete adjoint;
    value = sites x steps / (forward + backward device time)."""
    import torch
    import pytnl_lbm as pl
    from pytnl_lbm import adjoint_check as ac
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(world, local, "nccl")
    device = torch.device("cuda", local)
    spec = workload_spec(args.workload)
    steps = args.steps + (args.steps % 2)
    lat, m = ac.make(pl.STORE_F32)
    samples = ac.sample_sites(m)
    target = np.zeros((len(samples), 4))
    target[:, 0] = 1.0
    target[:, 1] = 0.01
    F = ac.bumps(seed=7)
    stream = torch.cuda.ExternalStream(lat.device_view().stream, device=device)
    every = int(math.ceil(math.sqrt(steps)))
    # warm-up with the timed run's sizes, so that the checkpoint and segment
    # buffers are allocated before the timed region
    lat.init_equilibrium()
    lat.adjoint_forward(F, steps, samples, target, checkpoint_every=every)
    lat.adjoint_backward()
    with ClockSampler(local) as clk:
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        lat.init_equilibrium()
        e0.record(stream)
        J = lat.adjoint_forward(F, steps, samples, target, checkpoint_every=every)
        e1.record(stream)
        g = lat.adjoint_backward()
        e2.record(stream)
        e2.synchronize()
    t_fwd, t_bwd = e0.elapsed_time(e1) / 1e3, e1.elapsed_time(e2) / 1e3
    secs = max_over_ranks(dist, t_fwd + t_bwd, device)
    sites = spec["X"] * spec["Y"] * spec["Z"]
    value = sites * steps * world / secs / 1e6
    v = lat.device_view()
    pop_bytes = v.sz * (spec["Z"] + 2) * v.elem_size  # all slots, ghost layer included
    lat.close()
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": steps,
            "warmup": 1, "ms_per_step": round(secs / steps * 1e3, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (gradient f64)",
            "data": "synthetic (seeded control field and target)",
            "config": {"workload": spec["workload"], "lattice": [spec["X"], spec["Y"], spec["Z"]],
                       "samples": int(len(samples)), "checkpoint_every": every,
                       "checkpoint_memory_gb": round((math.ceil(steps / every) + every + 2) * pop_bytes / 1e9, 2)},
            "gpu_launches": 3 * steps,
            "forward_s": round(t_fwd, 4), "backward_s": round(t_bwd, 4), "objective": J,
            "grad_max_abs": float(np.max(np.abs(g[0]))),
            "roofline": {"bound": "hbm", "achieved": None, "peak": read_peaks()[0], "unit": "GB/s", "frac": None,
                         "traffic": None,
                         "note": "per step: two primal A-A steps (216 B/site each), one adjoint step "
                                 "(27 FP32 primal reads + 27 FP64 adjoint reads + 27 FP64 adjoint writes, 540 B/site) "
                                 "and a 27-value FP32 copy per recomputed state (216 B/site)"},
            "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "per_run": "lbm_adjoint_forward + lbm_adjoint_backward through the C-ABI"},
            "clocks": clk.summary(),
        }
        bytes_per_site_step = 2 * 216 + 540 + 216
        line["roofline"]["achieved"] = round(bytes_per_site_step * sites * steps / secs / 1e9, 1)
        line["roofline"]["frac"] = round(line["roofline"]["achieved"] / line["roofline"]["peak"], 4)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


def run_ours(args):
    if workload_spec(args.workload)["kind"] == "adjoint":
        return run_adjoint(args)
    if workload_spec(args.workload)["kind"] == "ensemble":
        return run_ensemble(args)
    import torch
    import pytnl_lbm as pl
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(world, local, "nccl")
    device = torch.device("cuda", local)
    spec = workload_spec(args.workload)
    sites = spec["X"] * spec["Y"] * spec["Z"]
    lat, prof = make_lattice(pl, spec, args.storage, local, args.kernel)
    if args.autotune:
        lat.autotune(16)  # block shape and step kernel, 16 timed steps per candidate
    kernel_name = {pl.KERNEL_DIRECT: "direct", pl.KERNEL_TILE: "tile", pl.KERNEL_SPLIT: "split", pl.KERNEL_PAIR: "pair"}.get(
        lat.kernel, "direct")
    stream = torch.cuda.ExternalStream(lat.device_view().stream, device=device)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        secs = time_steps(pl, lat, args.steps, args.warmup, stream)
    block = lat.block()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    secs_max = max_over_ranks(dist, secs, device)
    ms_per_step = secs_max / args.steps * 1e3
    mlups_rank = sites * args.steps / secs / 1e6
    value = sites * args.steps * world / secs_max / 1e6

    # roofline of the step kernel (the only kernel of the timed region)
    bpe = BYTES_PER_ELEM[args.storage]
    # populations read and written once per update; a coupled scalar adds its 7
    bytes_per_site = 2 * 27 * bpe + (2 * 7 * bpe if spec.get("ade") else 0)
    alg_bytes = bytes_per_site * sites
    achieved = alg_bytes / (secs / args.steps) / 1e9
    peak, peak_kind = read_peaks()
    traffic = read_traffic(f"{args.workload}_{args.storage}_{kernel_name}")

    # e2e through the C-ABI with host buffers: per step an inlet-profile upload
    # from pinned host memory, one step with the FP64 sums, and the sums read
    # back to the host
    e2e_steps = max(10, min(args.steps // 4, 200))
    pinned = None
    if prof is not None:
        pinned = torch.from_numpy(np.ascontiguousarray(prof)).pin_memory().numpy()
    lat.step(2, sums=True)
    lat.sums()
    # each step's sums are read while the next step is already queued
    # (lbm_get_sums_of waits for that step only), so the host's per-step work
    # overlaps the device instead of idling it
    prev = None
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if pinned is not None:
            lat.set_inflow(pinned, None, None)
        lat.step(1, sums=True)
        it = lat.iteration
        if prev is not None:
            lat.sums_of(prev)
        prev = it
    lat.sums_of(prev)
    t1 = time.perf_counter()
    e2e_secs = max_over_ranks(dist, t1 - t0, device)
    e2e_value = sites * e2e_steps * world / e2e_secs / 1e6
    h2d = 0 if prof is None else int(prof.size) * (8 if args.storage == "f64" else 4)

    # FP16 / BF16 shifted storage on the same workload (the precision trade)
    variants = {}
    if args.variants and args.storage == "f32" and not spec.get("ade"):
        lat.close()
        for st in ("f16s", "bf16s", "f16sr", "bf16sr", "i16s"):
            vl, _ = make_lattice(pl, spec, st, local, args.kernel)
            if args.autotune:
                vl.autotune(16)
            vs = torch.cuda.ExternalStream(vl.device_view().stream, device=device)
            vsecs = time_steps(pl, vl, args.steps, args.warmup, vs)
            variants[st] = {"mlups": sites * args.steps / vsecs / 1e6,
                            "speedup_vs_f32": secs / vsecs,
                            "achieved_gbs": 2 * 27 * 2 * sites / (vsecs / args.steps) / 1e9}
            vl.close()
        # FP64 storage (the reference's default arithmetic), one-site kernel
        vl, _ = make_lattice(pl, spec, "f64", local, "direct")
        if args.autotune:
            vl.autotune(16)
        vs = torch.cuda.ExternalStream(vl.device_view().stream, device=device)
        vsecs = time_steps(pl, vl, args.steps, args.warmup, vs)
        gbs = 2 * 27 * 8 * sites / (vsecs / args.steps) / 1e9
        variants["f64"] = {"mlups": sites * args.steps / vsecs / 1e6, "achieved_gbs": gbs, "frac": gbs / peak}
        vl.close()
        for other in ("direct", "pair", "tile", "split"):
            if other == args.kernel or (other == "split" and spec["kind"] != "duct"):
                continue
            vl, _ = make_lattice(pl, spec, "f32", local, other)
            vs = torch.cuda.ExternalStream(vl.device_view().stream, device=device)
            vsecs = time_steps(pl, vl, args.steps, args.warmup, vs)
            variants[f"f32_{other}_kernel"] = {"mlups": sites * args.steps / vsecs / 1e6}
            vl.close()
        # the other collisions of the COLL slot (one-site kernel, autotuned
        # block), and a user-compiled collision through the plugin slot
        if spec["kind"] == "duct":
            for coll in ("srt", "bgk", "mrt", "plugin_trt"):
                vl, _ = make_lattice(pl, spec, "f32", local, "direct", coll)
                if args.autotune:
                    vl.autotune(16)
                vs = torch.cuda.ExternalStream(vl.device_view().stream, device=device)
                vsecs = time_steps(pl, vl, args.steps, args.warmup, vs)
                gbs = 216 * sites / (vsecs / args.steps) / 1e9
                variants[f"f32_{coll}"] = {"mlups": sites * args.steps / vsecs / 1e6, "achieved_gbs": gbs,
                                           "frac": gbs / peak}
                vl.close()
    else:
        lat.close()

    # the precision configuration: the Taylor-Green vortex at 256^3, Re 1600,
    # 20000 steps, kinetic energy and dissipation rate of every storage format
    # against the FP64-storage run (BF16 with round-to-nearest diverges on
    # this case and is left out)
    precision = None
    if args.precision and rank == 0:
        from pytnl_lbm import precision as prec
        precision = prec.study(256, 20000, 200, ("f32", "f16s", "f16sr", "bf16sr", "i16s"), local)
        precision.pop("series")
    # the duct configuration's FP32-against-FP64 comparison and the 512^3
    # Taylor-Green throughput
    duct_cmp = tgv512 = ens_block = None
    if args.configs and rank == 0 and spec["kind"] == "duct" and not spec.get("ade"):
        duct_cmp = duct_fp32_vs_fp64(pl, local)
        tgv512 = tgv512_throughput(pl, local, max(args.steps, 20), args.warmup)
        # the batching configuration: 64 Taylor-Green lattices, autotuned
        r = measure_ensemble(pl, local, workload_spec("ensemble64"), "f32", 200, args.warmup)
        ens_block = {"workload": workload_spec("ensemble64")["workload"], "steps": 200,
                     "mlups": round(r["value"], 1), "launch": GRID_POLICIES[r["shape"][1]],
                     "tile_sites": r["shape"][0], "shapes_mlups": r["shapes"],
                     "sequential_mlups": round(r["seq_value"], 1),
                     "speedup_vs_sequential": round(r["value"] / r["seq_value"], 3),
                     "kinetic_energy_max_rel_diff": r["ke_diff"]}

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE_LABEL[args.storage],
            "data": "synthetic (seeded initial state of the named configuration)",
            "config": workload_config(spec, args.storage, world),
            "launch": {"step_kernel": kernel_name, "autotuned": bool(args.autotune),
                       "block": (list(block) if kernel_name == "direct" or (kernel_name == "pair" and spec["kind"] != "duct")
                                 else f"{kernel_name} kernel, 128 threads")},
            # the split step of a lattice with a map launches two kernels per step
            "gpu_launches": args.steps * (2 if kernel_name == "split" and spec["kind"] == "duct" else 1),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s",
                         "algorithmic_bytes_per_site_update": bytes_per_site,
                         "achieved_vs_8TBs_spec": round(achieved / 8000.0, 4)},
            "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 48, "steps": e2e_steps,
                    "per_step": "lbm_set_inflow(pinned host) + lbm_step(1, LBM_STEP_SUMS) + lbm_get_sums_of "
                                "(the previous step's sums, read while this step runs; the last step's read closes "
                                "the timed region)"},
            "clocks": clk.summary(),
            "per_rank_mlups": round(mlups_rank, 2),
        }
        if variants:
            line["storage_variants"] = variants
        if precision is not None:
            line["precision"] = precision
        if duct_cmp is not None:
            line["duct_fp32_vs_fp64"] = duct_cmp
        if tgv512 is not None:
            line["tgv512"] = tgv512
        if ens_block is not None:
            line["ensemble64"] = ens_block
        if args.cpu_baseline and world == 1 and not spec.get("ade"):
            line["cpu_baseline"] = cpu_baseline(spec, args)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


def time_reference_cpu(spec, storage, sample_steps, warmup, min_seconds=10.0):
    """The reference's own per-site code (oracle/_ref, OpenMP on all host
    cores; the restatement in oracle/ if the reference was not built) on the
    workload: warm-up steps, then samples of `sample_steps` full-lattice A-A
    steps (at most ~60 s each) until at least `min_seconds` have been timed.
    Both the reference arm and the cpu_baseline leg of our arm use it, so
    that they measure the same thing."""
    sys.path.insert(0, ROOT)
    import oracle
    cores = os.cpu_count() or 1
    flags = spec["cum_flags"]
    use_ref = oracle.reference_available(flags)
    X, Y, Z = spec["X"], spec["Y"], spec["Z"]
    if spec["kind"] == "duct":
        m, prof, nu, fields = duct_setup(X, Y, Z)
        inflow = (prof, None, None)
    else:
        m = np.full((Z, Y, X), 9, np.uint8)
        nu = 0.05 * (X / (2 * math.pi)) / 1600.0
        inflow, fields = None, None
    prec = np.float64 if storage == "f64" else np.float32
    impl = oracle.Reference(flags, fast=True) if use_ref else oracle.Port()
    f = impl.allocate(X, Y, Z, prec)
    impl.init_equilibrium(f, X, Y, Z, eq="INV_CUM", fields=fields)
    m16 = m.astype(np.int16)

    def run(n, start):
        if use_ref:
            _, el = impl.aa_run(f, m16, coll="CUM", eq="INV_CUM", nu=nu, inflow=inflow, start_iter=start, nsteps=n,
                                nthreads=cores, return_time=True)
            return el
        t0 = time.perf_counter()
        impl.aa_run(f, m16, coll="CUM", eq="INV_CUM", cum_flags=flags, nu=nu, inflow=inflow, start_iter=start,
                    nsteps=n, nthreads=cores)
        return time.perf_counter() - t0

    warm = max(1, min(warmup, 2))
    per_step = run(warm, 0) / warm
    steps = int(max(2, min(sample_steps, 60.0 / max(per_step, 1e-6))))
    steps += steps % 2
    it, el, reps = warm, 0.0, 0
    while reps == 0 or el < min_seconds:
        el += run(steps, it)
        it += steps
        reps += 1
    value = X * Y * Z * steps * reps / el / 1e6
    cpu = cpu_description()
    sample = (f"{reps} samples of {steps} A-A steps of the full {X}x{Y}x{Z} workload ({prec.__name__}), {el:.1f} s in "
              f"all, OpenMP on {cores} threads, loop order of state.hpp:1388-1397, {cpu['isa']} build")
    return {"value": value, "steps": steps, "reps": reps, "seconds": el, "cores": cores,
            "kind": "reference" if use_ref else "port", "sample": sample, "cpu": cpu, "prec": prec}


def cpu_baseline(spec, args):
    """The cpu_baseline object of our arm's line (time_reference_cpu with the
    reference arm's sampling)."""
    r = time_reference_cpu(spec, args.storage, min(args.steps, 20), args.warmup)
    return {"value": round(r["value"], 3), "unit": "MLUPS", "cores": r["cores"], "kind": r["kind"],
            "sample": r["sample"], "cpu": r["cpu"]}


def run_reference(args):
    """The reference arm: TNL-LBM's per-site code on the host cores.

    Every timed step is one A-A update of the whole workload, as in our arm.
    Samples of `steps` steps (at most ~60 s each) repeat until at least 10 s
    have been timed, so that the figure does not rest on a short run."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    import oracle
    spec = workload_spec(args.workload)
    flags = spec["cum_flags"]
    cores = os.cpu_count() or 1
    if not oracle.reference_available(flags):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference sources)"}))
        return
    if spec["kind"] == "ensemble":
        return run_reference_ensemble(args, spec, oracle, cores)
    if spec["kind"] == "adjoint":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no time-dependent adjoint of this "
                          "workload (sim_adjoint solves a steady adjoint about a frozen flow)"}))
        return
    r = time_reference_cpu(spec, args.storage, args.steps, args.warmup)
    value = r["value"]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "MLUPS", "n_gpus": world,
        "steps": r["steps"], "warmup": args.warmup, "ms_per_step": round(r["seconds"] / (r["steps"] * r["reps"]) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if r["prec"] == np.float64 else "f32",
        "data": "synthetic (seeded initial state of the named configuration)",
        "config": workload_config(spec, args.storage, world),
        "implementation": "TNL-LBM per-site headers (oracle/_ref, %s build) + the reference's OpenMP loop" % r["cpu"]["isa"],
        "repetitions": r["reps"],
        "cpu_baseline": {"value": round(value, 3), "unit": "MLUPS", "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"], "cpu": r["cpu"]},
        "e2e": {"value": round(value, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="duct", choices=["duct", "duct_ade", "tgv512", "tgv256", "tgv64", "ensemble64", "ensemble_small", "adjoint"])
    ap.add_argument("--storage", default="f32", choices=list(BYTES_PER_ELEM))
    ap.add_argument("--no-variants", dest="variants", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-precision", dest="precision", action="store_false")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the duct FP32-vs-FP64 comparison and the 512^3 Taylor-Green throughput")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default block shape and kernel instead of lbm_autotune's choice")
    ap.add_argument("--kernel", default="direct", choices=["direct", "tile", "split", "pair"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
