"""CPU oracle for the D3Q27 A-A hot path (test infrastructure only).

Two checkers with the same call signatures:

* ``Port``      -- this project's C restatement (``oracle/lbm_oracle.c``),
  built into ``oracle/_build/liboracle.so``.
* ``Reference`` -- TNL-LBM's own per-site headers compiled from the reference
  tree through ``oracle/ref_harness.cpp`` into ``oracle/_ref/*.so``.  Present
  only where those libraries were built (they travel with the repository
  snapshot but cannot be rebuilt without the reference sources).

Only the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may use this package.  Nothing in the product imports it.

Array conventions (numpy, C order):
  populations  [27, Z+2, Y+2, X+2]  x fastest, one ghost layer
  map          [Z, Y, X]            int16 GEO values of D3Q27_BC_All
  macro        [4, Z, Y, X]         rho, vx, vy, vz
  inflow       [Z, Y]               per-direction velocity profile or None
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REFDIR = os.path.join(HERE, "_ref")

COLL = {"CUM": 0, "SRT": 1, "BGK": 2, "MRT": 3}
EQ = {"EQ": 0, "INV_CUM": 1}
ADE_COLL = {"SRT": 0, "MRT": 1, "CLBM": 2}
CUM_2017 = 1
CUM_ANTIALIAS = 2

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def build(quiet: bool = True, reference: str | None = None) -> None:
    """Compile the restatement, and the reference harness when a reference
    checkout is given (``reference`` or the TNL_LBM_REFERENCE environment
    variable) and holds the sources."""
    ref = reference or os.environ.get("TNL_LBM_REFERENCE", "")
    cmd = ["make", "-C", HERE, "all"] + ([f"REF={ref}"] if ref else [])
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _prec(dtype) -> int:
    dtype = np.dtype(dtype)
    if dtype == np.float64:
        return 0
    if dtype == np.float32:
        return 1
    raise TypeError(f"oracle supports float64/float32, not {dtype}")


def _profiles(inflow):
    if inflow is None:
        return None, None, None
    return tuple(None if p is None else np.ascontiguousarray(p, dtype=np.float64) for p in inflow)


class _Base:
    def allocate(self, X, Y, Z, dtype=np.float64):
        return np.zeros((27, Z + 2, Y + 2, X + 2), dtype=dtype)


class Port(_Base):
    """This project's C restatement of the reference algorithm."""

    def __init__(self):
        path = os.path.join(BUILD, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        for sfx in ("_f64", "_f32"):
            fn = getattr(self.lib, "orc_aa_run" + sfx)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _vp, _vp,
                           ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _vp,
                           ctypes.c_long, ctypes.c_int, ctypes.c_int]
            fn = getattr(self.lib, "orc_init_equilibrium" + sfx)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _vp, _dp, _dp, _dp, _dp,
                           ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
            fn = getattr(self.lib, "orc_collide" + sfx)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, _vp, _vp, ctypes.c_double,
                           ctypes.c_double, ctypes.c_double, ctypes.c_double]
            fn = getattr(self.lib, "orc_equilibrium" + sfx)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int, ctypes.c_long, _dp, _dp, _dp, _dp, _vp]

    @staticmethod
    def _sfx(dtype):
        return "_f64" if _prec(dtype) == 0 else "_f32"

    def aa_run(self, f, geo_map, coll="CUM", eq="INV_CUM", cum_flags=0, nu=0.01, force=(0.0, 0.0, 0.0), inflow=None,
               macro=None, start_iter=0, nsteps=1, nthreads=0):
        Z, Y, X = geo_map.shape
        assert f.shape == (27, Z + 2, Y + 2, X + 2) and f.flags.c_contiguous
        m = np.ascontiguousarray(geo_map, dtype=np.int16)
        vx, vy, vz = _profiles(inflow)
        if macro is not None:
            assert macro.shape == (4, Z, Y, X) and macro.dtype == f.dtype
        rc = getattr(self.lib, "orc_aa_run" + self._sfx(f.dtype))(
            COLL[coll], EQ[eq], cum_flags, X, Y, Z, _ptr(f), _ptr(m), nu, *force, _dptr(vx), _dptr(vy), _dptr(vz),
            _ptr(macro), start_iter, nsteps, nthreads)
        if rc != 0:
            raise RuntimeError(f"orc_aa_run failed with {rc}")
        return f

    def init_equilibrium(self, f, X, Y, Z, eq="INV_CUM", fields=None, uniform=(1.0, 0.0, 0.0, 0.0)):
        rho = vx = vy = vz = None
        if fields is not None:
            rho, vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64) for a in fields)
        rc = getattr(self.lib, "orc_init_equilibrium" + self._sfx(f.dtype))(
            EQ[eq], X, Y, Z, _ptr(f), _dptr(rho), _dptr(vx), _dptr(vy), _dptr(vz), *uniform)
        if rc != 0:
            raise RuntimeError("orc_init_equilibrium failed")
        return f

    def collide(self, f, coll="CUM", eq="INV_CUM", cum_flags=0, nu=0.01, force=(0.0, 0.0, 0.0)):
        """Per-site collision of f[n, 27] in place; returns macro [n, 4] (pre-collision rho, u)."""
        assert f.ndim == 2 and f.shape[1] == 27 and f.flags.c_contiguous
        macro = np.zeros((f.shape[0], 4), dtype=f.dtype)
        getattr(self.lib, "orc_collide" + self._sfx(f.dtype))(COLL[coll], EQ[eq], cum_flags, f.shape[0], _ptr(f),
                                                               _ptr(macro), nu, *force)
        return macro

    def equilibrium(self, rho, vx, vy, vz, eq="INV_CUM", dtype=np.float64):
        rho, vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (rho, vx, vy, vz))
        out = np.zeros((rho.size, 27), dtype=dtype)
        getattr(self.lib, "orc_equilibrium" + self._sfx(dtype))(EQ[eq], rho.size, _dptr(rho), _dptr(vx), _dptr(vy),
                                                                 _dptr(vz), _ptr(out))
        return out


_V4_FLAGS = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def host_isa_level() -> str:
    """x86-64 micro-architecture level of this host that the timed reference
    builds target: "x86-64-v4" with AVX-512 (F, BW, CD, DQ, VL), else
    "x86-64-v3"."""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return "x86-64-v4" if all(f in flags for f in _V4_FLAGS) else "x86-64-v3"
    except OSError:
        pass
    return "x86-64-v3"


_REF_VARIANTS = {0: "libref_cum_default", CUM_ANTIALIAS: "libref_cum_aa",
                 CUM_2017 | CUM_ANTIALIAS: "libref_cum_2017aa"}


def reference_available(cum_flags: int = 0) -> bool:
    name = _REF_VARIANTS.get(cum_flags)
    return name is not None and os.path.exists(os.path.join(REFDIR, name + ".so"))


class Reference(_Base):
    """TNL-LBM's own per-site code (one library per cumulant flag set)."""

    def __init__(self, cum_flags: int = 0, fast: bool = False):
        name = _REF_VARIANTS[cum_flags] + ("_fast" if fast else "")
        path = os.path.join(REFDIR, name + ".so")
        # the timed build: the AVX-512 one where the host has AVX-512
        v4 = os.path.join(REFDIR, name + "_v4.so")
        if fast and host_isa_level() == "x86-64-v4" and os.path.exists(v4):
            path = v4
        self.path = path
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.cum_flags = cum_flags
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_aa_run.restype = ctypes.c_int
        L.ref_aa_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _vp,
                                 _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp,
                                 _vp, ctypes.c_long, ctypes.c_int, ctypes.c_int, _dp]
        L.ref_init_equilibrium.restype = ctypes.c_int
        L.ref_init_equilibrium.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _vp, _dp,
                                           _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double]
        L.ref_collide.restype = ctypes.c_int
        L.ref_collide.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, _vp, _vp, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ref_equilibrium.restype = ctypes.c_int
        L.ref_equilibrium.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, _dp, _dp, _dp, _dp, _vp]
        L.ref_cum_flags.restype = ctypes.c_int
        assert L.ref_cum_flags() == cum_flags
        L.ref_srt_adjoint_collision.restype = ctypes.c_int
        L.ref_srt_adjoint_collision.argtypes = [ctypes.c_long, _dp, _dp, ctypes.c_double]
        L.ref_adjoint_data_term.restype = ctypes.c_int
        L.ref_adjoint_data_term.argtypes = [ctypes.c_long, _dp, _dp]
        L.ref_mean_update.restype = ctypes.c_int
        L.ref_mean_update.argtypes = [ctypes.c_int, ctypes.c_long, _vp, _vp, ctypes.c_int]
        L.ref_aa_ade_run.restype = ctypes.c_int
        L.ref_aa_ade_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long,
                                     ctypes.c_long, _vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, _dp, _dp, _dp, _vp, _vp, _vp, ctypes.c_double, _dp, ctypes.c_double,
                                     _vp, ctypes.c_long, ctypes.c_int]
        L.ref_ade_collide.restype = ctypes.c_int
        L.ref_ade_collide.argtypes = [ctypes.c_int, ctypes.c_long, _dp, _dp, _dp, ctypes.c_double]

    def aa_run(self, f, geo_map, coll="CUM", eq="INV_CUM", cum_flags=None, nu=0.01, force=(0.0, 0.0, 0.0), inflow=None,
               macro=None, start_iter=0, nsteps=1, nthreads=0, return_time=False):
        if cum_flags is not None and cum_flags != self.cum_flags:
            raise ValueError("this reference build has cumulant flags %d" % self.cum_flags)
        Z, Y, X = geo_map.shape
        assert f.shape == (27, Z + 2, Y + 2, X + 2) and f.flags.c_contiguous
        m = np.ascontiguousarray(geo_map, dtype=np.int16)
        vx, vy, vz = _profiles(inflow)
        el = ctypes.c_double(0.0)
        rc = self.lib.ref_aa_run(_prec(f.dtype), COLL[coll], EQ[eq], X, Y, Z, _ptr(f), _ptr(m), nu, *force, _dptr(vx),
                                 _dptr(vy), _dptr(vz), _ptr(macro), start_iter, nsteps, nthreads, ctypes.byref(el))
        if rc != 0:
            raise RuntimeError(f"ref_aa_run failed with {rc}")
        return (f, el.value) if return_time else f

    def init_equilibrium(self, f, X, Y, Z, eq="INV_CUM", fields=None, uniform=(1.0, 0.0, 0.0, 0.0)):
        rho = vx = vy = vz = None
        if fields is not None:
            rho, vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64) for a in fields)
        rc = self.lib.ref_init_equilibrium(_prec(f.dtype), EQ[eq], X, Y, Z, _ptr(f), _dptr(rho), _dptr(vx), _dptr(vy),
                                           _dptr(vz), *uniform)
        if rc != 0:
            raise RuntimeError("ref_init_equilibrium failed")
        return f

    def collide(self, f, coll="CUM", eq="INV_CUM", cum_flags=None, nu=0.01, force=(0.0, 0.0, 0.0)):
        macro = np.zeros((f.shape[0], 4), dtype=f.dtype)
        self.lib.ref_collide(_prec(f.dtype), COLL[coll], EQ[eq], f.shape[0], _ptr(f), _ptr(macro), nu, *force)
        return macro

    def equilibrium(self, rho, vx, vy, vz, eq="INV_CUM", dtype=np.float64):
        rho, vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (rho, vx, vy, vz))
        out = np.zeros((rho.size, 27), dtype=dtype)
        self.lib.ref_equilibrium(_prec(dtype), EQ[eq], rho.size, _dptr(rho), _dptr(vx), _dptr(vy), _dptr(vz), _ptr(out))
        return out

    def srt_adjoint_collision(self, fstar, u, nu):
        """D3Q27_SRT_ADJOINT::collision (col_srt_adjoint.h:50-109) of fstar[n, 27]
        about the primary velocity u[n, 3]; returns the updated copy."""
        out = np.ascontiguousarray(fstar, dtype=np.float64).copy()
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.lib.ref_srt_adjoint_collision(out.shape[0], _dptr(out), _dptr(u), nu)
        return out

    def aa_ade_run(self, f, geo_map, g, ade_map, coll="CUM", eq="INV_CUM", ade_coll="SRT", nu=0.01, D=0.01,
                   force=(0.0, 0.0, 0.0), inflow=None, dfield=None, inflow_phi=1.0, macro=None, phi=None, start_iter=0,
                   nsteps=1):
        """Coupled flow + D3Q7 scalar steps of cudaLBMKernel<NSE, ADE>
        (kernels.h:114-196): f [27, Z+2, Y+2, X+2] and g [7, Z+2, Y+2, X+2]
        updated in place; macro [4, Z, Y, X] and phi [Z, Y, X] outputs of every
        step (both or neither)."""
        Z, Y, X = geo_map.shape
        assert f.shape == (27, Z + 2, Y + 2, X + 2) and f.flags.c_contiguous
        assert g.shape == (7, Z + 2, Y + 2, X + 2) and g.flags.c_contiguous and g.dtype == f.dtype
        m = np.ascontiguousarray(geo_map, dtype=np.int16)
        am = np.ascontiguousarray(ade_map, dtype=np.int16)
        vx, vy, vz = _profiles(inflow)
        dfield = None if dfield is None else np.ascontiguousarray(dfield, dtype=np.float64)
        rc = self.lib.ref_aa_ade_run(_prec(f.dtype), COLL[coll], EQ[eq], ADE_COLL[ade_coll], X, Y, Z, _ptr(f), _ptr(m), nu,
                                     *force, _dptr(vx), _dptr(vy), _dptr(vz), _ptr(macro), _ptr(g), _ptr(am), D,
                                     _dptr(dfield), inflow_phi, _ptr(phi), start_iter, nsteps)
        if rc != 0:
            raise RuntimeError(f"ref_aa_ade_run failed with {rc}")
        return f, g

    def ade_collide(self, g, v, D, ade_coll="SRT"):
        """Per-site D3Q7 collision of g [n, 7] in place with velocities v [n, 3]; returns phi [n]."""
        assert g.dtype == np.float64 and g.flags.c_contiguous and g.shape[1] == 7
        v = np.ascontiguousarray(v, dtype=np.float64)
        phi = np.zeros(g.shape[0])
        self.lib.ref_ade_collide(ADE_COLL[ade_coll], g.shape[0], _dptr(g), _dptr(v), _dptr(phi), D)
        return phi

    def mean_update(self, macro, stats, counter):
        """D3Q27_MACRO_Mean::outputMacro (macro.h:117-171): one update of the
        running statistics stats [9, n] from the macro field macro [4, n]."""
        assert macro.dtype == stats.dtype and stats.flags.c_contiguous and stats.shape[0] == 9
        macro = np.ascontiguousarray(macro)
        self.lib.ref_mean_update(_prec(stats.dtype), stats.shape[1], _ptr(macro), _ptr(stats), counter)
        return stats

    def adjoint_data_term(self, macro):
        """D3Q27_EQ_ADJOINT::collisionWithData (eq_adjoint.h:30-33) of
        macro[n, 8] = (rho, vx, vy, vz, rho_m, vx_m, vy_m, vz_m) for every direction."""
        macro = np.ascontiguousarray(macro, dtype=np.float64)
        out = np.zeros((macro.shape[0], 27))
        self.lib.ref_adjoint_data_term(macro.shape[0], _dptr(macro), _dptr(out))
        return out


_REF_AB_VARIANTS = {0: "libref_ab_default", CUM_ANTIALIAS: "libref_ab_aa", CUM_2017 | CUM_ANTIALIAS: "libref_ab_2017aa"}


def reference_ab_available(cum_flags: int = 0) -> bool:
    name = _REF_AB_VARIANTS.get(cum_flags)
    return name is not None and os.path.exists(os.path.join(REFDIR, name + ".so"))


class ReferenceAB(_Base):
    """TNL-LBM's own per-site code with its A-B pull scheme (streaming_AB.h):
    two buffers swapped after every step, clamped neighbours at non-periodic
    boundary sites (kernels.h:48-55)."""

    def __init__(self, cum_flags: int = 0):
        path = os.path.join(REFDIR, _REF_AB_VARIANTS[cum_flags] + ".so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.cum_flags = cum_flags
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_ab_run.restype = ctypes.c_int
        L.ref_ab_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _vp,
                                 _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp,
                                 _vp, ctypes.c_long, ctypes.c_int, ctypes.c_int, _dp]
        L.ref_cum_flags.restype = ctypes.c_int
        assert L.ref_cum_flags() == cum_flags

    def ab_run(self, f, geo_map, coll="CUM", eq="INV_CUM", nu=0.01, force=(0.0, 0.0, 0.0), inflow=None, macro=None,
               nsteps=1, nthreads=0):
        """nsteps A-B steps of f [27, Z+2, Y+2, X+2] in place (the second buffer
        starts as a copy of f); macro [4, Z, Y, X] of the last step or None."""
        Z, Y, X = geo_map.shape
        assert f.shape == (27, Z + 2, Y + 2, X + 2) and f.flags.c_contiguous
        m = np.ascontiguousarray(geo_map, dtype=np.int16)
        vx, vy, vz = _profiles(inflow)
        el = ctypes.c_double(0.0)
        rc = self.lib.ref_ab_run(_prec(f.dtype), COLL[coll], EQ[eq], X, Y, Z, _ptr(f), _ptr(m), nu, *force, _dptr(vx),
                                 _dptr(vy), _dptr(vz), _ptr(macro), 0, nsteps, nthreads, ctypes.byref(el))
        if rc != 0:
            raise RuntimeError(f"ref_ab_run failed with {rc}")
        return f
