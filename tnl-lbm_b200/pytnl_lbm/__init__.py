"""pytnl_lbm -- Python binding of the B200 D3Q27 A-A hot path.

Counterpart of TNL-LBM's nanobind module (pytnl_lbm/pytnl_lbm.cpp:15-73).  The
binding is a thin ctypes layer over the C-ABI in include/tnl_lbm_b200.h; the
compute runs in the sm_100a kernels of lib/libtnl_lbm_b200.so.  There is no
CPU fallback: creating a lattice without the library or without a CUDA device
raises.  numpy arrays are exchanged with the host entry points; torch tensors
(the only place PyTorch is used) can wrap the device buffers without copies
through ``LBM.device_view()``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import (  # noqa: F401  (re-exported constants)
    COLL_BGK, COLL_CUM, COLL_MRT, COLL_PLUGIN_FIRST, COLL_PLUGIN_LAST, COLL_SRT, CUM_ANTIALIAS, CUM_GEIER_2017, EQ_INV_CUM, EQ_SECOND_ORDER,
    ADE_CLBM, ADE_GEO, ADE_MRT, ADE_SRT, GEO, KERNEL_DIRECT, KERNEL_PAIR, KERNEL_SPLIT, KERNEL_TILE, STREAMING_AA, STREAMING_AB, LAYOUT_GHOST, LAYOUT_INTERIOR, STATUS_TIMEOUT, STEP_MACRO, STEP_SUMS,
    STORE_BF16S, STORE_BF16SR, STORE_F16S, STORE_F16SR, STORE_F32, STORE_F32S, STORE_F64, STORE_I16S, LbmError, library,
    library_path)

__all__ = ["LBM", "Ensemble", "LbmError", "library", "library_path", "GEO", "macro_names", "kinetic_energy", "State", "execute", "Actions",
           "Counter", "MAX_COUNTER", "NSE", "macro_from_populations", "register_collision", "unregister_collision",
           "collision_name", "plugin_path"]

# D3Q27_MACRO_Default quantity order (include/lbm3d/d3q27/macro.h:61-68)
macro_names = ("rho", "vx", "vy", "vz")


@dataclass
class Config:
    """Composition of the plugin slots (LBM_CONFIG, include/lbm3d/defs.h:288-310)."""
    collision: int = COLL_CUM
    cum_flags: int = 0
    equilibrium: int = EQ_INV_CUM
    storage: int = STORE_F32


class LBM:
    """One lattice on one GPU (LBM_BLOCK + LBM of the reference, single block).

    Sizes are lattice sites per axis without the ghost layer.  ``periodic=True``
    makes every site GEO_PERIODIC and no map is needed.
    """

    def __init__(self, X, Y, Z, *, viscosity, collision=COLL_CUM, cum_flags=0, equilibrium=EQ_INV_CUM,
                 storage=STORE_F32, periodic=False, force=(0.0, 0.0, 0.0), device=0, use_graphs=True):
        self.lib = library()
        d = _abi.lbm_desc()
        d.X, d.Y, d.Z = int(X), int(Y), int(Z)
        d.storage, d.collision, d.cum_flags, d.equilibrium = storage, collision, cum_flags, equilibrium
        d.periodic = 1 if periodic else 0
        d.viscosity = float(viscosity)
        d.fx, d.fy, d.fz = (float(v) for v in force)
        d.device = int(device)
        d.use_graphs = 1 if use_graphs else 0
        self.desc = d
        self.shape = (int(Z), int(Y), int(X))
        self.X, self.Y, self.Z = int(X), int(Y), int(Z)
        self.storage = storage
        h = _abi.lbm_handle()
        _abi.check(self.lib.lbm_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h

    # -- lifetime -------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- setup ----------------------------------------------------------
    def set_map(self, geo_map):
        m = np.ascontiguousarray(geo_map, dtype=np.uint8)
        assert m.shape == self.shape, f"map shape {m.shape} != {self.shape}"
        _abi.check(self.lib.lbm_set_map(self.h, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    def get_map(self):
        """The map last set or loaded from a checkpoint, [Z][Y][X] uint8."""
        m = np.empty(self.shape, np.uint8)
        _abi.check(self.lib.lbm_get_map(self.h, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return m

    def set_inflow(self, vx=None, vy=None, vz=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (vx, vy, vz)]
        for a in arrs:
            if a is not None:
                assert a.shape == (self.Z, self.Y)
        _abi.check(self.lib.lbm_set_inflow(self.h, *[_abi.dptr(a) for a in arrs]))

    def set_viscosity(self, nu):
        _abi.check(self.lib.lbm_set_viscosity(self.h, float(nu)))

    def init_equilibrium(self, rho=None, vx=None, vy=None, vz=None, uniform=(1.0, 0.0, 0.0, 0.0)):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (rho, vx, vy, vz)]
        _abi.check(self.lib.lbm_init_equilibrium(self.h, *[_abi.dptr(a) for a in arrs], *map(float, uniform)))

    def init_taylor_green(self, u0, rho0=1.0):
        _abi.check(self.lib.lbm_init_taylor_green(self.h, float(u0), float(rho0)))

    def set_populations(self, f, layout=LAYOUT_GHOST):
        f = np.ascontiguousarray(f)
        dtype = 0 if f.dtype == np.float64 else 1
        assert f.dtype in (np.float64, np.float32)
        assert f.shape == self._pop_shape(layout), f"{f.shape} != {self._pop_shape(layout)}"
        _abi.check(self.lib.lbm_set_populations(self.h, f.ctypes.data_as(ctypes.c_void_p), layout, dtype))

    def get_populations(self, layout=LAYOUT_GHOST, dtype=np.float64):
        out = np.empty(self._pop_shape(layout), dtype=dtype)
        _abi.check(self.lib.lbm_get_populations(self.h, out.ctypes.data_as(ctypes.c_void_p), layout,
                                                0 if out.dtype == np.float64 else 1))
        return out

    def _pop_shape(self, layout):
        g = 2 if layout == LAYOUT_GHOST else 0
        return (27, self.Z + g, self.Y + g, self.X + g)

    # -- stepping -------------------------------------------------------
    def step(self, nsteps=1, macro=False, sums=False):
        flags = (STEP_MACRO if macro else 0) | (STEP_SUMS if sums else 0)
        _abi.check(self.lib.lbm_step(self.h, int(nsteps), flags))

    @property
    def iteration(self):
        return int(self.lib.lbm_iteration(self.h))

    @iteration.setter
    def iteration(self, it):
        _abi.check(self.lib.lbm_set_iteration(self.h, int(it)))

    def macro(self):
        out = np.empty((4,) + self.shape, dtype=np.float64)
        _abi.check(self.lib.lbm_get_macro(self.h, _abi.dptr(out)))
        return out

    def sums(self):
        out = np.zeros(6, dtype=np.float64)
        _abi.check(self.lib.lbm_get_sums(self.h, _abi.dptr(out)))
        return out

    def sums_of(self, iteration):
        """Sums of the observation step that ended at `iteration` (the last two
        are kept); waits for that step only."""
        out = np.zeros(6, dtype=np.float64)
        _abi.check(self.lib.lbm_get_sums_of(self.h, int(iteration), _abi.dptr(out)))
        return out

    def enstrophy_sum(self):
        v = ctypes.c_double(0)
        _abi.check(self.lib.lbm_enstrophy_sum(self.h, ctypes.byref(v)))
        return v.value

    def synchronize(self):
        _abi.check(self.lib.lbm_synchronize(self.h))

    def set_block(self, bx, by):
        _abi.check(self.lib.lbm_set_block(self.h, int(bx), int(by)))

    def block(self):
        bx, by = ctypes.c_int(0), ctypes.c_int(0)
        _abi.check(self.lib.lbm_get_block(self.h, ctypes.byref(bx), ctypes.byref(by)))
        return bx.value, by.value

    def set_kernel(self, kernel):
        _abi.check(self.lib.lbm_set_kernel(self.h, int(kernel)))

    def set_statistics(self, enable=True):
        """Running velocity mean and covariance of D3Q27_MACRO_Mean, updated every step."""
        _abi.check(self.lib.lbm_set_statistics(self.h, 1 if enable else 0))

    def statistics(self):
        """(mean [3, Z, Y, X], covariance [6, Z, Y, X] in the order xx, yy, zz, xy, xz, yz, count)."""
        out = np.empty((9,) + self.shape, np.float64)
        n = ctypes.c_int64(0)
        _abi.check(self.lib.lbm_get_statistics(self.h, _abi.dptr(out), ctypes.byref(n)))
        cov = out[3:] / max(n.value, 1)
        return out[:3], cov, n.value

    # -- coupled D3Q7 scalar (lbm_ade_*) ---------------------------------
    def ade_enable(self, diffusion, collision=ADE_SRT, inflow_phi=1.0):
        """Advance a scalar phi with the flow in every step (kernels.h:114-196)."""
        d = _abi.lbm_ade_desc(int(collision), float(diffusion), float(inflow_phi))
        _abi.check(self.lib.lbm_ade_enable(self.h, ctypes.byref(d)))

    def ade_disable(self):
        _abi.check(self.lib.lbm_ade_disable(self.h))

    def ade_set_map(self, geo_map):
        m = np.ascontiguousarray(geo_map, dtype=np.uint8)
        assert m.shape == self.shape, f"map shape {m.shape} != {self.shape}"
        _abi.check(self.lib.lbm_ade_set_map(self.h, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    def ade_set_diffusion(self, field=None):
        """Per-site diffusion coefficient [Z][Y][X]; None returns to the constant."""
        a = None if field is None else np.ascontiguousarray(field, dtype=np.float64)
        if a is not None:
            assert a.shape == self.shape
        _abi.check(self.lib.lbm_ade_set_diffusion(self.h, _abi.dptr(a)))

    def ade_init_equilibrium(self, phi=None, vx=None, vy=None, vz=None, uniform_phi=0.0):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (phi, vx, vy, vz)]
        _abi.check(self.lib.lbm_ade_init_equilibrium(self.h, *[_abi.dptr(a) for a in arrs], float(uniform_phi)))

    def _ade_shape(self, layout):
        g = 2 if layout == LAYOUT_GHOST else 0
        return (7, self.Z + g, self.Y + g, self.X + g)

    def ade_set_populations(self, g, layout=LAYOUT_GHOST):
        g = np.ascontiguousarray(g)
        assert g.shape == self._ade_shape(layout) and g.dtype in (np.float64, np.float32)
        _abi.check(self.lib.lbm_ade_set_populations(self.h, g.ctypes.data_as(ctypes.c_void_p), layout,
                                                    0 if g.dtype == np.float64 else 1))

    def ade_get_populations(self, layout=LAYOUT_GHOST, dtype=np.float64):
        out = np.empty(self._ade_shape(layout), dtype=dtype)
        _abi.check(self.lib.lbm_ade_get_populations(self.h, out.ctypes.data_as(ctypes.c_void_p), layout,
                                                    0 if out.dtype == np.float64 else 1))
        return out

    def ade_phi(self):
        """phi [Z][Y][X] of the last step with macro=True."""
        out = np.empty(self.shape, np.float64)
        _abi.check(self.lib.lbm_ade_get_phi(self.h, _abi.dptr(out)))
        return out

    def save_checkpoint(self, path):
        """Write the state (populations as stored, map, inflow, iteration) to ``path``."""
        _abi.check(self.lib.lbm_checkpoint_save(self.h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Resume from a checkpoint written by a lattice of the same description."""
        _abi.check(self.lib.lbm_checkpoint_load(self.h, os.fsencode(path)))

    def set_streaming(self, streaming):
        """STREAMING_AA (in place, default) or STREAMING_AB (two buffers, pull)."""
        _abi.check(self.lib.lbm_set_streaming(self.h, int(streaming)))

    @property
    def streaming(self):
        k = ctypes.c_int(0)
        _abi.check(self.lib.lbm_get_streaming(self.h, ctypes.byref(k)))
        return k.value

    @property
    def kernel(self):
        k = ctypes.c_int(0)
        _abi.check(self.lib.lbm_get_kernel(self.h, ctypes.byref(k)))
        return k.value

    def status(self):
        v = ctypes.c_int(0)
        _abi.check(self.lib.lbm_status(self.h, ctypes.byref(v)))
        return v.value

    def set_wait_limit(self, tries=-1):
        """Bound of the tile kernel's per-tile waits in tries (negative: the
        default); see lbm_set_wait_limit."""
        _abi.check(self.lib.lbm_set_wait_limit(self.h, int(tries)))

    def autotune(self, ntrials=4):
        _abi.check(self.lib.lbm_autotune(self.h, int(ntrials)))
        return self.block()

    # -- slabs of a lattice split along z (lbm_halo_*) -----------------------
    def set_distributed_z(self, distributed=True):
        _abi.check(self.lib.lbm_set_distributed_z(self.h, 1 if distributed else 0))

    def halo_bytes(self):
        """Bytes of one staged exchange: the nine slot planes that cross a z face."""
        return int(self.lib.lbm_halo_bytes(self.h))

    def halo_buffer(self):
        """A device buffer of halo_bytes() bytes on this lattice's device."""
        import torch
        return torch.empty(self.halo_bytes(), dtype=torch.uint8, device=torch.device("cuda", self.desc.device))

    def halo_pack(self, z, cz, buf):
        """Stage the slots with c_z = cz of plane z (ghost frame) into the device
        tensor ``buf``, on this lattice's stream."""
        _abi.check(self.lib.lbm_halo_pack(self.h, int(z), int(cz), ctypes.c_void_p(buf.data_ptr())))

    def halo_unpack(self, z, cz, buf):
        _abi.check(self.lib.lbm_halo_unpack(self.h, int(z), int(cz), ctypes.c_void_p(buf.data_ptr())))

    def halo_copy(self, z, src, src_z, cz):
        """Plane z of this lattice <- plane src_z of ``src`` (slots with c_z = cz)."""
        _abi.check(self.lib.lbm_halo_copy(self.h, int(z), src.h, int(src_z), int(cz)))

    def device_view(self):
        v = _abi.lbm_device_view()
        _abi.check(self.lib.lbm_device_view_get(self.h, ctypes.byref(v)))
        return v

    # -- discrete adjoint (SRT collision, per-site body force) -------------
    def adjoint_forward(self, force, nsteps, samples, target, checkpoint_every=0, rho_weight=0.0):
        """Run nsteps from the current state with the per-site force field
        ``force`` [3, Z, Y, X] (None: the uniform force of the lattice) and
        return J = sum_i 1/2 [rho_weight (rho_i - rho*_i)^2 + |u_i - u*_i|^2]
        at the sample sites (flat indices (z*Y + y)*X + x) against
        ``target`` [n, 4] = (rho*, u*x, u*y, u*z).  ``force`` may be a numpy
        array or a float64 torch tensor; a CUDA tensor is read in place on the
        device (no host round trip)."""
        samples = np.ascontiguousarray(samples, dtype=np.int64)
        target = np.ascontiguousarray(target, dtype=np.float64).reshape(len(samples), 4)
        fp = None
        keep = None
        if force is not None:
            if tuple(force.shape) != (3,) + self.shape:
                raise ValueError(f"force must have shape {(3,) + self.shape}")
            if _is_cuda_tensor(force):
                keep = force.detach().to(dtype=_torch().float64).contiguous()
                fp = ctypes.cast(ctypes.c_void_p(keep.data_ptr()), ctypes.POINTER(ctypes.c_double))
            else:
                keep = np.ascontiguousarray(force, dtype=np.float64)
                fp = _abi.dptr(keep)
        loss = ctypes.c_double(0.0)
        _abi.check(self.lib.lbm_adjoint_forward(
            self.h, fp, int(nsteps), int(checkpoint_every), samples.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            len(samples), _abi.dptr(target), float(rho_weight), ctypes.byref(loss)))
        return loss.value

    def adjoint_backward(self, seed=1.0, populations=False, layout=LAYOUT_GHOST, out=None):
        """seed * dJ/dF [3, Z, Y, X] and, with ``populations``, seed * dJ/d(initial
        populations) in the layout of get_populations.  ``out``: a contiguous
        float64 CUDA tensor [3, Z, Y, X] that receives dJ/dF on the device
        (returned in place of a numpy array)."""
        if out is not None:
            if not (_is_cuda_tensor(out) and out.dtype == _torch().float64 and out.is_contiguous()
                    and tuple(out.shape) == (3,) + self.shape):
                raise ValueError(f"out must be a contiguous float64 CUDA tensor of shape {(3,) + self.shape}")
            g = out
            gptr = ctypes.cast(ctypes.c_void_p(out.data_ptr()), ctypes.POINTER(ctypes.c_double))
        else:
            g = np.empty((3,) + self.shape, np.float64)
            gptr = _abi.dptr(g)
        gp = np.empty(self._pop_shape(layout), np.float64) if populations else None
        _abi.check(self.lib.lbm_adjoint_backward(self.h, float(seed), gptr,
                                                 gp.ctypes.data if gp is not None else None, layout, 0))
        return (g, gp) if populations else g

    def adjoint_release(self):
        _abi.check(self.lib.lbm_adjoint_release(self.h))

    def populations_tensor(self):
        """torch view of the raw population storage [27, Z+2, Y+2, pitch] (no copy;
        strides (sq, sz, sy, 1): the 27 slot rows of a lattice row lie side by side)."""
        import torch
        v = self.device_view()
        dt = {8: torch.float64, 4: torch.float32,
              2: torch.float16 if self.storage in (STORE_F16S, STORE_F16SR) else torch.bfloat16}[v.elem_size]
        flat = _wrap_device(v.populations, v.sz * (self.Z + 2), dt, self.desc.device)
        return flat.as_strided((27, self.Z + 2, self.Y + 2, v.sq), (v.sq, v.sz, v.sy, 1))


def _torch():
    import torch
    return torch


def _is_cuda_tensor(a):
    return hasattr(a, "is_cuda") and hasattr(a, "data_ptr") and bool(a.is_cuda)


def _wrap_device(ptr, n, dtype, device):
    import torch

    class _CudaArray:
        def __init__(self):
            self.__cuda_array_interface__ = {
                "shape": (n,), "typestr": {torch.float64: "<f8", torch.float32: "<f4", torch.float16: "<f2",
                                           torch.bfloat16: "<f2"}[dtype],
                "data": (int(ptr), False), "version": 3}

    t = torch.as_tensor(_CudaArray(), device=f"cuda:{device}")
    return t.view(dtype) if dtype == torch.bfloat16 else t


class Ensemble:
    """Many independent periodic lattices of different sizes and viscosities,
    advanced together by one launch per A-A step (lbm_ensemble_* of the C-ABI).

    ``sizes`` is a sequence of (X, Y, Z); ``viscosities`` one value per member.
    Each member evolves exactly as a periodic ``LBM`` of the same size and
    viscosity would.
    """

    def __init__(self, sizes, viscosities, *, collision=COLL_CUM, cum_flags=0, equilibrium=EQ_INV_CUM,
                 storage=STORE_F32, device=0, use_graphs=True):
        self.lib = library()
        sizes = [tuple(int(v) for v in s) for s in sizes]
        if len(sizes) != len(viscosities):
            raise ValueError("one viscosity per member")
        n = len(sizes)
        self._X = (ctypes.c_int32 * n)(*[s[0] for s in sizes])
        self._Y = (ctypes.c_int32 * n)(*[s[1] for s in sizes])
        self._Z = (ctypes.c_int32 * n)(*[s[2] for s in sizes])
        self._nu = (ctypes.c_double * n)(*[float(v) for v in viscosities])
        d = _abi.lbm_ensemble_desc()
        d.count = n
        d.X, d.Y, d.Z, d.viscosity = self._X, self._Y, self._Z, self._nu
        d.storage, d.collision, d.cum_flags, d.equilibrium = storage, collision, cum_flags, equilibrium
        d.device = int(device)
        d.use_graphs = 1 if use_graphs else 0
        self.sizes = sizes
        self.storage = storage
        h = ctypes.c_void_p()
        _abi.check(self.lib.lbm_ensemble_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h

    def __len__(self):
        return len(self.sizes)

    def close(self):
        if getattr(self, "h", None):
            self.lib.lbm_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_taylor_green(self, u0, rho0=1.0):
        _abi.check(self.lib.lbm_ensemble_init_taylor_green(self.h, float(u0), float(rho0)))

    def init_equilibrium(self, rho0=1.0, vx=0.0, vy=0.0, vz=0.0):
        _abi.check(self.lib.lbm_ensemble_init_equilibrium(self.h, float(rho0), float(vx), float(vy), float(vz)))

    def _pop_shape(self, member, layout):
        X, Y, Z = self.sizes[member]
        g = 2 if layout == LAYOUT_GHOST else 0
        return (27, Z + g, Y + g, X + g)

    def set_populations(self, member, f, layout=LAYOUT_GHOST):
        dtype = 0 if f.dtype == np.float64 else 1
        a = np.ascontiguousarray(f, dtype=np.float64 if dtype == 0 else np.float32)
        if a.shape != self._pop_shape(member, layout):
            raise ValueError(f"populations of member {member} must have shape {self._pop_shape(member, layout)}")
        _abi.check(self.lib.lbm_ensemble_set_populations(self.h, int(member), a.ctypes.data, layout, dtype))

    def get_populations(self, member, layout=LAYOUT_GHOST, dtype=np.float64):
        if not 0 <= int(member) < len(self.sizes):
            raise LbmError(1, f"member {member} out of range")
        out = np.empty(self._pop_shape(member, layout), dtype)
        _abi.check(self.lib.lbm_ensemble_get_populations(self.h, int(member), out.ctypes.data, layout,
                                                         0 if dtype == np.float64 else 1))
        return out

    def step(self, nsteps=1, sums=False):
        _abi.check(self.lib.lbm_ensemble_step(self.h, int(nsteps), STEP_SUMS if sums else 0))

    def sums(self):
        """[members, 6]: sum rho, rho vx, rho vy, rho vz, rho |u|^2, non-finite count."""
        out = np.empty((len(self.sizes), 6), np.float64)
        _abi.check(self.lib.lbm_ensemble_get_sums(self.h, _abi.dptr(out)))
        return out

    def kinetic_energy(self, rho0=1.0):
        """E = sum rho |u|^2 / (2 rho0 V) of every member after the last summed step."""
        vol = np.array([x * y * z for (x, y, z) in self.sizes], np.float64)
        return self.sums()[:, 4] / rho0 / 2.0 / vol

    @property
    def iteration(self):
        return int(self.lib.lbm_ensemble_iteration(self.h))

    @property
    def stream(self):
        """the ensemble's cudaStream_t as an integer"""
        s = ctypes.c_void_p()
        _abi.check(self.lib.lbm_ensemble_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self):
        _abi.check(self.lib.lbm_ensemble_synchronize(self.h))

    def set_shape(self, tile_sites, grid_policy):
        _abi.check(self.lib.lbm_ensemble_set_shape(self.h, int(tile_sites), int(grid_policy)))

    def shape(self):
        a, b = ctypes.c_int(0), ctypes.c_int(0)
        _abi.check(self.lib.lbm_ensemble_get_shape(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def autotune(self, ntrials=4):
        _abi.check(self.lib.lbm_ensemble_autotune(self.h, int(ntrials)))
        return self.shape()


# loaded plugin libraries, kept alive while their launchers are registered
_PLUGINS = {}


def plugin_path(name):
    """Path of a collision plugin built from tnl-lbm_b200/plugins/<name>.cu."""
    return os.path.join(os.path.dirname(_abi.library_path()), "plugins", name + ".so")


def register_collision(id, path, symbol, name=None):
    """Register the collision plugin launcher `symbol` of the shared library
    `path` (built with LBM_COLLISION_PLUGIN, tnl-lbm_b200/csrc/plugin.cuh)
    under `id` in [COLL_PLUGIN_FIRST, COLL_PLUGIN_LAST]; LBM(...,
    collision=id) then runs it.  Returns id."""
    lib = library()
    if not os.path.exists(path):
        raise LbmError(1, f"collision plugin {path} not found")
    so = ctypes.CDLL(os.path.abspath(path))
    fn = getattr(so, symbol)
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    addr = ctypes.cast(fn, ctypes.c_void_p).value
    label = (name or symbol).encode()
    _abi.check(lib.lbm_register_collision(int(id), addr, _abi.PLUGIN_ABI_VERSION, label))
    _PLUGINS[int(id)] = (so, fn)
    return int(id)


def unregister_collision(id):
    """Remove the plugin registered under `id`; lattices created with it keep
    their launcher, and the plugin library stays loaded."""
    _abi.check(library().lbm_register_collision(int(id), None, _abi.PLUGIN_ABI_VERSION, None))


def collision_name(id):
    """Name a plugin was registered under, or None."""
    n = library().lbm_collision_name(int(id))
    return None if n is None else n.decode()


def kinetic_energy(lbm: LBM, rho0=1.0):
    """Kinetic energy of the last summed step, E = sum rho |u|^2 / (2 rho0 V)
    (sim_NSE/sim_4.cu:257-275), in lattice units."""
    s = lbm.sums()
    return s[4] / rho0 / 2.0 / (lbm.X * lbm.Y * lbm.Z)


from ._state import MAX_COUNTER, NSE, Actions, Counter, State, execute, macro_from_populations  # noqa: E402,F401
