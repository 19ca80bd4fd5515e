"""ctypes declarations of include/tnl_lbm_b200.h and the library loader."""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

LBM_OK = 0
ERRORS = {1: "invalid argument", 2: "unsupported", 3: "CUDA error", 4: "non-finite density", 5: "size limit"}

STORE_F64, STORE_F32, STORE_F32S, STORE_F16S, STORE_BF16S, STORE_F16SR, STORE_BF16SR, STORE_I16S = 0, 1, 2, 3, 4, 5, 6, 7
COLL_CUM, COLL_SRT, COLL_BGK, COLL_MRT = 0, 1, 2, 3
COLL_PLUGIN_FIRST, COLL_PLUGIN_LAST = 16, 31
PLUGIN_ABI_VERSION = 2
CUM_GEIER_2017, CUM_ANTIALIAS = 1, 2
EQ_SECOND_ORDER, EQ_INV_CUM = 0, 1
LAYOUT_INTERIOR, LAYOUT_GHOST = 0, 1
STEP_MACRO, STEP_SUMS = 1, 2
KERNEL_DIRECT, KERNEL_TILE, KERNEL_SPLIT, KERNEL_PAIR = 0, 1, 3, 4
STREAMING_AA, STREAMING_AB = 0, 1
STATUS_TIMEOUT = 1
ADE_SRT, ADE_MRT, ADE_CLBM = 0, 1, 2

# scalar site types of D3Q7_BC_All (include/lbm3d/d3q7/bc.h:17-36) that the coupled step provides
ADE_GEO = dict(FLUID=0, WALL=1, WALL_BODY=2, SOLID=3, INFLOW=7, PERIODIC=9, NOTHING=10, SYM_TOP=12, SYM_BOTTOM=13,
               SYM_LEFT=14, SYM_RIGHT=15, SYM_BACK=16, SYM_FRONT=17)

# GEO site types of D3Q27_BC_All (include/lbm3d/d3q27/bc.h:17-43)
GEO = dict(FLUID=0, WALL=1, INFLOW=2, INFLOW_LEFT=3, INFLOW_BB_LEFT=4, INFLOW_EQ_LEFT=5, OUTFLOW_EQ=6,
           OUTFLOW_RIGHT=7, OUTFLOW_RIGHT_INTERP=8, PERIODIC=9, NOTHING=10, SYM_TOP=11, SYM_BOTTOM=12,
           SYM_LEFT=13, SYM_RIGHT=14, SYM_BACK=15, SYM_FRONT=16)


class LbmError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"[{ERRORS.get(code, code)}] {message}")
        self.code = code


class lbm_desc(ctypes.Structure):
    _fields_ = [("X", ctypes.c_int32), ("Y", ctypes.c_int32), ("Z", ctypes.c_int32),
                ("storage", ctypes.c_int32), ("collision", ctypes.c_int32), ("cum_flags", ctypes.c_int32),
                ("equilibrium", ctypes.c_int32), ("periodic", ctypes.c_int32),
                ("viscosity", ctypes.c_double), ("fx", ctypes.c_double), ("fy", ctypes.c_double),
                ("fz", ctypes.c_double), ("device", ctypes.c_int32), ("use_graphs", ctypes.c_int32)]


class lbm_device_view(ctypes.Structure):
    _fields_ = [("populations", ctypes.c_void_p), ("sq", ctypes.c_int64), ("sy", ctypes.c_int32),
                ("sz", ctypes.c_int32), ("x0", ctypes.c_int32), ("elem_size", ctypes.c_int32),
                ("macro", ctypes.c_void_p), ("macro_elem_size", ctypes.c_int32), ("stream", ctypes.c_void_p)]


class lbm_ensemble_desc(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32), ("X", ctypes.POINTER(ctypes.c_int32)),
                ("Y", ctypes.POINTER(ctypes.c_int32)), ("Z", ctypes.POINTER(ctypes.c_int32)),
                ("viscosity", ctypes.POINTER(ctypes.c_double)), ("storage", ctypes.c_int32),
                ("collision", ctypes.c_int32), ("cum_flags", ctypes.c_int32), ("equilibrium", ctypes.c_int32),
                ("device", ctypes.c_int32), ("use_graphs", ctypes.c_int32)]


class lbm_ade_desc(ctypes.Structure):
    _fields_ = [("collision", ctypes.c_int32), ("diffusion", ctypes.c_double), ("inflow_phi", ctypes.c_double)]


lbm_handle = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_H = lbm_handle

SIGNATURES = {
    "lbm_create": (ctypes.c_int, [ctypes.POINTER(lbm_desc), ctypes.POINTER(lbm_handle)]),
    "lbm_destroy": (ctypes.c_int, [_H]),
    "lbm_last_error": (ctypes.c_char_p, []),
    "lbm_set_map": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_uint8)]),
    "lbm_get_map": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_uint8)]),
    "lbm_set_inflow": (ctypes.c_int, [_H, _dp, _dp, _dp]),
    "lbm_set_viscosity": (ctypes.c_int, [_H, ctypes.c_double]),
    "lbm_init_equilibrium": (ctypes.c_int, [_H, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double]),
    "lbm_init_taylor_green": (ctypes.c_int, [_H, ctypes.c_double, ctypes.c_double]),
    "lbm_set_populations": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_get_populations": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_step": (ctypes.c_int, [_H, ctypes.c_int64, ctypes.c_int]),
    "lbm_iteration": (ctypes.c_int64, [_H]),
    "lbm_set_iteration": (ctypes.c_int, [_H, ctypes.c_int64]),
    "lbm_get_macro": (ctypes.c_int, [_H, _dp]),
    "lbm_get_sums": (ctypes.c_int, [_H, _dp]),
    "lbm_enstrophy_sum": (ctypes.c_int, [_H, _dp]),
    "lbm_synchronize": (ctypes.c_int, [_H]),
    "lbm_set_block": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int]),
    "lbm_get_block": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "lbm_autotune": (ctypes.c_int, [_H, ctypes.c_int]),
    "lbm_device_view_get": (ctypes.c_int, [_H, ctypes.POINTER(lbm_device_view)]),
    "lbm_set_kernel": (ctypes.c_int, [_H, ctypes.c_int]),
    "lbm_get_kernel": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    "lbm_status": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    "lbm_version": (ctypes.c_char_p, []),
    "lbm_set_statistics": (ctypes.c_int, [_H, ctypes.c_int]),
    "lbm_get_statistics": (ctypes.c_int, [_H, _dp, ctypes.POINTER(ctypes.c_int64)]),
    "lbm_checkpoint_save": (ctypes.c_int, [_H, ctypes.c_char_p]),
    "lbm_checkpoint_load": (ctypes.c_int, [_H, ctypes.c_char_p]),
    "lbm_set_streaming": (ctypes.c_int, [_H, ctypes.c_int]),
    "lbm_get_streaming": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    "lbm_adjoint_forward": (ctypes.c_int, [_H, _dp, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                           ctypes.c_int32, _dp, ctypes.c_double, _dp]),
    "lbm_adjoint_backward": (ctypes.c_int, [_H, ctypes.c_double, _dp, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_adjoint_release": (ctypes.c_int, [_H]),
    "lbm_get_sums_of": (ctypes.c_int, [_H, ctypes.c_int64, _dp]),
    "lbm_set_distributed_z": (ctypes.c_int, [_H, ctypes.c_int]),
    "lbm_halo_bytes": (ctypes.c_int64, [_H]),
    "lbm_halo_pack": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "lbm_halo_unpack": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "lbm_halo_copy": (ctypes.c_int, [_H, ctypes.c_int, _H, ctypes.c_int, ctypes.c_int]),
    "lbm_set_wait_limit": (ctypes.c_int, [_H, ctypes.c_int64]),
    "lbm_ade_enable": (ctypes.c_int, [_H, ctypes.POINTER(lbm_ade_desc)]),
    "lbm_ade_disable": (ctypes.c_int, [_H]),
    "lbm_ade_set_map": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_uint8)]),
    "lbm_ade_set_diffusion": (ctypes.c_int, [_H, _dp]),
    "lbm_ade_init_equilibrium": (ctypes.c_int, [_H, _dp, _dp, _dp, _dp, ctypes.c_double]),
    "lbm_ade_set_populations": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_ade_get_populations": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_ade_get_phi": (ctypes.c_int, [_H, _dp]),
    "lbm_ensemble_create": (ctypes.c_int, [ctypes.POINTER(lbm_ensemble_desc), ctypes.POINTER(ctypes.c_void_p)]),
    "lbm_ensemble_destroy": (ctypes.c_int, [_H]),
    "lbm_ensemble_init_taylor_green": (ctypes.c_int, [_H, ctypes.c_double, ctypes.c_double]),
    "lbm_ensemble_init_equilibrium": (ctypes.c_int, [_H, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double]),
    "lbm_ensemble_set_populations": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_ensemble_get_populations": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "lbm_ensemble_step": (ctypes.c_int, [_H, ctypes.c_int64, ctypes.c_int]),
    "lbm_ensemble_get_sums": (ctypes.c_int, [_H, _dp]),
    "lbm_ensemble_iteration": (ctypes.c_int64, [_H]),
    "lbm_ensemble_get_stream": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_void_p)]),
    "lbm_ensemble_synchronize": (ctypes.c_int, [_H]),
    "lbm_ensemble_set_shape": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int]),
    "lbm_ensemble_get_shape": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "lbm_ensemble_autotune": (ctypes.c_int, [_H, ctypes.c_int]),
    "lbm_register_collision": (ctypes.c_int, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_char_p]),
    "lbm_collision_name": (ctypes.c_char_p, [ctypes.c_int32]),
}

# lbm_collision_launcher: int32_t (*)(const void* step, int32_t storage)
COLLISION_LAUNCHER = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32)

_LIB = None


def library_path() -> str:
    return os.environ.get("TNL_LBM_B200_LIB", os.path.join(PKG, "lib", "libtnl_lbm_b200.so"))


def library():
    """Load the sm_100a library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise LbmError(3, f"{path} not found: build it with `python tnl-lbm_b200/build.py`")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def check(rc: int):
    if rc != LBM_OK:
        raise LbmError(rc, library().lbm_last_error().decode())


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)
