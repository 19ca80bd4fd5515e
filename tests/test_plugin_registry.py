"""The open collision slot on the host (CPU only): registration, the plugin
library's exported launchers and their storage query, and the lattice
descriptor checks that run before any device call."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NOT_SUPPORTED = 801  # cudaErrorNotSupported
LAUNCHERS = ("lbm_example_srt", "lbm_example_streaming", "lbm_example_trt")


@pytest.fixture
def pl():
    import pytnl_lbm
    yield pytnl_lbm
    for i in range(pytnl_lbm.COLL_PLUGIN_FIRST, pytnl_lbm.COLL_PLUGIN_LAST + 1):
        pytnl_lbm.unregister_collision(i)


def _abi_version(pl):
    from pytnl_lbm import _abi
    return _abi.PLUGIN_ABI_VERSION


def test_python_abi_version_matches_the_header():
    from pytnl_lbm import _abi
    text = open(os.path.join(ROOT, "include", "tnl_lbm_b200.h")).read()
    assert int(re.search(r"#define LBM_PLUGIN_ABI_VERSION (\d+)", text).group(1)) == _abi.PLUGIN_ABI_VERSION


def example_path(pl):
    path = pl.plugin_path("example_collisions")
    if not os.path.exists(path):
        pytest.skip("example plugins not built")
    return path


def test_plugin_library_exports_only_its_launchers(pl):
    out = subprocess.run(["nm", "-D", "--defined-only", example_path(pl)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)$", out, flags=re.M))
    assert set(LAUNCHERS) <= exported
    assert not [s for s in exported if "lbm" in s and s not in LAUNCHERS]


def test_launcher_answers_storage_queries_without_a_device(pl):
    so = ctypes.CDLL(example_path(pl))
    built = {"lbm_example_srt": range(8), "lbm_example_streaming": (0, 1), "lbm_example_trt": (0, 1)}
    for name in LAUNCHERS:
        fn = getattr(so, name)
        fn.restype = ctypes.c_int32
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        for storage in range(-1, 9):
            want = 0 if storage in built[name] else NOT_SUPPORTED
            assert fn(None, storage) == want, (name, storage)


def test_registration_checks_id_and_abi_version(pl):
    lib = pl.library()
    path = example_path(pl)
    for bad in (pl.COLL_PLUGIN_FIRST - 1, pl.COLL_PLUGIN_LAST + 1, 0, 3):
        with pytest.raises(pl.LbmError) as e:
            pl.register_collision(bad, path, "lbm_example_trt")
        assert e.value.code == 1
    so = ctypes.CDLL(path)
    addr = ctypes.cast(so.lbm_example_trt, ctypes.c_void_p).value
    bad_version = _abi_version(pl) + 1
    assert lib.lbm_register_collision(pl.COLL_PLUGIN_FIRST, addr, bad_version, b"trt") == 2
    assert f"plugin ABI {bad_version}".encode() in lib.lbm_last_error()
    assert pl.collision_name(pl.COLL_PLUGIN_FIRST) is None
    with pytest.raises(AttributeError):
        pl.register_collision(pl.COLL_PLUGIN_FIRST, path, "no_such_launcher")
    with pytest.raises(pl.LbmError):
        pl.register_collision(pl.COLL_PLUGIN_FIRST, os.path.join(ROOT, "missing.so"), "lbm_example_trt")


def test_register_name_and_remove(pl):
    path = example_path(pl)
    a = pl.register_collision(pl.COLL_PLUGIN_FIRST, path, "lbm_example_trt", name="TRT")
    b = pl.register_collision(pl.COLL_PLUGIN_LAST, path, "lbm_example_srt")
    assert pl.collision_name(a) == "TRT"
    assert pl.collision_name(b) == "lbm_example_srt"
    assert pl.collision_name(pl.COLL_PLUGIN_FIRST + 1) is None
    assert pl.collision_name(2) is None  # built-in ids carry no plugin name
    pl.register_collision(a, path, "lbm_example_streaming", name="streaming")  # replaces
    assert pl.collision_name(a) == "streaming"
    pl.unregister_collision(a)
    assert pl.collision_name(a) is None
    assert pl.collision_name(b) == "lbm_example_srt"


def test_descriptor_checks_for_plugin_ids(pl):
    from pytnl_lbm import _abi
    lib = pl.library()
    h = _abi.lbm_handle()
    cid = pl.COLL_PLUGIN_FIRST + 3
    d = _abi.lbm_desc(X=4, Y=4, Z=4, storage=pl.STORE_F64, collision=cid, viscosity=0.01)
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1  # nothing registered under the id
    assert b"no collision plugin registered" in lib.lbm_last_error()
    pl.register_collision(cid, example_path(pl), "lbm_example_trt")
    d.storage = pl.STORE_F16S  # the TRT example is built for FP64 and FP32 only
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 2
    assert b"not built for storage" in lib.lbm_last_error()
    d.storage, d.cum_flags = pl.STORE_F64, pl.CUM_ANTIALIAS
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert not h


USER_PLUGIN = r"""
#include "plugin.cuh"

struct Relax
{
    template <typename R>
    __device__ static void collision(lbm::Site<R>& s, const lbm::CollParams<R>& p)
    {
        R feq[27];
        lbm::set_equilibrium(feq, p.eq, s.rho, s.vx, s.vy, s.vz);
        for (int q = 0; q < 27; q++)
            s.f[q] += (feq[q] - s.f[q]) * p.inv_tau;
    }
};

LBM_COLLISION_PLUGIN(user_relax, Relax, LBM_PLUGIN_STORAGE(LBM_STORE_F64))
"""


def test_build_plugin_compiles_a_user_collision(pl, tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location("tnl_build", os.path.join(ROOT, "tnl-lbm_b200", "build.py"))
    build = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(build)
    if not os.path.exists(build.NVCC):
        pytest.skip("nvcc unavailable")
    src = tmp_path / "user_relax.cu"
    src.write_text(USER_PLUGIN)
    so = build.build_plugin(str(src), str(tmp_path / "user_relax.so"))
    lib = ctypes.CDLL(so)
    lib.user_relax.restype = ctypes.c_int32
    lib.user_relax.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    assert lib.user_relax(None, pl.STORE_F64) == 0
    assert lib.user_relax(None, pl.STORE_F32) == NOT_SUPPORTED
    pl.register_collision(pl.COLL_PLUGIN_FIRST + 5, so, "user_relax", name="relax")
    assert pl.collision_name(pl.COLL_PLUGIN_FIRST + 5) == "relax"
