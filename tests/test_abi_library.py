"""The C-ABI library: builds for sm_100a, loads, exports every declared entry
point, and validates arguments without a GPU (CPU only)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^LBM_API\s+[\w\s\*]+?\b(lbm_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "lbm_create" in names and "lbm_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    import pytnl_lbm
    lib = pytnl_lbm.library()
    path = pytnl_lbm.library_path()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (lbm_\w+)$", out, flags=re.M))
    assert set(declared_symbols()) <= exported


def test_library_is_built_for_sm100a():
    import pytnl_lbm
    out = subprocess.run(["cuobjdump", "--list-elf", pytnl_lbm.library_path()], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_argument_validation_without_gpu():
    import pytnl_lbm
    from pytnl_lbm import _abi
    lib = pytnl_lbm.library()
    h = _abi.lbm_handle()
    assert lib.lbm_create(None, ctypes.byref(h)) == 1
    d = _abi.lbm_desc(X=0, Y=4, Z=4, storage=1, viscosity=0.01)
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert b"positive" in lib.lbm_last_error()
    d = _abi.lbm_desc(X=4, Y=4, Z=4, storage=1, collision=0, cum_flags=1, viscosity=0.01)
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 2  # 2017 without anti-aliasing
    d = _abi.lbm_desc(X=4, Y=4, Z=4, storage=1, viscosity=-1.0)
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = _abi.lbm_desc(X=4, Y=4, Z=4, storage=1, viscosity=float("nan"))
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    # sizes beyond the launch limits, unknown slot values
    for X, Y, Z in ((65535 * 4 + 1, 4, 4), (4, 65536, 4), (4, 4, 65536)):
        d = _abi.lbm_desc(X=X, Y=Y, Z=Z, storage=1, viscosity=0.01)
        assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 5
    for field, value in (("storage", 8), ("storage", -1), ("collision", 4), ("equilibrium", 2)):
        d = _abi.lbm_desc(X=4, Y=4, Z=4, storage=1, viscosity=0.01)
        setattr(d, field, value)
        assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1, (field, value)
    assert not h
    assert lib.lbm_step(None, 1, 0) == 1


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import pytnl_lbm
    with pytest.raises(pytnl_lbm.LbmError) as e:
        pytnl_lbm.LBM(8, 8, 8, viscosity=0.01, periodic=True)
    assert "CUDA" in str(e.value)
