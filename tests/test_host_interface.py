"""The C++ host interface (tnl-lbm_b200/host/lbm_b200.hpp) and its example
solvers, built by tnl-lbm_b200/build.py against the C-ABI library."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tnl-lbm_b200", "lib")


def test_examples_are_built_and_linked():
    for name in ("sim_tgv", "sim_duct"):
        exe = os.path.join(LIB, name)
        assert os.path.exists(exe), f"{exe} missing: run python tnl-lbm_b200/build.py"
        out = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
        assert "libtnl_lbm_b200.so" in out and "not found" not in out


def test_header_compiles_standalone(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "lbm_b200.hpp"\n'
                   'using C = tnl_lbm_b200::LBM_CONFIG<tnl_lbm_b200::F32, tnl_lbm_b200::D3Q27_SRT, tnl_lbm_b200::D3Q27_EQ>;\n'
                   'static_assert(C::coll::id == LBM_COLL_SRT, "slot");\nint main() { return 0; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(ROOT, "tnl-lbm_b200", "host"), str(src), "-o", str(tmp_path / "t")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_sim_tgv_reproduces_reference_kinetic_energy(golden):
    """sim_tgv at 16^3 in FP64 prints the kinetic energy of the reference's own
    Taylor-Green run (tests/golden, probes after 2-step chunks)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = subprocess.run([os.path.join(LIB, "sim_tgv"), "16", "20", "2", "f64"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    rows = [line.split() for line in out.stdout.splitlines() if line and not line.startswith("#")]
    ke = np.array([float(r[1]) for r in rows])
    np.testing.assert_allclose(ke, golden["tgv16_ke"], rtol=1e-12)


@pytest.mark.gpu
def test_sim_duct_runs_and_conserves_mass_scale():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = subprocess.run([os.path.join(LIB, "sim_duct"), "96", "24", "24", "200"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    rows = np.array([[float(v) for v in line.split()] for line in out.stdout.splitlines()
                     if line and not line.startswith("#")])
    mass = rows[:, 1]
    assert np.all(np.isfinite(rows))
    assert np.all(np.abs(mass / (96 * 24 * 24) - 1) < 0.05)
    assert rows[-1, 2] > 0  # the inlet drives a positive mean flow
