"""Checkpoint / resume (lbm_checkpoint_save / lbm_checkpoint_load) on the GPU.

A run interrupted by a checkpoint and resumed in a fresh lattice must continue
bit for bit: the file holds the population buffer as stored (every storage
format), the A-A parity, the map, the inlet profiles and the streaming pattern.
"""
import numpy as np
import pytest

from helpers import GEO, duct_map, seeded_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    return pytnl_lbm


def make(pl, storage, streaming, X=36, Y=12, Z=10):
    lat = pl.LBM(X, Y, Z, viscosity=0.01, cum_flags=3, storage=getattr(pl, "STORE_" + storage))
    lat.set_streaming(streaming)
    return lat


@pytest.mark.parametrize("storage", ["F64", "F32", "F16S", "BF16S"])
@pytest.mark.parametrize("ab", [False, True])
@pytest.mark.parametrize("first", [10, 7])
def test_resume_continues_bit_for_bit(pl, port, tmp_path, storage, ab, first):
    X, Y, Z = 36, 12, 10
    rng = np.random.default_rng(first)
    streaming = pl.STREAMING_AB if ab else pl.STREAMING_AA
    outlet = GEO["OUTFLOW_RIGHT"] if ab else GEO["OUTFLOW_EQ"]
    m = duct_map(X, Y, Z, GEO["INFLOW_LEFT"], outlet)
    f0 = seeded_state(port, rng, X, Y, Z)
    a = make(pl, storage, streaming)
    a.set_map(m)
    a.set_inflow(0.02 * rng.random((Z, Y)), 0.001 * rng.random((Z, Y)), None)
    a.set_populations(f0)
    a.step(first)
    path = str(tmp_path / "state.ckpt")
    a.save_checkpoint(path)
    a.step(9, macro=True)
    ref_f, ref_m = a.get_populations(), a.macro()
    a.close()

    b = make(pl, storage, pl.STREAMING_AA)  # pattern, map and profiles come from the file
    b.load_checkpoint(path)
    assert b.iteration == first
    assert b.streaming == streaming
    b.step(9, macro=True)
    assert np.array_equal(b.get_populations(), ref_f)
    assert np.array_equal(b.macro(), ref_m)
    b.close()


def test_mismatched_or_damaged_checkpoints_are_rejected(pl, tmp_path):
    a = pl.LBM(16, 8, 6, viscosity=0.01, periodic=True)
    a.init_taylor_green(0.05)
    path = tmp_path / "a.ckpt"
    a.save_checkpoint(str(path))
    b = pl.LBM(16, 8, 7, viscosity=0.01, periodic=True)
    with pytest.raises(pl.LbmError):
        b.load_checkpoint(str(path))  # other size
    c = pl.LBM(16, 8, 6, viscosity=0.01, periodic=True, storage=pl.STORE_F64)
    with pytest.raises(pl.LbmError):
        c.load_checkpoint(str(path))  # other storage
    cut = tmp_path / "cut.ckpt"
    cut.write_bytes(path.read_bytes()[:-100])
    with pytest.raises(pl.LbmError):
        a.load_checkpoint(str(cut))
    junk = tmp_path / "junk.ckpt"
    junk.write_bytes(b"not a checkpoint" * 10)
    with pytest.raises(pl.LbmError):
        a.load_checkpoint(str(junk))
    d = pl.LBM(16, 8, 6, viscosity=0.02, periodic=True)
    d.load_checkpoint(str(path))  # the viscosity is restored
    for lat in (a, b, c, d):
        lat.close()
