"""User-compiled collisions in the open COLL slot (csrc/plugin.cuh) on the GPU.

* The library's SRT collision compiled as a plugin updates a mapped lattice
  (walls, inlet, outlet, periodic and symmetry sites) and a periodic one
  exactly as LBM_COLL_SRT does, on every storage, with the macro field and
  the FP64 sums of the observation step: the plugin runs the library's own
  per-site step with the collision inlined.
* A collision that does nothing leaves pure A-A streaming: after 2k steps
  slot q holds the initial populations shifted by 2k c_q (np.roll), exactly.
* A two-relaxation-time collision, which the built-ins do not have, matches a
  numpy restatement of collide-then-stream on a periodic lattice.
* With LBM_KERNEL_PAIR the plugins run on the two-site kernel (two sites per
  thread, packed FP32): the SRT plugin equals the built-in SRT's two-site
  step bit for bit, streaming stays exact, and TRT matches numpy; the sums of
  a sums-only step (which leaves the GEO_NOTHING sites to the finish kernel)
  agree with the one-site kernel's.
* Restrictions: plugin lattices run the one-site or the two-site kernel with
  A-A streaming and take no coupled scalar or adjoint; graphs and the host
  loop agree.
"""
import numpy as np
import pytest

from helpers import GEO, duct_map

pytestmark = pytest.mark.gpu

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])
OPP = np.array([0] + [q + 1 if q % 2 else q - 1 for q in range(1, 27)])
NNZ = np.abs(CX) + np.abs(CY) + np.abs(CZ)
W = np.where(NNZ == 0, 8 / 27, np.where(NNZ == 1, 2 / 27, np.where(NNZ == 2, 1 / 54, 1 / 216)))

SRT_ID, STREAM_ID, TRT_ID = 16, 17, 18


@pytest.fixture(scope="module")
def pl():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pytnl_lbm
    path = pytnl_lbm.plugin_path("example_collisions")
    pytnl_lbm.register_collision(SRT_ID, path, "lbm_example_srt", name="SRT (plugin)")
    pytnl_lbm.register_collision(STREAM_ID, path, "lbm_example_streaming", name="streaming only")
    pytnl_lbm.register_collision(TRT_ID, path, "lbm_example_trt", name="TRT")
    yield pytnl_lbm
    for i in (SRT_ID, STREAM_ID, TRT_ID):
        pytnl_lbm.unregister_collision(i)


def mixed_map(X, Y, Z):
    """Duct with a periodic z band and a symmetry plane: every kind of site the
    one-site step distinguishes."""
    m = duct_map(X, Y, Z)
    m[:, 2:-2, X // 2] = GEO["PERIODIC"]
    m[2, 2:-2, 2:X // 2] = GEO["SYM_BOTTOM"]
    m[3:5, 3:5, 3:5] = GEO["WALL"]
    return m


def make(pl, collision, storage, periodic, shape=(20, 12, 10), use_graphs=True, **kw):
    X, Y, Z = shape
    lat = pl.LBM(X, Y, Z, viscosity=0.02, collision=collision, equilibrium=pl.EQ_SECOND_ORDER,
                 storage=storage, periodic=periodic, use_graphs=use_graphs, **kw)
    if not periodic:
        lat.set_map(mixed_map(X, Y, Z))
        prof = np.full((Z, Y), 0.02)
        lat.set_inflow(prof)
        lat.init_equilibrium(uniform=(1.0, 0.01, 0.0, 0.0))
    else:
        rng = np.random.default_rng(5)
        rho = 1 + 0.01 * rng.standard_normal((Z, Y, X))
        u = 0.03 * rng.standard_normal((3, Z, Y, X))
        lat.init_equilibrium(rho, *u)
    return lat


@pytest.mark.parametrize("storage", ["F64", "F32", "F32S", "F16S", "BF16S", "F16SR", "BF16SR", "I16S"])
@pytest.mark.parametrize("periodic", [False, True])
def test_srt_plugin_equals_builtin_srt(pl, storage, periodic):
    st = getattr(pl, "STORE_" + storage)
    out = []
    for coll in (pl.COLL_SRT, SRT_ID):
        lat = make(pl, coll, st, periodic, force=(1e-5, 0.0, 2e-6))
        lat.step(21)
        lat.step(1, macro=True, sums=True)
        out.append((lat.get_populations(), lat.macro(), lat.sums()))
        lat.close()
    (f0, m0, s0), (f1, m1, s1) = out
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(m1, m0)
    np.testing.assert_array_equal(s1, s0)


@pytest.mark.parametrize("storage", ["F64", "F32"])
def test_streaming_plugin_is_pure_aa_streaming(pl, storage):
    X, Y, Z = 14, 10, 8
    dtype = np.float64 if storage == "F64" else np.float32
    lat = pl.LBM(X, Y, Z, viscosity=0.02, collision=STREAM_ID, storage=getattr(pl, "STORE_" + storage),
                 periodic=True)
    rng = np.random.default_rng(11)
    f0 = (rng.random((27, Z, Y, X)) + 0.5).astype(dtype)
    lat.set_populations(f0, layout=pl.LAYOUT_INTERIOR)
    for n in (2, 6):
        lat.iteration = 0
        lat.set_populations(f0, layout=pl.LAYOUT_INTERIOR)
        lat.step(n)
        f = lat.get_populations(layout=pl.LAYOUT_INTERIOR, dtype=dtype)
        for q in range(27):
            want = np.roll(f0[q], shift=(n * CZ[q], n * CY[q], n * CX[q]), axis=(0, 1, 2))
            np.testing.assert_array_equal(f[q], want, err_msg=f"q={q} after {n} steps")
    lat.close()


def trt_collide(f, nu):
    """Two-relaxation-time collision of [27, ...] populations towards the
    second-order equilibrium, Lambda = 3/16 (the plugin's definition)."""
    rho = f.sum(axis=0)
    vx = np.tensordot(CX, f, axes=1) / rho
    vy = np.tensordot(CY, f, axes=1) / rho
    vz = np.tensordot(CZ, f, axes=1) / rho
    usq = vx * vx + vy * vy + vz * vz
    cu = CX[:, None, None, None] * vx + CY[:, None, None, None] * vy + CZ[:, None, None, None] * vz
    feq = W[:, None, None, None] * rho * ((1 - 1.5 * usq + 3 * cu) + 4.5 * cu * cu)
    tau = 3 * nu + 0.5
    wp = 1 / tau
    wm = 1 / ((3 / 16) / (tau - 0.5) + 0.5)
    fb, eb = f[OPP], feq[OPP]
    return f - wp * 0.5 * ((f + fb) - (feq + eb)) - wm * 0.5 * ((f - fb) - (feq - eb))


def stream(f):
    return np.stack([np.roll(f[q], shift=(CZ[q], CY[q], CX[q]), axis=(0, 1, 2)) for q in range(27)])


@pytest.mark.parametrize("storage,tol", [("F64", 1e-13), ("F32", 2e-6)])
def test_trt_plugin_matches_numpy(pl, storage, tol):
    X, Y, Z = 12, 10, 8
    nu = 0.01
    rng = np.random.default_rng(3)
    lat = pl.LBM(X, Y, Z, viscosity=nu, collision=TRT_ID, equilibrium=pl.EQ_SECOND_ORDER,
                 storage=getattr(pl, "STORE_" + storage), periodic=True)
    rho = 1 + 0.01 * rng.standard_normal((Z, Y, X))
    u = 0.04 * rng.standard_normal((3, Z, Y, X))
    lat.init_equilibrium(rho, *u)
    f0 = lat.get_populations(layout=pl.LAYOUT_INTERIOR)
    f0 = f0 * (1 + 0.02 * rng.standard_normal(f0.shape))  # off equilibrium: both rates act
    lat.set_populations(f0, layout=pl.LAYOUT_INTERIOR)
    f0 = lat.get_populations(layout=pl.LAYOUT_INTERIOR)
    lat.step(4)
    f = lat.get_populations(layout=pl.LAYOUT_INTERIOR)
    want = f0
    for _ in range(4):
        want = stream(trt_collide(want, nu))
    err = np.max(np.abs(f - want)) / np.max(np.abs(want))
    assert err <= tol, err
    # the antisymmetric rate is not the symmetric one: TRT differs from SRT here
    srt = pl.LBM(X, Y, Z, viscosity=nu, collision=pl.COLL_SRT, equilibrium=pl.EQ_SECOND_ORDER,
                 storage=getattr(pl, "STORE_" + storage), periodic=True)
    srt.set_populations(f0, layout=pl.LAYOUT_INTERIOR)
    srt.step(4)
    assert np.max(np.abs(srt.get_populations(layout=pl.LAYOUT_INTERIOR) - f)) > 100 * tol
    lat.close()
    srt.close()


def test_graph_replay_equals_host_loop(pl):
    out = []
    for graphs in (True, False):
        lat = make(pl, TRT_ID, pl.STORE_F32, False, use_graphs=graphs)
        lat.step(37, sums=True)
        out.append((lat.get_populations(), lat.sums()))
        lat.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_plugin_lattice_restrictions(pl):
    lat = make(pl, SRT_ID, pl.STORE_F64, False)
    for kernel in (pl.KERNEL_TILE, pl.KERNEL_SPLIT):
        with pytest.raises(pl.LbmError) as e:
            lat.set_kernel(kernel)
        assert e.value.code == 2
    with pytest.raises(pl.LbmError) as e:
        lat.set_streaming(pl.STREAMING_AB)
    assert e.value.code == 2
    with pytest.raises(pl.LbmError) as e:
        lat.ade_enable(0.01)
    assert e.value.code == 2
    with pytest.raises(pl.LbmError) as e:
        lat.adjoint_forward(np.zeros((3, lat.Z, lat.Y, lat.X)), 4, np.zeros(0, np.int64), np.zeros((0, 3)))
    assert e.value.code == 2
    lat.set_kernel(pl.KERNEL_PAIR)  # accepted; FP64 arithmetic runs the one-site kernel
    lat.autotune(2)
    assert lat.kernel == pl.KERNEL_DIRECT  # FP64: no two-site candidate
    lat.step(4, sums=True)
    assert np.isfinite(lat.sums()).all()
    lat.close()


@pytest.mark.parametrize("storage", ["F32", "F32S", "F16S", "BF16SR", "I16S"])
@pytest.mark.parametrize("periodic", [False, True])
def test_srt_plugin_on_the_two_site_kernel_equals_builtin_srt(pl, storage, periodic):
    st = getattr(pl, "STORE_" + storage)
    out = []
    for coll in (pl.COLL_SRT, SRT_ID):
        lat = make(pl, coll, st, periodic, force=(1e-5, 0.0, 2e-6))
        lat.set_kernel(pl.KERNEL_PAIR)
        lat.step(21)
        lat.step(1, macro=True, sums=True)
        m = lat.macro()
        lat.step(1, sums=True)  # sums only: the GEO_NOTHING sites enter in the finish kernel
        out.append((lat.get_populations(), m, lat.sums()))
        lat.close()
    (f0, m0, s0), (f1, m1, s1) = out
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(m1, m0)
    np.testing.assert_array_equal(s1, s0)


def test_plugin_sums_on_the_two_site_kernel_match_the_one_site_kernel(pl):
    sums = []
    for kernel in (pl.KERNEL_DIRECT, pl.KERNEL_PAIR):
        lat = make(pl, TRT_ID, pl.STORE_F32, False, shape=(40, 14, 12))
        lat.set_kernel(kernel)
        lat.step(9, sums=True)
        sums.append(lat.sums())
        lat.close()
    # FP32 rounding of the two kernels differs (fused multiply-adds); the mass
    # also checks the GEO_NOTHING sites added by the finish kernel (about 7 %
    # of this lattice's sites)
    np.testing.assert_allclose(sums[1][:5], sums[0][:5], rtol=1e-6, atol=1e-6 * sums[0][0])
    assert sums[0][5] == sums[1][5] == 0


def test_streaming_plugin_on_the_two_site_kernel(pl):
    X, Y, Z = 14, 10, 8
    lat = pl.LBM(X, Y, Z, viscosity=0.02, collision=STREAM_ID, storage=pl.STORE_F32, periodic=True)
    lat.set_kernel(pl.KERNEL_PAIR)
    f0 = (np.random.default_rng(12).random((27, Z, Y, X)) + 0.5).astype(np.float32)
    lat.set_populations(f0, layout=pl.LAYOUT_INTERIOR)
    lat.step(4)
    f = lat.get_populations(layout=pl.LAYOUT_INTERIOR, dtype=np.float32)
    for q in range(27):
        np.testing.assert_array_equal(f[q], np.roll(f0[q], shift=(4 * CZ[q], 4 * CY[q], 4 * CX[q]), axis=(0, 1, 2)))
    lat.close()


def test_trt_plugin_on_the_two_site_kernel_matches_numpy(pl):
    X, Y, Z = 12, 10, 8
    nu = 0.01
    rng = np.random.default_rng(3)
    lat = pl.LBM(X, Y, Z, viscosity=nu, collision=TRT_ID, equilibrium=pl.EQ_SECOND_ORDER, storage=pl.STORE_F32,
                 periodic=True)
    lat.set_kernel(pl.KERNEL_PAIR)
    rho = 1 + 0.01 * rng.standard_normal((Z, Y, X))
    u = 0.04 * rng.standard_normal((3, Z, Y, X))
    lat.init_equilibrium(rho, *u)
    f0 = lat.get_populations(layout=pl.LAYOUT_INTERIOR)
    lat.set_populations(f0 * (1 + 0.02 * rng.standard_normal(f0.shape)), layout=pl.LAYOUT_INTERIOR)
    f0 = lat.get_populations(layout=pl.LAYOUT_INTERIOR)
    lat.step(4)
    f = lat.get_populations(layout=pl.LAYOUT_INTERIOR)
    want = f0
    for _ in range(4):
        want = stream(trt_collide(want, nu))
    assert np.max(np.abs(f - want)) / np.max(np.abs(want)) <= 2e-6
    lat.close()


def test_unregistering_keeps_live_lattices(pl, tmp_path):
    path = pl.plugin_path("example_collisions")
    cid = 30
    pl.register_collision(cid, path, "lbm_example_trt")
    lat = make(pl, cid, pl.STORE_F64, True)
    pl.unregister_collision(cid)
    lat.step(4, sums=True)
    s = lat.sums()
    ck = str(tmp_path / "plugin.ckpt")
    lat.save_checkpoint(ck)
    f = lat.get_populations()
    with pytest.raises(pl.LbmError):
        make(pl, cid, pl.STORE_F64, True)
    pl.register_collision(cid, path, "lbm_example_trt")
    other = make(pl, cid, pl.STORE_F64, True)
    other.load_checkpoint(ck)
    np.testing.assert_array_equal(other.get_populations(), f)
    lat.step(2, sums=True)
    other.step(2, sums=True)
    np.testing.assert_array_equal(other.sums(), lat.sums())
    assert s[0] > 0
    lat.close()
    other.close()
    pl.unregister_collision(cid)
