"""DistributedSlab (pytnl_lbm.slabs) across processes, on CPU with gloo.

One lattice split along z runs as one slab per process; around every odd A-A
step the slabs exchange the nine slot planes that cross each z face, as
staged buffers sent and received point to point.  These tests run that
transport with 2 and 3 gloo ranks on the host.  Each rank's slab is a numpy
lattice with the A-A semantics of the kernels (streaming_AA.h: the even step
writes the opposite slot of its own site, the odd step reads the opposite
slots of its neighbours and writes its neighbours) and the halo semantics of
lbm_halo_pack / lbm_halo_unpack / lbm_halo_copy (whole (y, x) planes of the
nine slots whose c_z matches).  After a run, every slab must equal, bit for
bit, its part of the same lattice stepped whole in one process.  A mistake in
the exchange order, the buffer bookkeeping or the self-copy of a single
periodic slab would corrupt the ghost planes and show up here.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])
OPP = np.array([0] + [q + 1 if q % 2 else q - 1 for q in range(1, 27)])
W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)


class NumpySlab:
    """A periodic (x, y) lattice of X x Y x Zs sites with a one-site ghost
    layer, stepped by the A-A pattern with a BGK-like relaxation as the
    collision.  z neighbours wrap inside the slab unless it is distributed
    along z, in which case they are the ghost planes."""

    def __init__(self, X, Y, Zs, f):
        self.X, self.Y, self.Zs = X, Y, Zs
        self.f = np.array(f, dtype=np.float64)
        assert self.f.shape == (27, Zs + 2, Y + 2, X + 2)
        self.iteration = 0
        self.distributed = False
        z, y, x = np.meshgrid(np.arange(Zs), np.arange(Y), np.arange(X), indexing="ij")
        self.site = (z, y, x)

    # -- the halo methods DistributedSlab calls ---------------------------
    def set_distributed_z(self, flag):
        self.distributed = bool(flag)

    def halo_buffer(self):
        return torch.zeros(9 * (self.Y + 2) * (self.X + 2) * 8, dtype=torch.uint8)

    def _planes(self, buf):
        return buf.numpy().view(np.float64).reshape(9, self.Y + 2, self.X + 2)

    def halo_pack(self, z, cz, buf):
        self._planes(buf)[:] = self.f[CZ == cz, z + 1]

    def halo_unpack(self, z, cz, buf):
        self.f[CZ == cz, z + 1] = self._planes(buf)

    def halo_copy(self, z, src, src_z, cz):
        self.f[CZ == cz, z + 1] = src.f[CZ == cz, src_z + 1]

    # -- the A-A step -------------------------------------------------------
    def _at(self, q, dz, dy, dx):
        """Ghost-frame index of the site shifted by (dx, dy, dz) for slot q."""
        z, y, x = self.site
        zz = z + dz if self.distributed else (z + dz) % self.Zs
        return (q, zz + 1, (y + dy) % self.Y + 1, (x + dx) % self.X + 1)

    def step(self, nsteps=1, macro=False, sums=False):
        for _ in range(nsteps):
            odd = self.iteration % 2 == 1
            F = np.empty((27,) + self.site[0].shape)
            for i in range(27):
                F[i] = self.f[self._at(OPP[i], -CZ[i], -CY[i], -CX[i])] if odd else self.f[self._at(i, 0, 0, 0)]
            rho = F.sum(0)
            ux, uy, uz = ((c[:, None, None, None] * F).sum(0) / rho for c in (CX, CY, CZ))
            cu = CX[:, None, None, None] * ux + CY[:, None, None, None] * uy + CZ[:, None, None, None] * uz
            F += 0.35 * (W[:, None, None, None] * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (ux * ux + uy * uy + uz * uz)) - F)
            for i in range(27):
                if odd:
                    self.f[self._at(i, CZ[i], CY[i], CX[i])] = F[i]
                else:
                    self.f[self._at(OPP[i], 0, 0, 0)] = F[i]
            self.iteration += 1


def initial_state(X, Y, Z, seed):
    rng = np.random.default_rng(seed)
    return W[:, None, None, None] * (1 + 0.1 * rng.standard_normal((27, Z + 2, Y + 2, X + 2)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, X, Y, Z, periodic, nsteps, seed, out):
    import torch.distributed as dist

    from pytnl_lbm.slabs import DistributedSlab, split_z
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        layout = split_z(Z, world)
        z0, zs = layout[rank]
        f0 = initial_state(X, Y, Z, seed)
        slab = NumpySlab(X, Y, zs, f0[:, z0:z0 + zs + 2])
        ds = DistributedSlab(slab, [s for _, s in layout], periodic_z=periodic, staging="host")
        ds.step(nsteps)
        out.put((rank, z0, zs, slab.f.copy()))
    finally:
        dist.destroy_process_group()


def run_ranks(world, X, Y, Z, periodic, nsteps, seed):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, X, Y, Z, periodic, nsteps, seed, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("world,Z,periodic,nsteps", [(2, 8, True, 7), (2, 9, False, 6), (3, 10, True, 9)])
def test_distributed_slabs_equal_the_whole_lattice(world, Z, periodic, nsteps):
    X, Y = 6, 5
    seed = 100 + Z
    whole = NumpySlab(X, Y, Z, initial_state(X, Y, Z, seed))
    # a non-periodic z axis reaches the lattice's own ghost planes, as a slab
    # at the end of the split does
    whole.distributed = not periodic
    whole.step(nsteps)
    for rank, z0, zs, f in run_ranks(world, X, Y, Z, periodic, nsteps, seed):
        np.testing.assert_array_equal(f[:, 1:zs + 1], whole.f[:, z0 + 1:z0 + zs + 1], err_msg=f"slab {rank}")


def test_single_periodic_slab_faces_itself():
    """One rank, periodic along z: the exchange is the self-copy branch and
    must reproduce the wrapped lattice."""
    X, Y, Z = 5, 4, 6
    seed = 7
    whole = NumpySlab(X, Y, Z, initial_state(X, Y, Z, seed))
    whole.step(5)
    (_, z0, zs, f), = run_ranks(1, X, Y, Z, True, 5, seed)
    np.testing.assert_array_equal(f[:, 1:Z + 1], whole.f[:, 1:Z + 1])
