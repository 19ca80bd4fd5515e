"""A lattice split along z into slabs, one lattice handle per slab.

The reference runs one lattice over MPI ranks and synchronises the subdomain
overlaps after every step (include/lbm3d/lattice_decomposition.h:16-55,
include/lbm3d/lbm.hpp:189-273).  Here each slab is an ``LBM`` handle marked
distributed along z (``lbm_set_distributed_z``), and the A-A pattern needs an
exchange only around odd steps: before the step every interface fills the
ghost planes with the nine slots that cross it, after the step it moves the
populations that left each slab into the neighbour's boundary plane
(``lbm_halo_*`` in include/tnl_lbm_b200.h).  Even steps are local.

``SlabLattice`` drives all slabs from one process: ``lbm_halo_copy`` moves the
planes with one kernel on the receiver's device (peer loads over NVLink when
the slabs sit on different GPUs).  ``exchange_plan`` lists the copies of one
phase; ``DistributedSlab`` runs one slab per process and carries the same
plan over torch.distributed point-to-point operations (NCCL on GPUs, or gloo
with the planes staged through host memory).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi

PRE, POST = 0, 1  # exchange phases around an odd step


def split_z(Z: int, nslabs: int):
    """(z0, Zs) of each slab: the first Z % nslabs slabs take one layer more."""
    if not 1 <= nslabs <= Z:
        raise ValueError("need 1 <= nslabs <= Z")
    base, extra = divmod(Z, nslabs)
    out, z0 = [], 0
    for s in range(nslabs):
        zs = base + (1 if s < extra else 0)
        out.append((z0, zs))
        z0 += zs
    return out


def interfaces(nslabs: int, periodic_z: bool):
    """(lower, upper) slab pairs that share a z face."""
    pairs = [(s, s + 1) for s in range(nslabs - 1)]
    if periodic_z:
        pairs.append((nslabs - 1, 0))  # a single periodic slab faces itself
    return pairs


def exchange_plan(sizes, periodic_z: bool, phase: int):
    """Copies of one phase as (dst slab, dst plane, src slab, src plane, c_z),
    planes in the ghost frame (-1 and Zs are the ghost planes)."""
    plan = []
    for lo, up in interfaces(len(sizes), periodic_z):
        zl = sizes[lo]
        if phase == PRE:
            plan.append((up, -1, lo, zl - 1, -1))
            plan.append((lo, zl, up, 0, +1))
        else:
            plan.append((lo, zl - 1, up, -1, -1))
            plan.append((up, 0, lo, zl, +1))
    return plan


class SlabLattice:
    """One lattice of X x Y x Z sites as ``nslabs`` z-slabs, driven from one
    process.  ``devices``: the device of each slab (all on device 0 by default).
    Keyword arguments are those of ``LBM``; ``periodic=True`` makes the whole
    lattice periodic (the last and first slabs share a face)."""

    def __init__(self, X, Y, Z, nslabs, *, devices=None, periodic=False, periodic_z=None, **kw):
        from . import LBM
        self.X, self.Y, self.Z = int(X), int(Y), int(Z)
        self.layout = split_z(self.Z, int(nslabs))
        self.periodic_z = bool(periodic if periodic_z is None else periodic_z)
        devices = devices or [0] * len(self.layout)
        self.slabs = []
        for (z0, zs), dev in zip(self.layout, devices):
            lat = LBM(self.X, self.Y, zs, periodic=periodic, device=dev, use_graphs=False, **kw)
            _abi.check(lat.lib.lbm_set_distributed_z(lat.h, 1))
            self.slabs.append(lat)
        self.lib = self.slabs[0].lib
        self.sizes = [zs for _, zs in self.layout]
        self._plans = {ph: exchange_plan(self.sizes, self.periodic_z, ph) for ph in (PRE, POST)}

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def set_kernel(self, kernel):
        """Step kernel of every slab (lbm_set_kernel)."""
        for lat in self.slabs:
            lat.set_kernel(kernel)

    # -- distribution of global arrays ------------------------------------
    def _zslices(self, arr, axis, ghost):
        """Per-slab views of a global array along its z axis (ghost: the array
        carries the ghost planes, so each slab takes its own plus one on each side)."""
        out = []
        for z0, zs in self.layout:
            sl = [slice(None)] * arr.ndim
            sl[axis] = slice(z0, z0 + zs + 2) if ghost else slice(z0, z0 + zs)
            out.append(np.ascontiguousarray(arr[tuple(sl)]))
        return out

    def set_map(self, geo_map):
        for lat, m in zip(self.slabs, self._zslices(np.asarray(geo_map, np.uint8), 0, False)):
            lat.set_map(m)

    def set_inflow(self, vx=None, vy=None, vz=None):
        parts = [None if a is None else self._zslices(np.asarray(a, np.float64), 0, False) for a in (vx, vy, vz)]
        for i, lat in enumerate(self.slabs):
            lat.set_inflow(*[None if p is None else p[i] for p in parts])

    def set_populations(self, f):
        """Global populations [27, Z+2, Y+2, X+2] (ghost layer included)."""
        for lat, part in zip(self.slabs, self._zslices(np.asarray(f), 1, True)):
            lat.set_populations(part)

    def get_populations(self, dtype=np.float64):
        parts = [lat.get_populations(dtype=dtype) for lat in self.slabs]
        out = np.empty((27, self.Z + 2, self.Y + 2, self.X + 2), dtype)
        for (z0, zs), p in zip(self.layout, parts):
            out[:, z0 + 1:z0 + zs + 1] = p[:, 1:zs + 1]
        out[:, 0] = parts[0][:, 0]
        out[:, -1] = parts[-1][:, -1]
        return out

    def macro(self):
        return np.concatenate([lat.macro() for lat in self.slabs], axis=1)

    def sums(self):
        return np.sum([lat.sums() for lat in self.slabs], axis=0)

    @property
    def iteration(self):
        return self.slabs[0].iteration

    @iteration.setter
    def iteration(self, it):
        for lat in self.slabs:
            lat.iteration = it

    # -- stepping ------------------------------------------------------------
    def exchange(self, phase):
        for dst, dz, src, sz, cz in self._plans[phase]:
            _abi.check(self.lib.lbm_halo_copy(self.slabs[dst].h, dz, self.slabs[src].h, sz, cz))

    def step(self, nsteps=1, macro=False, sums=False):
        for i in range(int(nsteps)):
            last = i == nsteps - 1
            odd = self.iteration % 2 == 1
            if odd:
                self.exchange(PRE)
            for lat in self.slabs:
                lat.step(1, macro=macro and last, sums=sums and last)
            if odd:
                self.exchange(POST)

    def synchronize(self):
        for lat in self.slabs:
            lat.synchronize()


class DistributedSlab:
    """One slab per process of a torch.distributed group (rank r owns slab r):
    the plan of ``exchange_plan`` carried by point-to-point sends and receives
    of staged planes.  ``lattice`` is this rank's slab (an ``LBM``, or any
    object with the same halo methods); ``sizes`` the z extent of every
    rank's slab.

    ``staging`` picks the transport buffers: ``"device"`` sends the staged
    device buffers themselves (NCCL between GPUs), ``"host"`` copies them
    through host memory first (gloo, or any backend without device tensors).
    A lattice whose halo buffers already live in host memory is sent as is."""

    def __init__(self, lattice, sizes, periodic_z, group=None, staging="device"):
        import torch
        if staging not in ("device", "host"):
            raise ValueError("staging must be 'device' or 'host'")
        self.lat = lattice
        self.sizes = list(sizes)
        self.periodic_z = bool(periodic_z)
        self.group = group
        self.staging = staging
        self.rank = torch.distributed.get_rank(group)
        if len(self.sizes) != torch.distributed.get_world_size(group):
            raise ValueError("one slab size per rank")
        lattice.set_distributed_z(True)
        self._plans = {ph: exchange_plan(self.sizes, self.periodic_z, ph) for ph in (PRE, POST)}
        # one staging buffer per copy of a phase this rank sends or receives
        # (keys (phase, k): k the copy's position in the plan), plus its host
        # mirror when staging through host memory
        self._bufs, self._host = {}, {}
        for ph in (PRE, POST):
            for k, (dst, _, src, _, _) in enumerate(self._plans[ph]):
                if self.rank in (dst, src) and dst != src:
                    buf = lattice.halo_buffer()
                    self._bufs[(ph, k)] = buf
                    if staging == "host" and buf.is_cuda:
                        self._host[(ph, k)] = torch.empty(buf.numel(), dtype=buf.dtype, pin_memory=True)
        self.stream = None
        if any(b.is_cuda for b in self._bufs.values()) or hasattr(lattice, "device_view"):
            dev = torch.device("cuda", lattice.desc.device)
            self.stream = torch.cuda.ExternalStream(lattice.device_view().stream, device=dev)

    def _wire(self, key):
        """The tensor that travels for copy `key`."""
        return self._host.get(key, self._bufs[key])

    def exchange(self, phase):
        import contextlib

        import torch
        import torch.distributed as dist
        ctx = torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()
        ops, unpack = [], []
        with ctx:
            for k, (dst, dz, src, sz, cz) in enumerate(self._plans[phase]):
                if src == self.rank and dst == self.rank:
                    self.lat.halo_copy(dz, self.lat, sz, cz)  # a slab facing itself
                elif src == self.rank:
                    self.lat.halo_pack(sz, cz, self._bufs[(phase, k)])
                    if (phase, k) in self._host:
                        self._host[(phase, k)].copy_(self._bufs[(phase, k)], non_blocking=True)
                    ops.append(dist.P2POp(dist.isend, self._wire((phase, k)), dst, self.group))
                elif dst == self.rank:
                    ops.append(dist.P2POp(dist.irecv, self._wire((phase, k)), src, self.group))
                    unpack.append((dz, cz, (phase, k)))
            if self._host and ops:
                self.stream.synchronize()  # staged planes in host memory before they are sent
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            for dz, cz, key in unpack:
                if key in self._host:
                    self._bufs[key].copy_(self._host[key], non_blocking=True)
                self.lat.halo_unpack(dz, cz, self._bufs[key])

    def step(self, nsteps=1, macro=False, sums=False):
        for i in range(int(nsteps)):
            last = i == nsteps - 1
            odd = self.lat.iteration % 2 == 1
            if odd:
                self.exchange(PRE)
            self.lat.step(1, macro=macro and last, sums=sums and last)
            if odd:
                self.exchange(POST)
