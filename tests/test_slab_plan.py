"""Host logic of the z-slab decomposition (pytnl_lbm.slabs) on CPU.

The exchange plan is applied to numpy slabs with the semantics of
lbm_halo_copy (the nine slots whose c_z matches, whole planes); after the
pre-step phase every slab's ghost planes must hold the slots that the
neighbouring slab (or, across the periodic face, the far end of the lattice)
holds at those global positions, and the post-step phase must move the slots
written into a ghost plane back to the slab that owns them.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tnl-lbm_b200"))

from pytnl_lbm.slabs import POST, PRE, exchange_plan, interfaces, split_z  # noqa: E402

CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])


def apply(plan, slabs):
    for dst, dz, src, sz, cz in plan:
        q = np.where(CZ == cz)[0]
        slabs[dst][q, dz + 1] = slabs[src][q, sz + 1]


@pytest.mark.parametrize("Z,n", [(21, 3), (8, 2), (5, 5), (7, 1)])
def test_split_covers_the_lattice(Z, n):
    parts = split_z(Z, n)
    assert sum(zs for _, zs in parts) == Z
    assert [z0 for z0, _ in parts] == list(np.cumsum([0] + [zs for _, zs in parts])[:-1])
    assert max(zs for _, zs in parts) - min(zs for _, zs in parts) <= 1


def test_interfaces():
    assert interfaces(3, False) == [(0, 1), (1, 2)]
    assert interfaces(3, True) == [(0, 1), (1, 2), (2, 0)]
    assert interfaces(1, True) == [(0, 0)]
    assert interfaces(1, False) == []


@pytest.mark.parametrize("Z,n,periodic", [(12, 3, True), (12, 3, False), (9, 2, True), (6, 1, True)])
def test_pre_phase_fills_ghosts_with_the_neighbours_slots(Z, n, periodic):
    rng = np.random.default_rng(Z + n)
    g = rng.random((27, Z))  # one value per slot and global plane
    parts = split_z(Z, n)
    slabs = [np.full((27, zs + 2), np.nan) for _, zs in parts]
    for s, (z0, zs) in enumerate(parts):
        slabs[s][:, 1:zs + 1] = g[:, z0:z0 + zs]
    apply(exchange_plan([zs for _, zs in parts], periodic, PRE), slabs)
    down, up = CZ == -1, CZ == 1
    for s, (z0, zs) in enumerate(parts):
        below, above = z0 - 1, z0 + zs
        if below >= 0 or periodic:
            np.testing.assert_array_equal(slabs[s][down, 0], g[down, below % Z])
        else:
            assert np.all(np.isnan(slabs[s][:, 0]))
        if above < Z or periodic:
            np.testing.assert_array_equal(slabs[s][up, zs + 1], g[up, above % Z])
        # only the crossing slots are touched
        assert np.all(np.isnan(slabs[s][~down, 0])) and np.all(np.isnan(slabs[s][~up, zs + 1]))


@pytest.mark.parametrize("Z,n,periodic", [(12, 3, True), (12, 4, False), (6, 1, True)])
def test_post_phase_returns_the_outgoing_populations(Z, n, periodic):
    parts = split_z(Z, n)
    slabs = [np.zeros((27, zs + 2)) for _, zs in parts]
    # a site at a face writes the slots that leave the slab into its ghost plane
    for s, (z0, zs) in enumerate(parts):
        slabs[s][CZ == -1, 0] = 1000 + s
        slabs[s][CZ == +1, zs + 1] = 2000 + s
    apply(exchange_plan([zs for _, zs in parts], periodic, POST), slabs)
    for s, (z0, zs) in enumerate(parts):
        up_nb = (s + 1) % n if (s + 1 < n or periodic) else None
        dn_nb = (s - 1) % n if (s > 0 or periodic) else None
        if up_nb is not None:
            assert np.all(slabs[s][CZ == -1, zs] == 1000 + up_nb)
        if dn_nb is not None:
            assert np.all(slabs[s][CZ == +1, 1] == 2000 + dn_nb)
