"""The reference's A-B pull scheme in the oracle harness (oracle/_ref/libref_ab_*).

Pinned by the exact relation between the two streaming patterns on a periodic
lattice: starting A-A from the streamed state S f0 (every direction shifted by
its velocity) gives, after an even number of steps, the streamed A-B result
S (A-B f0), bit for bit, since both run the same per-site operators in the
same evaluation order.
"""
import numpy as np
import pytest

import oracle
from helpers import GEO, tgv_fields


def stream(f):
    """S: f_q(x) <- f_q(x - c_q) on the interior of a periodic lattice."""
    from oracle.adjoint import CX, CY, CZ
    g = f.copy()
    for q in range(27):
        g[q, 1:-1, 1:-1, 1:-1] = np.roll(f[q, 1:-1, 1:-1, 1:-1], shift=(CZ[q], CY[q], CX[q]), axis=(0, 1, 2))
    return g


@pytest.mark.parametrize("coll,flags,eq", [("CUM", 3, "INV_CUM"), ("CUM", 0, "INV_CUM"), ("SRT", 0, "EQ"), ("MRT", 0, "EQ")])
def test_ab_and_aa_agree_bitwise_on_a_periodic_lattice(coll, flags, eq):
    if not (oracle.reference_available(flags) and oracle.reference_ab_available(flags)):
        pytest.skip("reference harness not built")
    aa, ab = oracle.Reference(flags), oracle.ReferenceAB(flags)
    X, Y, Z = 12, 10, 8
    f0 = aa.allocate(X, Y, Z)
    aa.init_equilibrium(f0, X, Y, Z, eq=eq, fields=tgv_fields(X, Y, Z, u0=0.05))
    f0 *= 1 + 0.01 * np.random.default_rng(1).standard_normal(f0.shape)
    m = np.full((Z, Y, X), GEO["PERIODIC"], np.int16)
    f_ab = np.ascontiguousarray(f0.copy())
    ab.ab_run(f_ab, m, coll=coll, eq=eq, nu=0.01, nsteps=6)
    f_aa = np.ascontiguousarray(stream(f0))
    aa.aa_run(f_aa, m, coll=coll, eq=eq, nu=0.01, nsteps=6)
    inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    assert np.array_equal(f_aa[inner], stream(f_ab)[inner])
