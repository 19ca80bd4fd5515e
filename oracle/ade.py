"""Numpy restatement of the D3Q7 advection-diffusion operators (test
infrastructure only: the checker of the coupled scalar, never the product).

Follows TNL-LBM include/lbm3d/d3q7/: the equilibrium of eq.h:17-54
(c_s^2 = 1/4, w_0 = 1/4, w_q = 1/8), phi as the sum of the populations
(common.h:15-26) and the collisions of col_srt.h:12-25, col_mrt.h:12-49 and
col_clbm.h:14-83 with omega = 1 / (1/2 + 4 D) and unit higher-order rates.
Directions in slot order zzz, pzz, mzz, zpz, zmz, zzp, zzm (defs.h:318-327).
"""
import numpy as np

C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=np.float64)
W = np.array([0.25] + [0.125] * 6)


def feq(phi, v):
    """Equilibrium [n, 7] of phi [n] and velocity v [n, 3]."""
    phi = np.asarray(phi, np.float64)
    v = np.asarray(v, np.float64)
    cu = v @ C.T
    u2 = (v * v).sum(axis=1)
    return W[None, :] * phi[:, None] * (1.0 - 2.0 * u2[:, None] + 4.0 * cu + 8.0 * cu * cu)


def collide(g, v, D, coll="SRT"):
    """One collision of g [n, 7] (returned as a new array) with velocity v [n, 3]."""
    g = np.array(g, np.float64)
    v = np.asarray(v, np.float64)
    phi = g.sum(axis=1)
    omega = 1.0 / (0.5 + 4.0 * D)
    if coll == "SRT":
        return g + omega * (feq(phi, v) - g), phi
    vx, vy, vz = v[:, 0], v[:, 1], v[:, 2]
    m100 = phi * vx + g[:, 2] - g[:, 1]
    m010 = phi * vy + g[:, 4] - g[:, 3]
    m001 = phi * vz + g[:, 6] - g[:, 5]
    if coll == "MRT":
        m200 = phi * (vx * vx + 0.25) - g[:, 2] - g[:, 1]
        m020 = phi * (vy * vy + 0.25) - g[:, 4] - g[:, 3]
        m002 = phi * (vz * vz + 0.25) - g[:, 6] - g[:, 5]
    else:
        m200 = phi * (0.25 - vx * vx) + 2 * vx * (g[:, 1] - g[:, 2]) - g[:, 2] - g[:, 1]
        m020 = phi * (0.25 - vy * vy) + 2 * vy * (g[:, 3] - g[:, 4]) - g[:, 4] - g[:, 3]
        m002 = phi * (0.25 - vz * vz) + 2 * vz * (g[:, 5] - g[:, 6]) - g[:, 6] - g[:, 5]
    m100, m010, m001 = omega * m100, omega * m010, omega * m001
    out = g.copy()
    if coll == "MRT":
        out[:, 0] += -m200 - m020 - m002
        out[:, 1] += 0.5 * (m200 + m100)
        out[:, 2] += 0.5 * (m200 - m100)
        out[:, 3] += 0.5 * (m020 + m010)
        out[:, 4] += 0.5 * (m020 - m010)
        out[:, 5] += 0.5 * (m002 + m001)
        out[:, 6] += 0.5 * (m002 - m001)
    else:
        out[:, 0] += -2 * (m100 * vx + m010 * vy + m001 * vz) - m200 - m020 - m002
        out[:, 1] += m100 * vx + 0.5 * (m200 + m100)
        out[:, 2] += m100 * vx + 0.5 * (m200 - m100)
        out[:, 3] += m010 * vy + 0.5 * (m020 + m010)
        out[:, 4] += m010 * vy + 0.5 * (m020 - m010)
        out[:, 5] += m001 * vz + 0.5 * (m002 + m001)
        out[:, 6] += m001 * vz + 0.5 * (m002 - m001)
    return out, phi
