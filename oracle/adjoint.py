"""CPU restatement of the per-site transpose of the SRT update (test
infrastructure only).

The GPU discrete adjoint (tnl-lbm_b200/csrc/adjoint.cuh) applies, at every
site and step, the transpose of the Jacobian of the SRT collision with a body
force (col_srt.h:14-105, velocity with the half-force shift of common.h:17-50,
second-order equilibrium of eq.h:13-130):

    out_q = f_q + (feq_q - f_q) / tau + (1 - 1/(2 tau)) S_q feq_q,
    S_q = 3 (c_q - u).F / rho,  u = (sum c f + F/2) / rho.

``srt_vjp`` restates that transpose in numpy; the tests pin it to the
reference's own adjoint collision (D3Q27_SRT_ADJOINT, col_srt_adjoint.h:50-109,
which assumes rho = 1 and F = 0) and to finite differences of the reference's
SRT collision.
"""
from __future__ import annotations

import numpy as np

# direction vectors and weights in slot order (include/lbm3d/defs.h:318-350)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])
C = np.stack([CX, CY, CZ], axis=1).astype(np.float64)
NNZ = np.abs(C).sum(axis=1)
W = np.where(NNZ == 0, 8 / 27, np.where(NNZ == 1, 2 / 27, np.where(NNZ == 2, 1 / 54, 1 / 216)))


def moments(f, F):
    rho = f.sum(axis=1)
    u = (f @ C + 0.5 * F) / rho[:, None]
    return rho, u


def feq(rho, u):
    cu = u @ C.T
    usq = (u * u).sum(axis=1)
    return W[None, :] * rho[:, None] * (1 - 1.5 * usq[:, None] + 3 * cu + 4.5 * cu * cu)


def srt_collide(f, F, nu):
    """The forward update out(f, F) for f[n, 27], F[n, 3]."""
    tau = 3 * nu + 0.5
    rho, u = moments(f, F)
    fe = feq(rho, u)
    S = 3 * ((C[None, :, :] - u[:, None, :]) * F[:, None, :]).sum(axis=2) / rho[:, None]
    return f + (fe - f) / tau + (1 - 0.5 / tau) * S * fe


def srt_vjp(f, F, nu, lam):
    """(d out / d f)^T lam and (d out / d F)^T lam at (f, F)."""
    tau = 3 * nu + 0.5
    it, k = 1 / tau, 1 - 0.5 / tau
    rho, u = moments(f, F)
    ir = 1 / rho
    fe = feq(rho, u)
    cmu = C[None, :, :] - u[:, None, :]                                      # c_q - u
    S = 3 * (cmu * F[:, None, :]).sum(axis=2) * ir[:, None]
    cu = u @ C.T
    dfeq = W[None, :, None] * rho[:, None, None] * (3 * C[None] * (1 + 3 * cu)[:, :, None] - 3 * u[:, None, :])
    lf = lam * fe
    A = it * lf.sum(axis=1) * ir
    B = (lam[:, :, None] * (it + k * S)[:, :, None] * dfeq).sum(axis=1) - 3 * k * lf.sum(axis=1)[:, None] * F * ir[:, None]
    g = (1 - it) * lam + A[:, None] + (cmu * B[:, None, :]).sum(axis=2) * ir[:, None]
    dF = B * (0.5 * ir)[:, None] + 3 * k * ir[:, None] * (lf[:, :, None] * cmu).sum(axis=1)
    return g, dF


def objective_gradient(f, F, target, w_rho):
    """J = 1/2 [w_rho (rho - rho*)^2 + |u - u*|^2] per site and its gradients
    with respect to f and F; target[n, 4] = (rho*, u*)."""
    rho, u = moments(f, F)
    dr = rho - target[:, 0]
    du = u - target[:, 1:4]
    J = 0.5 * (w_rho * dr * dr + (du * du).sum(axis=1))
    gf = w_rho * dr[:, None] + ((C[None, :, :] - u[:, None, :]) * du[:, None, :]).sum(axis=2) / rho[:, None]
    gF = du * (0.5 / rho)[:, None]
    return J, gf, gF
