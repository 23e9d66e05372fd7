"""Adjoint of the quench residual: a torch.autograd.Function over the GPU
VJP, and the sensitivity of a wall heat-flux functional through a GMRES
solve with the transposed temperature matrix.

Nothing here has a counterpart in the reference (it has no adjoint).  The
residual is the pair of FP64 right-hand sides that ``ovs_assemble`` writes
for the NS+VOF pass (RHSGu, RHSGp, RHSGls: (N, 5)) and the temperature pass
(RHSGtem: (N,)), as a function of the nodal velocity ug, pressure pg, VOF
field phig, temperature Tg and node coordinates xg, all other state held
fixed.  Its vector-Jacobian product is the CUDA kernel behind
``ovs_residual_vjp``: the element's Gauss-point quantities are recomputed in
forward-mode dual arithmetic for each nodal input; nothing is stored by the
forward pass.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _ffi as F
from .api import Context

_INPUTS = (("ug", F.OVS_VJP_UG, 3), ("pg", F.OVS_VJP_PG, 1), ("phig", F.OVS_VJP_PHIG, 1),
           ("tg", F.OVS_VJP_TG, 1), ("xg", F.OVS_VJP_XG, 3))


def _set_inputs(ctx: Context, tensors) -> None:
    for (name, _, width), t in zip(_INPUTS, tensors):
        a = t.detach().to("cpu", torch.float64).numpy()
        ctx.set_field(name, a.reshape(ctx.N, width) if width == 3 else a.reshape(ctx.N))


def residuals(ctx: Context) -> tuple[np.ndarray, np.ndarray]:
    """FP64 RHS of the NS+VOF pass (N, 5) and of the temperature pass (N,)
    for the context's current state (vectors only, no matrix)."""
    ctx.assemble(F.OVS_ASM_NSVOF, F.OVS_TENSOR_VEC, F.OVS_FP64)
    r1 = ctx.get_rhs(F.OVS_SYS_NSVOF, F.OVS_FP64)
    ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_VEC, F.OVS_FP64)
    r2 = ctx.get_rhs(F.OVS_SYS_TEM, F.OVS_FP64)[:, 0]
    return r1, r2


class QuenchResidual(torch.autograd.Function):
    """(ug (N,3), pg (N,), phig (N,), tg (N,), xg (N,3)) -> (RHS NS+VOF (N,5),
    RHS T (N,)), FP64, evaluated on the GPU context `ctx` (its other fields,
    parameters and IBC are held fixed).  Backward calls the GPU VJP with the
    forward inputs set again, so the context may be used in between."""

    @staticmethod
    def forward(fctx, ctx: Context, ug, pg, phig, tg, xg):
        _set_inputs(ctx, (ug, pg, phig, tg, xg))
        r1, r2 = residuals(ctx)
        fctx.ctx = ctx
        fctx.save_for_backward(ug, pg, phig, tg, xg)
        return torch.from_numpy(np.ascontiguousarray(r1)), torch.from_numpy(np.ascontiguousarray(r2))

    @staticmethod
    def backward(fctx, g1, g2):
        ctx = fctx.ctx
        _set_inputs(ctx, fctx.saved_tensors)
        g = np.zeros((ctx.N, F.OVS_VJP_COUNT))
        if g1 is not None:
            g += ctx.residual_vjp(F.OVS_ASM_NSVOF, g1.detach().to("cpu", torch.float64).numpy())
        if g2 is not None:
            g += ctx.residual_vjp(F.OVS_ASM_TEM, g2.detach().to("cpu", torch.float64).numpy())
        out = [None]
        for (name, col, width), t in zip(_INPUTS, fctx.saved_tensors):
            a = g[:, col:col + width] if width == 3 else g[:, col]
            out.append(torch.from_numpy(np.ascontiguousarray(a)).to(t.device, t.dtype).reshape(t.shape))
        return tuple(out)


def quench_residual(ctx: Context, ug, pg, phig, tg, xg):
    return QuenchResidual.apply(ctx, ug, pg, phig, tg, xg)


def heat_flux_after_step(ctx: Context, c: np.ndarray, tol: float = 1e-14, kspace: int = 200) -> float:
    """J = c . T_new with T_new = Tg + gami delt dT and A dT = RHS_T: the
    functional after one Newton update of the temperature pass (A and RHS
    assembled in FP64 for the current state, GMRES to `tol`)."""
    ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    dT, info = ctx.gmres(F.OVS_SYS_TEM, tol, kspace, 1, np.zeros((ctx.N, 1)))
    p = ctx.params
    tg = ctx.get_field("tg")
    return float(c @ (tg + p["gami"] * p["delt"] * dT[:, 0]))


def heat_flux_sensitivity(ctx: Context, c: np.ndarray, tol: float = 1e-14, kspace: int = 200):
    """dJ/dTg and dJ/drTg of J = heat_flux_after_step(ctx, c) by the adjoint:
    lambda = A^-T (gami delt c) from GMRES on the transposed temperature
    matrix, then dJ/dq = c dTg/dq + (dRHS_T/dq)^T lambda from the residual VJP.
    The temperature matrix does not depend on Tg or rTg (no phase change,
    no temperature discontinuity capturing in the quench configurations), so
    these two are exact.  Returns (dJ/dTg, dJ/drTg, lambda, gmres info)."""
    ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    p = ctx.params
    lam, info = ctx.gmres_transposed(F.OVS_SYS_TEM, p["gami"] * p["delt"] * c, tol, kspace)
    g = ctx.residual_vjp(F.OVS_ASM_TEM, lam)
    return c + g[:, F.OVS_VJP_TG], g[:, F.OVS_VJP_RTG], lam, info


def lhs_transpose_times(ctx: Context, v: np.ndarray) -> np.ndarray:
    """A^T v for the assembled FP64 NS+VOF block matrix (host arithmetic on
    the reference block arrays; v and the result (N, 5): u1 u2 u3 p phi).
    Blocks per slot (row node a, column node b): K(i,j) row u_i col u_j,
    G(i) row u_i col p, ULS(i) row u_i col phi, D(j) row p col u_j, M p-p,
    PLS row p col phi, LSU(j) row phi col u_j, LS phi-phi."""
    s = ctx.get_system(F.OVS_SYS_NSVOF, F.OVS_FP64)
    col, row = ctx.get_pattern()
    a = np.repeat(np.arange(ctx.N), np.diff(col))
    b = row - 1
    K = s["K11"].reshape(-1, 3, 3)          # [slot, i, j]: row comp i, col comp j
    y = np.zeros((ctx.N, 5))
    va = v[a]
    for j in range(3):
        np.add.at(y[:, j], b, np.einsum("ki,ki->k", K[:, :, j], va[:, 0:3]) + s["D1"][:, j] * va[:, 3]
                  + s["LSU"][:, j] * va[:, 4])
    np.add.at(y[:, 3], b, np.einsum("ki,ki->k", s["G"], va[:, 0:3]) + s["M"] * va[:, 3])
    np.add.at(y[:, 4], b, np.einsum("ki,ki->k", s["ULS"], va[:, 0:3]) + s["PLS"] * va[:, 3] + s["LS"] * va[:, 4])
    return y


def newton_jacobian_transpose_times(ctx: Context, v: np.ndarray) -> np.ndarray:
    """J^T v with J = -d RHS_NSVOF / d(Newton increment): acg += du,
    ug += gami delt du; pg += alfi gami delt dp; rphig += dphi,
    phig += gami delt dphi (src/solveFlow.f90:99-104) -- the matrix the
    assembled LHS stands for, from the VJP."""
    p = ctx.params
    g = ctx.residual_vjp(F.OVS_ASM_NSVOF, v)
    gd = p["gami"] * p["delt"]
    y = np.zeros((ctx.N, 5))
    y[:, 0:3] = g[:, F.OVS_VJP_ACG:F.OVS_VJP_ACG + 3] + gd * g[:, F.OVS_VJP_UG:F.OVS_VJP_UG + 3]
    y[:, 3] = p["alfi"] * gd * g[:, F.OVS_VJP_PG]
    y[:, 4] = g[:, F.OVS_VJP_RPHIG] + gd * g[:, F.OVS_VJP_PHIG]
    return -y
