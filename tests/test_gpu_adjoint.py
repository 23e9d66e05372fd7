"""Adjoint of the quench residual on the config-5 mesh (32^3 cells x6 tets).

* The VJP of the FP64 residual (NS+VOF and temperature RHS) with respect to
  nodal u, p, phi, T and coordinates against central finite differences
  along 20 seeded random directions, h = 1e-6 (inputs scaled to their field
  magnitudes): 1e-6 relative.
* The VJP against A^T v of the assembled temperature matrix: the
  temperature residual is linear in (T, dT/dt) for these physics and the
  matrix is its exact Jacobian with respect to the Newton increment
  (rTg += d, Tg += gami delt d), so the two agree to rounding.
* torch.autograd.Function plumbing: a loss through QuenchResidual against
  the directional derivative from the same differences.
* GMRES on the transposed temperature matrix and the sensitivity of the
  bottom-wall heat flux after one temperature Newton step to Tg and rTg,
  against central differences of the functional (affine in Tg and rTg, so
  taken with h = 1e-2).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCALES = {"ug": 0.01, "pg": 1.0, "phig": 0.1, "tg": 300.0, "xg": 1.0 / 32}


@pytest.fixture(scope="module")
def setup():
    from oversetdevfort_b200 import mesh as M
    from oversetdevfort_b200.api import Context

    case = M.adjoint_case(32)
    ctx = Context.from_case(case)
    yield case, ctx
    ctx.close()


def _state(ctx):
    return {n: ctx.get_field(n).copy() for n in SCALES}


def _set(ctx, st):
    for n, a in st.items():
        ctx.set_field(n, a)


def _vjp_all(ctx, v1, v2):
    from oversetdevfort_b200 import _ffi as F
    return ctx.residual_vjp(F.OVS_ASM_NSVOF, v1) + ctx.residual_vjp(F.OVS_ASM_TEM, v2)


def _cols():
    from oversetdevfort_b200 import _ffi as F
    return {"ug": slice(F.OVS_VJP_UG, F.OVS_VJP_UG + 3), "pg": F.OVS_VJP_PG, "phig": F.OVS_VJP_PHIG,
            "tg": F.OVS_VJP_TG, "xg": slice(F.OVS_VJP_XG, F.OVS_VJP_XG + 3)}


def test_vjp_matches_central_differences(setup):
    from oversetdevfort_b200.adjoint import residuals

    case, ctx = setup
    N = ctx.N
    rng = np.random.default_rng(20)
    st0 = _state(ctx)
    v1 = rng.standard_normal((N, 5))
    v2 = rng.standard_normal(N)
    g = _vjp_all(ctx, v1, v2)
    cols = _cols()
    h = 1e-6
    worst = 0.0
    for k in range(20):
        w = {n: SCALES[n] * rng.standard_normal(a.shape) for n, a in st0.items()}
        vals = []
        for sgn in (1.0, -1.0):
            _set(ctx, {n: st0[n] + sgn * h * w[n] for n in st0})
            r1, r2 = residuals(ctx)
            vals.append(np.sum(v1 * r1) + np.sum(v2 * r2))
        _set(ctx, st0)
        fd = (vals[0] - vals[1]) / (2 * h)
        ad = sum(np.sum(g[:, cols[n]] * w[n]) for n in st0)
        rel = abs(fd - ad) / max(abs(ad), 1e-300)
        worst = max(worst, rel)
        assert rel <= 1e-6, (k, fd, ad, rel)
    print(f"VJP vs central differences, 20 directions: worst relative error {worst:.2e}")


def test_vjp_matches_transposed_temperature_matrix(setup):
    from oversetdevfort_b200 import _ffi as F

    case, ctx = setup
    N = ctx.N
    p = ctx.params
    rng = np.random.default_rng(21)
    v = rng.standard_normal(N)
    ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    col, row = ctx.get_pattern()
    vals = ctx.get_lhs(F.OVS_SYS_TEM, F.OVS_FP64, F.OVS_BLK_TEM)
    rows = np.repeat(np.arange(N), np.diff(col))
    atv = np.zeros(N)
    np.add.at(atv, row - 1, vals * v[rows])
    g = ctx.residual_vjp(F.OVS_ASM_TEM, v)
    jtv = -(g[:, F.OVS_VJP_RTG] + p["gami"] * p["delt"] * g[:, F.OVS_VJP_TG])
    err = np.abs(atv - jtv).max() / np.abs(atv).max()
    print(f"A^T v vs VJP (temperature): relative error {err:.2e}")
    assert err <= 1e-10, err


def test_autograd_function(setup):
    import torch
    from oversetdevfort_b200.adjoint import quench_residual, residuals

    case, ctx = setup
    N = ctx.N
    st0 = _state(ctx)
    rng = np.random.default_rng(22)
    W1 = torch.from_numpy(rng.standard_normal((N, 5)))
    W2 = torch.from_numpy(rng.standard_normal(N))
    inp = {n: torch.from_numpy(st0[n].copy()).requires_grad_(True) for n in ("ug", "pg", "phig", "tg", "xg")}
    r1, r2 = quench_residual(ctx, inp["ug"], inp["pg"], inp["phig"], inp["tg"], inp["xg"])
    loss = (r1 * W1).sum() + (r2 * W2).sum()
    loss.backward()
    for n in inp:
        assert inp[n].grad is not None and inp[n].grad.shape == inp[n].shape
    h = 1e-6
    for k in range(3):
        w = {n: SCALES[n] * rng.standard_normal(st0[n].shape) for n in st0}
        vals = []
        for sgn in (1.0, -1.0):
            _set(ctx, {n: st0[n] + sgn * h * w[n] for n in st0})
            a1, a2 = residuals(ctx)
            vals.append(np.sum(W1.numpy() * a1) + np.sum(W2.numpy() * a2))
        _set(ctx, st0)
        fd = (vals[0] - vals[1]) / (2 * h)
        ad = sum(float((inp[n].grad * torch.from_numpy(w[n])).sum()) for n in inp)
        assert abs(fd - ad) <= 1e-6 * abs(ad), (k, fd, ad)


def test_transposed_gmres_and_heat_flux_sensitivity(setup):
    from oversetdevfort_b200 import _ffi as F
    from oversetdevfort_b200 import mesh as M
    from oversetdevfort_b200.adjoint import heat_flux_after_step, heat_flux_sensitivity

    case, ctx = setup
    N = ctx.N
    rng = np.random.default_rng(23)
    # A^T x = b through the transposed copy
    ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    b = rng.standard_normal(N)
    x, info = ctx.gmres_transposed(F.OVS_SYS_TEM, b, 1e-13, 200)
    col, row = ctx.get_pattern()
    vals = ctx.get_lhs(F.OVS_SYS_TEM, F.OVS_FP64, F.OVS_BLK_TEM)
    rows = np.repeat(np.arange(N), np.diff(col))
    atx = np.zeros(N)
    np.add.at(atx, row - 1, vals * x[rows])
    assert np.linalg.norm(atx - b) <= 1e-10 * np.linalg.norm(b), info.iterations
    # dJ/dTg, dJ/drTg of the bottom-wall heat flux after one T Newton step
    c = M.bottom_heat_flux_weights(case)
    dJ_dT, dJ_drT, lam, info = heat_flux_sensitivity(ctx, c)
    assert info.converged
    t0 = ctx.get_field("tg").copy()
    r0 = ctx.get_field("rtg").copy()
    for name, base, grad, scale in (("tg", t0, dJ_dT, 300.0), ("rtg", r0, dJ_drT, 10.0)):
        for k in range(2):
            w = scale * rng.standard_normal(N)
            # J is affine in Tg and rTg, so the step has no truncation error;
            # a larger step keeps the forward solves' residual (~1e-13) from
            # dominating the difference
            h = 1e-2
            ctx.set_field(name, base + h * w)
            Jp = heat_flux_after_step(ctx, c)
            ctx.set_field(name, base - h * w)
            Jm = heat_flux_after_step(ctx, c)
            ctx.set_field(name, base)
            fd = (Jp - Jm) / (2 * h)
            ad = float(grad @ w)
            assert abs(fd - ad) <= 1e-6 * abs(ad), (name, k, fd, ad)
