"""The device Newton loop of a quench time step (ovs_quench_newton,
solmultiphasethermofluid_stag src/solveFlow.f90:4-164) against the same
sequence driven from the host through the public calls: assemble, GMRES
cycle, Newton update, residual norms and the convergence test.  Both run
the same kernels in the same order, so the fields agree exactly.  The mixed
mode is checked to reduce the residuals and to converge."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context

pytestmark = pytest.mark.gpu

FIELDS = ("ug", "acg", "pg", "phig", "rphig", "tg", "rtg")


def _host_loop(ctx, newton_max, tol, kspace, utol, atol):
    def vec_all():
        ctx.assemble(F.OVS_ASM_NSVOF, F.OVS_TENSOR_VEC, F.OVS_FP64)
        ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_VEC, F.OVS_FP64)
        return ctx.residual_norms(F.OVS_FP64)
    r0 = vec_all()
    its = 0
    for it in range(1, newton_max + 1):
        for kernel, sysid, nf in ((F.OVS_ASM_NSVOF, F.OVS_SYS_NSVOF, 5), (F.OVS_ASM_TEM, F.OVS_SYS_TEM, 1)):
            ctx.assemble(kernel, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
            ctx.gmres(sysid, tol, kspace, 1, np.zeros((ctx.N, nf)))
            ctx.newton_update(sysid)
        r = vec_all()
        its = it
        if all((r[k] < utol[k] * r0[k]) or (r[k] < atol[k]) for k in range(4)):
            break
    return r0, r, its


def test_device_newton_matches_host_sequence():
    case = M.quench_case(M.box_tet(8, 8, 10, 1.0, 1.0, 1.25), "newton8")
    utol, atol = (1e-4,) * 4, (1e-30,) * 4
    a = Context.from_case(case)
    info = a.quench_newton(F.OVS_FP64, newton_max=3, kspace=50, tol_ns=1e-6, tol_tem=1e-6, utol=utol, atol=atol)
    b = Context.from_case(case)
    r0, r, its = _host_loop(b, 3, 1e-6, 50, utol, atol)
    assert info.iterations == its
    np.testing.assert_array_equal(np.array(info.residual0), r0)
    np.testing.assert_array_equal(np.array(info.residual), r)
    for f in FIELDS:
        np.testing.assert_array_equal(a.get_field(f), b.get_field(f))
    assert info.residual[0] < info.residual0[0] and info.residual[3] <= info.residual0[3]
    a.close()
    b.close()


def test_device_newton_mixed_mode_converges():
    case = M.quench_case(M.box_tet(8, 8, 10, 1.0, 1.0, 1.25), "newton8m")
    ctx = Context.from_case(case)
    info = ctx.quench_newton(F.OVS_FP32, newton_max=4, kspace=50, max_cycles=100, tol_ns=1e-8, tol_tem=1e-8,
                             utol=(1e-6,) * 4, atol=(1e-30,) * 4)
    assert info.iterations >= 1 and info.krylov_iterations_ns > 0
    assert info.residual[0] < 1e-3 * info.residual0[0], (list(info.residual), list(info.residual0))
    ctx.close()


def test_device_time_steps_match_host_driver():
    """ovs_quench_time_steps (driver.f90:70-100 around the Newton loop) against
    the host doing the predictor, quench_newton and the old-value copies."""
    case = M.quench_case(M.box_tet(6, 6, 8, 1.0, 1.0, 1.25), "steps6")
    kw = dict(mode=F.OVS_FP64, newton_max=2, kspace=40, tol_ns=1e-6, tol_tem=1e-6, utol=(1e-4,) * 4,
              atol=(1e-30,) * 4)
    a = Context.from_case(case)
    info, kt = a.quench_time_steps(0, 3, **kw)
    b = Context.from_case(case)
    g = case.params["gami"]
    for istep in range(3):
        b.set_field("ug", b.get_field("ugold"))
        b.set_field("acg", (g - 1.0) / g * b.get_field("acgold"))
        b.quench_newton(kw["mode"], 1 if istep <= 1 else kw["newton_max"], istep > 0, kw["kspace"], 1, 100,
                        kw["tol_ns"], kw["tol_tem"], kw["utol"], kw["atol"])
        for cur, old in (("ug", "ugold"), ("acg", "acgold"), ("dg", "dgold"), ("ugm", "ugmold"),
                         ("acgm", "acgmold")):
            b.set_field(old, b.get_field(cur))
    for f in FIELDS + ("ugold", "acgold", "phigold", "tgold"):
        np.testing.assert_array_equal(a.get_field(f), b.get_field(f))
    assert kt > 0
    a.close()
    b.close()


def _stirred_case(name):
    """A quench box with a seeded random velocity off the walls, so every
    Newton iteration has convective and stabilisation work to do."""
    case = M.quench_case(M.box_tet(6, 6, 8, 1.0, 1.0, 1.25), name)
    rng = np.random.default_rng(3)
    free = np.asarray(case.ibc)[:, 0] == 0
    for f in ("ug", "ugold"):
        case.state[f][free] = 0.05 * rng.standard_normal((int(free.sum()), 3))
    return case


NEWTON = dict(newton_max=3, solve_tem=True, kspace=150, kspace_min=1, tol_ns=1e-8, tol_tem=1e-8,
              utol=(1e-6,) * 4, atol=(1e-30,) * 4)


def _close(gpu, ref, tol, what):
    scale = max(np.abs(ref).max(), 1e-300)
    err = np.abs(np.asarray(gpu) - np.asarray(ref)).max()
    assert err <= tol * scale, f"{what}: {err:.3e} vs scale {scale:.3e}"


def test_device_newton_matches_oracle(oracle):
    """ovs_quench_newton (FP64) against the oracle's Newton loop of
    solmultiphasethermofluid_stag: the same Newton and Krylov iteration
    counts, the same convergence verdict, every state field to 1e-10."""
    case = _stirred_case("newton_oracle")
    ctx = Context.from_case(case)
    info = ctx.quench_newton(F.OVS_FP64, **NEWTON)
    oc = oracle.OracleCase(case)
    ref = oc.quench_newton(NEWTON["newton_max"], True, NEWTON["kspace"], 1, NEWTON["tol_ns"], NEWTON["tol_tem"],
                           NEWTON["utol"], NEWTON["atol"])
    assert info.iterations == ref["iterations"] and bool(info.converged) == bool(ref["converged"])
    assert info.krylov_iterations_ns == ref["krylov_ns"] and info.krylov_iterations_tem == ref["krylov_tem"]
    for f in FIELDS:
        _close(ctx.get_field(f), oc.state_arrays[f], 1e-10, f)
    _close(np.array(info.residual0), ref["residual0"], 1e-10, "residual0")
    ctx.close()


def test_device_time_steps_match_oracle(oracle):
    """ovs_quench_time_steps over steps 0-2 (driver.f90:70-100: predictor,
    Newton loop with the istep rules, old values) against the oracle's
    driver loop: the last step's iteration counts and every state field and
    old value to 1e-10."""
    case = _stirred_case("steps_oracle")
    ctx = Context.from_case(case)
    info, _ = ctx.quench_time_steps(0, 3, mode=F.OVS_FP64, max_cycles=1, **NEWTON)
    oc = oracle.OracleCase(case)
    ref = oc.quench_time_steps(0, 3, NEWTON["newton_max"], True, NEWTON["kspace"], 1, NEWTON["tol_ns"],
                               NEWTON["tol_tem"], NEWTON["utol"], NEWTON["atol"])
    assert info.iterations == ref["iterations"]
    assert info.krylov_iterations_ns == ref["krylov_ns"] and info.krylov_iterations_tem == ref["krylov_tem"]
    for f in FIELDS + ("ugold", "acgold"):
        _close(ctx.get_field(f), oc.state_arrays[f], 1e-10, f)
    ctx.close()


def test_device_newton_mixed_follows_fp64():
    """The OVS_MIXED Newton loop (FP64 assembly and residuals, every solve by
    the mixed refinement to the FP64 systems) against the same loop driven
    from the host with restarted FP64 GMRES solves (ovs_solve OVS_FP64) to
    the same true relative residual: the same Newton iterations and, with
    both linear solves tight (1e-11), the same state within 1e-5."""
    case = _stirred_case("newton_mixed")
    tol, utol, atol = 1e-11, NEWTON["utol"], NEWTON["atol"]
    b = Context.from_case(case)
    imx = b.quench_newton(F.OVS_MIXED, newton_max=3, solve_tem=True, kspace=50, kspace_min=1, max_cycles=400,
                          tol_ns=tol, tol_tem=tol, utol=utol, atol=atol)
    a = Context.from_case(case)

    def vec_all():
        a.assemble(F.OVS_ASM_NSVOF, F.OVS_TENSOR_VEC, F.OVS_FP64)
        a.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_VEC, F.OVS_FP64)
        return a.residual_norms(F.OVS_FP64)
    r0 = vec_all()
    its = 0
    for it in range(1, 4):
        for kernel, sysid in ((F.OVS_ASM_NSVOF, F.OVS_SYS_NSVOF), (F.OVS_ASM_TEM, F.OVS_SYS_TEM)):
            a.assemble(kernel, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
            _, info = a.solve(sysid, F.OVS_FP64, tol, kspace=50, max_cycles=400, want_solution=False)
            assert info.converged
            a.newton_update(sysid)
        r = vec_all()
        its = it
        if all((r[k] < utol[k] * r0[k]) or (r[k] < atol[k]) for k in range(4)):
            break
    assert imx.iterations == its
    for f in FIELDS:
        _close(b.get_field(f), a.get_field(f), 1e-5, f)
    a.close()
    b.close()
