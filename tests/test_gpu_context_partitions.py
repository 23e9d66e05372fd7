"""GPU checks of the partitioned Newton loop on device contexts and of the
context calls it is built from: distributed.ContextPartition
(ovs_set_solution, ovs_predictor, ovs_commit_old) against
ovs_quench_newton / ovs_quench_time_steps on one context, FP64 and mixed;
ovs_set_solution + ovs_newton_update against the update of an ovs_gmres
solution; ovs_predictor / ovs_commit_old against host arithmetic;
ovs_assemble_async / ovs_assemble_wait against ovs_assemble; the C driver's
cavity mode (one config-1 Newton step through the C ABI from plain C)."""
import numpy as np
import pytest
import torch

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import distributed as D
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import partition as P
from oversetdevfort_b200.api import Context

pytestmark = pytest.mark.gpu
OPTS = dict(newton_max=3, solve_tem=True, kspace=150, kspace_min=1, tol_ns=1e-8, tol_tem=1e-8,
            utol=(1e-6,) * 4, atol=(1e-30,) * 4)


def _case():
    case = M.quench_case(M.box_tet(6, 6, 8, 1.0, 1.0, 1.25), "gnewton")
    rng = np.random.default_rng(3)
    free = np.asarray(case.ibc)[:, 0] == 0
    for f in ("ug", "ugold"):
        case.state[f][free] = 0.05 * rng.standard_normal((int(free.sum()), 3))
    return case


@pytest.mark.parametrize("steps", [0, 3])
def test_partitioned_newton_on_contexts(steps):
    case = _case()
    g = Context.from_case(case)
    if steps:
        info, _ = g.quench_time_steps(0, steps, mode=F.OVS_FP64, max_cycles=1, **OPTS)
    else:
        info = g.quench_newton(mode=F.OVS_FP64, max_cycles=1, **OPTS)
    ref = {n: g.get_field(n) for n in ("ug", "acg", "pg", "phig", "tg", "ugold")}
    g.close()
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ctxs = [Context.from_case(P.local_case(case, p)) for p in parts]
    sp = {r: D.ContextPartition(c, plan.owned[r], device="cuda:0") for r, c in enumerate(ctxs)}
    if steps:
        out, _ = D.quench_time_steps(D.LocalComm(plan), sp, 0, steps, **OPTS)
    else:
        out = D.quench_newton(D.LocalComm(plan), sp, **OPTS)
    assert out["iterations"] == info.iterations
    assert out["krylov_iterations_ns"] == info.krylov_iterations_ns
    assert out["krylov_iterations_tem"] == info.krylov_iterations_tem
    for n, a in ref.items():
        for c, p in zip(ctxs, parts):
            np.testing.assert_allclose(c.get_field(n), a[p.nodes], rtol=0, atol=1e-10 * max(np.abs(a).max(), 1e-300))
    for c in ctxs:
        c.close()


def test_set_solution_then_update_equals_gmres_then_update():
    case = _case()
    a = Context.from_case(case)
    b = Context.from_case(case)
    for c in (a, b):
        c.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
    sol, info = a.gmres(F.OVS_SYS_NSVOF, 1e-8, 100, 1, np.zeros((a.N, 5)))
    a.newton_update(F.OVS_SYS_NSVOF)
    b.set_solution(F.OVS_SYS_NSVOF, sol)                                  # host array
    b.newton_update(F.OVS_SYS_NSVOF)
    for n in ("ug", "acg", "pg", "phig", "rphig"):
        np.testing.assert_array_equal(a.get_field(n), b.get_field(n))
    d = torch.as_tensor(np.ascontiguousarray(np.zeros((a.N, 5)).T), device="cuda:0")
    b.set_solution(F.OVS_SYS_NSVOF, d)                                    # device tensor, zero update
    b.newton_update(F.OVS_SYS_NSVOF)
    np.testing.assert_array_equal(a.get_field("ug"), b.get_field("ug"))
    a.close(); b.close()


def test_predictor_and_commit_old():
    case = _case()
    c = Context.from_case(case)
    rng = np.random.default_rng(1)
    for n in ("ugold", "acgold", "ug", "acg", "dg", "ugm", "acgm", "phig", "tg"):
        c.set_field(n, rng.standard_normal(c.get_field(n).shape))
    g = case.params["gami"]
    ugold, acgold = c.get_field("ugold"), c.get_field("acgold")
    c.predictor()
    np.testing.assert_array_equal(c.get_field("ug"), ugold)
    np.testing.assert_allclose(c.get_field("acg"), (g - 1.0) / g * acgold, rtol=1e-15)
    phigold = c.get_field("phigold")
    c.commit_old(False)
    for cur, old in (("ug", "ugold"), ("acg", "acgold"), ("dg", "dgold"), ("ugm", "ugmold"), ("acgm", "acgmold")):
        np.testing.assert_array_equal(c.get_field(cur), c.get_field(old))
    np.testing.assert_array_equal(c.get_field("phigold"), phigold)        # untouched without the flag
    c.commit_old(True)
    np.testing.assert_array_equal(c.get_field("phig"), c.get_field("phigold"))
    c.close()


def test_c_driver_cavity(tmp_path):
    import shutil, subprocess
    from pathlib import Path
    from oversetdevfort_b200 import build
    root = Path(__file__).resolve().parent.parent
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    exe = tmp_path / "drv"
    libdir = build.LIB.parent
    subprocess.run(["gcc", "-std=c99", "-O1", "-I", str(root / "include"), str(root / "tests/c/ovs_abi_driver.c"),
                    "-o", str(exe), "-L", str(libdir), f"-l:{build.LIB.name}", f"-Wl,-rpath,{libdir}", "-lm"],
                   check=True)
    res = subprocess.run([str(exe), "cavity", "8"], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "cavity checks: 0 failure(s)" in res.stdout


def test_assemble_async_equals_sync():
    case = _case()
    a = Context.from_case(case)
    b = Context.from_case(case)
    c1 = a.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP32)
    c2 = a.assemble(F.OVS_ASM_TEM, 6, F.OVS_FP32)
    b.assemble_async(F.OVS_ASM_NSVOF, 6, F.OVS_FP32)
    b.assemble_async(F.OVS_ASM_TEM, 6, F.OVS_FP32)
    cfl = b.assemble_wait()
    assert cfl == max(c1, c2) and b.last_status == F.OVS_OK
    for sysid in (F.OVS_SYS_NSVOF, F.OVS_SYS_TEM):
        np.testing.assert_array_equal(a.get_rhs(sysid, F.OVS_FP32), b.get_rhs(sysid, F.OVS_FP32))
    assert b.assemble_wait() == 0.0          # nothing queued
    for _ in range(16):
        b.assemble_async(F.OVS_ASM_TEM, 2, F.OVS_FP32)
    assert b.lib.ovs_assemble_async(b.h, F.OVS_ASM_TEM, 2, F.OVS_FP32) == F.OVS_ERR_STATE
    b.assemble_wait()
    a.close(); b.close()


def test_partitioned_newton_mixed_on_contexts():
    case = _case()
    g = Context.from_case(case)
    info = g.quench_newton(mode=F.OVS_FP32, max_cycles=40, **OPTS)
    ref = {n: g.get_field(n) for n in ("ug", "pg", "phig", "tg")}
    g.close()
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ctxs = [Context.from_case(P.local_case(case, p)) for p in parts]
    sp = {r: D.ContextPartition(c, plan.owned[r], device="cuda:0") for r, c in enumerate(ctxs)}
    out = D.quench_newton(D.LocalComm(plan), sp, mode=F.OVS_FP32, max_cycles=40, **OPTS)
    assert out["converged"] and abs(out["iterations"] - info.iterations) <= 1
    for n, a in ref.items():
        for c, p in zip(ctxs, parts):
            np.testing.assert_allclose(c.get_field(n), a[p.nodes], rtol=0, atol=1e-6 * max(np.abs(a).max(), 1e-300))
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("outer", [30, 0])
def test_partitioned_newton_mixed_fp64_system_on_contexts(outer):
    """The OVS_MIXED loop over three contexts (ContextPartition.round:
    ovs_round_matrix of each part's FP64 matrix as the inner operator, the
    FP64 parts outside) against ovs_quench_newton OVS_MIXED on one context,
    both with the flexible outer (30) and both with the restarted refinement
    (0): converged, the same Newton iterations within one, the state within
    1e-6."""
    case = _case()
    g = Context.from_case(case)
    g.set_option(F.OVS_OPT_MIXED_OUTER, outer)
    info = g.quench_newton(mode=F.OVS_MIXED, max_cycles=40, **OPTS)
    ref = {n: g.get_field(n) for n in ("ug", "pg", "phig", "tg")}
    g.close()
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ctxs = [Context.from_case(P.local_case(case, p)) for p in parts]
    sp = {r: D.ContextPartition(c, plan.owned[r], device="cuda:0") for r, c in enumerate(ctxs)}
    out = D.quench_newton(D.LocalComm(plan), sp, mode=F.OVS_MIXED, max_cycles=40, mixed_outer=outer, **OPTS)
    assert out["converged"] and abs(out["iterations"] - info.iterations) <= 1
    for n, a in ref.items():
        for c, p in zip(ctxs, parts):
            np.testing.assert_allclose(c.get_field(n), a[p.nodes], rtol=0, atol=1e-6 * max(np.abs(a).max(), 1e-300))
    for c in ctxs:
        c.close()


def test_round_matrix_is_the_fp32_rounding():
    """ovs_round_matrix writes the FP32 rounding of every FP64 matrix block
    into the FP32 store, and refuses a system without an FP64 matrix."""
    case = _case()
    c = Context.from_case(case)
    with pytest.raises(F.OvsError):
        c.round_matrix(F.OVS_SYS_NSVOF)
    c.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
    c.round_matrix(F.OVS_SYS_NSVOF)
    from oversetdevfort_b200.api import SYS_BLOCKS
    for b in SYS_BLOCKS[F.OVS_SYS_NSVOF]:
        a64 = c.get_lhs(F.OVS_SYS_NSVOF, F.OVS_FP64, b)
        np.testing.assert_array_equal(c.get_lhs(F.OVS_SYS_NSVOF, F.OVS_FP32, b), a64.astype(np.float32).astype(np.float64))
    c.close()
