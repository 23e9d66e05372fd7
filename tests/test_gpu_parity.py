"""GPU parity: every product entry point, called through the C ABI, against
the CPU oracle on the same seeded inputs (and against the committed golden
fixture).

Tolerances (normwise per block, |gpu - ref|_max <= tol * |ref|_max):
  * CSR pattern, slot maps, iteration counts: bit-exact / equal;
  * FP64 assembly, SpMV, GMRES: 1e-12 (assembly) / 1e-13 (SpMV) / 1e-10
    (GMRES solution, which amplifies the rounding differences of the
    assembly by the condition of the Krylov process);
  * FP32 assembly: 1e-5.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import (Context, genSparStruc, assembleQuenching, assembleNavSto,
                                     SparseGMRES_up, SparseGMRES_ns_conv, SparseGMRES_tem, SYS_BLOCKS,
                                     BLOCK_NAME)

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "quench_small.npz"
KIND = {F.OVS_SYS_NS: "ns", F.OVS_SYS_NSVOF: "nsvof", F.OVS_SYS_TEM: "tem"}


def close(gpu, ref, tol, what=""):
    gpu, ref = np.asarray(gpu, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    assert gpu.shape == ref.shape, (what, gpu.shape, ref.shape)
    scale = max(np.abs(ref).max(initial=0.0), 1e-300)
    err = np.abs(gpu - ref).max(initial=0.0)
    assert err <= tol * scale, f"{what}: max err {err:.3e} vs scale {scale:.3e} (tol {tol})"
    return err / scale


def _ctx(case):
    return Context.from_case(case)


# --------------------------------------------------------------- pattern
@pytest.mark.parametrize("mk", [lambda: M.box_tet(16, 16, 16), lambda: M.box_tet(4, 3, 3),
                                lambda: M.box_tet(7, 1, 3, 2.0, 0.5, 1.0), lambda: M.box_hex(3, 3, 2),
                                lambda: M.box_tet(1, 1, 1)])
def test_pattern_bit_exact(oracle, mk):
    m = mk()
    col_o, row_o = oracle.gen_spar_struc(m.ien, m.nnode)
    col_g, row_g = genSparStruc(m.ien, m.nnode)
    np.testing.assert_array_equal(col_g, col_o)
    np.testing.assert_array_equal(row_g, row_o)


def test_pattern_config2_size():
    m = M.box_tet(48, 48, 96, 1.0, 1.0, 2.0)
    col, row = genSparStruc(m.ien, m.nnode)
    assert m.nnode == 232897 and len(row) == 3398977 == M.expected_nnz_kuhn(48, 48, 96)
    assert np.all(np.diff(col) > 0)


# -------------------------------------------------------------- assembly
def _assemble_both(oracle, case, kernel, tensor_flag, prec):
    oc = oracle.OracleCase(case)
    ctx = _ctx(case)
    if kernel == F.OVS_ASM_NS:
        cfl_o = oc.assemble_navsto(tensor_flag)
        cfl_g = assembleNavSto(ctx, tensor_flag, prec)
        sysid, kind = F.OVS_SYS_NS, "ns"
    elif kernel == F.OVS_ASM_NSVOF:
        cfl_o = oc.assemble_quenching(tensor_flag, 3)
        cfl_g = assembleQuenching(ctx, tensor_flag, 3, prec)
        sysid, kind = F.OVS_SYS_NSVOF, "nsvof"
    else:
        cfl_o = oc.assemble_quenching(tensor_flag, 4)
        cfl_g = assembleQuenching(ctx, tensor_flag, 4, prec)
        sysid, kind = F.OVS_SYS_TEM, "tem"
    return oc, ctx, sysid, kind, cfl_o, cfl_g


def _compare_system(oc, ctx, sysid, kind, tensor_flag, prec, tol):
    ref = oc.system(kind)
    if tensor_flag & F.OVS_TENSOR_MAT:
        for b in SYS_BLOCKS[sysid]:
            name = BLOCK_NAME[b]
            close(ctx.get_lhs(sysid, prec, b), ref[name], tol, f"{kind}.{name}")
    if tensor_flag & F.OVS_TENSOR_VEC:
        g = ctx.get_rhs(sysid, prec)
        for f in range(g.shape[1]):
            close(g[:, f], ref["rhs"][:, f], tol, f"{kind}.rhs[{f}]")


CASES = [("nsvof", s) for s in (0, 1, 2)] + [("tem", s) for s in (0, 1)] + [("ns", s) for s in (0, 1)]


@pytest.mark.parametrize("kind,seed", CASES)
@pytest.mark.parametrize("tflag", [6, 4, 2])
def test_assembly_fp64_random(oracle, kind, seed, tflag):
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    case = M.random_case(nx=4 + seed, ny=3, nz=3 - (seed % 2), seed=seed, kernel=kernel)
    oc, ctx, sysid, k, cfl_o, cfl_g = _assemble_both(oracle, case, kernel, tflag, F.OVS_FP64)
    assert abs(cfl_g - cfl_o) <= 1e-12 * max(cfl_o, 1e-300)
    _compare_system(oc, ctx, sysid, k, tflag, F.OVS_FP64, 1e-12)


@pytest.mark.parametrize("kind,seed", CASES)
def test_assembly_fp32_random(oracle, kind, seed):
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    case = M.random_case(nx=4 + seed, ny=3, nz=3, seed=seed, kernel=kernel)
    oc, ctx, sysid, k, cfl_o, cfl_g = _assemble_both(oracle, case, kernel, 6, F.OVS_FP32)
    _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP32, 1e-5)


def test_assembly_config1_fp64_and_fp32(oracle):
    case = M.config1()
    oc, ctx, sysid, k, cfl_o, cfl_g = _assemble_both(oracle, case, F.OVS_ASM_NS, 6, F.OVS_FP64)
    assert abs(cfl_g - cfl_o) <= 1e-12 * cfl_o
    _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP64, 1e-12)
    assembleNavSto(ctx, 6, F.OVS_FP32)
    _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP32, 1e-5)


def test_assembly_quench_config_fp64(oracle):
    case = M.quench_case(M.box_tet(10, 10, 12, 1.0, 1.0, 1.2), "q10")
    for kernel in (F.OVS_ASM_NSVOF, F.OVS_ASM_TEM):
        oc, ctx, sysid, k, cfl_o, cfl_g = _assemble_both(oracle, case, kernel, 6, F.OVS_FP64)
        _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP64, 1e-12)
        ctx.assemble(kernel, 6, F.OVS_FP32)
        _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP32, 1e-5)


def test_assembly_against_golden_fixture():
    g = np.load(GOLDEN)
    case = M.random_case(nx=3, ny=2, nz=2, seed=11)
    ctx = _ctx(case)
    col, row = ctx.get_pattern()
    np.testing.assert_array_equal(col, g["q_col"])
    np.testing.assert_array_equal(row, g["q_row"])
    cfl = assembleQuenching(ctx, 6, 7)
    assert abs(cfl - g["q_cfl"][0]) <= 1e-12 * g["q_cfl"][0]
    for b in SYS_BLOCKS[F.OVS_SYS_NSVOF]:
        close(ctx.get_lhs(F.OVS_SYS_NSVOF, F.OVS_FP64, b), g["q_" + BLOCK_NAME[b]], 1e-12, BLOCK_NAME[b])
    close(ctx.get_lhs(F.OVS_SYS_TEM, F.OVS_FP64, F.OVS_BLK_TEM), g["q_TEM"], 1e-12, "TEM")
    r = ctx.get_rhs(F.OVS_SYS_NSVOF)
    close(r[:, :3], g["q_rhsu"], 1e-12, "rhsu")
    close(r[:, 3], g["q_rhsp"], 1e-12, "rhsp")
    close(r[:, 4], g["q_rhsls"], 1e-12, "rhsls")
    close(ctx.get_rhs(F.OVS_SYS_TEM)[:, 0], g["q_rhstem"], 1e-12, "rhstem")
    su, sp, sl, info = SparseGMRES_ns_conv(ctx, 1e-8, 20, 1, np.zeros((ctx.N, 3)), np.zeros(ctx.N),
                                           np.zeros(ctx.N))
    assert info.iterations == g["q_it_nsvof"][0]
    close(np.column_stack([su, sp, sl]), g["q_sol_nsvof"], 1e-10, "sol nsvof")
    st, info = SparseGMRES_tem(ctx, 1e-8, 20, 1, np.zeros(ctx.N))
    assert info.iterations == g["q_it_tem"][0]
    close(st, g["q_sol_tem"][:, 0], 1e-10, "sol tem")


def test_assembly_deterministic():
    case = M.random_case(nx=6, ny=5, nz=4, seed=9)
    ctx = _ctx(case)
    for prec in (F.OVS_FP64, F.OVS_FP32):
        runs = []
        for _ in range(3):
            ctx.assemble(F.OVS_ASM_NSVOF, 6, prec)
            runs.append((ctx.get_lhs(F.OVS_SYS_NSVOF, prec, F.OVS_BLK_K11), ctx.get_rhs(F.OVS_SYS_NSVOF, prec)))
        for k11, rhs in runs[1:]:
            assert np.array_equal(k11, runs[0][0]) and np.array_equal(rhs, runs[0][1])


# ------------------------------------------------------------ SpMV / GMRES
def _system_pair(oracle, seed, kind):
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    case = M.random_case(nx=5, ny=4, nz=3, seed=seed, kernel=kernel)
    case.mesh.elm_id[:] = 102
    case.ibc[:] = 0
    for f in range(6):
        case.ibc[case.mesh.faces[f], 0:3] = 1
    case.ibc[0, 3] = 1
    case.params["subdomain_flag"] = 1
    oc = oracle.OracleCase(case)
    if kind == "ns":
        oc.assemble_navsto(6)
    else:
        oc.assemble_quenching(6, 3 if kind == "nsvof" else 4)
    ctx = _ctx(case)
    sysid = {"ns": F.OVS_SYS_NS, "nsvof": F.OVS_SYS_NSVOF, "tem": F.OVS_SYS_TEM}[kind]
    ref = oc.system(kind)
    blocks = {k: v for k, v in ref.items() if k != "rhs"}
    ctx.set_system(sysid, F.OVS_FP64, blocks, ref["rhs"])
    return oc, ctx, sysid, ref


@pytest.mark.parametrize("kind", ["ns", "nsvof", "tem"])
def test_spmv_parity(oracle, kind):
    oc, ctx, sysid, ref = _system_pair(oracle, 21, kind)
    rng = np.random.default_rng(3)
    x = np.asfortranarray(rng.standard_normal(ref["rhs"].shape))
    close(ctx.spmv(sysid, F.OVS_FP64, x), oc.spmv(kind, x), 1e-13, f"spmv {kind}")
    # FP32 matrix: compare against the oracle on the FP32-rounded values
    blocks32 = {k: v.astype(np.float32).astype(np.float64) for k, v in ref.items() if k != "rhs"}
    ctx.set_system(sysid, F.OVS_FP32, blocks32, ref["rhs"])
    oc.load_system(kind, dict(blocks32, rhs=ref["rhs"]))
    close(ctx.spmv(sysid, F.OVS_FP32, x), oc.spmv(kind, x), 1e-13, f"spmv32 {kind}")


@pytest.mark.parametrize("kind", ["ns", "nsvof", "tem"])
@pytest.mark.parametrize("kspace,kmin,tol", [(40, 1, 1e-8), (25, 10, 1e-3), (60, 1, 1e-14)])
def test_gmres_reference_semantics(oracle, kind, kspace, kmin, tol):
    oc, ctx, sysid, ref = _system_pair(oracle, 22, kind)
    rng = np.random.default_rng(4)
    sol0 = np.asfortranarray(rng.standard_normal(ref["rhs"].shape)) * 1e-3
    so, it_o, er_o, r0_o = oc.gmres(kind, tol, kspace, kmin, sol0)
    sg, info = ctx.gmres(sysid, tol, kspace, kmin, sol0)
    assert info.iterations == it_o
    assert abs(info.res0 - r0_o) <= 1e-12 * r0_o
    close(sg, so, 1e-10, f"gmres {kind}")


def test_gmres_tem_zero_rhs_returns_zero(oracle):
    oc, ctx, sysid, ref = _system_pair(oracle, 23, "tem")
    ctx.set_rhs(F.OVS_SYS_TEM, F.OVS_FP64, np.zeros(ctx.N))
    s, info = SparseGMRES_tem(ctx, 1e-8, 20, 1, np.ones(ctx.N))
    assert np.all(s == 0.0)   # SparseGMRES_tem.f90:68-71 zeroes sol


@pytest.mark.parametrize("mk", [lambda: M.config1().mesh, lambda: M.box_hex(6, 5, 4),
                                lambda: M.box_tet(48, 48, 96, 1.0, 1.0, 2.0)],
                         ids=["config1", "hex", "config2_mesh"])
def test_slot_map_bit_exact(oracle, mk):
    """The element-slot -> CSR-slot map the assembly scatters through equals
    FillSparseMat_3D's k = SparseMatLoc_3D(...) + col(IEN(e,a)) - 1 for every
    (element, a, b), on config 1, a hexahedral box and the config-2 mesh
    (1,327,104 tets)."""
    m = mk()
    ctx = Context(m.nnode, m.nelem, m.ien.shape[1])
    ctx.upload_mesh(m)
    ctx.build_pattern()
    col, row = ctx.get_pattern()
    lmap = ctx.get_slot_map()
    ctx.close()
    ref = oracle.slot_map(m.ien, col, row)
    np.testing.assert_array_equal(lmap, ref)


def test_config1_newton_step(oracle):
    """Config 1 end to end: NS assembly, reference GMRES(50, 1e-6), Newton
    update - GPU vs oracle."""
    case = M.config1()
    oc = oracle.OracleCase(case)
    oc.assemble_navsto(6)
    ctx = _ctx(case)
    assembleNavSto(ctx, 6)
    so, it_o, er_o, r0_o = oc.gmres("ns", 1e-6, 50, 1)
    su, sp, info = SparseGMRES_up(ctx, 1e-6, 50, 1, np.zeros((ctx.N, 3)), np.zeros(ctx.N))
    assert info.iterations == it_o
    close(np.column_stack([su, sp]), so, 1e-9, "config1 sol")
    ctx.newton_update(F.OVS_SYS_NS)
    oc.newton_update(F.OVS_SYS_NS, so)
    for f in ("ug", "acg", "pg"):
        close(ctx.get_field(f), oc.state_arrays[f], 1e-12, f)
    r_g = ctx.residual_norms()
    oc.assemble_navsto(2)
    assembleNavSto(ctx, 2)
    r_o = oc.calculate_residual()
    close(ctx.residual_norms()[:2], r_o[:2], 1e-9, "residual after update")
    assert r_g[0] > 0


@pytest.mark.parametrize("mode", [F.OVS_FP64, F.OVS_FP32, F.OVS_MIXED])
def test_refined_solve_reaches_true_residual(oracle, mode):
    """The refined solve's own residual claim, rechecked with the oracle's
    SpMV on the system it refines against: the FP64 system for OVS_FP64 and
    OVS_MIXED, the FP32-assembled one for OVS_FP32."""
    case = M.quench_case(M.box_tet(8, 8, 8), "q8")
    ctx = _ctx(case)
    prec = F.OVS_FP32 if mode == F.OVS_FP32 else F.OVS_FP64
    ctx.assemble(F.OVS_ASM_NSVOF, 6, prec)
    sol, info = ctx.solve(F.OVS_SYS_NSVOF, mode, 1e-8, kspace=50, max_cycles=200)
    assert info.converged and info.rel_residual <= 1e-8
    # independent check of the true residual with the oracle's SpMV
    oc = oracle.OracleCase(case)
    sysblocks = ctx.get_system(F.OVS_SYS_NSVOF, prec)
    oc.load_system("nsvof", sysblocks)
    r = sysblocks["rhs"] - oc.spmv("nsvof", sol)
    assert np.linalg.norm(r) <= 1.05e-8 * np.linalg.norm(sysblocks["rhs"])


@pytest.mark.parametrize("sysid,kern,nf", [(F.OVS_SYS_NSVOF, F.OVS_ASM_NSVOF, 5), (F.OVS_SYS_TEM, F.OVS_ASM_TEM, 1)])
@pytest.mark.parametrize("outer", [30, 0])
def test_mixed_reaches_fp64_solution(oracle, sysid, kern, nf, outer):
    """OVS_MIXED solves the FP64 system, with the flexible FGMRES(30) outer
    (default) and with the restarted refinement (OVS_OPT_MIXED_OUTER = 0):
    its true residual on the FP64 system (rechecked with the oracle's SpMV)
    meets rtol, and every field of its solution is within 1e-5 (relative to
    the field's largest value) of the restarted FP64 GMRES solution.  Both
    run to rtol 1e-12: on this box a relative residual of 1e-10 leaves up to
    8e-4 of uncertainty in the VOF field of ANY solution (the pressure
    correction is ~1e7 and dominates the residual norm), so field-by-field
    agreement is only meaningful when both solves are tight.  The FP32
    rounding of the matrix is what the inner cycles used."""
    case = M.quench_case(M.box_tet(8, 8, 8), "q8")
    ctx = _ctx(case)
    ctx.set_option(F.OVS_OPT_MIXED_OUTER, outer)
    ctx.assemble(kern, 6, F.OVS_FP64)
    s64, i64 = ctx.solve(sysid, F.OVS_FP64, 1e-12, 50, 600)
    smx, imx = ctx.solve(sysid, F.OVS_MIXED, 1e-12, 50, 600)
    assert i64.converged and imx.converged and imx.rel_residual <= 1e-12
    oc = oracle.OracleCase(case)
    sysblocks = ctx.get_system(sysid, F.OVS_FP64)
    oc.load_system(KIND[sysid], sysblocks)
    r = sysblocks["rhs"] - oc.spmv(KIND[sysid], smx)
    assert np.linalg.norm(r) <= 2e-12 * np.linalg.norm(sysblocks["rhs"])
    for f in range(nf):
        scale = max(np.abs(s64[:, f]).max(), 1e-300)
        assert np.abs(smx[:, f] - s64[:, f]).max() <= 1e-5 * scale, f
    for b in SYS_BLOCKS[sysid]:
        a32 = ctx.get_lhs(sysid, F.OVS_FP32, b)
        np.testing.assert_array_equal(a32, sysblocks[BLOCK_NAME[b]].astype(np.float32).astype(np.float64))


def test_mixed_vs_fp64_solution_error(oracle):
    """The FP32-assembled system (OVS_FP32) is a different system: its
    solution has an FP64 residual far above what OVS_MIXED reaches on the
    same FP64 system, and stays within the FP32 assembly's rounding times the
    condition number of the FP64 solution."""
    case = M.quench_case(M.box_tet(8, 8, 8), "q8")
    ctx = _ctx(case)
    ctx.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
    s64, i64 = ctx.solve(F.OVS_SYS_NSVOF, F.OVS_FP64, 1e-12, 50, 600)
    smx, imx = ctx.solve(F.OVS_SYS_NSVOF, F.OVS_MIXED, 1e-12, 50, 600)
    sys64 = ctx.get_system(F.OVS_SYS_NSVOF, F.OVS_FP64)
    ctx.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP32)
    s32, i32 = ctx.solve(F.OVS_SYS_NSVOF, F.OVS_FP32, 1e-12, 50, 600)
    assert i64.converged and imx.converged and i32.converged
    oc = oracle.OracleCase(case)
    oc.load_system("nsvof", sys64)
    bn = np.linalg.norm(sys64["rhs"])
    res_mx = np.linalg.norm(sys64["rhs"] - oc.spmv("nsvof", smx)) / bn
    res_32 = np.linalg.norm(sys64["rhs"] - oc.spmv("nsvof", s32)) / bn
    assert res_mx <= 2e-12 and res_32 > 1e3 * res_mx, (res_mx, res_32)
    for f in range(5):
        scale = max(np.abs(s64[:, f]).max(), 1e-300)
        assert np.abs(smx[:, f] - s64[:, f]).max() <= 1e-5 * scale, f
        assert np.abs(s32[:, f] - s64[:, f]).max() <= 1e-2 * scale, f   # FP32 assembly: O(kappa * 1e-7)


# ------------------------------------------------------------ error paths
def test_error_paths():
    lib = F.load()
    case = M.random_case(seed=1)
    m = case.mesh
    ctx = Context(m.nnode, m.nelem, 4)
    with pytest.raises(F.OvsError) as e:
        ctx.assemble(F.OVS_ASM_NSVOF, 6)
    assert e.value.status == F.OVS_ERR_STATE
    ien = m.ien.copy(order="F")
    ien[0, 1] = ien[0, 0]  # degenerate element
    bad = M.Mesh(m.xg, ien, m.elm_id, m.faces, m.dims, m.lengths)
    with pytest.raises(F.OvsError) as e:
        ctx.upload_mesh(bad)
    assert e.value.status == F.OVS_ERR_ARG
    ctx.upload_mesh(m)
    ctx.build_pattern()
    ctx.set_params(case.params)
    ctx.set_state(case.state)
    with pytest.raises(F.OvsError):
        ctx.assemble(99, 6)
    with pytest.raises(F.OvsError) as e:
        ctx.gmres(F.OVS_SYS_NSVOF, 1e-6, 10, 1, np.zeros((m.nnode, 5)))
    assert e.value.status == F.OVS_ERR_STATE
    # an inverted element: warning status, results still written
    xg = m.xg.copy(order="F")
    n1, n2, n3, n4 = (m.ien[0] - 1)
    nrm = np.cross(xg[n3] - xg[n2], xg[n4] - xg[n2])
    nrm /= np.linalg.norm(nrm)
    xg[n1] -= 2.0 * np.dot(xg[n1] - xg[n2], nrm) * nrm   # mirror node 1 through face (2,3,4)
    ctx.set_field("xg", xg)
    ctx.assemble(F.OVS_ASM_NSVOF, 6)
    assert ctx.last_status == F.OVS_WARN_NEG_DETJ
    ctx.close()


def test_kdc_integer_dummy_quirk(oracle):
    """e3DC_beta2 declares ns_kdc INTEGER but receives real(8): the low 4
    bytes of the double become the multiplier.  With phi clamped to exactly 0
    the interpolated value is NS_kdc_w itself, so the quirk is reproducible:
    1 + 3 ulp has low word 3, i.e. k_dc = 3 |rL| / |G|."""
    case = M.random_case(nx=4, ny=3, nz=3, seed=12, kernel=F.OVS_ASM_NSVOF)
    for n in ("phig", "phigold"):
        case.state[n][:] = -0.5
    case.params["ns_kdc_w"] = np.nextafter(np.nextafter(np.nextafter(1.0, 2.0), 2.0), 2.0)
    assert np.frombuffer(np.float64(case.params["ns_kdc_w"]).tobytes()[:4], np.int32)[0] == 3
    oc, ctx, sysid, k, cfl_o, cfl_g = _assemble_both(oracle, case, F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
    _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP64, 1e-12)
    base = M.random_case(nx=4, ny=3, nz=3, seed=12, kernel=F.OVS_ASM_NSVOF)
    for n in ("phig", "phigold"):
        base.state[n][:] = -0.5
    ob = oracle.OracleCase(base)
    ob.assemble_quenching(6, 3)
    assert np.abs(ob.sys["K11"] - oc.sys["K11"]).max() > 0   # k_dc is active


@pytest.mark.parametrize("kind", ["nsvof", "tem", "ns"])
@pytest.mark.parametrize("prec", [F.OVS_FP64, F.OVS_FP32])
def test_row_pass_variants_bit_identical(kind, prec):
    """The chunked row pass (OVS_OPT_ROWS_GATHER = 0) with the element
    summaries staged through shared memory (OVS_OPT_ROWS_STAGED = 1) and
    read lane by lane from global memory (0) runs the same arithmetic in the
    same order: the assembled systems are bit-identical, matrix and
    right-hand side."""
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    sysid = {"nsvof": F.OVS_SYS_NSVOF, "tem": F.OVS_SYS_TEM, "ns": F.OVS_SYS_NS}[kind]
    case = M.random_case(nx=6, ny=5, nz=4, seed=21, kernel=kernel)
    out = []
    for staged in (0, 1):
        ctx = _ctx(case)
        ctx.set_option(F.OVS_OPT_ROWS_TILED, 0)
        ctx.set_option(F.OVS_OPT_ROWS_GATHER, 0)
        ctx.set_option(F.OVS_OPT_ROWS_STAGED, staged)
        ctx.assemble(kernel, 6, prec)
        out.append(ctx.get_system(sysid, prec))
        ctx.close()
    for k in out[0]:
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)


@pytest.mark.parametrize("kind", ["nsvof", "tem", "ns"])
@pytest.mark.parametrize("prec,tol", [(F.OVS_FP64, 1e-14), (F.OVS_FP32, 1e-6)])
def test_row_passes_agree(kind, prec, tol):
    """The tiled row pass (default: summaries staged per row tile in shared
    memory), the untiled gather pass (OVS_OPT_ROWS_TILED = 0) and the
    chunked pass (also OVS_OPT_ROWS_GATHER = 0).  Tiled and gather add every
    entry in the same order (each entry's list in pieces of consecutive
    elements, the pieces added in order); the chunked pass adds every entry
    in one ascending sweep.  The systems agree to rounding, normwise per
    block, and the tiled pass gives the same bits on a second run."""
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    sysid = {"nsvof": F.OVS_SYS_NSVOF, "tem": F.OVS_SYS_TEM, "ns": F.OVS_SYS_NS}[kind]
    case = M.random_case(nx=6, ny=5, nz=4, seed=23, kernel=kernel)
    out = []
    for tiled, gather in ((1, 1), (0, 1), (0, 0), (1, 1)):
        ctx = _ctx(case)
        ctx.set_option(F.OVS_OPT_ROWS_TILED, tiled)
        ctx.set_option(F.OVS_OPT_ROWS_GATHER, gather)
        ctx.assemble(kernel, 6, prec)
        out.append(ctx.get_system(sysid, prec))
        ctx.close()
    for k in out[0]:
        close(out[0][k], out[1][k], tol, k)
        close(out[1][k], out[2][k], tol, k)
        np.testing.assert_array_equal(out[0][k], out[3][k], err_msg=k)


@pytest.mark.parametrize("prec", [F.OVS_FP64, F.OVS_FP32])
@pytest.mark.parametrize("seed", [24, 25])
def test_quench_assembly_call_matches_two_passes(oracle, prec, seed):
    """OVS_ASM_QUENCH (assembleQuenching with NS, VOF and TEM flagged: the
    NS+VOF pass then the temperature pass under one status) against the two
    passes called apart: the same systems and CFL number, bit for bit on a
    second run, and the FP64 systems within 1e-12 of the oracle's."""
    case = M.random_case(nx=6, ny=5, nz=4, seed=seed, kernel=F.OVS_ASM_NSVOF)
    runs = []
    for fused in (True, False, True):
        ctx = _ctx(case)
        if fused:
            cfl = ctx.assemble(F.OVS_ASM_QUENCH, 6, prec)
        else:
            cfl = ctx.assemble(F.OVS_ASM_NSVOF, 6, prec)
            ctx.assemble(F.OVS_ASM_TEM, 6, prec)
        runs.append((cfl, ctx.get_system(F.OVS_SYS_NSVOF, prec), ctx.get_system(F.OVS_SYS_TEM, prec)))
        ctx.close()
    (c0, n0, t0), (c1, n1, t1), (c2, n2, t2) = runs
    assert c0 == c1 == c2
    for k in n0:
        np.testing.assert_array_equal(n0[k], n1[k], err_msg="nsvof." + k)
        np.testing.assert_array_equal(n0[k], n2[k], err_msg="nsvof." + k)
    for k in t0:
        np.testing.assert_array_equal(t0[k], t1[k], err_msg="tem." + k)
        np.testing.assert_array_equal(t0[k], t2[k], err_msg="tem." + k)
    if prec == F.OVS_FP64:
        oc = oracle.OracleCase(case)
        oc.assemble_quenching(6, 7)
        ctx = _ctx(case)
        ctx.assemble(F.OVS_ASM_QUENCH, 6, prec)
        _compare_system(oc, ctx, F.OVS_SYS_NSVOF, "nsvof", 6, prec, 1e-12)
        _compare_system(oc, ctx, F.OVS_SYS_TEM, "tem", 6, prec, 1e-12)
        ctx.close()


def _fan_case(kernel, m=40, seed=31):
    """A fan of m tets around the axis from node 0 to node 1 (ring nodes 2..):
    the two axis rows have degree m + 2 and m elements, more off-diagonal
    entries than the gather row pass has lanes for in one pass, and the
    entry (0, 1) lists all m elements."""
    base = M.random_case(nx=3, ny=3, nz=3, seed=seed, kernel=kernel)
    rng = np.random.default_rng(seed)
    ang = np.linspace(0.0, 2 * np.pi, m, endpoint=False) + rng.uniform(0.0, 0.02, m)
    ring = np.stack([np.cos(ang), np.sin(ang), 0.5 + 0.05 * rng.uniform(-1, 1, m)], axis=1)
    xg = np.asfortranarray(np.vstack([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0], ring]))
    ien = np.array([[0, 2 + i, 2 + (i + 1) % m, 1] for i in range(m)], dtype=np.int64)
    for t in ien:   # positive DetJ = det[x1 - x4, x2 - x4, x3 - x4]
        x = xg[t]
        if np.linalg.det(np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]])) < 0:
            t[0], t[1] = t[1], t[0]
    N = xg.shape[0]
    elm = np.where(rng.random(m) < 0.15, 101, 102).astype(np.int32)
    mesh = M.Mesh(xg, np.asfortranarray(ien.astype(np.int32) + 1), elm, [np.zeros(0, np.int64)] * 6,
                  (m, 1, 1), (1.0, 1.0, 1.0))
    st = {}
    for k, v in base.state.items():
        lo, hi = float(np.min(v)), float(np.max(v))
        st[k] = np.asfortranarray(rng.uniform(lo, hi, size=(N,) + v.shape[1:]).astype(v.dtype))
    ibc = np.asfortranarray((rng.random((N, 8)) < 0.2).astype(np.int32))
    return M.Case(f"fan{m}", mesh, base.params, st, ibc, kernel, kspace=30, gmres_tol=1e-8)


@pytest.mark.parametrize("kind", ["nsvof", "tem", "ns"])
@pytest.mark.parametrize("tile_elems", [0, 96, 16])
def test_assembly_high_degree_rows(oracle, kind, tile_elems):
    """Rows of degree 42 (two passes of the gather scheme's lanes, a
    40-element contribution list) against the oracle, FP64 1e-12,
    FP32 1e-5: the default gather pass (0), and the tiled pass with a 96-
    and a 16-element tile budget (with 16 the two 40-element rows take the
    untiled gather pass beside the tiles)."""
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    case = _fan_case(kernel)
    oc = oracle.OracleCase(case)
    ctx = _ctx(case)
    if tile_elems:
        ctx.set_option(F.OVS_OPT_ROWS_TILED, 1)
        ctx.set_option(F.OVS_OPT_TILE_ELEMS, tile_elems)
    if kernel == F.OVS_ASM_NS:
        oc.assemble_navsto(6)
        assembleNavSto(ctx, 6, F.OVS_FP64)
        sysid, k = F.OVS_SYS_NS, "ns"
    else:
        oc.assemble_quenching(6, 3 if kernel == F.OVS_ASM_NSVOF else 4)
        assembleQuenching(ctx, 6, 3 if kernel == F.OVS_ASM_NSVOF else 4, F.OVS_FP64)
        sysid, k = (F.OVS_SYS_NSVOF, "nsvof") if kernel == F.OVS_ASM_NSVOF else (F.OVS_SYS_TEM, "tem")
    ptr, cols = ctx.get_pattern()
    assert np.diff(ptr).max() == 42
    _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP64, 1e-12)
    ctx.assemble(kernel, 6, F.OVS_FP32)
    _compare_system(oc, ctx, sysid, k, 6, F.OVS_FP32, 1e-5)


@pytest.mark.parametrize("kind", ["nsvof", "tem", "ns"])
def test_element_pass_variants_bit_identical(kind):
    """The FP64 element pass with its node records in shared memory
    (OVS_OPT_ELEM_SMEM = 1) and in registers (0) evaluates the same
    formulas; the Gauss loop is rolled in one and unrolled in the other, so
    the compiler contracts multiply-adds differently and the results agree
    to rounding (1e-14 normwise per block), each within the oracle's 1e-12."""
    kernel = {"nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM, "ns": F.OVS_ASM_NS}[kind]
    sysid = {"nsvof": F.OVS_SYS_NSVOF, "tem": F.OVS_SYS_TEM, "ns": F.OVS_SYS_NS}[kind]
    case = M.random_case(nx=6, ny=5, nz=4, seed=22, kernel=kernel)
    out = []
    for sm in (0, 1):
        ctx = _ctx(case)
        ctx.set_option(F.OVS_OPT_ELEM_SMEM, sm)
        ctx.assemble(kernel, 6, F.OVS_FP64)
        out.append(ctx.get_system(sysid, F.OVS_FP64))
        ctx.close()
    for k in out[0]:
        close(out[1][k], out[0][k], 1e-14, k)


def _relabel(case, seed):
    """The same case with its nodes numbered by a random permutation (an
    unstructured numbering: rows far apart in memory share elements)."""
    import copy
    rng = np.random.default_rng(seed)
    m = case.mesh
    N = m.nnode
    new_of_old = rng.permutation(N)               # old node i -> new node new_of_old[i]
    old_of_new = np.argsort(new_of_old)
    ien = np.asfortranarray((new_of_old[np.asarray(m.ien) - 1] + 1).astype(np.int32))
    xg = np.asfortranarray(m.xg[old_of_new])
    faces = [np.sort(new_of_old[f]) for f in m.faces]
    mesh = M.Mesh(xg, ien, m.elm_id.copy(), faces, m.dims, m.lengths)
    state = {k: np.asfortranarray(np.asarray(v)[old_of_new]) for k, v in case.state.items()}
    ibc = np.asfortranarray(np.asarray(case.ibc)[old_of_new])
    c = copy.copy(case)
    c.mesh, c.state, c.ibc = mesh, state, ibc
    return c, old_of_new


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
@pytest.mark.parametrize("prec,tol", [(F.OVS_FP64, 1e-12), (F.OVS_FP32, 1e-5)])
def test_assembly_on_a_permuted_numbering(oracle, kind, prec, tol):
    """A random node numbering (rows that share an element far apart, the
    spatial row order a true permutation) assembles to the oracle's system
    on the same numbering, and its residual is the structured numbering's,
    permuted."""
    kernel = F.OVS_ASM_NSVOF if kind == "nsvof" else F.OVS_ASM_TEM
    base = M.random_case(nx=6, ny=5, nz=4, seed=40, kernel=kernel)
    case, old_of_new = _relabel(base, 7)
    oc, ctx, sysid, k, cfl_o, cfl_g = _assemble_both(oracle, case, kernel, 6, prec)
    _compare_system(oc, ctx, sysid, k, 6, prec, tol)
    col, row = ctx.get_pattern()
    col_o, row_o = oracle.gen_spar_struc(case.mesh.ien, case.mesh.nnode)
    np.testing.assert_array_equal(col, col_o)
    np.testing.assert_array_equal(row, row_o)
    np.testing.assert_array_equal(ctx.get_slot_map(), oracle.slot_map(case.mesh.ien, col, row))
    r_perm = ctx.get_rhs(sysid, prec)
    ctx.close()
    ctx2 = _ctx(base)
    ctx2.assemble(kernel, 6, prec)
    r_base = ctx2.get_rhs(sysid, prec)
    ctx2.close()
    close(r_perm, r_base[old_of_new], tol, "permuted residual")
