"""Hex path (config 4 family): trilinear hexahedra, 2x2x2 Gauss points.

The NS+VOF quench and temperature assembly on hexahedra against the oracle
(the same reference element routines with linhexshl and the 8-point rule):
FP64 to 1e-12 and FP32 to 1e-5 on random cases with every code path on
(solid elements, random Dirichlet flags, phase change, discontinuity
capturing, mesh motion) and on a quench box; bit-identical reassembly;
and the mixed-precision refined solve of a hex quench system to a true
relative residual of 1e-8.
"""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context, assembleQuenching

from test_gpu_parity import _compare_system

pytestmark = pytest.mark.gpu


def _both(oracle, case, kernel, tflag, prec):
    oc = oracle.OracleCase(case)
    ctx = Context.from_case(case)
    ff = 3 if kernel == F.OVS_ASM_NSVOF else 4
    cfl_o = oc.assemble_quenching(tflag, ff)
    cfl_g = assembleQuenching(ctx, tflag, ff, prec)
    sysid, kind = (F.OVS_SYS_NSVOF, "nsvof") if kernel == F.OVS_ASM_NSVOF else (F.OVS_SYS_TEM, "tem")
    return oc, ctx, sysid, kind, cfl_o, cfl_g


@pytest.mark.parametrize("kernel", [F.OVS_ASM_NSVOF, F.OVS_ASM_TEM])
@pytest.mark.parametrize("seed", [0, 1])
def test_hex_assembly_fp64_random(oracle, kernel, seed):
    case = M.random_case(nx=3 + seed, ny=3, nz=2, seed=seed, kernel=kernel, hex=True)
    oc, ctx, sysid, kind, cfl_o, cfl_g = _both(oracle, case, kernel, 6, F.OVS_FP64)
    assert abs(cfl_g - cfl_o) <= 1e-12 * max(cfl_o, 1e-300)
    _compare_system(oc, ctx, sysid, kind, 6, F.OVS_FP64, 1e-12)
    ctx.close()


@pytest.mark.parametrize("kernel", [F.OVS_ASM_NSVOF, F.OVS_ASM_TEM])
def test_hex_assembly_fp32_random(oracle, kernel):
    case = M.random_case(nx=4, ny=3, nz=3, seed=3, kernel=kernel, hex=True)
    oc, ctx, sysid, kind, cfl_o, cfl_g = _both(oracle, case, kernel, 6, F.OVS_FP32)
    _compare_system(oc, ctx, sysid, kind, 6, F.OVS_FP32, 1e-5)
    ctx.close()


def test_hex_quench_box_fp64_and_deterministic(oracle):
    case = M.quench_case(M.box_hex(8, 8, 10, 1.0, 1.0, 1.25), "hexq8")
    for kernel in (F.OVS_ASM_NSVOF, F.OVS_ASM_TEM):
        oc, ctx, sysid, kind, cfl_o, cfl_g = _both(oracle, case, kernel, 6, F.OVS_FP64)
        _compare_system(oc, ctx, sysid, kind, 6, F.OVS_FP64, 1e-12)
        a = ctx.get_system(sysid, F.OVS_FP32 if False else F.OVS_FP64)
        assembleQuenching(ctx, 6, 3 if kernel == F.OVS_ASM_NSVOF else 4, F.OVS_FP64)
        b = ctx.get_system(sysid, F.OVS_FP64)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
        ctx.close()


def test_hex_mixed_solve_reaches_true_residual():
    case = M.quench_case(M.box_hex(12, 12, 12), "hexq12")
    ctx = Context.from_case(case)
    ctx.assemble(F.OVS_ASM_NSVOF, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP32)
    ctx.assemble(F.OVS_ASM_NSVOF, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    sol, info = ctx.solve(F.OVS_SYS_NSVOF, F.OVS_FP32, 1e-8, kspace=100, max_cycles=200)
    assert info.converged and info.rel_residual <= 1e-8, (info.rel_residual, info.cycles)
    ctx.close()


@pytest.mark.parametrize("seed", [0, 5])
def test_hex_tensor_core_pass(oracle, seed):
    """FP32 NS+VOF hexahedra through the tcgen05 element-matrix pass (3xTF32)
    against the oracle at 1e-5 and against the CUDA-core expansion at 1e-5;
    reassembly is bit-identical."""
    case = M.random_case(nx=5, ny=4, nz=3, seed=seed, kernel=F.OVS_ASM_NSVOF, hex=True)
    oc, ctx, sysid, kind, cfl_o, cfl_g = _both(oracle, case, F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
    ctx.set_option(F.OVS_OPT_HEX_TC, 1)
    assembleQuenching(ctx, 6, 3, F.OVS_FP32)
    _compare_system(oc, ctx, sysid, kind, 6, F.OVS_FP32, 1e-5)
    tc = ctx.get_system(sysid, F.OVS_FP32)
    assembleQuenching(ctx, 6, 3, F.OVS_FP32)
    again = ctx.get_system(sysid, F.OVS_FP32)
    for k in tc:
        np.testing.assert_array_equal(tc[k], again[k])
    ctx.set_option(F.OVS_OPT_HEX_TC, 0)
    assembleQuenching(ctx, 6, 3, F.OVS_FP32)
    cc = ctx.get_system(sysid, F.OVS_FP32)
    for k in tc:
        scale = max(np.abs(cc[k]).max(), 1e-300)
        assert np.abs(tc[k] - cc[k]).max() <= 1e-5 * scale, k
    ctx.close()
