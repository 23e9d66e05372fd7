"""Face assemblies on the GPU against the oracle: FaceAssembly_NS_weak +
FaceAssembly_NS_outflow on the NS and NS+VOF systems and the convective
heat term on the temperature system, on random cases (solid elements,
subdomain selection, random Dirichlet flags on every IBC column, mesh
motion), FP64 to 1e-12 and FP32 to 1e-5 on the whole system; the face
contribution itself (system with faces minus system without) to 1e-12 of
its own size; MAT-only and VEC-only calls; bit-identical reassembly; the
argument checks of ovs_set_faces; a refined solve of a cavity whose walls
are all weak."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context, assembleNavSto, assembleQuenching

from test_gpu_parity import BLOCK_NAME, SYS_BLOCKS, _compare_system

pytestmark = pytest.mark.gpu

KERNEL = {"ns": F.OVS_ASM_NS, "nsvof": F.OVS_ASM_NSVOF, "tem": F.OVS_ASM_TEM}
SYSID = {"ns": F.OVS_SYS_NS, "nsvof": F.OVS_SYS_NSVOF, "tem": F.OVS_SYS_TEM}


def _case(kind, seed):
    case = M.random_case(nx=4 + seed, ny=3, nz=3, seed=seed, kernel=KERNEL[kind])
    case.bfaces = M.face_set(case.mesh, weak=(1, 4, 6), convective={2: (35.0, 310.0), 6: (8.0, 280.0)})
    return case


def _assemble(obj, kind, tflag, prec=None):
    if prec is None:   # oracle
        return obj.assemble_navsto(tflag) if kind == "ns" else \
            obj.assemble_quenching(tflag, 3 if kind == "nsvof" else 4)
    if kind == "ns":
        return assembleNavSto(obj, tflag, prec)
    return assembleQuenching(obj, tflag, 3 if kind == "nsvof" else 4, prec)


def _gpu_system(ctx, kind, tflag, prec):
    sysid = SYSID[kind]
    out = {}
    if tflag & F.OVS_TENSOR_MAT:
        for b in SYS_BLOCKS[sysid]:
            out[BLOCK_NAME[b]] = ctx.get_lhs(sysid, prec, b)
    if tflag & F.OVS_TENSOR_VEC:
        out["rhs"] = ctx.get_rhs(sysid, prec)
    return out


def _face_part_close(g1, g0, r1, r0, what):
    dg, dr = g1 - g0, r1 - r0
    noise = 64 * 2.2e-16 * max(np.abs(r0).max(initial=0.0), np.abs(r1).max(initial=0.0))
    scale = np.abs(dr).max(initial=0.0)
    err = np.abs(dg - dr).max(initial=0.0)
    assert err <= 1e-12 * scale + noise, f"{what}: face part err {err:.3e} (scale {scale:.3e}, noise {noise:.3e})"
    return scale


@pytest.mark.parametrize("kind", ["ns", "nsvof", "tem"])
@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("tflag", [6, 4, 2])
def test_face_assembly_fp64(oracle, kind, seed, tflag):
    case = _case(kind, seed)
    oc = oracle.OracleCase(case)
    ctx = Context.from_case(case)
    _assemble(oc, kind, tflag)
    _assemble(ctx, kind, tflag, F.OVS_FP64)
    _compare_system(oc, ctx, SYSID[kind], kind, tflag, F.OVS_FP64, 1e-12)
    g1, r1 = _gpu_system(ctx, kind, tflag, F.OVS_FP64), oc.system(kind)
    ctx.set_faces(None)
    case.bfaces = None
    oc0 = oracle.OracleCase(case)
    _assemble(oc0, kind, tflag)
    _assemble(ctx, kind, tflag, F.OVS_FP64)
    g0, r0 = _gpu_system(ctx, kind, tflag, F.OVS_FP64), oc0.system(kind)
    seen = 0.0
    for k in g1:
        seen = max(seen, _face_part_close(g1[k], g0[k], r1[k], r0[k], f"{kind}.{k}"))
    assert seen > 0.0   # the faces contributed
    ctx.close()


@pytest.mark.parametrize("kind", ["ns", "nsvof", "tem"])
def test_face_assembly_fp32(oracle, kind):
    case = _case(kind, 2)
    oc = oracle.OracleCase(case)
    ctx = Context.from_case(case)
    _assemble(oc, kind, 6)
    _assemble(ctx, kind, 6, F.OVS_FP32)
    _compare_system(oc, ctx, SYSID[kind], kind, 6, F.OVS_FP32, 1e-5)
    ctx.close()


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_face_assembly_deterministic(kind):
    case = _case(kind, 3)
    ctx = Context.from_case(case)
    for prec in (F.OVS_FP64, F.OVS_FP32):
        _assemble(ctx, kind, 6, prec)
        a = _gpu_system(ctx, kind, 6, prec)
        _assemble(ctx, kind, 6, prec)
        b = _gpu_system(ctx, kind, 6, prec)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
    ctx.close()


def test_set_faces_argument_checks():
    case = M.random_case(nx=3, ny=3, nz=2, seed=4)
    bf = M.face_set(case.mesh, weak=(1,), convective={2: (1.0, 300.0)})
    ctx = Context.from_case(case)
    lib, h = ctx.lib, ctx.h
    import ctypes as C

    def call(f2e, fo, fl, hc=None, ti=None):
        n = len(f2e)
        a = [np.ascontiguousarray(x, dtype=np.int32) for x in (f2e, fo, fl)]
        ip = [x.ctypes.data_as(C.POINTER(C.c_int)) for x in a]
        dp = [None if x is None else np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
              for x in (hc, ti)]
        return lib.ovs_set_faces(h, n, ip[0], ip[1], ip[2], dp[0], dp[1])

    one = np.ones(1)
    assert call([0], [1], [1]) == F.OVS_ERR_ARG                      # element ids are 1-based
    assert call([case.mesh.nelem + 1], [1], [1]) == F.OVS_ERR_ARG
    assert call([1], [5], [1]) == F.OVS_ERR_ARG                      # FACE_OR 1..4
    assert call([1], [1], [8]) == F.OVS_ERR_ARG                      # unknown flag
    assert call([1], [1], [F.OVS_FACE_CONVH]) == F.OVS_ERR_ARG       # h and T_inf required
    assert call([1], [1], [F.OVS_FACE_CONVH], one, one) == F.OVS_OK
    ctx.set_faces(bf)
    cot = np.zeros((case.mesh.nnode, 5))
    with pytest.raises(F.OvsError) as ei:
        ctx.residual_vjp(F.OVS_ASM_NSVOF, cot)
    assert ei.value.status == F.OVS_ERR_STATE
    ctx.set_faces(None)
    ctx.residual_vjp(F.OVS_ASM_NSVOF, cot)
    ctx.close()
    hexc = M.random_case(nx=2, ny=2, nz=2, seed=1, hex=True)
    hctx = Context.from_case(hexc)
    one_i = np.ones(1, dtype=np.int32)
    ip = one_i.ctypes.data_as(C.POINTER(C.c_int))
    assert hctx.lib.ovs_set_faces(hctx.h, 1, ip, ip, ip, None, None) == F.OVS_ERR_ARG
    hctx.close()


def test_weak_wall_cavity_refined_solve():
    """Lid-driven cavity with every wall weak (Nitsche): the lid moves through
    the wall velocity g = u_mesh on its nodes; pressure pinned at one node.
    The assembled NS system reaches a true relative residual of 1e-8 in the
    mixed-precision refined solve."""
    case = M.config1(n=10)
    m = case.mesh
    N = m.nnode
    case.ibc[:, :] = 0
    case.ibc[0, 3] = 1
    for n in ("ugm", "ugmold"):
        case.state[n][:] = 0.0
        case.state[n][m.faces[5], 0] = 1.0
    case.bfaces = M.face_set(m, weak=(1, 2, 3, 4, 5, 6))
    ctx = Context.from_case(case)
    for prec in (F.OVS_FP32, F.OVS_FP64):
        ctx.assemble(F.OVS_ASM_NS, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, prec)
    rhs = ctx.get_rhs(F.OVS_SYS_NS, F.OVS_FP64)
    assert np.abs(rhs[m.faces[5], 0]).max() > 0.0
    sol, info = ctx.solve(F.OVS_SYS_NS, F.OVS_FP32, 1e-8, kspace=100, max_cycles=200)
    assert info.converged and info.rel_residual <= 1e-8, (info.rel_residual, info.cycles)
    assert N == sol.shape[0]
    ctx.close()
