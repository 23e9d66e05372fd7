"""Distributed GMRES on the GPU: owner-computes partitions of a quench box,
each with its own context and local assembly, the local products on the
package's CUDA kernels (ovs_spmv_device / ovs_precond_device), two and three
partitions in one process on one GPU (LocalComm; no kernel waits on
another), against the single-context reference GMRES cycle (ovs_gmres) of
the same system: the same iteration count, the same solution to 1e-10."""
import numpy as np
import pytest
import torch

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import distributed as D
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import partition as P
from oversetdevfort_b200.api import Context

pytestmark = pytest.mark.gpu

SYS = {"nsvof": (F.OVS_SYS_NSVOF, F.OVS_ASM_NSVOF, 5), "tem": (F.OVS_SYS_TEM, F.OVS_ASM_TEM, 1)}


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_gmres_matches_one_context(kind, nparts):
    sysid, kern, nf = SYS[kind]
    case = M.quench_case(M.box_tet(10, 8, 12, 1.0, 1.0, 1.25), "dist_gpu")
    tol, kspace = 1e-8, 200
    g = Context.from_case(case)
    g.assemble(kern, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    sg, ig = g.gmres(sysid, tol, kspace, 1, np.zeros((case.mesh.nnode, nf)))
    assert ig.converged and np.isfinite(sg).all()
    g.close()
    parts = P.make_parts(case.mesh, nparts)
    plan = D.halo_plan(parts)
    ctxs, ops, rhs = [], {}, {}
    for r, p in enumerate(parts):
        c = Context.from_case(P.local_case(case, p))
        c.assemble(kern, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
        ctxs.append(c)
        ops[r] = D.DeviceOperator(c, sysid)
        rhs[r] = torch.as_tensor(np.ascontiguousarray(c.get_rhs(sysid, F.OVS_FP64).T), device="cuda:0")
    sol, info = D.gmres_cycle(D.LocalComm(plan), ops, rhs, tol, kspace, 1, tem=kind == "tem")
    assert info["converged"] and info["iterations"] == ig.iterations
    scale = np.abs(sg).max()
    for r, p in enumerate(parts):
        s = sol[r].cpu().numpy().T
        assert np.isfinite(s).all()
        np.testing.assert_allclose(s, sg[p.nodes], atol=1e-10 * scale, rtol=0)
    for c in ctxs:
        c.close()


def test_device_products_match_host_products():
    """ovs_spmv_device (plain and preconditioned) and ovs_precond_device on
    device vectors against ovs_spmv on host vectors and the preconditioned
    product composed from them."""
    case = M.quench_case(M.box_tet(6, 6, 8, 1.0, 1.0, 1.25), "dev_prod")
    c = Context.from_case(case)
    c.assemble(F.OVS_ASM_NSVOF, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    N = case.mesh.nnode
    x = np.random.default_rng(1).standard_normal((N, 5))
    host = c.spmv(F.OVS_SYS_NSVOF, F.OVS_FP64, x)
    op = D.DeviceOperator(c, F.OVS_SYS_NSVOF)
    xd = torch.as_tensor(np.ascontiguousarray(x.T), device="cuda:0")
    yd = torch.empty_like(xd)
    torch.cuda.synchronize()
    F.check(c.lib.ovs_spmv_device(c.h, F.OVS_SYS_NSVOF, F.OVS_FP64, 0, xd.data_ptr(), yd.data_ptr()), "spmv")
    np.testing.assert_allclose(yd.cpu().numpy().T, host, rtol=0, atol=1e-13 * np.abs(host).max())
    ad = torch.as_tensor(np.ascontiguousarray(host.T), device="cuda:0")
    pd, qd = torch.empty_like(xd), torch.empty_like(xd)
    op.precond(ad, pd)
    op.matvec(xd, qd)
    np.testing.assert_allclose(qd.cpu().numpy(), pd.cpu().numpy(), rtol=0, atol=1e-12 * pd.abs().max().item())
    assert c.lib.ovs_spmv_device(c.h, F.OVS_SYS_NSVOF, F.OVS_FP64, 4, xd.data_ptr(), yd.data_ptr()) == F.OVS_ERR_ARG
    c.close()


def test_row_list_products_match_the_full_product():
    """ovs_spmv_device_rows on a partition's interior and boundary rows
    (split_rows): every listed row equals the full product's bit for bit,
    the unlisted rows keep what they held, an index outside [0, N) is
    skipped; plain and preconditioned, NS+VOF and T, FP64 and FP32 values."""
    case = M.quench_case(M.box_tet(8, 7, 10, 1.0, 1.0, 1.25), "rows_prod")
    parts = P.make_parts(case.mesh, 3)
    p = parts[1]
    c = Context.from_case(P.local_case(case, p))
    n = p.nodes.size
    col, row = c.get_pattern()
    inner, bnd = D.split_rows(col, row, p.owned, n)
    assert inner.size > 0 and bnd.size > 0
    rng = np.random.default_rng(4)
    for kern, sysid, nf in ((F.OVS_ASM_NSVOF, F.OVS_SYS_NSVOF, 5), (F.OVS_ASM_TEM, F.OVS_SYS_TEM, 1)):
        for prec in (F.OVS_FP64, F.OVS_FP32):
            c.assemble(kern, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, prec)
            F.check(c.lib.ovs_build_precond(c.h, sysid, prec), "precond")
            xd = torch.as_tensor(rng.standard_normal((nf, n)), device="cuda:0")
            for flags in (0, F.OVS_SPMV_PRECOND):
                full = torch.empty_like(xd)
                torch.cuda.synchronize()
                F.check(c.lib.ovs_spmv_device(c.h, sysid, prec, flags, xd.data_ptr(), full.data_ptr()), "full")
                part = torch.full_like(xd, -3.5)
                for rows in (inner, bnd):
                    rd = torch.as_tensor(rows.astype(np.int32), device="cuda:0")
                    F.check(c.lib.ovs_spmv_device_rows(c.h, sysid, prec, flags, xd.data_ptr(), part.data_ptr(),
                                                       rd.data_ptr(), int(rd.numel())), "rows")
                own = torch.as_tensor(np.sort(np.asarray(p.owned)), device="cuda:0")
                assert torch.equal(part[:, own], full[:, own])
                ghost = torch.as_tensor(np.setdiff1d(np.arange(n), p.owned), device="cuda:0")
                assert bool((part[:, ghost] == -3.5).all())
    # an index outside [0, N) is skipped, nrows = 0 does nothing, bad arguments are refused
    y = torch.full_like(xd, 2.0)
    bad = torch.as_tensor(np.array([-1, n, n + 7], dtype=np.int32), device="cuda:0")
    F.check(c.lib.ovs_spmv_device_rows(c.h, F.OVS_SYS_TEM, F.OVS_FP32, 0, xd.data_ptr(), y.data_ptr(),
                                       bad.data_ptr(), 3), "skipped")
    F.check(c.lib.ovs_spmv_device_rows(c.h, F.OVS_SYS_TEM, F.OVS_FP32, 0, xd.data_ptr(), y.data_ptr(), 0, 0), "none")
    assert bool((y == 2.0).all())
    assert c.lib.ovs_spmv_device_rows(c.h, F.OVS_SYS_TEM, F.OVS_FP32, 0, xd.data_ptr(), y.data_ptr(),
                                      bad.data_ptr(), -1) == F.OVS_ERR_ARG
    assert c.lib.ovs_spmv_device_rows(c.h, F.OVS_SYS_TEM, F.OVS_FP32, 0, xd.data_ptr(), y.data_ptr(), 0, 3) == F.OVS_ERR_ARG
    assert c.lib.ovs_spmv_device_rows(c.h, F.OVS_SYS_TEM, F.OVS_FP32, 8, xd.data_ptr(), y.data_ptr(),
                                      bad.data_ptr(), 3) == F.OVS_ERR_ARG
    c.close()


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_overlapped_partitioned_gmres_is_the_same_cycle(kind):
    """The partitioned cycle with the product split around the halo exchange
    (interior rows, exchange, boundary rows) against the product taken
    whole after the exchange: the same iterations, the same solution bit
    for bit, on three partitions with the CUDA products."""
    sysid, kern, nf = SYS[kind]
    case = M.quench_case(M.box_tet(10, 8, 12, 1.0, 1.0, 1.25), "dist_gpu_ov")
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ctxs, ops, rhs = [], {}, {}
    for r, p in enumerate(parts):
        c = Context.from_case(P.local_case(case, p))
        c.assemble(kern, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
        ctxs.append(c)
        ops[r] = D.DeviceOperator(c, sysid)
        rhs[r] = torch.as_tensor(np.ascontiguousarray(c.get_rhs(sysid, F.OVS_FP64).T), device="cuda:0")
    (s1, i1), (s2, i2) = [D.gmres_cycle(D.LocalComm(plan), ops, rhs, 1e-8, 200, 1, tem=kind == "tem", overlap=ov)
                          for ov in (True, False)]
    assert i1["converged"] and i1["iterations"] == i2["iterations"]
    for r in s1:
        assert torch.equal(s1[r], s2[r])
    for c in ctxs:
        c.close()
