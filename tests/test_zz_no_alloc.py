"""The allocation-free GMRES entry point against the context-based one.

ovs_gmres_tem_noalloc serves callers that cannot allocate device memory at
solve time (code inside a framework's memory pool, time-critical loops,
plug-in hosts): they pass their own device buffers and the solver keeps its
temporaries in a fixed array inside the library.  Here it solves the same
temperature system as ovs_gmres (OVS_SYS_TEM) twice in a row, through the C
ABI, and both results must match the context-based solve within the GMRES
tolerance of the other tests (1e-10 normwise, same iteration count).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("dims", [(8, 6, 5), (16, 12, 10)], ids=["n378", "n2431"])
def test_noalloc_matches_context_gmres_on_two_calls(dims):
    """Two calls in a row against ovs_gmres; the larger case (2,431
    unknowns) runs every strided loop of the 1024-thread block more than
    twice.  After the first call, a call changes neither the device's free
    memory nor torch's allocations."""
    import torch
    from oversetdevfort_b200 import _ffi as F
    from oversetdevfort_b200 import mesh as M
    from oversetdevfort_b200.api import Context

    case = M.random_case(nx=dims[0], ny=dims[1], nz=dims[2], seed=31, kernel=F.OVS_ASM_TEM)
    ctx = Context.from_case(case)
    ctx.assemble(F.OVS_ASM_TEM, F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, F.OVS_FP64)
    N = ctx.N
    col, row = ctx.get_pattern()
    vals = ctx.get_lhs(F.OVS_SYS_TEM, F.OVS_FP64, F.OVS_BLK_TEM)
    rhs = ctx.get_rhs(F.OVS_SYS_TEM)[:, 0]
    tol, kspace, kmin = 1e-10, 40, 1
    ref, info_ref = ctx.gmres(F.OVS_SYS_TEM, tol, kspace, kmin, np.zeros((N, 1)))
    ref = ref[:, 0]
    ctx.close()

    dev = torch.device("cuda:0")
    d_rowptr = torch.tensor(col - 1, dtype=torch.int32, device=dev)
    d_colidx = torch.tensor(row - 1, dtype=torch.int32, device=dev)
    d_vals = torch.tensor(vals, dtype=torch.float64, device=dev)
    d_rhs = torch.tensor(rhs, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    lib = F.load()
    sols = [torch.zeros(N, dtype=torch.float64, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    mem = []
    for call in range(2):
        d_sol = sols[call]
        info = F.OvsGmresInfo()
        st = lib.ovs_gmres_tem_noalloc(N, _ptr(d_rowptr), _ptr(d_colidx), _ptr(d_vals), _ptr(d_rhs),
                                       _ptr(d_sol), tol, kspace, kmin, None, ctypes.byref(info))
        assert st == F.OVS_OK, (call, st)
        torch.cuda.synchronize()
        mem.append((torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)))
        sol = d_sol.cpu().numpy()
        assert info.iterations == info_ref.iterations, (call, info.iterations, info_ref.iterations)
        err = np.abs(sol - ref).max() / np.abs(ref).max()
        assert err <= 1e-10, (call, err)
        assert abs(info.res0 - info_ref.res0) <= 1e-12 * info_ref.res0

    assert mem[1] == mem[0], mem          # the second call allocated nothing

    # requests beyond the fixed scratch are refused with a clear status
    d_sol = torch.zeros(N, dtype=torch.float64, device=dev)
    st = lib.ovs_gmres_tem_noalloc(F.OVS_NOALLOC_MAX_N + 1, _ptr(d_rowptr), _ptr(d_colidx), _ptr(d_vals),
                                   _ptr(d_rhs), _ptr(d_sol), tol, kspace, kmin, None, None)
    assert st == F.OVS_ERR_ARG
    st = lib.ovs_gmres_tem_noalloc(N, _ptr(d_rowptr), _ptr(d_colidx), _ptr(d_vals), _ptr(d_rhs), _ptr(d_sol),
                                   tol, F.OVS_NOALLOC_MAX_KSPACE + 1, kmin, None, None)
    assert st == F.OVS_ERR_ARG


def test_noalloc_zero_hessenberg_column_ends_the_cycle():
    """A right-hand side on a node whose row and column are zero (a zero
    diagonal: the Jacobi factor is 1): P^-1 A v_1 = 0, the first Hessenberg
    column is zero and the reference's rotation would be 0/0.  The cycle
    ends after no iteration with breakdown = 1 and the solution untouched."""
    import torch
    from oversetdevfort_b200 import _ffi as F

    dev = torch.device("cuda:0")
    # 3 unknowns; row/column 1 hold only a zero diagonal entry
    rowptr = torch.tensor([0, 2, 3, 5], dtype=torch.int32, device=dev)
    colidx = torch.tensor([0, 2, 1, 0, 2], dtype=torch.int32, device=dev)
    vals = torch.tensor([4.0, 1.0, 0.0, 1.0, 3.0], dtype=torch.float64, device=dev)
    rhs = torch.tensor([0.0, 2.0, 0.0], dtype=torch.float64, device=dev)
    sol = torch.full((3,), 7.0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    info = F.OvsGmresInfo()
    st = F.load().ovs_gmres_tem_noalloc(3, _ptr(rowptr), _ptr(colidx), _ptr(vals), _ptr(rhs), _ptr(sol), 1e-10,
                                        10, 1, None, ctypes.byref(info))
    assert st == F.OVS_OK
    assert info.iterations == 0 and info.breakdown == 1 and info.converged == 0
    assert info.res0 == 2.0 and np.isfinite(info.ercheck)
    assert sol.cpu().tolist() == [7.0, 7.0, 7.0]
