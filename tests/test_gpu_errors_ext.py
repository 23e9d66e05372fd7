"""Error statuses of the later entry points: the NS-only kernel and the
adjoint on a hex context, the transposed solve on a block system or before
the temperature matrix exists, and bad Newton-loop options."""
import ctypes as C

import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context

pytestmark = pytest.mark.gpu


def test_extension_error_statuses():
    hexc = Context.from_case(M.random_case(nx=2, ny=2, nz=2, seed=4, kernel=F.OVS_ASM_NSVOF, hex=True))
    cfl = C.c_double(0.0)
    assert hexc.lib.ovs_assemble(hexc.h, F.OVS_ASM_NS, 6, F.OVS_FP64, C.byref(cfl)) == F.OVS_ERR_ARG
    cot = np.zeros((hexc.N, 5))
    grad = np.zeros((hexc.N, F.OVS_VJP_COUNT))
    dp = C.POINTER(C.c_double)
    assert hexc.lib.ovs_residual_vjp(hexc.h, F.OVS_ASM_NSVOF, cot.ctypes.data_as(dp),
                                     grad.ctypes.data_as(dp)) == F.OVS_ERR_ARG
    hexc.close()

    ctx = Context.from_case(M.random_case(nx=3, ny=2, nz=2, seed=5, kernel=F.OVS_ASM_TEM))
    b = np.ones(ctx.N)
    x = np.zeros(ctx.N)
    info = F.OvsGmresInfo()
    st = ctx.lib.ovs_gmres_transposed(ctx.h, F.OVS_SYS_NSVOF, b.ctypes.data_as(dp), 1e-8, 20, 1,
                                      x.ctypes.data_as(dp), C.byref(info))
    assert st == F.OVS_ERR_ARG
    st = ctx.lib.ovs_gmres_transposed(ctx.h, F.OVS_SYS_TEM, b.ctypes.data_as(dp), 1e-8, 20, 1,
                                      x.ctypes.data_as(dp), C.byref(info))
    assert st == F.OVS_ERR_STATE   # no temperature matrix assembled yet
    g2 = np.zeros((ctx.N, F.OVS_VJP_COUNT))
    assert ctx.lib.ovs_residual_vjp(ctx.h, F.OVS_ASM_NS, b.ctypes.data_as(dp), g2.ctypes.data_as(dp)) == F.OVS_ERR_ARG
    o = F.OvsNewtonOpts(7, 1, 1, 30, 1, 10, 1e-6, 1e-6, (C.c_double * 4)(*[1e-3] * 4), (C.c_double * 4)(*[0.0] * 4))
    ni = F.OvsNewtonInfo()
    assert ctx.lib.ovs_quench_newton(ctx.h, C.byref(o), C.byref(ni)) == F.OVS_ERR_ARG
    o.mode, o.kspace = F.OVS_FP64, 0
    assert ctx.lib.ovs_quench_newton(ctx.h, C.byref(o), C.byref(ni)) == F.OVS_ERR_ARG
    ctx.close()
