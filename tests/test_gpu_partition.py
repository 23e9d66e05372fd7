"""Sharded assembly on the GPU: each owner-computes partition assembled in
its own context (here one after another on one GPU) gives the owned rows
bit-identical to the single-context assembly, FP64 and FP32, tets and
hexahedra."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import partition as P
from oversetdevfort_b200.api import BLOCK_NAME, SYS_BLOCKS, Context

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("hexm", [False, True])
@pytest.mark.parametrize("prec", [F.OVS_FP64, F.OVS_FP32])
def test_partitioned_owned_rows_bit_identical(hexm, prec):
    case = M.random_case(nx=6, ny=4, nz=3, seed=13, hex=hexm)
    g = Context.from_case(case)
    gcol, grow = g.get_pattern()
    gcol = gcol.astype(np.int64) - 1
    out = {}
    for kernel, sysid in ((F.OVS_ASM_NSVOF, F.OVS_SYS_NSVOF), (F.OVS_ASM_TEM, F.OVS_SYS_TEM)):
        g.assemble(kernel, 6, prec)
        out[sysid] = g.get_system(sysid, prec)
    g.close()
    for part in P.make_parts(case.mesh, 3):
        ctx = Context.from_case(P.local_case(case, part))
        col, row = ctx.get_pattern()
        for kernel, sysid in ((F.OVS_ASM_NSVOF, F.OVS_SYS_NSVOF), (F.OVS_ASM_TEM, F.OVS_SYS_TEM)):
            ctx.assemble(kernel, 6, prec)
            loc = ctx.get_system(sysid, prec)
            for b in SYS_BLOCKS[sysid]:
                name = BLOCK_NAME[b]
                rp, gcols, vals = P.owned_rows(col, row, loc[name], part)
                for i, A in enumerate(part.global_rows):
                    a, e = gcol[A], gcol[A + 1]
                    np.testing.assert_array_equal(gcols[rp[i]:rp[i + 1]], grow[a:e] - 1)
                    np.testing.assert_array_equal(vals[rp[i]:rp[i + 1]], out[sysid][name][a:e])
            np.testing.assert_array_equal(loc["rhs"][part.owned], out[sysid]["rhs"][part.global_rows])
        ctx.close()
