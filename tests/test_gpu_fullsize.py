"""The full config-3 workload (128^3 cells x6 Kuhn tets: 12,582,912 tets,
2,146,689 nodes, 31,802,497 CSR slots) through the C ABI against the oracle
at full size: the pattern and the element-slot -> CSR-slot map bit for bit,
and one FP64 assembly of the NS+VOF and temperature systems (every block and
right-hand side, 1e-12 normwise) - the large-index paths (offsets past 2^31
bytes) and the one-byte slot map on every row.  About a minute of oracle
time on one core."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context, SYS_BLOCKS, BLOCK_NAME

pytestmark = pytest.mark.gpu


def _close(gpu, ref, tol, what):
    scale = max(float(np.abs(ref).max(initial=0.0)), 1e-300)
    err = float(np.abs(gpu - ref).max(initial=0.0))
    assert err <= tol * scale, f"{what}: {err:.3e} vs scale {scale:.3e}"


def test_config3_pattern_slots_and_fp64_assembly(oracle):
    case = M.config3(128)
    m = case.mesh
    assert (m.nelem, m.nnode) == (12582912, 2146689)
    ctx = Context.from_case(case)
    col, row = ctx.get_pattern()
    assert len(row) == 31802497 == M.expected_nnz_kuhn(128, 128, 128)
    ctx.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
    gsys = {"nsvof": {BLOCK_NAME[b]: ctx.get_lhs(F.OVS_SYS_NSVOF, F.OVS_FP64, b) for b in SYS_BLOCKS[F.OVS_SYS_NSVOF]}}
    gsys["nsvof"]["rhs"] = ctx.get_rhs(F.OVS_SYS_NSVOF, F.OVS_FP64)
    ctx.assemble(F.OVS_ASM_TEM, 6, F.OVS_FP64)
    gsys["tem"] = {"TEM": ctx.get_lhs(F.OVS_SYS_TEM, F.OVS_FP64, F.OVS_BLK_TEM),
                   "rhs": ctx.get_rhs(F.OVS_SYS_TEM, F.OVS_FP64)}
    lmap = ctx.get_slot_map()
    ctx.close()

    col_o, row_o = oracle.gen_spar_struc(m.ien, m.nnode)
    np.testing.assert_array_equal(col, col_o)
    np.testing.assert_array_equal(row, row_o)
    del row_o
    np.testing.assert_array_equal(lmap, oracle.slot_map(m.ien, col, row))
    del lmap

    oc = oracle.OracleCase(case)
    oc.assemble_quenching(6, 3)
    ref = oc.system("nsvof")
    for name, g in gsys["nsvof"].items():
        if name == "rhs":
            for f in range(g.shape[1]):
                _close(g[:, f], ref["rhs"][:, f], 1e-12, f"nsvof.rhs[{f}]")
        else:
            _close(g, ref[name], 1e-12, f"nsvof.{name}")
    del ref, gsys["nsvof"]
    oc.assemble_quenching(6, 4)
    _close(gsys["tem"]["TEM"], oc.sys["TEM"], 1e-12, "tem.TEM")
    _close(gsys["tem"]["rhs"][:, 0], oc.sys["rhstem"], 1e-12, "tem.rhs")
