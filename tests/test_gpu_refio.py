"""The reference's on-disk inputs through the GPU path: a partition mesh
(part.<id>.dat, input_mesh src/input.f90:15-214) and a restart
(restart.<step>.<id>, readSol src/iosol.f90:122-194, with step.dat) are
written by refio, read back the way the driver starts a rank
(refio.load_rank, src/driver.f90:39-60) and assembled and solved through the
C ABI.  The text formats round-trip FP64 exactly, so the pattern, both
assembled systems and the GMRES solutions equal those of the same case held
in memory bit for bit."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import refio
from oversetdevfort_b200.api import Context

pytestmark = pytest.mark.gpu


def test_part_and_restart_files_assemble_and_solve_like_memory(tmp_path):
    case = M.quench_case(M.box_tet(6, 5, 7, 1.0, 0.8, 1.1), "refio_gpu")
    m = case.mesh
    rng = np.random.default_rng(11)
    # a state as writeSol leaves it: current fields plus the old temperatures
    written = {k: np.array(v, copy=True) for k, v in case.state.items()}
    free = np.asarray(case.ibc)[:, 0] == 0
    written["ug"][free] = 0.05 * rng.standard_normal((int(free.sum()), 3))
    written["acg"][:] = rng.standard_normal(written["acg"].shape)
    written["pg"][:] = rng.uniform(-1, 1, m.nnode)
    written["rphig"][:] = 0.1 * rng.standard_normal(m.nnode)
    written["rtgold"][:] = rng.standard_normal(m.nnode)
    rank, step = 2, 9
    refio.write_part(tmp_path / refio.part_name(rank + 1), refio.part_from_mesh(m))
    refio.write_restart(tmp_path / refio.restart_name(step, rank), step, 0.009, written)
    refio.write_step(tmp_path / "step.dat", step, 0.0)
    loaded, st, time, _ = refio.load_rank(tmp_path, rank, case.params)
    assert st == step and time == 0.009
    loaded.ibc[...] = case.ibc                       # setBCs' IBC, as in memory

    # the same start in memory: readSol's arrays are writeSol's, then the predictor
    arrays = {old: written[cur] for old, cur in zip(refio.RESTART_READ, refio.RESTART_WRITE)}
    mem = M.Case("memory", m, case.params, refio.state_from_restart(arrays, case.params["gami"]), case.ibc,
                 F.OVS_ASM_NSVOF)

    out = []
    for c in (loaded, mem):
        ctx = Context.from_case(c)
        col, row = ctx.get_pattern()
        ctx.assemble(F.OVS_ASM_NSVOF, 6, F.OVS_FP64)
        ctx.assemble(F.OVS_ASM_TEM, 6, F.OVS_FP64)
        sys_ns = ctx.get_system(F.OVS_SYS_NSVOF, F.OVS_FP64)
        sys_t = ctx.get_system(F.OVS_SYS_TEM, F.OVS_FP64)
        s_ns, i_ns = ctx.gmres(F.OVS_SYS_NSVOF, 1e-8, 100, 1, np.zeros((ctx.N, 5)))
        s_t, i_t = ctx.gmres(F.OVS_SYS_TEM, 1e-10, 60, 1, np.zeros((ctx.N, 1)))
        out.append((col, row, sys_ns, sys_t, s_ns, s_t, i_ns.iterations, i_t.iterations))
        ctx.close()
    a, b = out
    for x, y in zip(a[:2], b[:2]):
        np.testing.assert_array_equal(x, y)
    for d1, d2 in zip(a[2:4], b[2:4]):
        assert d1.keys() == d2.keys()
        for k in d1:
            np.testing.assert_array_equal(d1[k], d2[k])
    np.testing.assert_array_equal(a[4], b[4])
    np.testing.assert_array_equal(a[5], b[5])
    assert a[6:] == b[6:] and a[6] > 0
