"""setBCs_NSVOF / setBCs_Tem on the device (ovs_apply_bcs) against the
oracle, bit for bit on the state and IBC (random state, NodeID 101 nodes,
boundaries sharing edges, a permuted FACE_ID table, each `which`), the
argument checks of ovs_set_bc_spec, and the placement inside the device
Newton loop (the BCs a registered spec applies equal the same BCs applied
beforehand)."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context

pytestmark = pytest.mark.gpu

STATE = ("ug", "acg", "phig", "rphig", "tg", "rtg", "ugold", "acgold")


def _spec(m, seed):
    rng = np.random.default_rng(seed)
    nid = np.where(rng.random(m.nnode) < 0.05, 101, 0).astype(np.int32)
    u = {b: tuple(float(rng.uniform(-1, 1)) if rng.random() < 0.6 else None for _ in range(3)) for b in range(1, 7)}
    phi = {b: float(rng.uniform(0, 1)) for b in (2, 5) }
    T = {b: float(rng.uniform(300, 400)) for b in (1, 5, 6)}
    return M.box_bc_spec(m, u=u, phi=phi, T=T, node_id=nid, face_ids=(3, 1, 2, 6, 4, 5))


@pytest.mark.parametrize("which", [1, 2, 3])
@pytest.mark.parametrize("seed", [0, 1])
def test_apply_bcs_matches_oracle(oracle, which, seed):
    case = M.random_case(nx=4, ny=3, nz=3, seed=seed)
    spec = _spec(case.mesh, seed)
    ctx = Context.from_case(case)
    ctx.set_bc_spec(spec)
    ctx.apply_bcs(which)
    oc = oracle.OracleCase(case)
    oc.set_bcs(spec, which)
    for f in STATE:
        np.testing.assert_array_equal(ctx.get_field(f), oc.state_arrays[f], err_msg=f)
    np.testing.assert_array_equal(ctx.get_ibc(8), oc.ibc)
    ctx.close()


def test_bc_spec_argument_checks():
    case = M.random_case(nx=3, ny=2, nz=2, seed=3)
    ctx = Context.from_case(case)
    assert ctx.lib.ovs_apply_bcs(ctx.h, 3) == F.OVS_ERR_STATE          # nothing registered
    m = case.mesh
    good = M.box_bc_spec(m, u={1: (0.0, 0.0, 0.0)})
    bad_fid = M.box_bc_spec(m, u={1: (0.0, 0.0, 0.0)})
    bad_fid.face_id = bad_fid.face_id.copy()
    bad_fid.face_id[0] = 7                                                # beyond the type tables
    bad_node = M.box_bc_spec(m)
    bad_node.bnodes = [b.copy() for b in bad_node.bnodes]
    bad_node.bnodes[2][0] = m.nnode + 1
    dup = M.box_bc_spec(m)
    dup.bnodes = [b.copy() for b in dup.bnodes]
    dup.bnodes[3][1] = dup.bnodes[3][0]                                   # a node twice in one boundary
    for sp in (bad_fid, bad_node, dup):
        keep, cs = sp.to_c()
        import ctypes as C
        assert ctx.lib.ovs_set_bc_spec(ctx.h, C.byref(cs)) == F.OVS_ERR_ARG
    ctx.set_bc_spec(good)
    assert ctx.lib.ovs_apply_bcs(ctx.h, 0) == F.OVS_ERR_ARG
    assert ctx.lib.ovs_apply_bcs(ctx.h, 4) == F.OVS_ERR_ARG
    ctx.apply_bcs(3)
    ctx.set_bc_spec(None)
    assert ctx.lib.ovs_apply_bcs(ctx.h, 3) == F.OVS_ERR_STATE
    ctx.close()


def test_newton_applies_registered_bcs():
    """quench_newton with a registered spec equals the BCs applied first and
    the Newton loop run without a spec (one Newton iteration: the spec is
    applied before the first residual and again before the iteration, and
    both applications give the same state)."""
    case = M.quench_case(M.box_tet(6, 6, 8, 1.0, 1.0, 1.25), "bc6")
    m = case.mesh
    spec = M.box_bc_spec(m, u={b: (0.0, 0.0, 0.0) for b in range(1, 6)}, T={5: 380.0}, phi={6: 1.0})
    kw = dict(mode=F.OVS_FP64, newton_max=1, solve_tem=True, kspace=40, kspace_min=1, max_cycles=100,
              tol_ns=1e-6, tol_tem=1e-6, utol=(1e-4,) * 4, atol=(1e-30,) * 4)
    a = Context.from_case(case)
    a.set_bc_spec(spec)
    ia = a.quench_newton(**kw)
    b = Context.from_case(case)
    b.set_bc_spec(spec)
    b.apply_bcs(3)
    b.set_bc_spec(None)
    ib = b.quench_newton(**kw)
    for f in F.FIELDS:
        np.testing.assert_array_equal(a.get_field(f), b.get_field(f), err_msg=f)
    np.testing.assert_array_equal(a.get_ibc(), b.get_ibc())
    assert ia.krylov_iterations_ns == ib.krylov_iterations_ns > 0
    a.close()
    b.close()
