"""setBCs_NSVOF / setBCs_Tem in the oracle (CPU): IBC from NodeID 101,
Dirichlet values and the rates ((v - vold)/Delt + (gami - 1) rate_old)/gami,
later boundaries winning on shared nodes, and the reference's mix of
FACE_ID-indexed types with boundary-indexed values."""
import numpy as np

from oversetdevfort_b200 import mesh as M


def _case():
    m = M.box_tet(3, 2, 2)
    rng = np.random.default_rng(7)
    N = m.nnode
    st = M.empty_state(N)
    for k, a in st.items():
        a[...] = rng.standard_normal(a.shape)
    ibc = np.asfortranarray(rng.integers(0, 2, size=(N, 8)).astype(np.int32))
    return M.Case("bc", m, M.base_params(delt=0.01), st, ibc, 2)


def _rate(v, vold, rold, p):
    return ((v - vold) * (1.0 / p["delt"]) + (p["gami"] - 1.0) * rold) / p["gami"]


def test_set_bcs_known_answers(oracle):
    case = _case()
    m, p = case.mesh, case.params
    nid = np.zeros(m.nnode, np.int32)
    nid[[0, 5]] = 101
    spec = M.box_bc_spec(m, u={1: (0.0, 0.0, 0.0), 6: (1.0, None, 0.0)}, phi={5: 1.0}, T={5: 400.0, 6: 300.0},
                         node_id=nid)
    oc = oracle.OracleCase(case)
    old = {k: v.copy() for k, v in oc.state_arrays.items()}
    oc.set_bcs(spec, 3)
    ibc, s = oc.ibc, oc.state_arrays
    top, x0, bot = m.faces[5], m.faces[0], m.faces[4]
    assert np.all(ibc[:, 6:] == 0) and np.all(ibc[[0, 5], :5] == 1)
    assert np.all(ibc[x0, :3] == 1) and np.all(ibc[top, 0] == 1) and np.all(ibc[top, 2] == 1)
    free = np.setdiff1d(np.arange(m.nnode), np.concatenate([x0, top, [0, 5]]))
    assert np.all(ibc[free, :3] == 0) and np.all(ibc[free, 3] == 0)
    np.testing.assert_array_equal(s["ug"][top, 0], 1.0)                 # the lid wins on the shared edge
    np.testing.assert_array_equal(s["ug"][np.setdiff1d(x0, top), 0], 0.0)
    np.testing.assert_array_equal(s["acg"][top, 0], _rate(1.0, old["ugold"][top, 0], old["acgold"][top, 0], p))
    np.testing.assert_array_equal(s["ug"][np.setdiff1d(top, x0), 1], old["ug"][np.setdiff1d(top, x0), 1])
    np.testing.assert_array_equal(s["phig"][bot], 1.0)
    np.testing.assert_array_equal(ibc[bot, 4], 1)
    np.testing.assert_array_equal(s["tg"][top], 300.0)
    np.testing.assert_array_equal(s["tg"][np.setdiff1d(bot, top)], 400.0)
    np.testing.assert_array_equal(s["rtg"][top], _rate(300.0, old["tgold"][top], old["rtgold"][top], p))
    np.testing.assert_array_equal(ibc[np.union1d(bot, top), 5], 1)


def test_set_bcs_face_id_and_boundary_indexing(oracle):
    """Types by FACE_ID, values by boundary number (src/setBCs.f90:212-216)."""
    case = _case()
    m = case.mesh
    spec = M.BcSpec(face_id=np.array([2, 1], np.int32),
                    bnodes=[(np.asarray(m.faces[0]) + 1).astype(np.int32), (np.asarray(m.faces[1]) + 1).astype(np.int32)],
                    bcug_type=np.array([[1, 0, 0], [0, 1, 0]], np.int32),
                    bcug_valu=np.array([[5.0, 6.0, 7.0], [8.0, 9.0, 10.0]]),
                    bcphig_type=np.zeros(2, np.int32), bcphig_valu=np.zeros(2),
                    bctg_type=np.array([0, 1], np.int32), bctg_valu=np.array([111.0, 222.0]))
    oc = oracle.OracleCase(case)
    old_ug = oc.state_arrays["ug"].copy()
    oc.set_bcs(spec, 3)
    s, ibc = oc.state_arrays, oc.ibc
    x0, x1 = m.faces[0], m.faces[1]
    # boundary 1 (x0 nodes, FACE_ID 2): type row 2 -> y component, value row 1 -> 6
    np.testing.assert_array_equal(s["ug"][x0, 1], 6.0)
    np.testing.assert_array_equal(s["ug"][x0, 0], old_ug[x0, 0])
    # boundary 2 (x1 nodes, FACE_ID 1): type row 1 -> x component, value row 2 -> 8
    np.testing.assert_array_equal(s["ug"][x1, 0], 8.0)
    np.testing.assert_array_equal(ibc[x0, 1], 1)
    np.testing.assert_array_equal(ibc[x1, 0], 1)
    # T: type row 2 (FACE_ID 2) is Dirichlet -> boundary 1 with value 111
    np.testing.assert_array_equal(s["tg"][x0], 111.0)
    np.testing.assert_array_equal(ibc[x1, 5], 0)


def test_bc_spec_checks_without_a_device(lib):
    """ovs_check_bc_spec, the checks ovs_set_bc_spec makes, on the host:
    the box spec passes (boundaries sharing edge nodes are fine); a FACE_ID
    beyond the type tables, a node id outside 1..N, a node twice in one
    boundary, offsets not starting at 0 and a missing table are rejected."""
    import ctypes as C
    from oversetdevfort_b200 import _ffi as F
    from oversetdevfort_b200 import api
    m = M.box_tet(3, 2, 2)
    good = M.box_bc_spec(m, u={1: (0.0, 0.0, 0.0), 6: (1.0, None, 0.0)}, phi={5: 1.0}, T={5: 300.0},
                         face_ids=(2, 1, 3, 4, 6, 5))
    assert api.check_bc_spec(good, m.nnode) == F.OVS_OK
    assert api.check_bc_spec(good, m.nnode - 1) == F.OVS_ERR_ARG      # the last node is out of range
    bad_fid = M.box_bc_spec(m)
    bad_fid.face_id = bad_fid.face_id.copy()
    bad_fid.face_id[0] = 7
    assert api.check_bc_spec(bad_fid, m.nnode) == F.OVS_ERR_ARG
    bad_node = M.box_bc_spec(m)
    bad_node.bnodes = [b.copy() for b in bad_node.bnodes]
    bad_node.bnodes[2][0] = 0
    assert api.check_bc_spec(bad_node, m.nnode) == F.OVS_ERR_ARG
    dup = M.box_bc_spec(m)
    dup.bnodes = [b.copy() for b in dup.bnodes]
    dup.bnodes[3][1] = dup.bnodes[3][0]
    assert api.check_bc_spec(dup, m.nnode) == F.OVS_ERR_ARG
    keep, cs = good.to_c()
    keep["ptr"][0] = 1                                                # offsets must start at 0
    assert lib.ovs_check_bc_spec(C.byref(cs), m.nnode) == F.OVS_ERR_ARG
    keep, cs = good.to_c()
    cs.bctg_type = None                                               # a missing table
    assert lib.ovs_check_bc_spec(C.byref(cs), m.nnode) == F.OVS_ERR_ARG
    assert lib.ovs_check_bc_spec(None, m.nnode) == F.OVS_ERR_ARG
    empty = M.BcSpec(np.zeros(0, np.int32), [], np.zeros((0, 3), np.int32), np.zeros((0, 3)), np.zeros(0, np.int32),
                     np.zeros(0), np.zeros(0, np.int32), np.zeros(0), None)
    assert api.check_bc_spec(empty, m.nnode) == F.OVS_OK              # no boundaries
