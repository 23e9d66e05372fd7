"""The reference's mesh and restart files (oversetdevfort_b200.refio): round
trips of box meshes through part.dat (the CSR pattern of the read mesh is
the original's, by the oracle's genSparStruc), the non-FEM and NURBS
branches of input_mesh on a hand-written file, and restart round trips
including writeSol's old-temperature quirk.  CPU only."""
import numpy as np
import pytest

from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import refio


@pytest.mark.parametrize("mk", [lambda: M.box_tet(3, 2, 2, 1.0, 0.5, 2.0), lambda: M.box_hex(2, 3, 2)])
def test_part_round_trip_and_pattern(tmp_path, oracle, mk):
    m = mk()
    m.elm_id[::3] = 101
    pm = refio.part_from_mesh(m)
    pm.node_id[:] = np.arange(m.nnode) % 5
    path = tmp_path / "part1.dat"
    refio.write_part(path, pm)
    back = refio.read_part(path)
    np.testing.assert_array_equal(back.xg, m.xg)
    np.testing.assert_array_equal(back.ien, m.ien)
    np.testing.assert_array_equal(back.elm_id, m.elm_id)
    np.testing.assert_array_equal(back.node_id, pm.node_id)
    m2 = refio.mesh_from_part(back)
    for a, b in zip(m2.faces, m.faces):
        np.testing.assert_array_equal(a, b)
    c1, r1 = oracle.gen_spar_struc(m.ien, m.nnode)
    c2, r2 = oracle.gen_spar_struc(m2.ien, m2.nnode)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(r1, r2)


def test_part_non_fem_and_nurbs_records(tmp_path):
    # one tet with one boundary and NURBS data: every branch of input_mesh
    text = """3 4 3
4 1 1 1
0.0 0.0 0.0
1.0D0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
4 1 2 3 4
7 1 3
3 1 2 3
1 4
1
2
3
1.0
0.5D0
1.0
1.0
1 0 0 0
"""
    path = tmp_path / "part2.dat"
    path.write_text(text)
    pm = refio.read_part(path, fem_flag=0)
    assert (pm.nsd, pm.nshl, pm.nshlb_max) == (3, 4, 3)
    assert pm.xg[1, 0] == 1.0 and pm.ien.tolist() == [[1, 2, 3, 4]]
    b = pm.bounds[0]
    assert b.face_id == 7 and b.nshlb.tolist() == [3] and b.face_ien.tolist() == [[1, 2, 3]]
    assert b.f2e.tolist() == [1] and b.face_or.tolist() == [4] and b.bnodes.tolist() == [1, 2, 3]
    assert pm.wg.tolist() == [1.0, 0.5, 1.0, 1.0] and pm.epid.tolist() == [1] and pm.eijk.tolist() == [[0, 0, 0]]
    back = tmp_path / "part3.dat"
    refio.write_part(back, pm, fem_flag=0)
    pm2 = refio.read_part(back, fem_flag=0)
    np.testing.assert_array_equal(pm2.xg, pm.xg)
    np.testing.assert_array_equal(pm2.wg, pm.wg)
    assert pm2.bounds[0].nshlb.tolist() == [3]


def test_restart_round_trip_and_predictor(tmp_path):
    rng = np.random.default_rng(3)
    N = 17
    st = M.empty_state(N)
    for k, a in st.items():
        a[...] = rng.standard_normal(a.shape)
    path = tmp_path / "restart1"
    refio.write_restart(path, 12, 0.125, st)
    step, time, arr = refio.read_restart(path, N)
    assert step == 12 and time == 0.125
    # writeSol stores the current fields but the OLD temperature arrays;
    # readSol puts every record into the *old fields
    for rd, wr in zip(refio.RESTART_READ, refio.RESTART_WRITE):
        np.testing.assert_array_equal(arr[rd], st[wr])
    s2 = refio.state_from_restart(arr, gami=0.8)
    np.testing.assert_array_equal(s2["ug"], st["ug"])
    np.testing.assert_array_equal(s2["pg"], st["pg"])
    np.testing.assert_allclose(s2["acg"], (0.8 - 1.0) / 0.8 * st["acg"])
    np.testing.assert_array_equal(s2["tg"], st["tgold"])


def test_part_faces_round_trip_to_face_set(tmp_path):
    """Boundary triangles written to part.dat (FACE_IEN, F2E, FACE_OR) come
    back as the same face set the box enumeration gives, in file order."""
    m = M.box_tet(3, 2, 2, 1.0, 0.5, 2.0)
    pm = refio.part_from_mesh(m)
    path = tmp_path / "part4.dat"
    refio.write_part(path, pm)
    back = refio.read_part(path)
    for b, nodes in zip(back.bounds, m.faces):
        assert np.isin(b.face_ien - 1, nodes).all()
    bf = refio.faces_from_part(back, weak=(2, 6), convective={5: (4.0, 300.0)})
    ref = M.face_set(m, weak=(2, 6), convective={5: (4.0, 300.0)})
    for a, b in zip((bf.f2e, bf.face_or, bf.flags, bf.hconv, bf.tinf),
                    (ref.f2e, ref.face_or, ref.flags, ref.hconv, ref.tinf)):
        np.testing.assert_array_equal(a, b)


def test_bc_spec_from_part_drives_setbcs_like_the_box_spec(tmp_path, oracle):
    """setBCs on a mesh read back from part.dat, with the boundaries and
    NodeID of the file, gives the state and IBC of the same BCs given on the
    box mesh directly."""
    m = M.box_tet(3, 2, 2, 1.0, 0.5, 2.0)
    pm = refio.part_from_mesh(m)
    pm.node_id[:] = 0
    pm.node_id[[1, 7]] = 101
    path = tmp_path / "part5.dat"
    refio.write_part(path, pm)
    back = refio.read_part(path)
    ut = np.zeros((6, 3), np.int32)
    uv = np.zeros((6, 3))
    ut[5] = (1, 0, 1)
    uv[5] = (1.0, 0.0, -0.5)
    ut[0] = (1, 1, 1)
    pt, pv = np.zeros(6, np.int32), np.zeros(6)
    pt[4], pv[4] = 1, 1.0
    tt, tv = np.zeros(6, np.int32), np.zeros(6)
    tt[4], tv[4] = 1, 420.0
    spec_file = refio.bc_spec_from_part(back, ut, uv, pt, pv, tt, tv)
    spec_box = M.box_bc_spec(m, u={6: (1.0, None, -0.5), 1: (0.0, 0.0, 0.0)}, phi={5: 1.0}, T={5: 420.0},
                             node_id=pm.node_id)
    rng = np.random.default_rng(4)
    st = M.empty_state(m.nnode)
    for k, a in st.items():
        a[...] = rng.standard_normal(a.shape)
    ibc = np.asfortranarray(np.zeros((m.nnode, 8), dtype=np.int32))
    a = oracle.OracleCase(M.Case("f", m, M.base_params(), {k: v.copy() for k, v in st.items()}, ibc.copy(), 2))
    b = oracle.OracleCase(M.Case("b", m, M.base_params(), {k: v.copy() for k, v in st.items()}, ibc.copy(), 2))
    a.set_bcs(spec_file, 3)
    b.set_bcs(spec_box, 3)
    for k in a.state_arrays:
        np.testing.assert_array_equal(a.state_arrays[k], b.state_arrays[k])
    np.testing.assert_array_equal(a.ibc, b.ibc)
    with pytest.raises(ValueError):
        refio.bc_spec_from_part(back, ut[:3], uv, pt, pv, tt, tv)


def test_reference_file_names_and_step_file(tmp_path):
    """cname (src/cname.f90:4-37) and the names built from it: part.<id>.dat
    (src/input.f90:31), restart.<step>.<rank+1> (src/iosol.f90:137, 390);
    step.dat written and read back (readStep, a missing file gives step 0)."""
    assert refio.cname(0) == ".0" and refio.cname(7) == ".7" and refio.cname(120) == ".120"
    assert refio.cname(123456789) == ".123456789" and refio.cname(1234567890) == ".234567890"
    assert refio.part_name(3) == "part.3.dat"
    assert refio.restart_name(250, 0) == "restart.250.1" and refio.restart_name(0, 11) == "restart.0.12"
    assert refio.read_step(tmp_path / "step.dat") == (0, None)
    refio.write_step(tmp_path / "step.dat", 42, 0.125)
    assert refio.read_step(tmp_path / "step.dat") == (42, 0.125)
    # the list-directed record a Fortran compiler writes reads the same
    (tmp_path / "step2.dat").write_text("          17   1.2500000000000000D-01\n")
    assert refio.read_step(tmp_path / "step2.dat") == (17, 0.125)


def test_load_rank_follows_the_driver_start_up(tmp_path):
    """refio.load_rank reads what rank r of the reference reads at start-up:
    part.<r+1>.dat, step.dat and restart.<step>.<r+1>, giving the state of
    the first resumed step after the predictor; without step.dat it starts
    at step 0 from the given initial state."""
    case = M.quench_case(M.box_tet(3, 2, 4, 1.0, 1.0, 1.25), "load_rank")
    m = case.mesh
    refio.write_part(tmp_path / refio.part_name(2), refio.part_from_mesh(m))
    rng = np.random.default_rng(4)
    st = {k: rng.standard_normal(np.shape(v)) for k, v in case.state.items()}
    # step 0: no step.dat, the caller's initial state
    c0, step, time, pm = refio.load_rank(tmp_path, 1, case.params, {"tg": case.state["tg"]})
    assert step == 0 and time == 0.0 and c0.name == "part2"
    np.testing.assert_array_equal(c0.mesh.ien, m.ien)
    np.testing.assert_array_equal(c0.state["tg"], case.state["tg"])
    assert not c0.ibc.any()
    # a restart at step 7
    refio.write_restart(tmp_path / refio.restart_name(7, 1), 7, 0.007, st)
    refio.write_step(tmp_path / "step.dat", 7, 0.0)
    c7, step, time, _ = refio.load_rank(tmp_path, 1, case.params)
    assert step == 7 and time == 0.007
    g = case.params["gami"]
    np.testing.assert_array_equal(c7.state["ugold"], st["ug"])          # writeSol's ug is readSol's ugold
    np.testing.assert_array_equal(c7.state["ug"], st["ug"])             # predictor ug = ugold
    np.testing.assert_allclose(c7.state["acg"], (g - 1.0) / g * st["acg"], rtol=1e-15)
    np.testing.assert_array_equal(c7.state["tgold"], st["tgold"])       # writeSol writes Tgold
    np.testing.assert_array_equal(c7.state["pg"], st["pg"])
