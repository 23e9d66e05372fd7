"""Face assemblies in the oracle (CPU): the box-face enumeration, and known
answers that pin the face rule, outward normals and surface Jacobian of
eval_faceshape_tet, the weak-Dirichlet coupling blocks and backflow terms
(FaceAssembly_NS_weak + FaceAssembly_NS_outflow) and the convective heat
term, on uniform states where the face integrals have closed forms."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M

LX, LY, LZ = 1.5, 1.0, 2.0
NORMALS = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
AREAS = [LY * LZ, LY * LZ, LX * LZ, LX * LZ, LX * LY, LX * LY]


def test_box_face_enumeration():
    nx, ny, nz = 3, 2, 4
    m = M.box_tet(nx, ny, nz, LX, LY, LZ)
    fs = M.box_boundary_faces(m)
    assert [f.size for f, _ in fs] == [2 * ny * nz] * 2 + [2 * nx * nz] * 2 + [2 * nx * ny] * 2
    ien0 = np.asarray(m.ien) - 1
    for (f2e, fo), nodes in zip(fs, m.faces):
        assert np.all(np.diff(f2e) >= 0)
        for e, o in zip(f2e, fo):
            loc = M.TET_FACE_NODES[o - 1]
            assert np.isin(ien0[e - 1, list(loc)], nodes).all()
    bf = M.face_set(m, weak=(1, 6), convective={6: (5.0, 300.0)})
    assert len(bf.f2e) == 2 * (2 * ny * nz) // 2 + 2 * nx * ny
    assert set(bf.flags.tolist()) == {F.OVS_FACE_WEAK, F.OVS_FACE_WEAK | F.OVS_FACE_CONVH}


def _uniform_case(kernel, U, Um, p0, T0, **par):
    m = M.box_tet(3, 2, 4, LX, LY, LZ)
    N = m.nnode
    st = M.empty_state(N)
    for n in ("ug", "ugold"):
        st[n][:] = U
    for n in ("ugm", "ugmold"):
        st[n][:] = Um
    st["pg"][:] = p0
    for n in ("tg", "tgold"):
        st[n][:] = T0
    p = M.base_params(**par)
    ibc = np.asfortranarray(np.zeros((N, 8), dtype=np.int32))
    return M.Case("uniform", m, p, st, ibc, kernel)


def _with_and_without(oracle, case, bf, kind):
    out = []
    for faces in (None, bf):
        case.bfaces = faces
        oc = oracle.OracleCase(case)
        if kind == "ns":
            oc.assemble_navsto(6)
        else:
            oc.assemble_quenching(6, 3 if kind == "nsvof" else 4)
        out.append(oc.system(kind))
    return out


@pytest.mark.parametrize("kind", ["ns", "nsvof"])
@pytest.mark.parametrize("fid", range(1, 7))
def test_weak_face_known_answers(oracle, kind, fid):
    U, Um, p0 = np.array([0.3, -0.2, 0.5]), np.array([0.05, 0.1, -0.02]), 2.5
    kernel = F.OVS_ASM_NS if kind == "ns" else F.OVS_ASM_NSVOF
    case = _uniform_case(kernel, U, Um, p0, 350.0, mua=0.0, muw=0.0)
    bf = M.face_set(case.mesh, weak=(fid,))
    s0, s1 = _with_and_without(oracle, case, bf, kind)
    par = case.params
    fact2 = par["alfi"] * par["gami"] * par["delt"]
    n, area = np.array(NORMALS[fid - 1], dtype=float), AREAS[fid - 1]
    dG = (s1["G"] - s0["G"]).sum(axis=0)
    dD = (s1["D1"] - s0["D1"]).sum(axis=0)
    np.testing.assert_allclose(dG, fact2 * area * n, atol=1e-14)
    np.testing.assert_allclose(dD, -fact2 * area * n, atol=1e-14)
    drhs = (s1["rhs"] - s0["rhs"]).sum(axis=0)
    w = U - Um
    uneg = min(float(w @ n), 0.0)
    rho = par["rhoa"]
    # weak: -int (p n + (tauB - rho u_n^-) w) with mu = 0 (tauB = 0); outflow: +int rho u_n^- w
    # (differences of residuals that also hold the element terms: roundoff of their size)
    np.testing.assert_allclose(drhs[:3], area * (-p0 * n + 2.0 * rho * uneg * w), rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(drhs[3], area * float(w @ n), rtol=1e-10, atol=1e-12)
    # backflow on the velocity diagonal: -2 fact2 rho u_n^- area per component
    dK = (s1["K11"] - s0["K11"]).sum(axis=0)
    np.testing.assert_allclose(dK[[0, 4, 8]], -2.0 * fact2 * rho * uneg * area, atol=1e-14)
    np.testing.assert_allclose(dK[[1, 2, 3, 5, 6, 7]], 0.0, atol=1e-14)
    if kind == "nsvof":
        for b in ("LS", "LSU", "ULS", "PLS"):
            np.testing.assert_array_equal(s1[b], s0[b])
        np.testing.assert_array_equal(s1["rhs"][:, 4], s0["rhs"][:, 4])


@pytest.mark.parametrize("fid", [1, 4, 5])
def test_convective_heat_known_answers(oracle, fid):
    T0, h, tinf = 350.0, 12.5, 290.0
    case = _uniform_case(F.OVS_ASM_NSVOF, np.zeros(3), np.zeros(3), 0.0, T0)
    bf = M.face_set(case.mesh, convective={fid: (h, tinf)})
    s0, s1 = _with_and_without(oracle, case, bf, "tem")
    par = case.params
    fact2 = par["alfi"] * par["gami"] * par["delt"]
    area = AREAS[fid - 1]
    # differences of systems that also hold the element terms (rho cp ~ 4e6):
    # roundoff of their size, not of the face terms'
    eps_m = 1e-14 * np.abs(s0["TEM"]).max() * len(s0["TEM"])
    eps_r = 1e-14 * np.abs(s0["rhs"]).max() * len(s0["rhs"])
    np.testing.assert_allclose((s1["TEM"] - s0["TEM"]).sum(), fact2 * h * area, atol=eps_m)
    np.testing.assert_allclose((s1["rhs"] - s0["rhs"]).sum(), -h * (T0 - tinf) * area, atol=eps_r)
    # the convective term is a weighted face mass matrix: symmetric, couples face nodes only
    oc = oracle.OracleCase(case)
    col, row = oc.col.astype(np.int64) - 1, oc.row.astype(np.int64) - 1
    dT = s1["TEM"] - s0["TEM"]
    on = np.zeros(case.mesh.nnode, dtype=bool)
    on[case.mesh.faces[fid - 1]] = True
    for i in range(case.mesh.nnode):
        for k in range(col[i], col[i + 1]):
            j = row[k]
            if abs(dT[k]) > 1e-3 * fact2 * h * area / len(case.mesh.faces[fid - 1]):
                assert on[i] and on[j]
                kt = col[j] + np.nonzero(row[col[j]:col[j + 1]] == i)[0][0]
                assert abs(dT[kt] - dT[k]) <= 1e-13 * np.abs(s0["TEM"]).max()


def test_constrained_nodes_get_face_diagonal(oracle):
    """BCLhs_3D runs on each face routine's arrays too: every weak face
    touching a node with a velocity Dirichlet flag adds 1 to that node's
    diagonal once in FaceAssembly_NS_weak and once in _outflow."""
    case = _uniform_case(F.OVS_ASM_NS, np.array([0.1, 0.0, 0.0]), np.zeros(3), 1.0, 300.0)
    node = int(case.mesh.faces[4][3])
    case.ibc[node, 0] = 1
    bf = M.face_set(case.mesh, weak=(5,))
    s0, s1 = _with_and_without(oracle, case, bf, "ns")
    oc = oracle.OracleCase(case)
    col, row = oc.col.astype(np.int64) - 1, oc.row.astype(np.int64) - 1
    kd = col[node] + np.nonzero(row[col[node]:col[node + 1]] == node)[0][0]
    f2e = bf.f2e - 1
    touching = np.isin(np.asarray(case.mesh.ien)[f2e] - 1, node).any(axis=1).sum()
    assert touching > 0
    assert s1["K11"][kd, 0] - s0["K11"][kd, 0] == 2 * touching
    assert np.all(s1["rhs"][node, 0] == 0.0)


def test_weak_face_matrix_is_its_residual_jacobian(oracle):
    """FaceAssembly_NS_weak + _outflow at a uniform flow carried by the mesh
    (every wall weak): the face terms are linear in u and p there (the
    backflow term is second order), so with them the NS momentum rows stay
    the Jacobian of the residual under the Newton update, and the continuity
    rows' departure (the NS routine's missing PSPG residual) is the same as
    without faces."""
    m = M.box_tet(3, 3, 3, 1.0, 1.0, 1.0)
    p = M.base_params(gravvec=(0.0, 0.0, 0.0), rhoa=1.3, mua=0.05, ns_kdc_a=0.0, subdomain_flag=1,
                      elm_id_set=(102, 0))
    st = M.empty_state(m.nnode)
    rng = np.random.default_rng(5)
    for f in ("ug", "ugold", "ugm", "ugmold"):
        st[f][:] = np.array([0.3, -0.2, 0.1])
    for f in ("acg", "acgold"):
        st[f][:] = rng.standard_normal((m.nnode, 3))
    st["pg"][:] = rng.standard_normal(m.nnode)
    ibc = np.asfortranarray(np.zeros((m.nnode, 8), dtype=np.int32))
    bf = M.face_set(m, weak=(1, 2, 3, 4, 5, 6))

    def miss(d, faces):
        case = M.Case("fjac", m, p, {k: v.copy() for k, v in st.items()}, ibc, F.OVS_ASM_NS)
        case.bfaces = bf if faces else None
        oc = oracle.OracleCase(case)
        oc.assemble_navsto(6)
        r0 = np.concatenate([oc.sys["rhsu"], oc.sys["rhsp"][:, None]], axis=1)
        kd = oc.spmv("ns", np.asfortranarray(d))
        oc.newton_update(F.OVS_SYS_NS, np.asfortranarray(d))
        oc.assemble_navsto(2)
        return np.concatenate([oc.sys["rhsu"], oc.sys["rhsp"][:, None]], axis=1) - r0 + kd, kd

    du = np.zeros((m.nnode, 4))
    du[:, :3] = 1e-6 * rng.standard_normal((m.nnode, 3))
    dp = np.zeros((m.nnode, 4))
    dp[:, 3] = rng.standard_normal(m.nnode)
    for d, tol in ((du, 1e-8), (dp, 1e-11)):
        e1, k1 = miss(d, True)
        e0, k0 = miss(d, False)
        assert np.abs(k1 - k0).max() > 0.0                         # the faces are in the matrix
        assert np.abs(e1[:, :3]).max() <= tol * np.abs(k1).max()    # momentum rows: Jacobian
        assert np.abs(e1[:, 3] - e0[:, 3]).max() <= 1e-9 * np.abs(k1).max()


def test_convective_face_matrix_is_its_residual_jacobian(oracle):
    """The convective heat term is linear in T: with it on three walls the
    temperature matrix stays the exact Jacobian of the temperature residual
    under the Newton update (rT += d, T += gamma Delt d)."""
    m = M.box_tet(3, 3, 3, 1.0, 0.9, 1.1)
    p = M.base_params(c_evap=0.0, c_cond=0.0, tem_kdc=0.0)
    st = M.empty_state(m.nnode)
    rng = np.random.default_rng(11)
    for f in ("tg", "tgold"):
        st[f][:] = 320.0 + 10.0 * rng.standard_normal(m.nnode)
    for f in ("rtg", "rtgold"):
        st[f][:] = rng.standard_normal(m.nnode)
    ibc = np.asfortranarray(np.zeros((m.nnode, 8), dtype=np.int32))
    case = M.Case("cjac", m, p, st, ibc, F.OVS_ASM_NSVOF)
    case.bfaces = M.face_set(m, convective={1: (40.0, 290.0), 4: (15.0, 300.0), 6: (80.0, 280.0)})
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(6, 4)
    r0 = oc.sys["rhstem"].copy()
    d = rng.standard_normal(m.nnode)
    kd = oc.spmv("tem", np.asfortranarray(d[:, None]))[:, 0]
    oc.newton_update(F.OVS_SYS_TEM, np.asfortranarray(d[:, None]))
    oc.assemble_quenching(2, 4)
    np.testing.assert_allclose(oc.sys["rhstem"] - r0, -kd, rtol=0, atol=1e-11 * np.abs(kd).max())


def test_face_set_checks_without_a_device(lib):
    """ovs_check_faces, the checks ovs_set_faces makes, on the host: the box
    face set passes; an owning element beyond the mesh, a FACE_OR of 5, an
    unknown flag bit and convective faces without their tables are
    rejected; an empty set passes."""
    from oversetdevfort_b200 import api
    m = M.box_tet(3, 2, 2)
    bf = M.face_set(m, weak=(1, 6), convective={6: (5.0, 300.0)})
    assert api.check_faces(bf, m.nelem) == F.OVS_OK
    assert api.check_faces(bf, int(bf.f2e.max()) - 1) == F.OVS_ERR_ARG
    for field, bad in (("face_or", 5), ("flags", 8)):
        b2 = M.BoundaryFaces(*(np.array(getattr(bf, k), copy=True) for k in ("f2e", "face_or", "flags", "hconv", "tinf")))
        getattr(b2, field)[0] = bad
        assert api.check_faces(b2, m.nelem) == F.OVS_ERR_ARG, field
    b3 = M.BoundaryFaces(bf.f2e, bf.face_or, bf.flags, np.zeros(0), np.zeros(0))
    assert api.check_faces(b3, m.nelem) == F.OVS_ERR_ARG                # convective faces, no tables
    z = np.zeros(0, dtype=np.int32)
    assert api.check_faces(M.BoundaryFaces(z, z, z, np.zeros(0), np.zeros(0)), m.nelem) == F.OVS_OK
    assert lib.ovs_check_faces(0, 0, None, None, None, None, None) == F.OVS_ERR_ARG
