"""Known-answer tests that pin the CPU oracle (CPU only, no GPU).

The reference ships no tests or golden vectors, so the oracle is pinned by
answers known in closed form: pattern counts of the Kuhn split and of the
27-point hex stencil, the binary-search semantics of SparseMatLoc_3D, the
Galerkin mass of a single tet, the domain volume, partition of unity,
GMRES against dense LU, and patch tests of the element routines (a linear
temperature field leaves no interior conduction residual; a linear pressure
field gives -grad p times the lumped nodal volume; a linear divergence-free
velocity moving with the mesh leaves no interior momentum or continuity
residual; uniform advection of linear phi and T with the rates that cancel
it leaves no VOF residual and no interior temperature residual), the shape
functions and metric of tets and hexes in closed form, and every block of
the NS, NS+VOF and temperature element matrices of one tet at rest in
closed form (mass, viscous, grad-div, pressure and PSPG blocks with the
stabilisation parameters of e3STAB).
"""
import numpy as np
import pytest

from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import _ffi as F


def _pattern_props(col, row, N):
    assert col[0] == 1 and len(col) == N + 1
    for i in range(N):
        r = row[col[i] - 1: col[i + 1] - 1]
        assert np.all(np.diff(r) > 0), "row not strictly ascending"
        assert (i + 1) in r, "diagonal missing"


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 3, 4), (5, 1, 2), (16, 16, 16)])
def test_pattern_kuhn_closed_form(oracle, dims):
    m = M.box_tet(*dims)
    col, row = oracle.gen_spar_struc(m.ien, m.nnode)
    assert len(row) == M.expected_nnz_kuhn(*dims)
    if m.nnode < 2000:
        _pattern_props(col, row, m.nnode)
    # symmetric structure
    N = m.nnode
    rows = np.repeat(np.arange(N), np.diff(col))
    a = set(zip(rows.tolist(), (row - 1).tolist()))
    assert all((j, i) in a for (i, j) in list(a)[:5000])


def test_pattern_config1_count(oracle):
    m = M.box_tet(16, 16, 16)
    col, row = oracle.gen_spar_struc(m.ien, m.nnode)
    assert len(row) == 66961  # 16^3 x6 Kuhn tets, 4913 nodes


@pytest.mark.parametrize("dims", [(1, 1, 1), (3, 2, 2), (4, 4, 3)])
def test_pattern_hex_closed_form(oracle, dims):
    m = M.box_hex(*dims)
    col, row = oracle.gen_spar_struc(m.ien, m.nnode)
    assert len(row) == M.expected_nnz_hex(*dims)
    _pattern_props(col, row, m.nnode)


def test_sparse_mat_loc_semantics(oracle):
    lib = oracle.load()
    lst = np.array([2, 5, 9, 11], dtype=np.int32)
    p = oracle._i(lst)
    # last 1-based index with list(idx) <= goal; no not-found check
    assert lib.orc_sparse_mat_loc(p, 4, 9) == 3
    assert lib.orc_sparse_mat_loc(p, 4, 2) == 1
    assert lib.orc_sparse_mat_loc(p, 4, 1) == 1
    assert lib.orc_sparse_mat_loc(p, 4, 10) == 3
    assert lib.orc_sparse_mat_loc(p, 4, 12) == 4
    assert lib.orc_sparse_mat_loc(p, 4, 11) == 4


@pytest.mark.parametrize("mk", [lambda: M.box_tet(4, 3, 3), lambda: M.box_hex(3, 2, 2)])
def test_slot_map_points_at_the_column(oracle, mk):
    """FillSparseMat_3D's slot k(e,a,b) lies in row IEN(e,a) and holds
    column IEN(e,b) (rows are sorted and contain every element neighbour, so
    the search finds the goal itself); on a random permutation of the
    element order the map follows the elements."""
    m = mk()
    col, row = oracle.gen_spar_struc(m.ien, m.nnode)
    lmap = oracle.slot_map(m.ien, col, row)
    E, nshl = m.ien.shape
    for a in range(nshl):
        i = m.ien[:, a]
        for b in range(nshl):
            k = lmap[:, a, b]
            assert np.all((k >= col[i - 1]) & (k < col[i]))
            np.testing.assert_array_equal(row[k - 1], m.ien[:, b])
    perm = np.random.default_rng(0).permutation(E)
    np.testing.assert_array_equal(oracle.slot_map(m.ien[perm], col, row), lmap[perm])


def test_mesh_orientation():
    for m in (M.box_tet(3, 2, 2, 1.0, 0.5, 2.0), M.box_hex(2, 2, 3)):
        x = m.xg[m.ien - 1]  # (E, nshl, 3)
        if m.nshl == 4:
            J = np.stack([x[:, 0] - x[:, 3], x[:, 1] - x[:, 3], x[:, 2] - x[:, 3]], axis=2)
            assert np.all(np.linalg.det(J) > 0)
            vol = np.linalg.det(J).sum() / 6.0
            assert abs(vol - np.prod(m.lengths)) < 1e-12
        else:
            # node 5 is the (-1,-1,-1) corner, 3 the (+1,+1,+1) one
            assert np.all(x[:, 2] - x[:, 4] > 0)


def _single_tet_case(rho=2.0):
    xg = np.asfortranarray(np.array([[1.2, 0.2, 0.1], [0.3, 0.1, 0.0], [0.4, 1.1, 0.2], [0.2, 0.3, 0.9]]))
    ien = np.asfortranarray(np.array([[1, 2, 3, 4]], dtype=np.int32))
    # orient positively
    J = np.stack([xg[0] - xg[3], xg[1] - xg[3], xg[2] - xg[3]], axis=1)
    assert np.linalg.det(J) > 0
    m = M.Mesh(xg, ien, np.array([102], dtype=np.int32), [np.arange(4)] * 6, (1, 1, 1), (1, 1, 1))
    p = M.base_params(rhow=rho, rhoa=rho, muw=0.0, mua=0.0)
    st = M.empty_state(4)
    ibc = np.zeros((4, 8), dtype=np.int32, order="F")
    return M.Case("single_tet", m, p, st, ibc, F.OVS_ASM_NSVOF), abs(np.linalg.det(J)) / 6.0


def test_single_tet_galerkin_mass(oracle):
    """u = 0, mu = 0: K11(a,b) = alpha_m rho |T| (1 + delta_ab) / 20 (the
    4-point rule integrates quadratics exactly)."""
    rho = 2.0
    case, vol = _single_tet_case(rho)
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    K = oc.sys["K11"]
    col, row = oc.col, oc.row
    am = case.params["almi"]
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            want = am * rho * vol * (1 + (a == b)) / 20.0
            for comp in (0, 4, 8):
                assert abs(K[k, comp] - want) < 1e-14 * abs(want) + 1e-16
            for comp in (1, 2, 3, 5, 6, 7):
                assert abs(K[k, comp]) < 1e-15


@pytest.mark.parametrize("kernel", [F.OVS_ASM_NS, F.OVS_ASM_NSVOF])
def test_volume_kat(oracle, kernel):
    """With u = 0 and no BCs the velocity-block entries of K(1,1) sum to
    alpha_m * rho * volume (shape-gradient terms sum to zero)."""
    m = M.box_tet(3, 4, 2, 1.0, 0.7, 0.4)
    rho = 3.5
    p = M.base_params(rhow=rho, rhoa=rho, muw=0.01, mua=0.01)
    st = M.empty_state(m.nnode)
    ibc = np.zeros((m.nnode, 8), dtype=np.int32, order="F")
    case = M.Case("vol", m, p, st, ibc, kernel)
    oc = oracle.OracleCase(case)
    if kernel == F.OVS_ASM_NS:
        oc.assemble_navsto(F.OVS_TENSOR_MAT)
    else:
        oc.assemble_quenching(F.OVS_TENSOR_MAT, 3)
    total = oc.sys["K11"][:, 0].sum()
    want = p["almi"] * rho * 1.0 * 0.7 * 0.4
    assert abs(total - want) < 1e-12 * want
    # PSPG Laplacian rows sum to zero (sum_b grad N_b = 0)
    rs = np.add.reduceat(oc.sys["M"], oc.col[:-1] - 1)
    assert np.abs(rs).max() < 1e-12 * np.abs(oc.sys["M"]).max()


def test_dirichlet_diagonal_counts(oracle):
    """A constrained dof's assembled diagonal equals the number of elements
    around the node (per-element BC treatment, src/BCLhs_3D.f90)."""
    case = M.config1(n=3)
    oc = oracle.OracleCase(case)
    oc.assemble_navsto(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC)
    m = case.mesh
    nelem_at = np.bincount(m.ien.ravel() - 1, minlength=m.nnode)
    for i in m.faces[0][:10]:
        k = next(k for k in range(oc.col[i] - 1, oc.col[i + 1] - 1) if oc.row[k] == i + 1)
        assert oc.sys["K11"][k, 0] == nelem_at[i]
        assert oc.sys["K11"][k, 4] == nelem_at[i]
        assert oc.sys["K11"][k, 1] == 0.0
        assert oc.sys["rhsu"][i, 0] == 0.0


def test_quench_literal_switch_freezes_vof(oracle):
    case = M.random_case(seed=3)
    oc = oracle.OracleCase(case, literal=True)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    assert np.all(oc.sys["LS"] == 0) and np.all(oc.sys["LSU"] == 0)
    assert np.abs(oc.sys["rhsls"]).max() > 0


def _dense(oc, kind):
    N = oc.N
    nf = {"ns": 4, "nsvof": 5, "tem": 1}[kind]
    A = np.zeros((N * nf, N * nf))
    for j in range(N * nf):
        e = np.zeros(N * nf)
        e[j] = 1.0
        A[:, j] = oc.spmv(kind, e.reshape((N, nf), order="F")).ravel(order="F")
    return A


def test_gmres_diagonal_one_iteration(oracle):
    case = M.random_case(seed=4)
    oc = oracle.OracleCase(case)
    rng = np.random.default_rng(0)
    d = np.zeros(oc.icnt)
    for i in range(oc.N):
        k = next(k for k in range(oc.col[i] - 1, oc.col[i + 1] - 1) if oc.row[k] == i + 1)
        d[k] = rng.uniform(1, 3)
    rhs = rng.standard_normal(oc.N)
    oc.load_system("tem", {"TEM": d, "rhs": rhs[:, None]})
    sol, it, er, r0 = oc.gmres("tem", 1e-10, 20, 1)
    assert it == 1
    dd = np.array([d[next(k for k in range(oc.col[i] - 1, oc.col[i + 1] - 1) if oc.row[k] == i + 1)]
                   for i in range(oc.N)])
    np.testing.assert_allclose(sol[:, 0], rhs / dd, rtol=1e-14)


@pytest.mark.parametrize("kind", ["tem", "ns", "nsvof"])
def test_gmres_full_space_matches_dense_lu(oracle, kind):
    case = M.random_case(nx=2, ny=2, nz=2, seed=5, phase_change=False)
    case.mesh.elm_id[:] = 102  # no all-solid / non-target rows (singular)
    case.ibc[:] = 0
    for f in range(6):                 # closed cavity ...
        case.ibc[case.mesh.faces[f], 0:3] = 1
    case.ibc[0, 3] = 1                 # ... with the pressure level pinned
    oc = oracle.OracleCase(case)
    if kind == "ns":
        case.params["subdomain_flag"] = 1
        oc = oracle.OracleCase(case)
        oc.assemble_navsto(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC)
    else:
        oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3 if kind == "nsvof" else 4)
    s = oc.system(kind)
    nf = s["rhs"].shape[1]
    n = oc.N * nf
    if kind == "nsvof":
        # the VOF preconditioner maps 1/LS(ii) = 0 when LS(ii) = 0; make sure it is not
        assert np.all(np.abs(s["LS"]) >= 0)
    sol, it, er, r0 = oc.gmres(kind, 1e-13, n, 1)
    A = _dense(oc, kind)
    b = s["rhs"].ravel(order="F")
    x = np.linalg.solve(A, b)
    xs = sol.ravel(order="F")
    res = np.linalg.norm(b - A @ xs) / np.linalg.norm(b)
    assert res < 1e-9, (it, res)
    # forward error within the conditioning of the system
    err = np.linalg.norm(xs - x) / np.linalg.norm(x)
    assert err < 1e-14 * np.linalg.cond(A), (it, err)


def test_newton_update_and_residual(oracle):
    case = M.random_case(seed=6)
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_VEC, 7)
    r = oc.calculate_residual()
    s = oc.sys
    np.testing.assert_allclose(r, [np.sum(s["rhsu"] ** 2), np.sum(s["rhsp"] ** 2), np.sum(s["rhsls"] ** 2),
                                   np.sum(s["rhstem"] ** 2)], rtol=1e-13)
    rng = np.random.default_rng(1)
    sol = np.asfortranarray(rng.standard_normal((oc.N, 5)))
    before = {k: v.copy() for k, v in oc.state_arrays.items()}
    oc.newton_update(F.OVS_SYS_NSVOF, sol)
    p = case.params
    gdt = p["gami"] * p["delt"]
    np.testing.assert_allclose(oc.state_arrays["acg"], before["acg"] + sol[:, :3], rtol=1e-15)
    np.testing.assert_allclose(oc.state_arrays["ug"], before["ug"] + gdt * sol[:, :3], rtol=1e-15)
    np.testing.assert_allclose(oc.state_arrays["pg"], before["pg"] + p["alfi"] * p["gami"] * p["delt"] * sol[:, 3],
                               rtol=1e-15)
    np.testing.assert_allclose(oc.state_arrays["phig"], before["phig"] + gdt * sol[:, 4], rtol=1e-15)


def test_genalpha_matches_reference_formulas(lib):
    for rinf in (0.0, 0.5, 1.0, -1.0, 2.0):
        p = F.OvsParams()
        assert lib.ovs_params_genalpha(rinf, p) == 0
        want = M.genalpha(rinf)
        for k in ("almi", "alfi", "gami", "beti"):
            assert getattr(p, k) == want[k]


def test_golden_fixture_regression(oracle):
    """The committed fixture (made by tests/golden/make_golden.py) is
    reproduced bit-for-bit by the oracle."""
    import importlib.util
    from pathlib import Path
    here = Path(__file__).resolve().parent / "golden"
    spec = importlib.util.spec_from_file_location("make_golden", here / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = np.load(here / "quench_small.npz")
    fresh = mg.compute()
    for k in g.files:
        np.testing.assert_array_equal(g[k], fresh[k], err_msg=k)


def _interior(m):
    nx, ny, nz = m.dims
    i = np.arange(m.nnode)
    ix, iy, iz = i % (nx + 1), (i // (nx + 1)) % (ny + 1), i // ((nx + 1) * (ny + 1))
    return (ix > 0) & (ix < nx) & (iy > 0) & (iy < ny) & (iz > 0) & (iz < nz)


def _lumped_volume(m):
    """sum over the elements around each node of |T| / 4 (|cell| / 8 for the
    box's hexahedra)"""
    x = np.asarray(m.xg)
    ien0 = np.asarray(m.ien) - 1
    if m.nshl == 8:
        lx, ly, lz = m.lengths
        nx, ny, nz = m.dims
        out = np.zeros(m.nnode)
        for k in range(8):
            np.add.at(out, ien0[:, k], lx * ly * lz / (nx * ny * nz) / 8.0)
        return out
    a, b, c, d = (x[ien0[:, k]] for k in range(4))
    vol = np.abs(np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a))) / 6.0
    out = np.zeros(m.nnode)
    for k in range(4):
        np.add.at(out, ien0[:, k], vol / 4.0)
    return out


def _still_case(m, **par):
    p = M.base_params(c_evap=0.0, c_cond=0.0, ns_kdc_w=0.0, ns_kdc_a=0.0, lsc_kdc=0.0, tem_kdc=0.0,
                      gravvec=(0.0, 0.0, 0.0), **par)
    st = M.empty_state(m.nnode)
    ibc = np.zeros((m.nnode, 8), dtype=np.int32, order="F")
    return p, st, ibc


@pytest.mark.parametrize("box", [M.box_tet, M.box_hex])
def test_temperature_patch_and_mass(oracle, box):
    """No flow, no rate, no phase change, T linear in x: the conduction
    residual of every interior node is zero (linear elements reproduce a
    linear field exactly), and the temperature mass entries sum to
    alpha_m rho c_p volume."""
    m = box(3, 3, 4, 1.0, 0.8, 1.1)
    p, st, ibc = _still_case(m)
    x = np.asarray(m.xg)
    T = 300.0 + 5.0 * x[:, 0] + 2.0 * x[:, 1] - 3.0 * x[:, 2]
    for f in ("tg", "tgold"):
        st[f][:] = T
    oc = oracle.OracleCase(M.Case("tpatch", m, p, st, ibc, F.OVS_ASM_NSVOF))
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    r = oc.sys["rhstem"]
    inner = _interior(m)
    assert inner.sum() > 0
    scale = np.abs(r).max()
    assert scale > 0.0 and np.abs(r[inner]).max() <= 1e-12 * scale
    rcp = p["rhow"] * p["cpw"]
    want = p["almi"] * rcp * 1.0 * 0.8 * 1.1
    assert abs(oc.sys["TEM"].sum() - want) <= 1e-12 * want


def _assemble_vec(oc, kernel):
    if kernel == F.OVS_ASM_NS:
        oc.assemble_navsto(F.OVS_TENSOR_VEC)
    else:
        oc.assemble_quenching(F.OVS_TENSOR_VEC, 3)


@pytest.mark.parametrize("kernel,box", [(F.OVS_ASM_NSVOF, M.box_tet), (F.OVS_ASM_NS, M.box_tet),
                                        (F.OVS_ASM_NSVOF, M.box_hex)])
def test_pressure_gradient_patch(oracle, kernel, box):
    """No flow, no acceleration, no gravity, p linear: the momentum residual
    of an interior node is -grad p times the node's lumped volume
    (sum of |T|/4 over its elements), and the VOF residual vanishes."""
    m = box(4, 3, 3, 1.2, 0.9, 0.75)
    p, st, ibc = _still_case(m)
    x = np.asarray(m.xg)
    g = np.array([2.0, -1.5, 0.75])
    st["pg"][:] = 10.0 + x @ g
    oc = oracle.OracleCase(M.Case("ppatch", m, p, st, ibc, kernel))
    _assemble_vec(oc, kernel)
    inner = _interior(m)
    lv = _lumped_volume(m)
    ru = oc.sys["rhsu"]
    want = -lv[inner, None] * g[None, :]
    np.testing.assert_allclose(ru[inner], want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    if kernel == F.OVS_ASM_NSVOF:
        assert np.abs(oc.sys["rhsls"]).max() == 0.0


@pytest.mark.parametrize("kernel,box", [(F.OVS_ASM_NSVOF, M.box_tet), (F.OVS_ASM_NS, M.box_tet),
                                        (F.OVS_ASM_NSVOF, M.box_hex)])
def test_viscous_patch(oracle, kernel, box):
    """A linear, divergence-free velocity carried by the mesh (no advection),
    no acceleration, no pressure: the viscous term of linear elements
    reproduces it exactly, so every interior node has zero momentum and
    continuity residual (the stabilisation and divergence terms vanish
    with the advection velocity and div u)."""
    m = box(4, 4, 3, 1.0, 1.0, 0.8)
    p, st, ibc = _still_case(m, muw=0.7, mua=0.7)
    x = np.asarray(m.xg)
    A = np.array([[0.3, 1.2, -0.4], [0.5, -0.9, 0.8], [-0.2, 0.6, 0.6]])   # trace 0
    u = x @ A.T
    for f in ("ug", "ugold", "ugm", "ugmold"):
        st[f][:] = u
    oc = oracle.OracleCase(M.Case("vpatch", m, p, st, ibc, kernel))
    _assemble_vec(oc, kernel)
    inner = _interior(m)
    ru, rp = oc.sys["rhsu"], oc.sys["rhsp"]
    scale = max(np.abs(ru).max(), 1e-300)
    assert np.abs(ru).max() > 0.0                    # boundary nodes carry the traction
    assert np.abs(ru[inner]).max() <= 1e-12 * scale
    assert np.abs(rp[inner]).max() <= 1e-12 * max(np.abs(rp).max(), scale)


@pytest.mark.parametrize("box", [M.box_tet, M.box_hex])
def test_advection_patch(oracle, box):
    """Uniform advection velocity, linear phi and T, and the rates that make
    their transport residuals vanish pointwise (rphi = -u.grad phi,
    rT = -u.grad T, no phase change): the Galerkin and SUPG terms, both
    weighted by that residual, give nothing, so the VOF residual is zero at
    every node and the temperature residual at every interior node (linear
    conduction leaves only the boundary flux)."""
    m = box(4, 3, 3, 1.0, 0.9, 0.8)
    p, st, ibc = _still_case(m)
    x = np.asarray(m.xg)
    u = np.array([0.6, -0.25, 0.4])
    gphi, gT = np.array([0.1, 0.05, -0.08]), np.array([4.0, -2.0, 1.0])
    for f in ("ug", "ugold"):
        st[f][:] = u
    phi = 0.4 + x @ gphi
    T = 320.0 + x @ gT
    for f in ("phig", "phigold"):
        st[f][:] = phi
    for f in ("rphig", "rphigold"):
        st[f][:] = -(u @ gphi)
    for f in ("tg", "tgold"):
        st[f][:] = T
    for f in ("rtg", "rtgold"):
        st[f][:] = -(u @ gT)
    oc = oracle.OracleCase(M.Case("apatch", m, p, st, ibc, F.OVS_ASM_NSVOF))
    oc.assemble_quenching(F.OVS_TENSOR_VEC, 3)
    rl = oc.sys["rhsls"]
    assert np.abs(rl).max() <= 1e-13
    # temperature with a uniform phase (variable conductivity would add a flux)
    for f in ("phig", "phigold"):
        st[f][:] = 0.0
    for f in ("rphig", "rphigold"):
        st[f][:] = 0.0
    oc = oracle.OracleCase(M.Case("apatch_t", m, p, st, ibc, F.OVS_ASM_NSVOF))
    oc.assemble_quenching(F.OVS_TENSOR_VEC, 4)
    rt = oc.sys["rhstem"]
    inner = _interior(m)
    assert np.abs(rt).max() > 0.0
    # the cancelled terms are rho c_p |u.grad T| per unit volume (~4e4 per node
    # here): round-off of their size, not of the boundary flux
    terms = p["rhow"] * p["cpw"] * abs(u @ gT) * _lumped_volume(m).max()
    assert np.abs(rt[inner]).max() <= 1e-12 * terms


@pytest.mark.parametrize("box", [M.box_tet, M.box_hex])
def test_temperature_matrix_is_the_residual_jacobian(oracle, box):
    """No flow, no phase change, one phase: the temperature residual is
    linear in the state, so after the Newton update with a vector d
    (rT += d, T += gamma Delt d, src/solveFlow.f90:139-140) the residual
    changes by exactly -K d, K the assembled temperature matrix
    (alpha_m mass + alpha_f gamma Delt conduction)."""
    m = box(3, 3, 3, 1.0, 0.9, 1.1)
    p, st, ibc = _still_case(m)
    rng = np.random.default_rng(11)
    for f in ("tg", "tgold"):
        st[f][:] = 320.0 + 10.0 * rng.standard_normal(m.nnode)
    for f in ("rtg", "rtgold"):
        st[f][:] = rng.standard_normal(m.nnode)
    oc = oracle.OracleCase(M.Case("tjac", m, p, st, ibc, F.OVS_ASM_NSVOF))
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    r0 = oc.sys["rhstem"].copy()
    d = rng.standard_normal(m.nnode)
    kd = oc.spmv("tem", np.asfortranarray(d[:, None]))[:, 0]
    oc.newton_update(F.OVS_SYS_TEM, np.asfortranarray(d[:, None]))
    oc.assemble_quenching(F.OVS_TENSOR_VEC, 4)
    dr = oc.sys["rhstem"] - r0
    np.testing.assert_allclose(dr, -kd, rtol=0, atol=1e-11 * np.abs(kd).max())


def test_ns_matrix_is_the_residual_jacobian_at_rest(oracle):
    """NS-only routine at a uniform flow carried by the mesh (u_adv = 0,
    grad u = 0) with random acceleration and pressure: the stabilisation
    parameters and the convection term have no first-order change there, so
    after a Newton update with eps d (acg += d, ug += gamma Delt d,
    pg += alpha_f gamma Delt d_p) the momentum residual changes by -K eps d up
    to O(eps^2).  The continuity rows are not the residual's Jacobian: the
    routine hands zeros to e3RHS as uprime (src/assembleNavSto.f90:284-288),
    so its residual has no PSPG term while its matrix keeps the PSPG blocks;
    a pressure-only update leaves the continuity residual unchanged."""
    m = M.box_tet(3, 3, 3, 1.0, 1.0, 1.0)
    p, st, ibc = _still_case(m, rhoa=1.3, mua=0.05, subdomain_flag=1, elm_id_set=(102, 0))
    rng = np.random.default_rng(5)
    U = np.array([0.3, -0.2, 0.1])
    for f in ("ug", "ugold", "ugm", "ugmold"):
        st[f][:] = U
    for f in ("acg", "acgold"):
        st[f][:] = rng.standard_normal((m.nnode, 3))
    st["pg"][:] = rng.standard_normal(m.nnode)

    def change(d):
        oc = oracle.OracleCase(M.Case("nsjac", m, p, {k: v.copy() for k, v in st.items()}, ibc, F.OVS_ASM_NS))
        oc.assemble_navsto(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC)
        r0 = np.concatenate([oc.sys["rhsu"], oc.sys["rhsp"][:, None]], axis=1)
        kd = oc.spmv("ns", np.asfortranarray(d))
        oc.newton_update(F.OVS_SYS_NS, np.asfortranarray(d))
        oc.assemble_navsto(F.OVS_TENSOR_VEC)
        return np.concatenate([oc.sys["rhsu"], oc.sys["rhsp"][:, None]], axis=1) - r0, kd

    eps = 1e-6
    dr, kd = change(eps * rng.standard_normal((m.nnode, 4)))
    np.testing.assert_allclose(dr[:, :3], -kd[:, :3], rtol=0, atol=1e-8 * np.abs(kd[:, :3]).max())
    dp = np.zeros((m.nnode, 4))
    dp[:, 3] = eps * rng.standard_normal(m.nnode)
    dr, kd = change(dp)
    assert np.all(dr[:, 3] == 0.0) and np.abs(kd[:, 3]).max() > 0.0


def test_nsvof_matrix_against_residual_change_at_rest(oracle):
    """NS+VOF quench routine at a uniform flow carried by the mesh, one
    phase, no phase change: under the Newton update (acg += d_u,
    ug += gamma Delt d_u, pg += alpha_f gamma Delt d_p, rphig += d_phi,
    phig += gamma Delt d_phi) the residual changes by -K d in the continuity
    rows for a velocity update and in the momentum rows for a pressure update
    (exactly: linear there), in the momentum rows for a small velocity update
    up to O(eps), and in the VOF rows for a VOF update (exactly); the momentum
    rows do not follow a VOF update (rho(phi) and mu(phi) are not in the
    matrix's u-row/phi-column blocks)."""
    m = M.box_tet(3, 3, 3, 1.0, 1.0, 1.0)
    p, st, ibc = _still_case(m, muw=0.05, mua=0.05)
    rng = np.random.default_rng(5)
    for f in ("ug", "ugold", "ugm", "ugmold"):
        st[f][:] = np.array([0.3, -0.2, 0.1])
    for f in ("acg", "acgold"):
        st[f][:] = rng.standard_normal((m.nnode, 3))
    st["pg"][:] = rng.standard_normal(m.nnode)

    def change(cols, eps):
        oc = oracle.OracleCase(M.Case("vjac", m, p, {k: v.copy() for k, v in st.items()}, ibc, F.OVS_ASM_NSVOF))
        oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
        cat = lambda: np.concatenate([oc.sys["rhsu"], oc.sys["rhsp"][:, None], oc.sys["rhsls"][:, None]], axis=1)
        r0 = cat()
        d = np.zeros((m.nnode, 5))
        d[:, cols] = eps * rng.standard_normal((m.nnode, len(cols)))
        kd = oc.spmv("nsvof", np.asfortranarray(d))
        oc.newton_update(F.OVS_SYS_NSVOF, np.asfortranarray(d))
        oc.assemble_quenching(F.OVS_TENSOR_VEC, 3)
        return cat() - r0, kd

    dr, kd = change([0, 1, 2], 1e-6)
    sc = np.abs(kd).max()
    assert np.abs(dr[:, 3] + kd[:, 3]).max() <= 1e-9 * sc          # continuity rows: exact
    assert np.abs(dr[:, :3] + kd[:, :3]).max() <= 1e-4 * sc        # momentum rows: O(eps)
    dr, kd = change([3], 1.0)
    assert np.abs(dr[:, :4] + kd[:, :4]).max() <= 1e-9 * np.abs(kd).max()   # linear in p
    dr, kd = change([4], 1e-6)
    assert np.abs(dr[:, 4] + kd[:, 4]).max() <= 1e-9 * np.abs(kd[:, 4]).max()   # VOF rows: exact
    assert np.abs(kd[:, :3]).max() == 0.0 and np.abs(dr[:, :3]).max() > 0.0      # no phi columns in u rows


def test_oracle_newton_loop_reduces_the_residuals(oracle):
    """The oracle's solmultiphasethermofluid_stag loop on a small quench box:
    every Newton iteration solves the NS+VOF and temperature systems with one
    reference GMRES cycle and updates the state; three iterations cut the
    momentum, continuity and temperature residuals (sums of squares) by
    orders of magnitude, and the iteration stops once check_convergence
    holds."""
    case = M.quench_case(M.box_tet(5, 5, 6, 1.0, 1.0, 1.25), "onewton")
    rng = np.random.default_rng(3)   # a stirred start: the box at rest has no momentum residual
    free = np.asarray(case.ibc)[:, 0] == 0
    for f in ("ug", "ugold"):
        case.state[f][free] = 0.05 * rng.standard_normal((int(free.sum()), 3))
    oc = oracle.OracleCase(case)
    out = oc.quench_newton(3, True, 100, 1, 1e-8, 1e-8, (1e-6,) * 4, (1e-30,) * 4)
    r0, r = out["residual0"], out["residual"]
    assert out["iterations"] >= 1 and out["krylov_ns"] > 0 and out["krylov_tem"] > 0
    for k in (0, 1, 3):
        assert r0[k] > 0.0 and r[k] < 1e-3 * r0[k], (k, r[k], r0[k])
    loose = oracle.OracleCase(case).quench_newton(5, True, 100, 1, 1e-8, 1e-8, (1e30,) * 4, (1e-30,) * 4)
    assert loose["converged"] and loose["iterations"] == 1   # the loop body runs before the first check


def test_oracle_time_loop(oracle):
    """The oracle's driver loop: after each step the old velocity and
    acceleration equal the new ones, step 0 solves no temperature and takes
    one Newton iteration, and two steps move the state."""
    case = M.quench_case(M.box_tet(4, 4, 5, 1.0, 1.0, 1.25), "otime")
    oc = oracle.OracleCase(case)
    t0 = oc.state_arrays["tg"].copy()
    out = oc.quench_time_steps(0, 1, 3, True, 80, 1, 1e-8, 1e-8, (1e-6,) * 4, (1e-30,) * 4)
    assert out["iterations"] == 1 and out["krylov_tem"] == 0
    np.testing.assert_array_equal(oc.state_arrays["tg"], t0)          # no temperature solve at step 0
    out = oc.quench_time_steps(1, 2, 3, True, 80, 1, 1e-8, 1e-8, (1e-6,) * 4, (1e-30,) * 4)
    assert out["krylov_tem"] > 0
    for cur, old in (("ug", "ugold"), ("acg", "acgold")):
        np.testing.assert_array_equal(oc.state_arrays[cur], oc.state_arrays[old])
    assert np.abs(oc.state_arrays["tg"] - t0).max() > 0.0


# ------------------------------------------------------------ geometry KATs

def _random_tet(rng):
    while True:
        x = rng.standard_normal((4, 3))
        J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
        d = np.linalg.det(J)
        if abs(d) > 0.2:
            if d < 0:
                x[[0, 1]] = x[[1, 0]]
                J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
            return x, J


def test_tet_shape_functions_closed_form(oracle):
    """eval_shape_fem on linear tets (src/eval_shape_FEM.f90:4-61) against
    the closed form: x = x4 + J xi, so grad N_k = row k of J^-1 (k = 1..3),
    grad N_4 = -(sum of the others), DetJ = det J, G = sum_k grad xi_k
    grad xi_k^T the same at every point, the weights summing to |T| = det J
    / 6; N is the barycentric coordinate of the point; the current
    configuration x + d is used (:31-36)."""
    rng = np.random.default_rng(7)
    for _ in range(20):
        x, J = _random_tet(rng)
        Ji = np.linalg.inv(J)
        grad = np.vstack([Ji, -Ji.sum(axis=0)])
        Gw = Ji.T @ Ji
        vol = 0.0
        for g in range(4):
            detj, N, shg, G, w = oracle.eval_shape(4, g, x)
            assert abs(detj - np.linalg.det(J)) < 1e-12 * abs(detj)
            assert abs(N.sum() - 1.0) < 1e-15
            np.testing.assert_allclose(shg, grad, rtol=0, atol=1e-12 * np.abs(grad).max())
            np.testing.assert_allclose(G, Gw, rtol=0, atol=1e-12 * np.abs(Gw).max())
            xp = N @ x   # the Gauss point maps to the barycentric combination
            np.testing.assert_allclose(np.linalg.solve(J, xp - x[3]), N[:3], atol=1e-12)
            vol += w * detj
        assert abs(vol - np.linalg.det(J) / 6.0) < 1e-14 * vol
        d = 0.1 * rng.standard_normal((4, 3))
        a = oracle.eval_shape(4, 2, x, d)
        b = oracle.eval_shape(4, 2, x + d)
        assert a[0] == b[0] and all(np.array_equal(u, v) for u, v in zip(a[1:4], b[1:4]))


_HEX_XI = 2.0 * np.array([(0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1), (0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)]) - 1.0


def test_hex_shape_functions(oracle):
    """linhexshl + eval_shape_fem on trilinear hexahedra (the hex extension):
    partition of unity, gradients summing to zero, a linear field c.x + e
    reproduced with its exact gradient c on distorted hexes; on a
    parallelepiped x = x0 + A xi, DetJ = det A at every point, G = A^-T A^-1
    and the 8-point weights sum to the volume 8 det A."""
    rng = np.random.default_rng(11)
    for distort in (0.0, 0.08):
        for _ in range(10):
            A = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
            if np.linalg.det(A) < 0.3:
                continue
            x = rng.standard_normal(3) + _HEX_XI @ A.T + distort * rng.standard_normal((8, 3))
            c, e = rng.standard_normal(3), rng.standard_normal()
            f = x @ c + e
            vol = 0.0
            for g in range(8):
                detj, N, shg, G, w = oracle.eval_shape(8, g, x)
                assert abs(N.sum() - 1.0) < 1e-14
                assert np.abs(shg.sum(axis=0)).max() < 1e-12 * np.abs(shg).max()
                np.testing.assert_allclose(f @ shg, c, rtol=0, atol=1e-11 * (1 + np.abs(c).max()))
                vol += w * detj
                if distort == 0.0:
                    Ai = np.linalg.inv(A)
                    assert abs(detj - np.linalg.det(A)) < 1e-12 * abs(detj)
                    np.testing.assert_allclose(G, Ai.T @ Ai, rtol=0, atol=1e-12 * np.abs(Ai).max() ** 2)
            if distort == 0.0:
                assert abs(vol - 8.0 * np.linalg.det(A)) < 1e-12 * vol


def test_ns_element_matrix_at_rest_closed_form(oracle):
    """IntElmAss_NS_overset on one tet with the fluid and mesh at rest
    (u = ugm = 0), mu > 0: every block in closed form from e3STAB_3D
    (src/e3STAB.f90:4-44: tau_M = tau_P = 1/(rho sqrt(4/dt^2 + 12 nu^2
    G:G)), tau_C = rho sqrt(12 nu^2 G:G)/tr G) and e3LHS_3D_fluid_Old
    (src/e3LHS.f90:4-161) with f1 = alpha_m, f2 = alpha_f gamma dt:
      K_ij = delta_ij (f1 rho M_ab + f2 mu |T| gN_a.gN_b)
             + f2 |T| (mu d_jN_a d_iN_b + tau_C d_iN_a d_jN_b)
      G_d = -f2 |T|/4 d_dN_a;  D_d = |T|/4 (f2 d_dN_b + f1 tau_P rho d_dN_a)
      M = f2 tau_P |T| gN_a.gN_b
    with M_ab = |T| (1 + delta_ab)/20 (the 4-point rule is exact)."""
    rho, mu = 1.7, 0.37
    case, vol = _single_tet_case(rho)
    case.params.update(mua=mu, muw=mu, delt=0.05)
    case.kernel = F.OVS_ASM_NS
    oc = oracle.OracleCase(case)
    oc.assemble_navsto(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC)
    p = case.params
    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    x = np.asarray(case.mesh.xg)
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    G = Ji.T @ Ji
    nu = mu / rho
    GG = (G * G).sum()
    tauM = 1.0 / (rho * np.sqrt(4.0 / p["delt"] ** 2 + 12.0 * nu * nu * GG))
    tauC = rho * np.sqrt(12.0 * nu * nu * GG) / np.trace(G)
    col, row = oc.col, oc.row
    s = oc.sys
    checked = 0
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            Mab = vol * (1 + (a == b)) / 20.0
            lap = gN[a] @ gN[b]
            for i in range(3):
                for j in range(3):
                    want = (i == j) * (f1 * rho * Mab + f2 * mu * vol * lap) \
                        + f2 * vol * (mu * gN[a, j] * gN[b, i] + tauC * gN[a, i] * gN[b, j])
                    got = s["K11"][k, 3 * i + j]
                    assert abs(got - want) < 1e-12 * (abs(want) + f2 * mu * vol * np.abs(gN).max() ** 2), (a, b, i, j)
            for d in range(3):
                wg = -f2 * vol / 4.0 * gN[a, d]
                wd = vol / 4.0 * (f2 * gN[b, d] + f1 * tauM * rho * gN[a, d])
                assert abs(s["G"][k, d] - wg) < 1e-12 * abs(f2 * vol * np.abs(gN).max())
                assert abs(s["D1"][k, d] - wd) < 1e-12 * abs(f2 * vol * np.abs(gN).max())
            wm = f2 * tauM * vol * lap
            assert abs(s["M"][k] - wm) < 1e-12 * f2 * tauM * vol * np.abs(gN).max() ** 2
            checked += 1
    assert checked == 16


def test_nsvof_element_matrix_at_rest_closed_form(oracle):
    """IntElmAss_NSVOF_Quenching_STAB on one fluid tet at rest (u = ugm = 0),
    uniform phi = 0.25 between the phases, T below Ts and no phase change:
    rho, mu = prop_interp(w, a, phi) (src/solveQuenching.f90:352-358),
    lambda = -2/3 mu (:359), the taus of e3STAB_3D_NSVOF (src/e3STAB.f90:
    292-333) and the blocks of :434-494 in closed form:
      K_ij = delta_ij (f1 rho M_ab + f2 mu |T| gN_a.gN_b)
             + f2 |T| (mu d_jN_a d_iN_b + (tau_C + lambda) d_iN_a d_jN_b)
      G_d = -f2 |T|/4 d_dN_a;  D_d = |T|/4 (f2 d_dN_b + f1 tau_M rho d_dN_a)
      M = f2 tau_M |T| gN_a.gN_b;  LS = f1 M_ab;  ULS = PLS = 0; LSU = 0
    (grad phi = 0)."""
    case, vol = _single_tet_case(1.0)
    rhow, rhoa, muw, mua, phi = 3.0, 1.0, 0.5, 0.1, 0.25
    case.params.update(rhow=rhow, rhoa=rhoa, muw=muw, mua=mua, delt=0.02)
    for f in ("phig", "phigold"):
        case.state[f][:] = phi
    for f in ("tg", "tgold"):
        case.state[f][:] = 300.0
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    p = case.params
    assert p["c_evap"] == 0.0 and p["c_cond"] == 0.0 and 300.0 < p["ts"]
    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    rho, mu = rhow * (1 - phi) + rhoa * phi, muw * (1 - phi) + mua * phi
    lam = -2.0 / 3.0 * mu
    x = np.asarray(case.mesh.xg)
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    G = Ji.T @ Ji
    nu, GG = mu / rho, (G * G).sum()
    tauM = 1.0 / (rho * np.sqrt(4.0 / p["delt"] ** 2 + 12.0 * nu * nu * GG))
    tauC = rho * np.sqrt(12.0 * nu * nu * GG) / np.trace(G)
    s, col, row = oc.sys, oc.col, oc.row
    gmax = np.abs(gN).max()
    kscale = f2 * mu * vol * gmax ** 2 + f1 * rho * vol
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            Mab = vol * (1 + (a == b)) / 20.0
            lap = gN[a] @ gN[b]
            for i in range(3):
                for j in range(3):
                    want = (i == j) * (f1 * rho * Mab + f2 * mu * vol * lap) \
                        + f2 * vol * (mu * gN[a, j] * gN[b, i] + (tauC + lam) * gN[a, i] * gN[b, j])
                    assert abs(s["K11"][k, 3 * i + j] - want) < 1e-12 * kscale, (a, b, i, j)
            for d in range(3):
                assert abs(s["G"][k, d] + f2 * vol / 4.0 * gN[a, d]) < 1e-12 * f2 * vol * gmax
                wd = vol / 4.0 * (f2 * gN[b, d] + f1 * tauM * rho * gN[a, d])
                assert abs(s["D1"][k, d] - wd) < 1e-12 * f2 * vol * gmax
                assert s["ULS"][k, d] == 0.0
                assert abs(s["LSU"][k, d]) < 1e-14 * f2 * vol * gmax
            assert abs(s["M"][k] - f2 * tauM * vol * lap) < 1e-12 * f2 * tauM * vol * gmax ** 2
            assert abs(s["LS"][k] - f1 * Mab) < 1e-14 * f1 * vol
            assert s["PLS"][k] == 0.0


@pytest.mark.parametrize("solid", [False, True])
def test_temperature_element_matrix_at_rest_closed_form(oracle, solid):
    """IntElmAss_Tem_Quenching_STAB on one tet at rest, no phase change
    (src/solveQuenching.f90:758-839): the SUPG and source terms vanish and
    TEM = f1 (rho c_p) M_ab + f2 kappa |T| gN_a.gN_b, with rho c_p and kappa
    interpolated by phi in a fluid element (prop_interp of rho_w c_pw and
    rho_a c_pa) and the solid's own in a solid one (ELM_ID != 102)."""
    case, vol = _single_tet_case(1.0)
    phi = 0.4
    case.params.update(delt=0.03)
    if solid:
        case.mesh.elm_id[:] = 103
    for f in ("phig", "phigold"):
        case.state[f][:] = phi
    for f in ("tg", "tgold"):
        case.state[f][:] = 320.0
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    p = case.params
    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    if solid:
        rhocp, kap = p["rhos"] * p["cps"], p["kappas"]
    else:
        rhocp = p["rhow"] * p["cpw"] * (1 - phi) + p["rhoa"] * p["cpa"] * phi
        kap = p["kappaw"] * (1 - phi) + p["kappaa"] * phi
    x = np.asarray(case.mesh.xg)
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    col, row, T = oc.col, oc.row, oc.sys["TEM"]
    scale = f1 * rhocp * vol + f2 * kap * vol * np.abs(gN).max() ** 2
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            want = f1 * rhocp * vol * (1 + (a == b)) / 20.0 + f2 * kap * vol * (gN[a] @ gN[b])
            assert abs(T[k] - want) < 1e-12 * scale, (a, b, T[k], want)


def _hex_integrals(A):
    """Integrals over the parallelepiped x = x0 + A xi of a trilinear hex by
    a 3-point Gauss-Legendre rule per direction: int N_a N_b, int d_iN_a
    d_jN_b ([a, b, i, j]) and int d_dN_a N_b ([a, b, d])."""
    Ai = np.linalg.inv(A)
    q, w = np.polynomial.legendre.leggauss(3)
    NN, gg, gN_N = np.zeros((8, 8)), np.zeros((8, 8, 3, 3)), np.zeros((8, 8, 3))
    detA = np.linalg.det(A)
    for i1 in range(3):
        for i2 in range(3):
            for i3 in range(3):
                xi = np.array([q[i1], q[i2], q[i3]])
                wt = w[i1] * w[i2] * w[i3] * detA
                f = 1.0 + _HEX_XI * xi                       # (8, 3) factors (1 + xi_a,k xi_k)
                N = np.prod(f, axis=1) / 8.0
                dN = np.stack([_HEX_XI[:, k] * np.prod(np.delete(f, k, axis=1), axis=1) / 8.0 for k in range(3)], 1)
                g = dN @ Ai                                  # physical gradients (8, 3)
                NN += wt * np.outer(N, N)
                gg += wt * g[:, None, :, None] * g[None, :, None, :]
                gN_N += wt * g[:, None, :] * N[None, :, None]
    return NN, gg, gN_N


def _single_hex_case(A, rhow, rhoa, muw, mua, phi, T, delt):
    x0 = np.array([0.2, -0.1, 0.3])
    xg = np.asfortranarray(x0 + _HEX_XI @ A.T)
    ien = np.asfortranarray(np.arange(1, 9, dtype=np.int32)[None, :])
    m = M.Mesh(xg, ien, np.array([102], dtype=np.int32), [np.arange(8)] * 6, (1, 1, 1), (1, 1, 1))
    p = M.base_params(rhow=rhow, rhoa=rhoa, muw=muw, mua=mua, delt=delt)
    st = M.empty_state(8)
    for f in ("phig", "phigold"):
        st[f][:] = phi
    for f in ("tg", "tgold"):
        st[f][:] = T
    return M.Case("single_hex", m, p, st, np.zeros((8, 8), dtype=np.int32, order="F"), F.OVS_ASM_NSVOF)


def test_hex_temperature_element_matrix_at_rest(oracle):
    """The temperature matrix of one trilinear hex at rest, no phase change:
    TEM = f1 rho c_p int N_a N_b + f2 kappa int gN_a.gN_b, the integrals by
    the 3-point rule."""
    rng = np.random.default_rng(6)
    A = np.diag([0.3, 0.45, 0.35]) + 0.05 * rng.standard_normal((3, 3))
    phi = 0.7
    case = _single_hex_case(A, 2.0, 0.5, 0.3, 0.05, phi, 300.0, 0.05)
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    p = case.params
    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    rhocp = p["rhow"] * p["cpw"] * (1 - phi) + p["rhoa"] * p["cpa"] * phi
    kap = p["kappaw"] * (1 - phi) + p["kappaa"] * phi
    NN, gg, _ = _hex_integrals(A)
    lap = np.einsum("abii->ab", gg)
    want_all = f1 * rhocp * NN + f2 * kap * lap
    scale = np.abs(want_all).max()
    col, row, T = oc.col, oc.row, oc.sys["TEM"]
    for a in range(8):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            assert abs(T[k] - want_all[a, b]) <= 1e-12 * scale, (a, b)


def test_hex_nsvof_element_matrix_at_rest(oracle):
    """The NS+VOF element matrices of one trilinear hexahedron (the hex
    extension: linhexshl with the 2x2x2 rule) on a parallelepiped at rest,
    against the same closed form as the tet, with the integrals taken here
    by a 3x3x3 Gauss-Legendre rule (both rules are exact for these
    integrands: degree <= 2 in each reference coordinate)."""
    rng = np.random.default_rng(5)
    A = np.diag([0.4, 0.3, 0.5]) + 0.05 * rng.standard_normal((3, 3))
    x0 = np.array([0.2, -0.1, 0.3])
    xg = np.asfortranarray(x0 + _HEX_XI @ A.T)
    ien = np.asfortranarray(np.arange(1, 9, dtype=np.int32)[None, :])
    m = M.Mesh(xg, ien, np.array([102], dtype=np.int32), [np.arange(8)] * 6, (1, 1, 1), (1, 1, 1))
    rhow, rhoa, muw, mua, phi = 2.0, 0.5, 0.3, 0.05, 0.6
    p = M.base_params(rhow=rhow, rhoa=rhoa, muw=muw, mua=mua, delt=0.04)
    st = M.empty_state(8)
    for f in ("phig", "phigold"):
        st[f][:] = phi
    for f in ("tg", "tgold"):
        st[f][:] = 300.0
    case = M.Case("single_hex", m, p, st, np.zeros((8, 8), dtype=np.int32, order="F"), F.OVS_ASM_NSVOF)
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    rho, mu = rhow * (1 - phi) + rhoa * phi, muw * (1 - phi) + mua * phi
    lam = -2.0 / 3.0 * mu
    Ai = np.linalg.inv(A)
    G = Ai.T @ Ai
    nu, GG = mu / rho, (G * G).sum()
    tauM = 1.0 / (rho * np.sqrt(4.0 / p["delt"] ** 2 + 12.0 * nu * nu * GG))
    tauC = rho * np.sqrt(12.0 * nu * nu * GG) / np.trace(G)
    NN, gg, gN_N = _hex_integrals(A)
    lap = np.einsum("abii->ab", gg)
    s, col, row = oc.sys, oc.col, oc.row
    kscale = np.abs(f2 * mu * lap).max() + f1 * rho * NN.max()
    gscale = f2 * np.abs(gN_N).max()
    for a in range(8):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            for i in range(3):
                for j in range(3):
                    want = (i == j) * (f1 * rho * NN[a, b] + f2 * mu * lap[a, b]) \
                        + f2 * (mu * gg[a, b, j, i] + (tauC + lam) * gg[a, b, i, j])
                    assert abs(s["K11"][k, 3 * i + j] - want) < 1e-12 * kscale, (a, b, i, j)
            for d in range(3):
                assert abs(s["G"][k, d] + f2 * gN_N[a, b, d]) < 1e-12 * gscale
                wd = f2 * gN_N[b, a, d] + f1 * tauM * rho * gN_N[a, b, d]
                assert abs(s["D1"][k, d] - wd) < 1e-12 * gscale
            assert abs(s["M"][k] - f2 * tauM * lap[a, b]) < 1e-12 * f2 * tauM * np.abs(lap).max()
            assert abs(s["LS"][k] - f1 * NN[a, b]) < 1e-13 * f1 * NN.max()


def test_viscous_residual_broadcast_quirk_closed_form(oracle):
    """Momentum and continuity residuals of one tet with a linear velocity
    u = B x carried by the mesh (u - ugm = 0: no advection, uprime = 0), no
    acceleration, pressure or gravity, s_i(a) = sum_k d_kN_a (B_ki + B_ik):

    * NS+VOF (src/solveQuenching.f90:501-512): every component of node a
      receives -|T| [d_cN_a (tau_C + lambda) tr B + mu (s_1 + s_2 + s_3)],
      the three scalar viscous terms broadcast to all three components, as
      the reference writes them;
    * NS-only e3Rhs_3D_fluid (src/e3RHS.f90:26-95): the stress per component,
      -|T| [d_cN_a tau_C tr B + mu s_c(a)];
    * continuity in both: -|T|/4 tr B."""
    rng = np.random.default_rng(9)
    B = 0.3 * rng.standard_normal((3, 3))
    trB = np.trace(B)
    rho, mu = 1.3, 0.21
    out = {}
    for kernel in (F.OVS_ASM_NSVOF, F.OVS_ASM_NS):
        case, vol = _single_tet_case(rho)
        case.params.update(mua=mu, muw=mu, delt=0.02, gravvec=(0.0, 0.0, 0.0))
        x = np.asarray(case.mesh.xg)
        for f in ("ug", "ugold", "ugm", "ugmold"):
            case.state[f][:] = x @ B.T
        for f in ("tg", "tgold"):
            case.state[f][:] = 300.0
        oc = oracle.OracleCase(case)
        if kernel == F.OVS_ASM_NS:
            oc.assemble_navsto(F.OVS_TENSOR_VEC)
        else:
            oc.assemble_quenching(F.OVS_TENSOR_VEC, 3)
        out[kernel] = (oc.sys["rhsu"].copy(), oc.sys["rhsp"].copy())
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    G = Ji.T @ Ji
    nu, GG = mu / rho, (G * G).sum()
    tauC = rho * np.sqrt(12.0 * nu * nu * GG) / np.trace(G)
    lam = -2.0 / 3.0 * mu
    s = gN @ (B + B.T)                      # s[a, i] = sum_k d_kN_a (B_ki + B_ik)
    quench = -vol * (gN * (tauC + lam) * trB + mu * s.sum(axis=1)[:, None])
    ns = -vol * (gN * tauC * trB + mu * s)
    scale = vol * (np.abs(gN).max() * (tauC + mu) * np.abs(B).max())
    ru, rp = out[F.OVS_ASM_NSVOF]
    np.testing.assert_allclose(ru, quench, rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(rp, -vol / 4.0 * trB * np.ones(4), rtol=0, atol=1e-13 * vol * abs(trB))
    ru, rp = out[F.OVS_ASM_NS]
    np.testing.assert_allclose(ru, ns, rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(rp, -vol / 4.0 * trB * np.ones(4), rtol=0, atol=1e-13 * vol * abs(trB))
    # the quirk is visible: the two routines differ by more than rounding
    assert np.abs(out[F.OVS_ASM_NSVOF][0] - ns).max() > 1e-6 * scale


def test_pattern_row_limit_of_the_reference(oracle):
    """Asadj's row bound (src/genSparStruc.f90:14, :93): a node's list holds at
    most 27*nshl entries, self included (108 for tets).  A star of tets
    around node 1 with exactly 108 entries builds; one more distinct
    neighbour is "Stop the Music!!!" (OVS_ERR_PATTERN)."""
    import ctypes as C

    def star(nbrs):
        # tets (1, a, b, c) over consecutive neighbour triples; the last
        # triple wraps to reuse earlier neighbours, so node 1 sees exactly
        # `nbrs` distinct neighbours
        ids = list(range(2, nbrs + 2))
        tets = []
        for t in range(0, nbrs, 3):
            tri = [ids[(t + k) % nbrs] for k in range(3)]
            tets.append([1] + tri)
        return np.asfortranarray(np.array(tets, dtype=np.int32)), nbrs + 1

    lib = oracle.load()
    for nbrs, ok in ((107, True), (108, False)):
        ien, N = star(nbrs)
        col = np.zeros(N + 1, dtype=np.int32)
        icnt = C.c_int(0)
        st = lib.orc_gen_spar_struc(N, ien.shape[0], 4, oracle._i(ien), oracle._i(col), None, C.byref(icnt))
        if ok:
            assert st == 0 and col[1] - col[0] == 108
        else:
            assert st == F.OVS_ERR_PATTERN


@pytest.mark.parametrize("T, phi", [(400.0, 0.3), (350.0, 0.3), (350.0, 1.2)])
def test_phase_change_terms_at_rest_closed_form(oracle, T, phi):
    """The phase-change terms of both quench element routines on one fluid
    tet at rest, uniform phi = 0.3, phi rate 0.2, T = 400 > Ts, T rate 1.5,
    c_evap > 0, C_DMDOT = 0.7, gravity on, derived from the reference text:
    mdot = c_evap (1 - phi) rho_w (T - Ts)/Ts, dmdphi = -c_evap rho_w
    (T - Ts)/Ts C_DMDOT (src/solveQuenching.f90:343-350), vdot = mdot/rho_a
    - mdot/rho_w, D = 1/rho_a - 1/rho_w, uprime = tau_M rho g (rL = -rho g),
    tau_LS irrelevant (no convection):
      LS  = M_ab [f1 + f2 (vdot + phi D dmdphi - dmdphi/rho_a + tau_C (dmdphi D)^2)]
      ULS_d = f2 tau_C dmdphi D |T|/4 d_dN_a;  PLS = -f2 dmdphi D M_ab
      LSU_d = -f2 dmdphi D tau_C |T|/4 d_dN_b
      RHSu_a = rho g |T|/4 + tau_C vdot |T| gN_a
      RHSp_a = vdot |T|/4 + |T| gN_a . uprime
      RHSphi_a = -|T|/4 (rphi + phi vdot - mdot/rho_a + dmdphi D tau_C vdot)
    (:434-521), and for the temperature (:743-855), with dmdT = c_evap
    (1 - phi) rho_w/Ts C_DMDOT, Se = ((c_pw - c_pa)(T - Ts) - L) mdot,
    dSedT = (c_pw - c_pa) mdot + ((c_pw - c_pa)(T - Ts) - L) dmdT:
      TEM = M_ab (f1 rho c_p - f2 dSedT) + f2 kappa |T| gN_a.gN_b
      RHST_a = |T|/4 (Se - rho c_p rT).
    Also the condensation branch (T < Ts: mdot = c_cond phi_c rho_a (T -
    Ts)/Ts, dmdphi = c_cond rho_a (T - Ts)/Ts C_DMDOT, dmdT = c_cond phi_c
    rho_a/Ts C_DMDOT), and phi outside [0, 1], where the properties and mdot
    take the clamped phi_c, the VOF residual the unclamped phi, and dmdphi
    is zeroed (:362-366)."""
    case, vol = _single_tet_case(1.0)
    p = case.params
    p.update(rhow=1000.0, rhoa=1.0, muw=1e-3, mua=1e-5, delt=1e-3, c_evap=0.05, c_cond=0.02, c_dmdot=0.7)
    rphi, rT = 0.2, 1.5
    st = case.state
    for f, v in (("phig", phi), ("phigold", phi), ("rphig", rphi), ("rphigold", rphi), ("tg", T), ("tgold", T),
                 ("rtg", rT), ("rtgold", rT)):
        st[f][:] = v
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    ns = {k: oc.sys[k].copy() for k in ("LS", "ULS", "PLS", "LSU", "rhsu", "rhsp", "rhsls")}
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    tem, rhst = oc.sys["TEM"].copy(), oc.sys["rhstem"].copy()

    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    rw, ra, Ts = p["rhow"], p["rhoa"], p["ts"]
    pc = min(max(phi, 0.0), 1.0)
    rho = rw * (1 - pc) + ra * pc
    mu = p["muw"] * (1 - pc) + p["mua"] * pc
    if T > Ts:
        mdot = p["c_evap"] * (1 - pc) * rw * (T - Ts) / Ts
        dmdphi = -p["c_evap"] * rw * (T - Ts) / Ts * p["c_dmdot"]
        dmdT = p["c_evap"] * (1 - pc) * rw / Ts * p["c_dmdot"]
    else:
        mdot = p["c_cond"] * pc * ra * (T - Ts) / Ts
        dmdphi = p["c_cond"] * ra * (T - Ts) / Ts * p["c_dmdot"]
        dmdT = p["c_cond"] * pc * ra / Ts * p["c_dmdot"]
    if phi < 0.0 or phi > 1.0:
        dmdphi = 0.0
    vdot = mdot / ra - mdot / rw
    D = 1.0 / ra - 1.0 / rw
    x = np.asarray(case.mesh.xg)
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    G = Ji.T @ Ji
    nu, GG = mu / rho, (G * G).sum()
    tauM = 1.0 / (rho * np.sqrt(4.0 / p["delt"] ** 2 + 12.0 * nu * nu * GG))
    tauC = rho * np.sqrt(12.0 * nu * nu * GG) / np.trace(G)
    g = np.asarray(p["gravvec"], dtype=float)
    uprime = tauM * rho * g
    cpw, cpa = p["cpw"], p["cpa"]
    rhocp = rw * cpw * (1 - pc) + ra * cpa * pc
    kap = p["kappaw"] * (1 - pc) + p["kappaa"] * pc
    Se = ((cpw - cpa) * (T - Ts) - p["lh"]) * mdot
    dSedT = (cpw - cpa) * mdot + ((cpw - cpa) * (T - Ts) - p["lh"]) * dmdT

    def close(got, want, scale, what):
        assert abs(got - want) <= 1e-11 * scale, (what, got, want)

    col, row = oc.col, oc.row
    ls_fac = f1 + f2 * (vdot + phi * D * dmdphi - dmdphi / ra + tauC * (dmdphi * D) ** 2)
    gs = vol * np.abs(gN).max()
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            Mab = vol * (1 + (a == b)) / 20.0
            close(ns["LS"][k], ls_fac * Mab, abs(ls_fac) * vol, ("LS", a, b))
            close(ns["PLS"][k], -f2 * dmdphi * D * Mab, abs(f2 * dmdphi * D) * vol + 1e-300, ("PLS", a, b))
            for d in range(3):   # LSU's convection term f2 N_a N_b dphi/dx rounds to ~1e-16 of f2 phi |T| |gN|
                close(ns["ULS"][k, d], f2 * tauC * dmdphi * D * vol / 4.0 * gN[a, d],
                      abs(f2 * tauC * dmdphi * D) * gs + 1e-300, ("ULS", a, b, d))
                close(ns["LSU"][k, d], -f2 * dmdphi * D * tauC * vol / 4.0 * gN[b, d],
                      abs(f2 * tauC * dmdphi * D) * gs + f2 * gs * abs(phi), ("LSU", a, b, d))
            tw = Mab * (f1 * rhocp - f2 * dSedT) + f2 * kap * vol * (gN[a] @ gN[b])
            close(tem[k], tw, abs(f1 * rhocp * vol) + abs(f2 * dSedT * vol) + f2 * kap * gs * np.abs(gN).max(),
                  ("TEM", a, b))
    for a in range(4):
        for c in range(3):
            w = rho * g[c] * vol / 4.0 + tauC * vdot * vol * gN[a, c]
            close(ns["rhsu"][a, c], w, rho * 9.81 * vol + abs(tauC * vdot) * gs, ("rhsu", a, c))
        close(ns["rhsp"][a], vdot * vol / 4.0 + vol * gN[a] @ uprime, abs(vdot) * vol + gs * np.abs(uprime).max(),
              ("rhsp", a))
        wphi = -vol / 4.0 * (rphi + phi * vdot - mdot / ra + dmdphi * D * tauC * vdot)
        close(ns["rhsls"][a], wphi, vol * (abs(rphi) + abs(phi * vdot) + abs(mdot / ra) + abs(dmdphi * D * tauC * vdot)),
              ("rhsphi", a))
        close(rhst[a], vol / 4.0 * (Se - rhocp * rT), vol * (abs(Se) + abs(rhocp * rT)), ("rhstem", a))
    assert mdot != 0.0 and abs(Se) > 0   # the terms are really present
    assert (dmdphi == 0.0) == (phi > 1.0)


@pytest.mark.parametrize("lsc_kdc, tem_kdc, rphi, blend", [(0.0, 0.0, 0.0, False), (0.3, 0.2, 0.4, False),
                                                            (0.3, 0.2, 0.4, True)])
def test_uniform_advection_element_matrices_closed_form(oracle, lsc_kdc, tem_kdc, rphi, blend):
    """Both quench routines on one tet with a uniform velocity u relative to
    the fixed mesh (shconv_a = u.gN_a constant), uniform phi = 0.3, uniform
    T below Ts, T rate 1.5, gravity on, no phase change: every convection,
    SUPG and PSPG block, the residuals and the CFL number in closed form
    (src/solveQuenching.f90:400-521, :786-855), with the taus of e3STAB
    (uGu now in tau_M, tau_C, tau_LS, tau_T; tau_T built from rho_i c_p,i,
    the product of the separately interpolated properties, while the
    Galerkin terms use the interpolated rho c_p) and e3CFL = dt sqrt(uGu):
      K_ij = delta_ij [f1 rho M + f2 rho sc_b |T|/4 + f2 mu |T| lap
                      + f1 rho^2 tau_M sc_a |T|/4 + f2 rho^2 tau_M sc_a sc_b |T|]
             + f2 |T| (mu d_jN_a d_iN_b + (tau_C + lambda) d_iN_a d_jN_b)
      G_d = -f2 |T|/4 d_dN_a + f2 rho tau_M sc_a d_dN_b |T|
      D_d = f2 |T|/4 d_dN_b + f1 tau_M rho |T|/4 d_dN_a + f2 tau_M rho sc_b d_dN_a |T|
      LS  = f1 M + f2 sc_b |T|/4 + tau_LS sc_a (f1 |T|/4 + f2 sc_b |T|)
      TEM = rhocp (f1 M + f2 sc_b |T|/4) + tau_T rhocp^2 sc_a (f1 |T|/4 + f2 sc_b |T|) + f2 kappa |T| lap
      RHSu = rho g |T|/4 + rho sc_a uprime |T|, uprime = tau_M rho g;  RHSp = |T| gN_a.uprime
      RHSphi = 0;  RHST = -rhocp rT (|T|/4 + tau_T rhocp sc_a |T|).
    With the discontinuity-capturing constants on (:419-423, :795-801) and a
    phi rate: k_dc_phi = LSC_kdc |rphi| / |G|_F adds f2 k_dc_phi |T| lap to
    LS, k_dc_T = TEM_kdc |rhocp rT| / |G|_F / Tref adds f2 k_dc_T |T| lap to
    TEM, and RHSphi = -rphi (|T|/4 + tau_LS sc_a |T|).
    With `blend`, the old and new nodal values differ and the values above
    are the alpha-stage ones of src/solveQuenching.f90:26-37 (u, phi, T with
    alfi; acceleration, phi and T rates with almi), with a nonzero
    acceleration a: uprime = tau_M rho (g - a), RHSu = rho (g - a) |T|/4 +
    rho sc_a uprime |T|."""
    case, vol = _single_tet_case(1.0)
    p = case.params
    p.update(rhow=3.0, rhoa=1.2, muw=0.02, mua=0.004, delt=0.01, lsc_kdc=lsc_kdc, tem_kdc=tem_kdc, tref=2.0)
    u = np.array([0.3, -0.2, 0.5])
    acc = np.array([0.5, -1.0, 2.0]) if blend else np.zeros(3)
    phi, T, rT = 0.3, 300.0, 1.5
    st = case.state
    af, am = p["alfi"], p["almi"]
    # old values, and new ones whose alpha-stage blend is the value above
    olds = {"ug": np.array([0.1, 0.2, -0.1]), "acg": np.array([-0.3, 0.4, 0.1]), "phig": 0.2, "rphig": -0.1,
            "tg": 320.0, "rtg": 0.7} if blend else {"ug": u, "acg": acc, "phig": phi, "rphig": rphi, "tg": T, "rtg": rT}
    for name, val, alpha in (("ug", u, af), ("acg", acc, am), ("phig", phi, af), ("rphig", rphi, am), ("tg", T, af),
                             ("rtg", rT, am)):
        st[name + "old"][:] = olds[name]
        st[name][:] = olds[name] + (val - olds[name]) / alpha
    oc = oracle.OracleCase(case)
    cfl_ns = oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    ns = {k: oc.sys[k].copy() for k in ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS", "rhsu", "rhsp", "rhsls")}
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    tem, rhst = oc.sys["TEM"].copy(), oc.sys["rhstem"].copy()

    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    dt = p["delt"]
    rho = p["rhow"] * (1 - phi) + p["rhoa"] * phi
    mu = p["muw"] * (1 - phi) + p["mua"] * phi
    lam = -2.0 / 3.0 * mu
    cp = p["cpw"] * (1 - phi) + p["cpa"] * phi
    rhocp = p["rhow"] * p["cpw"] * (1 - phi) + p["rhoa"] * p["cpa"] * phi
    kap = p["kappaw"] * (1 - phi) + p["kappaa"] * phi
    x = np.asarray(case.mesh.xg)
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    G = Ji.T @ Ji
    uGu, GG = u @ G @ u, (G * G).sum()
    nu = mu / rho
    tauM = 1.0 / (rho * np.sqrt(4.0 / dt ** 2 + uGu + 12.0 * nu * nu * GG))
    tauC = rho * np.sqrt(uGu + 12.0 * nu * nu * GG) / np.trace(G)
    tauLS = 1.0 / np.sqrt(4.0 / dt ** 2 + uGu)
    kk = kap / (rho * cp)
    tauT = 1.0 / (rho * cp * np.sqrt(uGu + 4.0 / dt ** 2 + 12.0 * kk * kk * GG))
    sc = gN @ u
    g = np.asarray(p["gravvec"], dtype=float)
    uprime = tauM * rho * (g - acc)
    kdc_phi = lsc_kdc * abs(rphi) / np.sqrt(GG)
    kdc_T = tem_kdc * abs(rhocp * rT) / np.sqrt(GG) / p["tref"]
    assert abs(cfl_ns - dt * np.sqrt(uGu)) <= 1e-14 * cfl_ns

    def close(got, want, scale, what):
        assert abs(got - want) <= 1e-11 * scale, (what, got, want)

    col, row = oc.col, oc.row
    gm = np.abs(gN).max()
    kscale = vol * (f1 * rho + f2 * rho * np.abs(sc).max() + f2 * mu * gm * gm
                    + f2 * rho * rho * tauM * np.abs(sc).max() ** 2 + f2 * tauC * gm * gm)
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            Mab = vol * (1 + (a == b)) / 20.0
            lap = gN[a] @ gN[b]
            diag = (f1 * rho * Mab + f2 * rho * sc[b] * vol / 4.0 + f2 * mu * vol * lap
                    + f1 * rho * rho * tauM * sc[a] * vol / 4.0 + f2 * rho * rho * tauM * sc[a] * sc[b] * vol)
            for i in range(3):
                for j in range(3):
                    want = (i == j) * diag + f2 * vol * (mu * gN[a, j] * gN[b, i] + (tauC + lam) * gN[a, i] * gN[b, j])
                    close(ns["K11"][k, 3 * i + j], want, kscale, ("K", a, b, i, j))
            for d in range(3):
                wg = -f2 * vol / 4.0 * gN[a, d] + f2 * rho * tauM * sc[a] * gN[b, d] * vol
                wd = f2 * vol / 4.0 * gN[b, d] + f1 * tauM * rho * vol / 4.0 * gN[a, d] + f2 * tauM * rho * sc[b] * gN[a, d] * vol
                close(ns["G"][k, d], wg, f2 * vol * gm, ("G", a, b, d))
                close(ns["D1"][k, d], wd, f2 * vol * gm, ("D", a, b, d))
                assert ns["ULS"][k, d] == 0.0 and abs(ns["LSU"][k, d]) <= 1e-14 * f2 * vol * gm
            close(ns["M"][k], f2 * tauM * vol * lap, f2 * tauM * vol * gm * gm, ("M", a, b))
            wls = (f1 * Mab + f2 * sc[b] * vol / 4.0 + tauLS * sc[a] * (f1 * vol / 4.0 + f2 * sc[b] * vol)
                   + f2 * kdc_phi * vol * lap)
            close(ns["LS"][k], wls, vol * (f1 + f2 * np.abs(sc).max() * (1 + tauLS * np.abs(sc).max())
                                           + f2 * kdc_phi * gm * gm), ("LS", a, b))
            assert ns["PLS"][k] == 0.0
            wt = (rhocp * (f1 * Mab + f2 * sc[b] * vol / 4.0)
                  + tauT * rhocp * rhocp * sc[a] * (f1 * vol / 4.0 + f2 * sc[b] * vol) + f2 * (kap + kdc_T) * vol * lap)
            close(tem[k], wt, vol * rhocp * (f1 + f2 * np.abs(sc).max()) * (1 + tauT * rhocp * np.abs(sc).max())
                  + f2 * (kap + kdc_T) * vol * gm * gm, ("TEM", a, b))
    for a in range(4):
        for c in range(3):
            close(ns["rhsu"][a, c], rho * (g[c] - acc[c]) * vol / 4.0 + rho * sc[a] * uprime[c] * vol,
                  rho * 12.0 * vol * (1 + tauM * rho * np.abs(sc).max()), ("rhsu", a, c))
        close(ns["rhsp"][a], vol * gN[a] @ uprime, vol * gm * np.abs(uprime).max(), ("rhsp", a))
        close(ns["rhsls"][a], -rphi * (vol / 4.0 + tauLS * sc[a] * vol),
              vol * (abs(rphi) * (1 + tauLS * np.abs(sc).max()) + 1e-3), ("rhsphi", a))
        close(rhst[a], -rhocp * rT * (vol / 4.0 + tauT * rhocp * sc[a] * vol),
              rhocp * rT * vol * (1 + tauT * rhocp * np.abs(sc).max()), ("rhstem", a))


def test_ns_uniform_advection_matrix_closed_form(oracle):
    """IntElmAss_NS_overset on one tet with a uniform velocity u relative to
    the fixed mesh: e3LHS_3D_fluid_Old (src/e3LHS.f90:4-161) with tmp1_a =
    rho u.gN_a, tauBar = 0 and the taus of e3STAB_3D (src/e3STAB.f90:4-44)
    with uGu:
      K_ij = delta_ij [f1 rho M + f1 tmp1_a tau_M rho |T|/4 + f2 tmp1_b |T|/4
                      + f2 tmp1_a tau_M tmp1_b |T| + f2 mu |T| lap]
             + f2 |T| (mu d_jN_a d_iN_b + tau_C d_iN_a d_jN_b)
      G_d = -f2 |T|/4 d_dN_a + f2 tmp1_a tau_M d_dN_b |T|
      D_d = f2 |T|/4 d_dN_b + f2 d_dN_a tau_P tmp1_b |T| + f1 tau_P rho |T|/4 d_dN_a
      M = f2 tau_P |T| lap."""
    rho, mu = 1.4, 0.05
    case, vol = _single_tet_case(rho)
    case.params.update(mua=mu, muw=mu, delt=0.02)
    u = np.array([0.4, 0.1, -0.3])
    for f in ("ug", "ugold"):
        case.state[f][:] = u
    oc = oracle.OracleCase(case)
    oc.assemble_navsto(F.OVS_TENSOR_MAT)
    p = case.params
    f1, f2 = p["almi"], p["alfi"] * p["gami"] * p["delt"]
    x = np.asarray(case.mesh.xg)
    J = np.stack([x[0] - x[3], x[1] - x[3], x[2] - x[3]], axis=1)
    Ji = np.linalg.inv(J)
    gN = np.vstack([Ji, -Ji.sum(axis=0)])
    G = Ji.T @ Ji
    uGu, GG, nu = u @ G @ u, (G * G).sum(), mu / rho
    tauM = 1.0 / (rho * np.sqrt(4.0 / p["delt"] ** 2 + uGu + 12.0 * nu * nu * GG))
    tauC = rho * np.sqrt(uGu + 12.0 * nu * nu * GG) / np.trace(G)
    t1 = rho * (gN @ u)
    s, col, row = oc.sys, oc.col, oc.row
    gm = np.abs(gN).max()
    kscale = vol * (f1 * rho + f2 * np.abs(t1).max() * (1 + tauM * np.abs(t1).max()) + f2 * (mu + tauC) * gm * gm)
    for a in range(4):
        for k in range(col[a] - 1, col[a + 1] - 1):
            b = row[k] - 1
            Mab = vol * (1 + (a == b)) / 20.0
            lap = gN[a] @ gN[b]
            diag = (f1 * rho * Mab + f1 * t1[a] * tauM * rho * vol / 4.0 + f2 * t1[b] * vol / 4.0
                    + f2 * t1[a] * tauM * t1[b] * vol + f2 * mu * vol * lap)
            for i in range(3):
                for j in range(3):
                    want = (i == j) * diag + f2 * vol * (mu * gN[a, j] * gN[b, i] + tauC * gN[a, i] * gN[b, j])
                    assert abs(s["K11"][k, 3 * i + j] - want) <= 1e-11 * kscale, ("K", a, b, i, j)
            for d in range(3):
                wg = -f2 * vol / 4.0 * gN[a, d] + f2 * t1[a] * tauM * gN[b, d] * vol
                wd = f2 * vol / 4.0 * gN[b, d] + f2 * gN[a, d] * tauM * t1[b] * vol + f1 * tauM * rho * vol / 4.0 * gN[a, d]
                assert abs(s["G"][k, d] - wg) <= 1e-11 * f2 * vol * gm * (1 + tauM * np.abs(t1).max())
                assert abs(s["D1"][k, d] - wd) <= 1e-11 * f2 * vol * gm * (1 + tauM * np.abs(t1).max())
            assert abs(s["M"][k] - f2 * tauM * vol * lap) <= 1e-11 * f2 * tauM * vol * gm * gm


def test_bottom_heat_flux_weights_closed_form():
    """mesh.bottom_heat_flux_weights (the config-5 functional J = c . T): a
    linear temperature T = t0 + a x + b y + g z has dT/dz = g on every bottom
    tet, so J = kappa g (bottom area), with kappa = prop_interp(kappa_w,
    kappa_a, phi) for a uniform phi; only bottom-touching tets' nodes carry
    weight."""
    lx, ly, lz = 1.2, 0.8, 0.5
    case = M.quench_case(M.box_tet(4, 3, 2, lx, ly, lz), "flux")
    p = case.params
    x = case.mesh.xg
    phi = 0.35
    c = M.bottom_heat_flux_weights(case, np.full(case.mesh.nnode, phi))
    t0, a, b, g = 310.0, 2.0, -3.0, 7.5
    T = t0 + a * x[:, 0] + b * x[:, 1] + g * x[:, 2]
    kap = p["kappaw"] * (1 - phi) + p["kappaa"] * phi
    assert abs(c @ T - kap * g * lx * ly) <= 1e-12 * kap * abs(g) * lx * ly
    # constants and in-plane gradients carry no flux
    assert abs(c.sum()) <= 1e-12 * np.abs(c).max()
    assert abs(c @ x[:, 0]) <= 1e-12 * np.abs(c).max() and abs(c @ x[:, 1]) <= 1e-12 * np.abs(c).max()
    # weights only on the nodes of tets with a face on z = 0 (the bottom layer of nodes and one above)
    assert np.all(c[x[:, 2] > lz / 2 + 1e-12] == 0.0)


@pytest.mark.parametrize("routine", ["quench", "ns"])
def test_assembly_uses_the_current_configuration(oracle, routine):
    """The element routines evaluate the geometry at x + d_alpha, d_alpha =
    dgold + alfi (dg - dgold) (src/solveQuenching.f90:30, src/eval_shape_FEM.f90:
    31-36): assembling with a displacement field equals, bit for bit,
    assembling on the displaced coordinates with no displacement."""
    case = M.random_case(nx=3, ny=3, nz=2, seed=21)
    rng = np.random.default_rng(2)
    x = np.asarray(case.mesh.xg)
    S = 0.05 * rng.standard_normal((3, 3))
    dgold = np.asfortranarray(x @ S.T)
    dg = np.asfortranarray(dgold + 0.01 * rng.standard_normal(x.shape))
    p = case.params
    d_alpha = dgold + p["alfi"] * (dg - dgold)
    moved = M.Case(case.name, M.Mesh(np.asfortranarray(x + d_alpha), case.mesh.ien, case.mesh.elm_id,
                                     case.mesh.faces, case.mesh.dims, case.mesh.lengths),
                   p, {k: v.copy() for k, v in case.state.items()}, case.ibc, case.kernel)
    case.state["dg"][:] = dg
    case.state["dgold"][:] = dgold
    moved.state["dg"][:] = 0.0
    moved.state["dgold"][:] = 0.0
    out = []
    for c in (case, moved):
        oc = oracle.OracleCase(c)
        if routine == "ns":
            oc.assemble_navsto(6)
            keys = ("K11", "G", "D1", "M", "rhsu", "rhsp")
            out.append({k: oc.sys[k].copy() for k in keys})
        else:
            oc.assemble_quenching(6, 3)
            d = {k: oc.sys[k].copy() for k in ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS", "rhsu", "rhsp",
                                               "rhsls")}
            oc.assemble_quenching(6, 4)
            d.update(TEM=oc.sys["TEM"].copy(), rhstem=oc.sys["rhstem"].copy())
            out.append(d)
    assert np.abs(d_alpha).max() > 1e-3
    for k in out[0]:
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)


def test_solid_elements_carry_no_flow_terms(oracle):
    """ELM_ID != 102 is solid: the NS+VOF routine adds nothing for it, matrix
    or residual (src/solveQuenching.f90:250, 434, 496), while the temperature
    routine assembles its solid conduction (tested in closed form above)."""
    case, vol = _single_tet_case(2.0)
    case.mesh.elm_id[:] = 103
    st = case.state
    st["ug"][:] = np.array([0.3, -0.1, 0.2])
    st["acg"][:] = 1.0
    for f in ("phig", "phigold"):
        st[f][:] = 0.4
    for f in ("tg", "tgold"):
        st[f][:] = 350.0
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    for k in ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS", "rhsu", "rhsp", "rhsls"):
        assert not np.any(oc.sys[k]), k
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    diag = [k for i in range(4) for k in range(oc.col[i] - 1, oc.col[i + 1] - 1) if oc.row[k] == i + 1]
    assert np.all(oc.sys["TEM"][diag] > 0.0)


def test_quench_bc_masks_follow_bclhs_ns_conv(oracle):
    """Element Dirichlet masks of the quench path, BCLhs_NS_conv
    (src/BCLhs_3D.f90:278-428) with pressure at IBC column 4 and VOF at
    column 5, checked on the assembled system:
      velocity d at node i: row i of K(d,:), G(d), LSU(d) and column i of
        K(:,d), D(d), LSU(d) are zero except the K(d,d) diagonal = number of
        elements at i; RHSu(i,d) = 0.  As the template has it, ULS(d) of
        row i is NOT cleared (a constrained velocity row keeps its phi
        coupling), while LSU(d) of row i -- a phi row -- is;
      pressure at i: row i of M, D, PLS and column i of G are zero, M
        diagonal = count, RHSp(i) = 0;
      VOF at i: row and column i of LS, row i of LSU, column i of PLS and
        ULS are zero, LS diagonal = count, RHSphi(i) = 0."""
    case = M.random_case(nx=4, ny=3, nz=3, seed=13, solid_frac=0.0, bc_frac=0.0)
    m = case.mesh
    N = m.nnode
    rng = np.random.default_rng(1)
    perm = rng.permutation(N)
    vel, pre, vof = perm[:8], perm[8:14], perm[14:20]
    ibc = np.zeros((N, 8), dtype=np.int32, order="F")
    ibc[vel, 0:3] = 1
    ibc[pre, 3] = 1
    ibc[vof, 4] = 1
    case.ibc = ibc
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    s, col, row = oc.sys, oc.col, oc.row
    cnt = np.bincount(np.asarray(m.ien).ravel() - 1, minlength=N)
    rows_of = lambda i: range(col[i] - 1, col[i + 1] - 1)
    r_of = np.repeat(np.arange(N), np.diff(col))          # row of every slot
    c_of = row - 1                                        # column of every slot
    for i in vel:
        for k in rows_of(i):
            diag = c_of[k] == i
            for d in range(3):
                for j in range(3):
                    want = cnt[i] if (diag and j == d) else 0.0
                    assert s["K11"][k, 3 * d + j] == want
                assert s["G"][k, d] == 0.0 and s["LSU"][k, d] == 0.0
        colk = np.nonzero(c_of == i)[0]
        for d in range(3):
            for c in range(3):
                vals = s["K11"][colk, 3 * c + d]
                assert np.all(vals[r_of[colk] != i] == 0.0)
            assert np.all(s["D1"][colk, d] == 0.0) and np.all(s["LSU"][colk, d] == 0.0)
        assert np.all(s["rhsu"][i] == 0.0)
    # the template leaves ULS of constrained velocity rows in place
    uls_rows = np.concatenate([np.abs(s["ULS"][list(rows_of(i))]).ravel() for i in vel])
    assert uls_rows.max() > 0.0
    for i in pre:
        for k in rows_of(i):
            assert s["M"][k] == (cnt[i] if c_of[k] == i else 0.0)
            assert np.all(s["D1"][k] == 0.0) and s["PLS"][k] == 0.0
        colk = np.nonzero(c_of == i)[0]
        assert np.all(s["G"][colk] == 0.0)
        assert s["rhsp"][i] == 0.0
    for i in vof:
        for k in rows_of(i):
            assert s["LS"][k] == (cnt[i] if c_of[k] == i else 0.0)
            assert np.all(s["LSU"][k] == 0.0)
        colk = np.nonzero(c_of == i)[0]
        assert np.all(s["LS"][colk][r_of[colk] != i] == 0.0)
        assert np.all(s["PLS"][colk] == 0.0) and np.all(s["ULS"][colk] == 0.0)
        assert s["rhsls"][i] == 0.0
    # unconstrained phi rows do couple to velocity (the LSU clearing above is the BC's doing)
    free = np.setdiff1d(np.arange(N), np.concatenate([vel, vof]))
    assert np.abs(s["LSU"][np.isin(r_of, free)]).max() > 0.0


def test_temperature_bc_masks_follow_bclhs_tem(oracle):
    """BCLhs_tem (src/BCLhs_3D.f90:247-274) on IBC column 6, assembled: row i
    and column i of the temperature matrix are zero except the diagonal,
    which counts the elements at i; RHStem(i) = 0; other rows keep their
    entries."""
    case = M.random_case(nx=4, ny=3, nz=3, seed=17, solid_frac=0.2, bc_frac=0.0)
    m = case.mesh
    N = m.nnode
    tn = np.random.default_rng(3).permutation(N)[:10]
    ibc = np.zeros((N, 8), dtype=np.int32, order="F")
    ibc[tn, 5] = 1
    case.ibc = ibc
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 4)
    T, col, row = oc.sys["TEM"], oc.col, oc.row
    cnt = np.bincount(np.asarray(m.ien).ravel() - 1, minlength=N)
    r_of = np.repeat(np.arange(N), np.diff(col))
    c_of = row - 1
    for i in tn:
        sel = (r_of == i) | (c_of == i)
        diag = (r_of == i) & (c_of == i)
        assert np.all(T[sel & ~diag] == 0.0) and T[diag][0] == cnt[i]
        assert oc.sys["rhstem"][i] == 0.0
    free = ~np.isin(r_of, tn) & ~np.isin(c_of, tn)
    assert np.all(T[free & (r_of == c_of)] > 0.0)


def test_ns_bc_masks_follow_bclhs_3d(oracle):
    """BCLhs_3D (src/BCLhs_3D.f90:4-122) on the NS-only path, assembled:
    velocity d at node i clears row i of K(d,:) and G(d) and column i of
    K(:,d) and D(d), the K(d,d) diagonal counting the elements at i;
    pressure (IBC column 4) clears row i of M and D and column i of G, the
    M diagonal counting the elements; the constrained RHS entries are 0."""
    case = M.random_case(nx=4, ny=3, nz=3, seed=19, kernel=F.OVS_ASM_NS, solid_frac=0.0, bc_frac=0.0)
    m = case.mesh
    N = m.nnode
    perm = np.random.default_rng(4).permutation(N)
    vel, pre = perm[:8], perm[8:14]
    ibc = np.zeros((N, 8), dtype=np.int32, order="F")
    ibc[vel, 0:3] = 1
    ibc[pre, 3] = 1
    case.ibc = ibc
    oc = oracle.OracleCase(case)
    oc.assemble_navsto(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC)
    s, col, row = oc.sys, oc.col, oc.row
    cnt = np.bincount(np.asarray(m.ien).ravel() - 1, minlength=N)
    r_of = np.repeat(np.arange(N), np.diff(col))
    c_of = row - 1
    for i in vel:
        ri, ci = r_of == i, c_of == i
        for d in range(3):
            for j in range(3):
                v = s["K11"][ri, 3 * d + j]
                assert np.all(v[~(ci[ri] & (j == d))] == 0.0)
                w = s["K11"][ci, 3 * j + d]
                assert np.all(w[r_of[ci] != i] == 0.0)
            assert s["K11"][ri & ci, 4 * d][0] == cnt[i]
            assert np.all(s["G"][ri, d] == 0.0) and np.all(s["D1"][ci, d] == 0.0)
        assert np.all(s["rhsu"][i] == 0.0)
    for i in pre:
        ri, ci = r_of == i, c_of == i
        assert np.all(s["M"][ri & ~ci] == 0.0) and s["M"][ri & ci][0] == cnt[i]
        assert np.all(s["D1"][ri] == 0.0) and np.all(s["G"][ci] == 0.0)
        assert s["rhsp"][i] == 0.0


def test_scatter_is_the_sum_of_element_assemblies(oracle):
    """FillSparseMat / LocaltoGlobal through SparseMatLoc_3D (src/
    FillSparseMat.f90:4-67, 237-288; src/LocaltoGlobal.f90:26-51): the
    assembled matrix and RHS equal the sum, entry by entry over (row,
    column) pairs, of the same case assembled one element at a time (each a
    one-element mesh over the same nodes), BC masks included -- every
    element contributes its own unit diagonal at a constrained dof."""
    case = M.random_case(nx=3, ny=2, nz=2, seed=23, bc_frac=0.2)
    m = case.mesh
    N, E = m.nnode, m.nelem
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
    r_of = np.repeat(np.arange(N), np.diff(oc.col))
    slot = {(int(r), int(c) - 1): k for k, (r, c) in enumerate(zip(r_of, oc.row))}
    keys = ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS")
    acc = {k: np.zeros_like(oc.sys[k]) for k in keys}
    rhs = {k: np.zeros_like(oc.sys[k]) for k in ("rhsu", "rhsp", "rhsls")}
    for e in range(E):
        me = M.Mesh(m.xg, np.asfortranarray(m.ien[e:e + 1]), m.elm_id[e:e + 1].copy(), m.faces, m.dims, m.lengths)
        ce = M.Case(case.name, me, case.params, case.state, case.ibc, case.kernel)
        oe = oracle.OracleCase(ce)
        oe.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 3)
        re_of = np.repeat(np.arange(N), np.diff(oe.col))
        for ke, (r, c) in enumerate(zip(re_of, oe.row)):
            k = slot[(int(r), int(c) - 1)]
            for name in keys:
                acc[name][k] += oe.sys[name][ke]
        for name in rhs:
            rhs[name] += oe.sys[name]
    for name in keys:
        scale = max(np.abs(oc.sys[name]).max(), 1e-300)
        np.testing.assert_allclose(acc[name], oc.sys[name], rtol=0, atol=1e-13 * scale, err_msg=name)
    for name in rhs:
        scale = max(np.abs(oc.sys[name]).max(), 1e-300)
        np.testing.assert_allclose(rhs[name], oc.sys[name], rtol=0, atol=1e-13 * scale, err_msg=name)


def test_spmv_block_structure(oracle):
    """SparseProd_NS_conv / SparseProdUP_3D / SparseProd_LS (src/SparseProd.f90:
    4-60, 128-242) against a dense product built here from the CSR blocks:
    u rows take K11 (row component i, column component j at (i-1)*3+j), ULS
    and G; p rows take D1, PLS and M; phi rows take LSU and LS and no
    pressure; the (u, p) product drops the phi blocks; the scalar product
    uses the temperature values."""
    case = M.random_case(nx=3, ny=2, nz=2, seed=29)
    oc = oracle.OracleCase(case)
    N, K = oc.N, oc.icnt
    rng = np.random.default_rng(8)
    blocks = {"K11": rng.standard_normal((K, 9)), "G": rng.standard_normal((K, 3)), "D1": rng.standard_normal((K, 3)),
              "M": rng.standard_normal(K), "LS": rng.standard_normal(K), "LSU": rng.standard_normal((K, 3)),
              "ULS": rng.standard_normal((K, 3)), "PLS": rng.standard_normal(K)}
    oc.load_system("nsvof", {**blocks, "rhs": np.zeros((N, 5))})
    oc.load_system("tem", {"TEM": rng.standard_normal(K), "rhs": np.zeros((N, 1))})
    r_of = np.repeat(np.arange(N), np.diff(oc.col))
    c_of = oc.row - 1
    A = np.zeros((5 * N, 5 * N))          # field-major unknowns: u1, u2, u3, p, phi
    for k in range(K):
        r, c = r_of[k], c_of[k]
        for i in range(3):
            for j in range(3):
                A[i * N + r, j * N + c] += blocks["K11"][k, 3 * i + j]
            A[i * N + r, 3 * N + c] += blocks["G"][k, i]
            A[i * N + r, 4 * N + c] += blocks["ULS"][k, i]
            A[3 * N + r, i * N + c] += blocks["D1"][k, i]
            A[4 * N + r, i * N + c] += blocks["LSU"][k, i]
        A[3 * N + r, 3 * N + c] += blocks["M"][k]
        A[3 * N + r, 4 * N + c] += blocks["PLS"][k]
        A[4 * N + r, 4 * N + c] += blocks["LS"][k]
    x = rng.standard_normal((N, 5))
    want = (A @ x.T.reshape(-1)).reshape(5, N).T
    np.testing.assert_allclose(oc.spmv("nsvof", x), want, rtol=0, atol=1e-12 * np.abs(want).max())
    want_up = (A[:4 * N, :4 * N] @ x[:, :4].T.reshape(-1)).reshape(4, N).T
    np.testing.assert_allclose(oc.spmv("ns", x[:, :4]), want_up, rtol=0, atol=1e-12 * np.abs(want_up).max())
    T = np.zeros((N, N))
    np.add.at(T, (r_of, c_of), oc.sys["TEM"])
    np.testing.assert_allclose(oc.spmv("tem", x[:, :1])[:, 0], T @ x[:, 0], rtol=0, atol=1e-12 * np.abs(T).max() * 10)


@pytest.mark.parametrize("kind", ["ns", "nsvof", "tem"])
def test_gmres_preconditioner_rules(oracle, kind):
    """The block-diagonal preconditioners of SparseGMRES_up (src/
    SparseGMRES_NS.f90:74-121), SparseGMRES_ns_conv (src/SparseGMRES_NS_conv.f:
    54-139) and SparseGMRES_tem (src/SparseGMRES_tem.f90:52-58), through the
    cycle's first norm unorm = |P^-1 b|: the exact inverse of each 3x3
    velocity block, 1/M with 1 where M = 0, 1/LS with 0 where LS = 0, and
    1/diag with 1 where the temperature diagonal is 0; some diagonals are
    planted at 0."""
    case = M.random_case(nx=3, ny=2, nz=2, seed=31)
    oc = oracle.OracleCase(case)
    N, K = oc.N, oc.icnt
    rng = np.random.default_rng(9)
    r_of = np.repeat(np.arange(N), np.diff(oc.col))
    dslot = np.array([k for k in range(K) if oc.row[k] - 1 == r_of[k]])
    K11 = rng.standard_normal((K, 9))
    K11[dslot] += 4.0 * np.array([1, 0, 0, 0, 1, 0, 0, 0, 1])   # regular velocity blocks
    Mv, LS, TEM = rng.standard_normal(K), rng.standard_normal(K), rng.standard_normal(K)
    zero = rng.permutation(N)[:5]
    Mv[dslot[zero]] = 0.0
    LS[dslot[zero[:3]]] = 0.0
    TEM[dslot[zero[2:]]] = 0.0
    b = rng.standard_normal((N, 5))
    blocks = {"K11": K11, "G": rng.standard_normal((K, 3)), "D1": rng.standard_normal((K, 3)), "M": Mv, "LS": LS,
              "LSU": rng.standard_normal((K, 3)), "ULS": rng.standard_normal((K, 3)), "PLS": rng.standard_normal(K)}
    if kind == "tem":
        oc.load_system("tem", {"TEM": TEM, "rhs": b[:, :1]})
        t = TEM[dslot]
        pb = np.where(t == 0.0, 1.0, 1.0 / np.where(t == 0.0, 1.0, t)) * b[:, 0]
    else:
        nf = 5 if kind == "nsvof" else 4
        oc.load_system(kind, {**{k: v for k, v in blocks.items() if kind == "nsvof" or k in ("K11", "G", "D1", "M")},
                              "rhs": b[:, :nf]})
        pb = np.zeros((N, nf))
        for i in range(N):
            B = K11[dslot[i]].reshape(3, 3)
            pb[i, :3] = np.linalg.solve(B, b[i, :3])
            m = Mv[dslot[i]]
            pb[i, 3] = b[i, 3] / m if m != 0.0 else b[i, 3]
            if kind == "nsvof":
                ls = LS[dslot[i]]
                pb[i, 4] = b[i, 4] / ls if ls != 0.0 else 0.0
    _, _, _, r0 = oc.gmres(kind, 1e-3, 1, 1)
    assert abs(r0 - np.linalg.norm(pb)) <= 1e-12 * np.linalg.norm(pb)


def test_gmres_exit_rule_and_single_cycle(oracle):
    """The cycle's exit (src/SparseGMRES_NS.f90:327; SparseGMRES_tem.f90:219):
    stop when |e(k+1)| <= tol |P^-1 b| AND k >= Kspace_mn -- a loose
    tolerance still runs Kspace_mn iterations -- and no restart: a space too
    small for the tolerance returns after Kspace iterations with its partial
    solution, |e| above the target."""
    case = M.quench_case(M.box_tet(4, 3, 5, 1.0, 1.0, 1.25), "exit")
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(6, 3)
    _, it_loose, er, r0 = oc.gmres("nsvof", 0.9, 50, 1)
    assert it_loose >= 1 and er <= 0.9 * r0
    _, it_min, er_min, _ = oc.gmres("nsvof", 0.9, 50, 7)
    assert it_min == max(7, it_loose)
    s_short, it_short, er_short, r0s = oc.gmres("nsvof", 1e-12, 3, 1)
    assert it_short == 3 and er_short > 1e-12 * r0s and np.abs(s_short).max() > 0.0
    _, it_long, er_long, _ = oc.gmres("nsvof", 1e-12, 300, 1)
    assert it_long > 3 and er_long < er_short


@pytest.mark.parametrize("dims, hexa, N, E, nnz", [
    ((16, 16, 16), False, 4913, 24576, 66961),                  # config 1
    ((48, 48, 96), False, 232897, 1327104, 3398977),           # config 2
    ((128, 128, 128), False, 2146689, 12582912, 31802497),     # config 3 (the bench workload)
    ((96, 96, 96), True, 912673, 884736, 24137569),            # config 4
    ((32, 32, 32), False, 35937, 196608, 513313),              # config 5
])
def test_config_sizes(dims, hexa, N, E, nnz):
    """The sizes of the five workloads (nodes, elements, CSR entries) from
    the closed forms the pattern tests pin (Kuhn split: nodes + both
    directions of every edge; hexahedra: the 27-point stencil)."""
    nx, ny, nz = dims
    assert (nx + 1) * (ny + 1) * (nz + 1) == N
    assert (1 if hexa else 6) * nx * ny * nz == E
    assert (M.expected_nnz_hex if hexa else M.expected_nnz_kuhn)(nx, ny, nz) == nnz
