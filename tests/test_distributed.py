"""Distributed GMRES over owner-computes partitions (oversetdevfort_b200.
distributed), CPU: the halo plan, and the reference GMRES cycle run on
partitions -- three in one process (LocalComm) and two gloo ranks
(TorchComm) -- against the oracle's single-domain GMRES of the same system:
the same iteration count and the same solution to 1e-10, ghosts included.
The local products here use the oracle's local system (test stand-in for
the GPU operator, which tests/test_gpu_distributed.py covers), with the
interior / boundary split of the overlapped product: on the gloo ranks the
interior rows are computed while the halo messages are in flight."""
import os
import socket

import numpy as np
import pytest
import torch

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import distributed as D
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import partition as P

NF = {"nsvof": 5, "tem": 1, "ns": 4}


class OracleOperator:
    """P^-1 A and P^-1 of a partition's local system assembled by the oracle
    (block-diagonal preconditioner of SparseGMRES_*, as gm_setup_precond)."""

    def __init__(self, oc, kind):
        self.oc, self.kind = oc, kind
        N = oc.N
        col, row = oc.col.astype(np.int64) - 1, oc.row.astype(np.int64) - 1
        dslot = np.zeros(N, dtype=np.int64)
        for i in range(N):
            j = np.nonzero(row[col[i]:col[i + 1]] == i)[0][0]
            dslot[i] = col[i] + j
        with np.errstate(divide="ignore", invalid="ignore"):   # singular ghost blocks, overwritten before use
            self._setup(oc.sys, dslot, kind)

    def _setup(self, s, dslot, kind):
        if kind == "tem":
            md = s["TEM"][dslot]
            self.pinv = np.where(md == 0.0, 1.0, 1.0 / np.where(md == 0.0, 1.0, md))
            return
        K = s["K11"][dslot]
        b11 = K[:, 4] * K[:, 8] - K[:, 7] * K[:, 5]
        b12 = K[:, 7] * K[:, 2] - K[:, 1] * K[:, 8]
        b13 = K[:, 1] * K[:, 5] - K[:, 2] * K[:, 4]
        tmp = 1.0 / (b11 * K[:, 0] + b12 * K[:, 3] + b13 * K[:, 6])
        B = np.stack([b11 * tmp, b12 * tmp, b13 * tmp,
                      (K[:, 5] * K[:, 6] - K[:, 3] * K[:, 8]) * tmp, (K[:, 0] * K[:, 8] - K[:, 6] * K[:, 2]) * tmp,
                      (K[:, 3] * K[:, 2] - K[:, 0] * K[:, 5]) * tmp, (K[:, 3] * K[:, 7] - K[:, 4] * K[:, 6]) * tmp,
                      (K[:, 6] * K[:, 1] - K[:, 0] * K[:, 7]) * tmp, (K[:, 0] * K[:, 4] - K[:, 1] * K[:, 3]) * tmp], 1)
        self.B = B
        md = s["M"][dslot]
        self.pinv = np.where(md == 0.0, 1.0, 1.0 / np.where(md == 0.0, 1.0, md))
        if kind == "nsvof":
            ld = s["LS"][dslot]
            self.lsinv = np.where(ld == 0.0, 0.0, 1.0 / np.where(ld == 0.0, 1.0, ld))

    def _pre(self, x):   # x (nf, N) numpy; ghost rows are incomplete and may be singular
        if self.kind == "tem":
            return self.pinv[None, :] * x
        y = np.empty_like(x)
        for g in range(3):
            y[g] = self.B[:, 3 * g] * x[0] + self.B[:, 3 * g + 1] * x[1] + self.B[:, 3 * g + 2] * x[2]
        y[3] = x[3] * self.pinv
        if self.kind == "nsvof":
            y[4] = x[4] * self.lsinv
        return y

    def precond(self, x, y):
        with np.errstate(invalid="ignore"):
            y.copy_(torch.from_numpy(self._pre(x.numpy())))

    def matvec(self, x, y):
        ax = self.oc.spmv(self.kind, np.asfortranarray(x.numpy().T))
        with np.errstate(invalid="ignore"):
            y.copy_(torch.from_numpy(self._pre(np.ascontiguousarray(ax.T))))

    def split(self, owned):
        inner, bnd = D.split_rows(self.oc.col, self.oc.row, owned, self.oc.N)
        self.parts = {"interior": torch.as_tensor(inner), "boundary": torch.as_tensor(bnd)}

    def matvec_part(self, x, y, part):
        # the product from x as it is now (its ghosts may still be stale),
        # only the part's rows written
        full = torch.empty_like(y)
        self.matvec(x, full)
        idx = self.parts[part]
        y[:, idx] = full[:, idx]


def _case(kind):
    # a quench box: every node in fluid elements, so every diagonal block is
    # regular (random cases with solid-only nodes give singular blocks, and
    # the reference preconditioner NaNs on them in one domain or many)
    return M.quench_case(M.box_tet(6, 5, 8, 1.0, 1.0, 1.25), "dist")


def _local(oracle, case, part, kind):
    oc = oracle.OracleCase(P.local_case(case, part))
    oc.assemble_quenching(6, 4 if kind == "tem" else 3)
    return oc


def _global(oracle, case, kind, tol, kspace):
    og = oracle.OracleCase(case)
    og.assemble_quenching(6, 4 if kind == "tem" else 3)
    s, it, er, r0 = og.gmres(kind, tol, kspace, 1)
    assert np.isfinite(s).all() and it < kspace   # converged inside the cycle
    return s, it


def test_halo_plan_and_exchange():
    case = _case("nsvof")
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    N = case.mesh.nnode
    covered = np.zeros(N, dtype=int)
    for r, p in enumerate(parts):
        covered[p.nodes[plan.owned[r]]] += 1
        ghosts = np.setdiff1d(np.arange(p.nodes.size), plan.owned[r])
        got = np.concatenate([plan.recv[r][s] for s in range(3) if s != r])
        np.testing.assert_array_equal(np.sort(got), ghosts)
        for s in range(3):
            if s != r:   # what s sends to r are the same global nodes, in the same order
                np.testing.assert_array_equal(parts[s].nodes[plan.send[s][r]], p.nodes[plan.recv[r][s]])
    assert np.all(covered == 1)
    g = np.random.default_rng(0).standard_normal((2, N))
    vecs = {r: torch.from_numpy(np.where(np.isin(np.arange(p.nodes.size), plan.owned[r]), g[:, p.nodes], -7.0))
            for r, p in enumerate(parts)}
    D.LocalComm(plan).halo(vecs)
    for r, p in enumerate(parts):
        np.testing.assert_array_equal(vecs[r].numpy(), g[:, p.nodes])


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_local_comm_gmres_matches_single_domain(oracle, kind):
    case = _case(kind)
    tol, kspace = 1e-8, 200
    sg, itg = _global(oracle, case, kind, tol, kspace)
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ops, rhs = {}, {}
    for r, p in enumerate(parts):
        oc = _local(oracle, case, p, kind)
        ops[r] = OracleOperator(oc, kind)
        rhs[r] = torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))
    sol, info = D.gmres_cycle(D.LocalComm(plan), ops, rhs, tol, kspace, 1, tem=kind == "tem")
    assert info["converged"] and info["iterations"] == itg
    scale = np.abs(sg).max()
    for r, p in enumerate(parts):
        np.testing.assert_allclose(sol[r].numpy().T, sg[p.nodes], atol=1e-10 * scale, rtol=0)


def test_split_rows_interior_and_boundary(oracle):
    """Owned rows with every column owned are interior, the others
    boundary; ghost rows are in neither; each list ascending."""
    # 5 local nodes, 0-2 owned, 3-4 ghosts; rows (0-based columns):
    # 0: {0,1}  1: {0,1,3}  2: {2}  3: {1,3}  4: {4,2}
    rows = [[0, 1], [0, 1, 3], [2], [1, 3], [2, 4]]
    col = np.cumsum([0] + [len(r) for r in rows]) + 1
    row = np.concatenate([np.asarray(r) for r in rows]) + 1
    inner, bnd = D.split_rows(col, row, [2, 0, 1], 5)
    np.testing.assert_array_equal(inner, [0, 2])
    np.testing.assert_array_equal(bnd, [1])
    # one part owning every node: all rows interior; no owned node: nothing
    inner, bnd = D.split_rows(col, row, np.arange(5), 5)
    np.testing.assert_array_equal(inner, np.arange(5))
    assert bnd.size == 0
    inner, bnd = D.split_rows(col, row, np.zeros(0, dtype=np.int64), 5)
    assert inner.size == 0 and bnd.size == 0
    case = _case("nsvof")
    parts = P.make_parts(case.mesh, 3)
    for p in parts:
        oc = oracle.OracleCase(P.local_case(case, p))
        inner, bnd = D.split_rows(oc.col, oc.row, p.owned, p.nodes.size)
        assert inner.size + bnd.size == np.asarray(p.owned).size and inner.size > 0 and bnd.size > 0
        ghost = np.ones(p.nodes.size, bool)
        ghost[p.owned] = False
        c0, r0 = oc.col.astype(np.int64) - 1, oc.row.astype(np.int64) - 1
        for i in inner:
            assert not ghost[r0[c0[i]:c0[i + 1]]].any()
        for i in bnd:
            assert ghost[r0[c0[i]:c0[i + 1]]].any()


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_overlapped_products_give_the_same_cycle(oracle, kind):
    """Interior rows while the halo is in flight, boundary rows after it:
    the same iterations and the same solution bit for bit as the product
    taken whole after the halo exchange."""
    case = _case(kind)
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ops, rhs = {}, {}
    for r, p in enumerate(parts):
        oc = _local(oracle, case, p, kind)
        ops[r] = OracleOperator(oc, kind)
        rhs[r] = torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))
    out = [D.gmres_cycle(D.LocalComm(plan), ops, rhs, 1e-8, 200, 1, tem=kind == "tem", overlap=ov)
           for ov in (True, False)]
    (s1, i1), (s2, i2) = out
    assert i1["iterations"] == i2["iterations"] and i1["converged"]
    for r in s1:
        np.testing.assert_array_equal(s1[r].numpy(), s2[r].numpy())

    class WholeHaloComm:
        """A comm with the whole-vector exchange only (no halo_start):
        the cycle takes each product whole after it."""

        def __init__(self, plan):
            self.plan, self._c = plan, D.LocalComm(plan)

        def __getattr__(self, name):
            if name in ("halo_start", "halo_finish"):
                raise AttributeError(name)
            return getattr(self._c, name)

    s3, i3 = D.gmres_cycle(WholeHaloComm(plan), ops, rhs, 1e-8, 200, 1, tem=kind == "tem")
    assert i3["iterations"] == i1["iterations"]
    for r in s1:
        np.testing.assert_array_equal(s3[r].numpy(), s1[r].numpy())


def test_cgs2_orthogonalization_converges_to_the_same_solution(oracle):
    """The batched (classical, twice) Gram-Schmidt variant: two vector sums
    per Arnoldi step instead of k + 1 scalar ones; it reaches the tolerance
    within a few iterations of the reference's modified Gram-Schmidt and the
    same solution to the tolerance's order."""
    kind = "nsvof"
    case = _case(kind)
    tol, kspace = 1e-8, 200
    sg, itg = _global(oracle, case, kind, tol, kspace)
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ops, rhs = {}, {}
    for r, p in enumerate(parts):
        oc = _local(oracle, case, p, kind)
        ops[r] = OracleOperator(oc, kind)
        rhs[r] = torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))
    sol, info = D.gmres_cycle(D.LocalComm(plan), ops, rhs, tol, kspace, 1, orthog="cgs2")
    assert info["converged"] and abs(info["iterations"] - itg) <= 3
    scale = np.abs(sg).max()
    for r, p in enumerate(parts):
        np.testing.assert_allclose(sol[r].numpy().T, sg[p.nodes], atol=1e-6 * scale, rtol=0)
    with pytest.raises(ValueError):
        D.gmres_cycle(D.LocalComm(plan), ops, rhs, tol, kspace, 1, orthog="householder")


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q, orthog="mgs"):
    import datetime
    import torch.distributed as dist
    from oracle import pyoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    kind, tol, kspace = "nsvof", 1e-8, 200
    case = _case(kind)
    parts = P.make_parts(case.mesh, world)
    plan = D.halo_plan(parts)
    oc = _local(pyoracle, case, parts[rank], kind)
    ops = {rank: OracleOperator(oc, kind)}
    rhs = {rank: torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))}
    sol, info = D.gmres_cycle(D.TorchComm(plan, rank), ops, rhs, tol, kspace, 1, orthog=orthog)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object((parts[rank].nodes, sol[rank].numpy(), info["iterations"]), gathered, dst=0)
    if rank == 0:
        sg, itg = _global(pyoracle, case, kind, tol, kspace)
        scale = np.abs(sg).max()
        if orthog == "mgs":   # the reference's order: the same iterations, the same solution
            ok = all(it == itg and np.isfinite(s).all() and np.abs(s.T - sg[nodes]).max() <= 1e-10 * scale
                     for nodes, s, it in gathered)
        else:                 # batched Gram-Schmidt: converged to the tolerance's order
            ok = all(abs(it - itg) <= 3 and np.isfinite(s).all() and np.abs(s.T - sg[nodes]).max() <= 1e-6 * scale
                     for nodes, s, it in gathered)
        q.put(bool(ok))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("orthog", ["mgs", "cgs2"])
def test_two_gloo_ranks_gmres(oracle, orthog):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q, orthog)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ok


# ------------------------------------------------- partitioned Newton loop

class OraclePartition:
    """A partition's local system on the oracle, with the methods
    distributed.quench_newton calls (stand-in for ContextPartition)."""

    def __init__(self, oc, owned):
        self.oc, self.owned = oc, np.asarray(owned)

    def assemble(self, tensor_flag, field_flag):
        self.oc.assemble_quenching(tensor_flag, field_flag)

    def residual_sq(self):
        s, o = self.oc.sys, self.owned
        return np.array([np.sum(s["rhsu"][o] ** 2), np.sum(s["rhsp"][o] ** 2), np.sum(s["rhsls"][o] ** 2),
                         np.sum(s["rhstem"][o] ** 2)])

    def rhs(self, kind):
        return torch.from_numpy(np.ascontiguousarray(self.oc.system(kind)["rhs"].T))

    def operator(self, kind):
        return OracleOperator(self.oc, kind)

    def update(self, kind, sol):
        self.oc.newton_update(F.OVS_SYS_NSVOF if kind == "nsvof" else F.OVS_SYS_TEM,
                              np.asfortranarray(sol.numpy().T))


NEWTON = dict(newton_max=3, solve_tem=True, kspace=150, kspace_min=1, tol_ns=1e-8, tol_tem=1e-8,
              utol=(1e-6,) * 4, atol=(1e-30,) * 4)


def _stirred_case():
    case = M.quench_case(M.box_tet(5, 5, 6, 1.0, 1.0, 1.25), "dnewton")
    rng = np.random.default_rng(3)   # the box at rest has no momentum residual
    free = np.asarray(case.ibc)[:, 0] == 0
    for f in ("ug", "ugold"):
        case.state[f][free] = 0.05 * rng.standard_normal((int(free.sum()), 3))
    return case


def _one_domain_newton(oracle, case):
    og = oracle.OracleCase(case)
    n = NEWTON
    out = og.quench_newton(n["newton_max"], n["solve_tem"], n["kspace"], n["kspace_min"], n["tol_ns"],
                           n["tol_tem"], n["utol"], n["atol"])
    return og, out


def _compare_newton(out, ref, states, og, parts, r0_rtol=1e-12):
    """Same iterations and Krylov counts; the residuals to 1e-4 relative
    (the temperature residual ends 24 orders below its start, where the
    summation order of the dots shows) plus 1e-16 of the initial one; the
    state of every local node (ghosts too) to 1e-10 (measured: 2e-13).
    residual0 agrees to r0_rtol: 1e-12 for a first step, looser after
    earlier steps whose states already differ in the last digits."""
    assert out["iterations"] == ref["iterations"] >= 1
    assert out["krylov_iterations_ns"] == ref["krylov_ns"] > 0
    assert out["krylov_iterations_tem"] == ref["krylov_tem"] > 0
    assert out["converged"] == ref["converged"]
    np.testing.assert_allclose(out["residual0"], ref["residual0"], rtol=r0_rtol)
    r0, r, rr = (np.asarray(ref["residual0"]), np.asarray(out["residual"]), np.asarray(ref["residual"]))
    assert np.all(np.abs(r - rr) <= 1e-4 * np.abs(rr) + 1e-16 * r0), (r, rr)
    for name in ("ug", "acg", "pg", "phig", "rphig", "tg", "rtg"):
        g = og.state_arrays[name]
        scale = max(np.abs(g).max(), 1e-300)
        for st, p in zip(states, parts):
            np.testing.assert_allclose(st[name], g[p.nodes], rtol=0, atol=1e-10 * scale, err_msg=name)


@pytest.mark.parametrize("nparts", [2, 3, 4])
def test_partitioned_newton_matches_one_domain(oracle, nparts):
    """distributed.quench_newton over partitions in one process against the
    oracle's one-domain solmultiphasethermofluid_stag loop."""
    case = _stirred_case()
    og, ref = _one_domain_newton(oracle, case)
    parts = P.make_parts(case.mesh, nparts)
    plan = D.halo_plan(parts)
    ocs = {r: oracle.OracleCase(P.local_case(case, p)) for r, p in enumerate(parts)}
    sys_parts = {r: OraclePartition(ocs[r], plan.owned[r]) for r in ocs}
    with np.errstate(divide="ignore", invalid="ignore"):
        out = D.quench_newton(D.LocalComm(plan), sys_parts, **NEWTON)
    _compare_newton(out, ref, [ocs[r].state_arrays for r in ocs], og, parts)
    assert out["residual"][0] < 1e-3 * out["residual0"][0]


def _newton_rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from oracle import pyoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    case = _stirred_case()
    parts = P.make_parts(case.mesh, world)
    plan = D.halo_plan(parts)
    oc = pyoracle.OracleCase(P.local_case(case, parts[rank]))
    with np.errstate(divide="ignore", invalid="ignore"):
        out = D.quench_newton(D.TorchComm(plan, rank), {rank: OraclePartition(oc, plan.owned[rank])}, **NEWTON)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object({k: oc.state_arrays[k] for k in ("ug", "acg", "pg", "phig", "rphig", "tg", "rtg")},
                       gathered, dst=0)
    if rank == 0:
        try:
            og, ref = _one_domain_newton(pyoracle, case)
            _compare_newton(out, ref, gathered, og, parts)
            q.put(True)
        except AssertionError as e:
            q.put(str(e))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_newton(oracle):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_newton_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ok is True, ok


class OracleBcPartition(OraclePartition):
    """OraclePartition whose BC producers run on its part of the setBCs input."""

    def __init__(self, oc, owned, spec):
        super().__init__(oc, owned)
        self.spec = spec

    def apply_bcs(self):
        self.oc.set_bcs(self.spec, 3)


def test_partitioned_newton_with_bc_producers(oracle):
    """quench_newton(bcs=True): setBCs_NSVOF/setBCs_Tem on every part's own
    boundary nodes (partition.local_bc_spec) where the reference calls them;
    three parts follow the one-part run: Newton and Krylov iterations equal,
    the state of every local node to 1e-10, IBC equal."""
    case = _stirred_case()
    m = case.mesh
    # walls and floor no-slip, the top free (its natural condition fixes the
    # pressure level), the floor at 300 K, the top kept gas
    spec = M.box_bc_spec(m, u={b: (0.0, 0.0, 0.0) for b in range(1, 6)}, phi={6: 1.0}, T={5: 300.0},
                         face_ids=(2, 1, 3, 4, 6, 5))
    runs = {}
    for nparts in (1, 3):
        parts = P.make_parts(m, nparts)
        plan = D.halo_plan(parts)
        ocs = {r: oracle.OracleCase(P.local_case(case, p)) for r, p in enumerate(parts)}
        sp = {r: OracleBcPartition(ocs[r], plan.owned[r], P.local_bc_spec(spec, parts[r])) for r in ocs}
        with np.errstate(divide="ignore", invalid="ignore"):
            out = D.quench_newton(D.LocalComm(plan), sp, bcs=True, **NEWTON)
        runs[nparts] = (out, ocs, parts)
    (o1, oc1, p1), (o3, oc3, p3) = runs[1], runs[3]
    assert o1["iterations"] >= 1 and o1["krylov_iterations_ns"] > 0 and o1["krylov_iterations_tem"] > 0
    assert np.all(np.isfinite(o1["residual"])) and o1["residual"][0] < 1e-3 * o1["residual0"][0]
    assert (o3["iterations"], o3["krylov_iterations_ns"], o3["krylov_iterations_tem"]) == \
        (o1["iterations"], o1["krylov_iterations_ns"], o1["krylov_iterations_tem"])
    g = oc1[0].state_arrays
    for r, p in enumerate(p3):
        np.testing.assert_array_equal(oc3[r].ibc, oc1[0].ibc[p.nodes])
        for name in ("ug", "acg", "pg", "phig", "rphig", "tg", "rtg"):
            scale = max(np.abs(g[name]).max(), 1e-300)
            np.testing.assert_allclose(oc3[r].state_arrays[name], g[name][p.nodes], rtol=0, atol=1e-10 * scale,
                                       err_msg=name)
    # the producers ran: the floor holds 300 K and the top phi = 1
    floor, top = np.asarray(m.faces[4]), np.asarray(m.faces[5])
    np.testing.assert_array_equal(g["tg"][floor], 300.0)
    np.testing.assert_array_equal(g["phig"][top], 1.0)


class OracleStepPartition(OraclePartition):
    """OraclePartition with the driver's predictor and old-value copies."""

    def predictor(self):
        st, g = self.oc.state_arrays, self.oc.params.gami
        st["ug"][...] = st["ugold"]
        st["acg"][...] = (g - 1.0) / g * st["acgold"]

    def commit_old(self, update_vof_tem_old):
        st = self.oc.state_arrays
        pairs = [("ug", "ugold"), ("acg", "acgold"), ("dg", "dgold"), ("ugm", "ugmold"), ("acgm", "acgmold")]
        if update_vof_tem_old:
            pairs += [("phig", "phigold"), ("rphig", "rphigold"), ("tg", "tgold"), ("rtg", "rtgold")]
        for cur, old in pairs:
            st[old][...] = st[cur]


def test_partitioned_time_loop_matches_one_domain(oracle):
    """distributed.quench_time_steps over three parts against the oracle's
    one-domain driver loop: steps 0-2 (one Newton iteration and no
    temperature solve at step 0, one iteration at step 1, up to three at
    step 2); the last step's record and every local node's state, old
    values included, agree."""
    case = _stirred_case()
    n = dict(NEWTON)
    og = oracle.OracleCase(case)
    ref = og.quench_time_steps(0, 3, n["newton_max"], n["solve_tem"], n["kspace"], n["kspace_min"], n["tol_ns"],
                               n["tol_tem"], n["utol"], n["atol"])
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    ocs = {r: oracle.OracleCase(P.local_case(case, p)) for r, p in enumerate(parts)}
    sp = {r: OracleStepPartition(ocs[r], plan.owned[r]) for r in ocs}
    with np.errstate(divide="ignore", invalid="ignore"):
        last, kt = D.quench_time_steps(D.LocalComm(plan), sp, 0, 3, **n)
    _compare_newton(last, ref, [ocs[r].state_arrays for r in ocs], og, parts, r0_rtol=1e-8)
    assert kt >= last["krylov_iterations_ns"] + last["krylov_iterations_tem"]
    for r, p in enumerate(parts):
        for name in ("ugold", "acgold"):
            g = og.state_arrays[name]
            np.testing.assert_allclose(ocs[r].state_arrays[name], g[p.nodes], rtol=0,
                                       atol=1e-10 * np.abs(g).max(), err_msg=name)


class OracleApply(OracleOperator):
    """OracleOperator with the plain product y = A x (refinement residual)."""

    def apply(self, x, y):
        y.copy_(torch.from_numpy(np.ascontiguousarray(self.oc.spmv(self.kind, np.asfortranarray(x.numpy().T)).T)))


def _fp32_copy(oracle, case, part, kind, oc64):
    """The same local system with every matrix value rounded to FP32 (the
    inner operator of the mixed-precision refinement)."""
    oc = oracle.OracleCase(P.local_case(case, part))
    d = oc64.system(kind)
    oc.load_system(kind, {k: (v if k == "rhs" else v.astype(np.float32).astype(np.float64)) for k, v in d.items()})
    return oc


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_partitioned_refined_solve_reaches_true_residual(oracle, kind):
    """distributed.solve_refined over three parts: inner GMRES cycles on the
    FP32-rounded system (floor 1e-6 per cycle), the FP64 residual outside;
    the true relative residual, recomputed here on the one-domain FP64
    system from the gathered owned rows, is below 1e-8, and it took more
    than one cycle."""
    case = _case(kind)
    rtol = 1e-8
    parts = P.make_parts(case.mesh, 3)
    plan = D.halo_plan(parts)
    inner, outer, rhs = {}, {}, {}
    for r, p in enumerate(parts):
        oc = _local(oracle, case, p, kind)
        outer[r] = OracleApply(oc, kind)
        inner[r] = OracleOperator(_fp32_copy(oracle, case, p, kind, oc), kind)
        rhs[r] = torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))
    x, info = D.solve_refined(D.LocalComm(plan), inner, outer, rhs, rtol, kspace=60, max_cycles=50,
                              tem=kind == "tem")
    assert info["converged"] and info["cycles"] > 1 and info["rel_residual"] <= rtol
    og = oracle.OracleCase(case)
    og.assemble_quenching(6, 4 if kind == "tem" else 3)
    nf = NF[kind]
    xg = np.zeros((case.mesh.nnode, nf))
    for r, p in enumerate(parts):
        xg[p.nodes[plan.owned[r]]] = x[r].numpy().T[plan.owned[r]]
    for r, p in enumerate(parts):   # ghosts hold their owners' values exactly
        np.testing.assert_array_equal(x[r].numpy().T, xg[p.nodes])
    b = og.system(kind)["rhs"]
    res = b - og.spmv(kind, np.asfortranarray(xg))
    true_rel = np.linalg.norm(res) / np.linalg.norm(b)
    assert true_rel <= 1.01 * rtol, true_rel
    assert abs(true_rel - info["rel_residual"]) <= 1e-3 * rtol


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_partitioned_flexible_solve_reaches_true_residual(oracle, kind):
    """distributed.solve_flexible over three parts: an FGMRES(30) outer on the
    FP64 operators, each direction one GMRES cycle on the FP32-rounded
    system; the true relative residual, recomputed on the one-domain FP64
    system from the gathered owned rows, is below 1e-8, and three parts
    follow one part (cycles and iterations equal, solution to 1e-10)."""
    case = _case(kind)
    rtol = 1e-8
    og = oracle.OracleCase(case)
    og.assemble_quenching(6, 4 if kind == "tem" else 3)
    nf = NF[kind]
    res = {}
    for nparts in (1, 3):
        parts = P.make_parts(case.mesh, nparts)
        plan = D.halo_plan(parts)
        inner, outer, rhs = {}, {}, {}
        for r, p in enumerate(parts):
            oc = _local(oracle, case, p, kind)
            outer[r] = OracleApply(oc, kind)
            inner[r] = OracleOperator(_fp32_copy(oracle, case, p, kind, oc), kind)
            rhs[r] = torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))
        comm = D.LocalComm(plan)
        x, info = D.solve_flexible(comm, inner, outer, rhs, rtol, kspace=60, max_cycles=50, tem=kind == "tem")
        assert info["converged"] and info["rel_residual"] <= rtol
        xg = np.zeros((case.mesh.nnode, nf))
        for r, p in enumerate(parts):
            xg[p.nodes[plan.owned[r]]] = x[r].numpy().T[plan.owned[r]]
        for r, p in enumerate(parts):   # ghosts hold their owners' values exactly
            np.testing.assert_array_equal(x[r].numpy().T, xg[p.nodes])
        b = og.system(kind)["rhs"]
        true_rel = np.linalg.norm(b - og.spmv(kind, np.asfortranarray(xg))) / np.linalg.norm(b)
        assert true_rel <= 1.01 * rtol, true_rel
        assert abs(true_rel - info["rel_residual"]) <= 1e-3 * rtol
        res[nparts] = (xg, info)
    (x1, i1), (x3, i3) = res[1], res[3]
    assert (i1["cycles"], i1["iterations"]) == (i3["cycles"], i3["iterations"])
    np.testing.assert_allclose(x3, x1, rtol=0, atol=1e-10 * np.abs(x1).max())


def _refined_rank_main(rank, world, port, q, solver="refined"):
    import datetime
    import torch.distributed as dist
    from oracle import pyoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    kind, rtol = "nsvof", 1e-8
    case = _case(kind)
    parts = P.make_parts(case.mesh, world)
    plan = D.halo_plan(parts)
    oc = _local(pyoracle, case, parts[rank], kind)
    inner = {rank: OracleOperator(_fp32_copy(pyoracle, case, parts[rank], kind, oc), kind)}
    outer = {rank: OracleApply(oc, kind)}
    rhs = {rank: torch.from_numpy(np.ascontiguousarray(oc.system(kind)["rhs"].T))}
    solve = D.solve_flexible if solver == "flexible" else D.solve_refined
    with np.errstate(divide="ignore", invalid="ignore"):
        x, info = solve(D.TorchComm(plan, rank), inner, outer, rhs, rtol, kspace=60, max_cycles=50)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object((parts[rank].nodes, plan.owned[rank], x[rank].numpy(), info), gathered, dst=0)
    if rank == 0:
        og = pyoracle.OracleCase(case)
        og.assemble_quenching(6, 3)
        xg = np.zeros((case.mesh.nnode, NF[kind]))
        for nodes, owned, xl, _ in gathered:
            xg[nodes[owned]] = xl.T[owned]
        b = og.system(kind)["rhs"]
        true_rel = np.linalg.norm(b - og.spmv(kind, np.asfortranarray(xg))) / np.linalg.norm(b)
        same = len({(i["cycles"], i["iterations"]) for *_, i in gathered}) == 1
        q.put(bool(info["converged"] and (info["cycles"] > 1 or solver == "flexible") and true_rel <= 1.01 * rtol
                   and same))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("solver", ["refined", "flexible"])
def test_two_gloo_ranks_refined_solve(oracle, solver):
    """solve_refined and solve_flexible on two gloo ranks reach the true
    residual, both ranks reporting the same cycles and iterations."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_refined_rank_main, args=(r, 2, port, q, solver)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ok


_ROUND32 = ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS", "TEM", "rhsu", "rhsp", "rhsls", "rhstem")


class OracleMixedPartition(OraclePartition):
    """OraclePartition with a precision argument: FP32 assembly emulated by
    rounding the assembled matrix and right-hand sides to FP32."""

    def assemble(self, tensor_flag, field_flag, precision=F.OVS_FP64):
        self.oc.assemble_quenching(tensor_flag, field_flag)
        if precision == F.OVS_FP32:
            for k in _ROUND32:
                a = self.oc.sys[k]
                a[...] = a.astype(np.float32).astype(np.float64)

    def residual_sq(self, precision=F.OVS_FP64):
        return super().residual_sq()

    def rhs(self, kind, precision=F.OVS_FP64):
        return super().rhs(kind)

    def operator(self, kind, precision=F.OVS_FP64):
        return OracleApply(self.oc, kind)


def test_partitioned_newton_mixed_mode(oracle):
    """quench_newton(mode=OVS_FP32): FP32 assembly and refined solves to
    tol_ns / tol_tem over the partitions.  Three parts follow one part
    (Newton and Krylov iterations equal, state to 1e-10), take the Newton
    iterations of the FP64 one-domain loop, and end within 1e-4 of its state
    (FP32 rounding of the system: measured 2.2e-5 for u)."""
    case = _stirred_case()
    og, ref = _one_domain_newton(oracle, case)
    runs = {}
    for nparts in (1, 3):
        parts = P.make_parts(case.mesh, nparts)
        plan = D.halo_plan(parts)
        ocs = {r: oracle.OracleCase(P.local_case(case, p)) for r, p in enumerate(parts)}
        sp = {r: OracleMixedPartition(ocs[r], plan.owned[r]) for r in ocs}
        with np.errstate(divide="ignore", invalid="ignore"):
            out = D.quench_newton(D.LocalComm(plan), sp, mode=F.OVS_FP32, max_cycles=40, **NEWTON)
        runs[nparts] = (out, ocs, parts)
    (o1, oc1, _), (o3, oc3, p3) = runs[1], runs[3]
    assert o1["converged"] and o1["iterations"] == ref["iterations"]
    assert (o3["iterations"], o3["krylov_iterations_ns"], o3["krylov_iterations_tem"]) == \
        (o1["iterations"], o1["krylov_iterations_ns"], o1["krylov_iterations_tem"])
    assert o3["residual"][0] < 1e-3 * o3["residual0"][0]
    for name in ("ug", "pg", "phig", "tg"):
        g1, g = oc1[0].state_arrays[name], og.state_arrays[name]
        scale = np.abs(g).max()
        np.testing.assert_allclose(g1, g, rtol=0, atol=1e-4 * scale, err_msg=name)
        for r, p in enumerate(p3):
            np.testing.assert_allclose(oc3[r].state_arrays[name], g1[p.nodes], rtol=0, atol=1e-10 * scale,
                                       err_msg=name)


class OracleStepBcPartition(OracleStepPartition):
    def __init__(self, oc, owned, spec):
        super().__init__(oc, owned)
        self.spec = spec

    def apply_bcs(self):
        self.oc.set_bcs(self.spec, 3)


def test_partitioned_time_loop_with_bc_producers(oracle):
    """quench_time_steps(bcs=True) over steps 0-2: three parts, each with its
    own part of the setBCs input, follow the one-part run (iterations,
    Krylov counts, state and old values to 1e-10, IBC equal)."""
    case = _stirred_case()
    m = case.mesh
    spec = M.box_bc_spec(m, u={b: (0.0, 0.0, 0.0) for b in range(1, 6)}, phi={6: 1.0}, T={5: 300.0})
    runs = {}
    for nparts in (1, 3):
        parts = P.make_parts(m, nparts)
        plan = D.halo_plan(parts)
        ocs = {r: oracle.OracleCase(P.local_case(case, p)) for r, p in enumerate(parts)}
        sp = {r: OracleStepBcPartition(ocs[r], plan.owned[r], P.local_bc_spec(spec, parts[r])) for r in ocs}
        with np.errstate(divide="ignore", invalid="ignore"):
            last, kt = D.quench_time_steps(D.LocalComm(plan), sp, 0, 3, bcs=True, **NEWTON)
        runs[nparts] = (last, kt, ocs, parts)
    (l1, k1, o1, _), (l3, k3, o3, p3) = runs[1], runs[3]
    assert k1 == k3 and l1["iterations"] == l3["iterations"] and np.isfinite(l1["residual"]).all()
    g = o1[0].state_arrays
    for r, p in enumerate(p3):
        np.testing.assert_array_equal(o3[r].ibc, o1[0].ibc[p.nodes])
        for name in ("ug", "acg", "pg", "phig", "tg", "ugold", "acgold"):
            scale = max(np.abs(g[name]).max(), 1e-300)
            np.testing.assert_allclose(o3[r].state_arrays[name], g[name][p.nodes], rtol=0, atol=1e-10 * scale,
                                       err_msg=name)


class OracleRoundPartition(OracleMixedPartition):
    """OracleMixedPartition for mode OVS_MIXED: FP64 assembly, and `round`
    makes the FP32 rounding of the FP64 local matrix the inner operator
    (as ContextPartition.round does with ovs_round_matrix)."""

    def __init__(self, oracle, case, part, owned):
        super().__init__(oracle.OracleCase(P.local_case(case, part)), owned)
        self.oracle, self.case, self.part, self.rounded = oracle, case, part, {}

    def round(self, kind):
        self.rounded[kind] = _fp32_copy(self.oracle, self.case, self.part, kind, self.oc)

    def operator(self, kind, precision=F.OVS_FP64):
        if precision == F.OVS_FP32:
            return OracleOperator(self.rounded[kind], kind)
        return OracleApply(self.oc, kind)


def test_partitioned_newton_mixed_on_the_fp64_system(oracle):
    """quench_newton(mode=OVS_MIXED): FP64 assembly and residuals, every solve
    refined against the FP64 local operators with inner cycles on their FP32
    rounding.  Three parts follow one part (Newton and Krylov iterations
    equal, state to 1e-10) and take the FP64 one-domain loop's Newton
    iterations, ending within 1e-4 of its state (measured 2.2e-5 for u: the
    linear solves stop at different points, a true residual of 1e-8 here and
    the reference cycle's preconditioned estimate there)."""
    case = _stirred_case()
    og, ref = _one_domain_newton(oracle, case)
    runs = {}
    for nparts in (1, 3):
        parts = P.make_parts(case.mesh, nparts)
        plan = D.halo_plan(parts)
        sp = {r: OracleRoundPartition(oracle, case, p, plan.owned[r]) for r, p in enumerate(parts)}
        with np.errstate(divide="ignore", invalid="ignore"):
            out = D.quench_newton(D.LocalComm(plan), sp, mode=F.OVS_MIXED, max_cycles=40, **NEWTON)
        runs[nparts] = (out, sp, parts)
    (o1, sp1, _), (o3, sp3, p3) = runs[1], runs[3]
    assert o1["converged"] and o1["iterations"] == ref["iterations"]
    assert (o3["iterations"], o3["krylov_iterations_ns"], o3["krylov_iterations_tem"]) == \
        (o1["iterations"], o1["krylov_iterations_ns"], o1["krylov_iterations_tem"])
    for name in ("ug", "pg", "phig", "tg"):
        g1, g = sp1[0].oc.state_arrays[name], og.state_arrays[name]
        scale = np.abs(g).max()
        np.testing.assert_allclose(g1, g, rtol=0, atol=1e-4 * scale, err_msg=name)
        for r, p in enumerate(p3):
            np.testing.assert_allclose(sp3[r].oc.state_arrays[name], g1[p.nodes], rtol=0, atol=1e-10 * scale,
                                       err_msg=name)
