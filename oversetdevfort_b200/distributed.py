"""Distributed Krylov solve over owner-computes partitions (one rank per GPU).

The reference runs SparseGMRES_ns_conv / SparseGMRES_up / SparseGMRES_tem on
METIS element partitions and keeps shared nodes consistent with commu: after
each product the partial rows of shared nodes are summed on their master
('in') and the master values are copied back ('out'), and every dot product
is an MPI_ALLREDUCE (src/SparseGMRES_NS_conv.f:65-76, 169-176, 210-251,
287-308, 391-395; src/commu.f90:118-266).

Here every rank owns a contiguous range of nodes and holds every element
touching them (`partition.make_parts`), so the rows of its owned nodes are
complete after a purely local assembly.  The same GMRES cycle then needs two
exchanges per Arnoldi step:

* a halo update before each product: the ghost entries of the vector (local
  nodes owned by another rank) receive their owners' values; the product's
  owned rows are then exact;
* a global sum for every dot product, over owned entries only (each node
  counted once).

The algebra of the cycle is the reference's, step for step (modified
Gram-Schmidt with the norm as the last dot, Givens rotations, back
substitution), as in `ovs_gmres` for one context; only the summation order
of the dot products differs.  `LocalComm` runs several partitions in one
process (one GPU, or the host); `TorchComm` runs one partition per process
over `torch.distributed` (NCCL between GPUs, gloo on the host), with
point-to-point halo messages and one all-reduce per dot product (or, with
orthog="cgs2", two vector all-reduces and one norm per Arnoldi step).  The local
products are this package's CUDA kernels (`DeviceOperator`, through
`ovs_spmv_device` / `ovs_precond_device`); the exchanges and the small
Hessenberg algebra run on the host side of each rank.  Each product is
split around its halo exchange: the rows that read no ghost entry run
while the messages are in flight, the others after the ghosts land
(`split_rows`, `ovs_spmv_device_rows`).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _ffi as F
from .api import check_convergence


@dataclass
class HaloPlan:
    owned: list     # per part: local indices of the owned nodes (ascending global id)
    send: list      # send[r][s]: local indices (in r) of r's owned nodes that part s holds as ghosts
    recv: list      # recv[r][s]: local indices (in r) of r's ghosts owned by part s
    nlocal: list    # per part: local node count


def halo_plan(parts) -> HaloPlan:
    """Exchange lists of a set of `partition.Part`s (all parts of the mesh)."""
    nparts = len(parts)
    N = int(max(int(p.nodes.max()) for p in parts if p.nodes.size)) + 1
    owner = np.full(N, -1, dtype=np.int64)
    loc = []
    for r, p in enumerate(parts):
        owner[p.nodes[p.owned]] = r
        lr = np.full(N, -1, dtype=np.int64)
        lr[p.nodes] = np.arange(p.nodes.size)
        loc.append(lr)
    if np.any(owner < 0):
        raise ValueError("every node must be owned by one part")
    send = [[np.zeros(0, np.int64) for _ in range(nparts)] for _ in range(nparts)]
    recv = [[np.zeros(0, np.int64) for _ in range(nparts)] for _ in range(nparts)]
    for r, p in enumerate(parts):
        own_of = owner[p.nodes]
        for s in range(nparts):
            if s == r:
                continue
            g = np.nonzero(own_of == s)[0]          # r's ghosts owned by s, ascending global id
            recv[r][s] = g
            send[s][r] = loc[s][p.nodes[g]]
    return HaloPlan([np.asarray(p.owned, dtype=np.int64) for p in parts], send, recv,
                    [int(p.nodes.size) for p in parts])


def split_rows(col, row, owned, nlocal: int):
    """The owned rows of a partition's local CSR pattern (col: row pointer,
    row: column indices, both 1-based, as ovs_get_pattern gives them) split
    into interior rows, whose columns are all owned nodes, and boundary rows,
    which read at least one ghost; each ascending.  The interior part of a
    product needs no halo values, so it can run while the halo exchange is
    in flight."""
    col = np.asarray(col, dtype=np.int64) - 1
    row = np.asarray(row, dtype=np.int64) - 1
    ghost = np.ones(nlocal, dtype=bool)
    ghost[np.asarray(owned, dtype=np.int64)] = False
    rid = np.repeat(np.arange(nlocal), np.diff(col))
    reads_ghost = np.bincount(rid, weights=ghost[row].astype(np.float64), minlength=nlocal) > 0
    own = np.sort(np.asarray(owned, dtype=np.int64))
    return own[~reads_ghost[own]], own[reads_ghost[own]]


class _Index:
    """Index tensors of a plan on a device, made once."""

    def __init__(self, plan: HaloPlan):
        self.plan = plan
        self.cache = {}

    def get(self, key, arr, device):
        import torch
        k = (key, str(device))
        if k not in self.cache:
            self.cache[k] = torch.as_tensor(arr, dtype=torch.long, device=device)
        return self.cache[k]


class LocalComm:
    """All partitions in this process: halo copies between their vectors,
    global sums as plain sums in part order."""

    def __init__(self, plan: HaloPlan):
        self.plan = plan
        self.idx = _Index(plan)

    def parts(self):
        return list(range(len(self.plan.owned)))

    def allreduce(self, vals):
        s = 0.0
        for v in vals:
            s += v
        return s

    def allreduce_vec(self, vals):
        s = np.zeros_like(vals[0])
        for v in vals:
            s = s + v
        return s

    def allreduce_t(self, vals):
        """Sum of 0-dim tensors (one per part) as a tensor on the first
        part's device, in part order, without a host round trip."""
        s = vals[0]
        for v in vals[1:]:
            s = s + v.to(s.device)
        return s

    def halo_start(self, vecs: dict):
        """In one process the halo copies are done at once."""
        self.halo(vecs)

    def halo_finish(self, handle):
        pass

    def halo(self, vecs: dict):
        pl = self.plan
        for r in vecs:
            for s in vecs:
                if s == r or pl.recv[r][s].size == 0:
                    continue
                dev = vecs[r].device
                vecs[r][:, self.idx.get(("r", r, s), pl.recv[r][s], dev)] = \
                    vecs[s][:, self.idx.get(("s", s, r), pl.send[s][r], vecs[s].device)].to(dev)


class TorchComm:
    """One partition per process over torch.distributed (rank = part)."""

    def __init__(self, plan: HaloPlan, rank: int, device=None):
        """device: where the all-reduce buffers live; by default the current
        CUDA device with the NCCL backend, the host otherwise."""
        self.plan = plan
        self.rank = rank
        if device is None:
            import torch
            import torch.distributed as dist
            nccl = dist.is_initialized() and dist.get_backend() == "nccl"
            device = f"cuda:{torch.cuda.current_device()}" if nccl else "cpu"
        self.device = device
        self.idx = _Index(plan)

    def parts(self):
        return [self.rank]

    def allreduce(self, vals):
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(vals[0])], dtype=torch.float64, device=self.device)
        dist.all_reduce(t)
        return float(t.item())

    def allreduce_vec(self, vals):
        import torch
        import torch.distributed as dist
        t = torch.as_tensor(np.asarray(vals[0], dtype=np.float64), device=self.device).clone()
        dist.all_reduce(t)
        return t.cpu().numpy()

    def allreduce_t(self, vals):
        """The global sum of this rank's 0-dim tensor, left on the device:
        with NCCL the all-reduce is queued on the current stream and nothing
        waits on the host."""
        import torch.distributed as dist
        t = vals[0].to(self.device).reshape(1).clone()
        dist.all_reduce(t)
        return t[0]

    def halo(self, vecs: dict):
        self.halo_finish(self.halo_start(vecs))

    def halo_start(self, vecs: dict):
        """Posts this rank's halo messages (the owned values its neighbours
        hold as ghosts out, its ghosts' values in) and returns at once; the
        ghosts are written by halo_finish.  Between the two, work that reads
        no ghost entry can run."""
        import torch
        import torch.distributed as dist
        r, pl = self.rank, self.plan
        x = vecs[r]
        ops, bufs = [], []
        for s in range(len(pl.owned)):
            if s == r:
                continue
            if pl.send[r][s].size:
                sb = x[:, self.idx.get(("s", r, s), pl.send[r][s], x.device)].contiguous()
                ops.append(dist.P2POp(dist.isend, sb, s))
            if pl.recv[r][s].size:
                rb = torch.empty((x.shape[0], pl.recv[r][s].size), dtype=x.dtype, device=x.device)
                ops.append(dist.P2POp(dist.irecv, rb, s))
                bufs.append((s, rb))
        reqs = dist.batch_isend_irecv(ops) if ops else []
        return reqs, bufs, x

    def halo_finish(self, handle):
        reqs, bufs, x = handle
        r, pl = self.rank, self.plan
        for q in reqs:
            q.wait()
        for s, rb in bufs:
            x[:, self.idx.get(("r", r, s), pl.recv[r][s], x.device)] = rb


class DeviceOperator:
    """P^-1 A and P^-1 of one partition's assembled system on its context
    (FP64 device vectors of shape (nf, N_local), field-major)."""

    def __init__(self, ctx, system: int, precision: int = F.OVS_FP64):
        self.ctx, self.system, self.precision = ctx, system, precision
        self._parts = None
        F.check(ctx.lib.ovs_build_precond(ctx.h, system, precision), "ovs_build_precond")

    def split(self, owned):
        """Interior and boundary owned rows of this partition (split_rows on
        the context's pattern), for matvec_part; made once."""
        if self._parts is None:
            col, row = self.ctx.get_pattern()
            inner, bnd = split_rows(col, row, owned, self.ctx.N)
            self._parts = {"interior": inner.astype(np.int32), "boundary": bnd.astype(np.int32)}
            self._dev = {}

    def matvec_part(self, x, y, part: str):
        """P^-1 A x on the interior or the boundary rows only
        (ovs_spmv_device_rows); the other rows of y are left as they are."""
        import torch
        key = (part, str(x.device))
        if key not in self._dev:
            self._dev[key] = torch.as_tensor(self._parts[part], device=x.device)
        rows = self._dev[key]
        self._sync()
        F.check(self.ctx.lib.ovs_spmv_device_rows(self.ctx.h, self.system, self.precision, F.OVS_SPMV_PRECOND,
                                                  x.data_ptr(), y.data_ptr(), rows.data_ptr(), int(rows.numel())),
                "ovs_spmv_device_rows")

    @staticmethod
    def _sync():
        import torch
        torch.cuda.current_stream().synchronize()

    def matvec(self, x, y):
        self._sync()
        F.check(self.ctx.lib.ovs_spmv_device(self.ctx.h, self.system, self.precision, F.OVS_SPMV_PRECOND,
                                             x.data_ptr(), y.data_ptr()), "ovs_spmv_device")

    def precond(self, x, y):
        self._sync()
        F.check(self.ctx.lib.ovs_precond_device(self.ctx.h, self.system, self.precision, x.data_ptr(),
                                                y.data_ptr()), "ovs_precond_device")

    def apply(self, x, y):
        """y = A x without the preconditioner (the refinement residual)."""
        self._sync()
        F.check(self.ctx.lib.ovs_spmv_device(self.ctx.h, self.system, self.precision, 0, x.data_ptr(),
                                             y.data_ptr()), "ovs_spmv_device")


def gmres_cycle(comm, ops: dict, rhs: dict, tol: float, kspace: int, kspace_min: int = 1, tem: bool = False,
                orthog: str = "mgs", rhs_pre: bool = False, overlap: bool = True):
    """One GMRES(kspace) cycle from a zero start on the partitions of `comm`
    (SparseGMRES_ns_conv / _up / _tem semantics): `ops[r]` the operator of
    part r, `rhs[r]` its right-hand side (nf, N_local) with the owned rows
    valid.  orthog "mgs" is the reference's modified Gram-Schmidt (one global
    sum per dot, k + 1 at step k); "cgs2" orthogonalizes with classical
    Gram-Schmidt twice (two vector sums and one norm per step, whatever k),
    for ranks where the latency of a collective outweighs its size.
    rhs_pre: rhs is already P^-1 times the right-hand side (the cycle then
    solves P^-1 A x = rhs).  overlap: where every operator has split /
    matvec_part and comm has halo_start / halo_finish, each product runs
    its interior rows while the halo exchange is in flight and its boundary
    rows after it (the owned rows are the same bit for bit, so is the
    cycle); otherwise the product is taken whole after the exchange.  Returns (solution per part
    with ghosts filled, info dict)."""
    if orthog not in ("mgs", "cgs2"):
        raise ValueError("orthog must be 'mgs' or 'cgs2'")
    import torch
    P = comm.parts()
    pl = comm.plan
    ow = {r: torch.as_tensor(pl.owned[r], dtype=torch.long, device=rhs[r].device) for r in P}

    def gdot(a, b):
        return comm.allreduce([float((a[r][:, ow[r]] * b[r][:, ow[r]]).sum()) for r in P])

    sol = {r: torch.zeros_like(rhs[r]) for r in P}
    info = {"iterations": 0, "converged": False, "ercheck": 0.0, "res0": 0.0}
    split = (overlap and hasattr(comm, "halo_start") and hasattr(comm, "halo_finish")
             and all(hasattr(ops[r], "matvec_part") and hasattr(ops[r], "split") for r in P))
    if split:
        for r in P:
            ops[r].split(pl.owned[r])
    if tem and gdot(rhs, rhs) == 0.0:   # SparseGMRES_tem.f90:68-71
        info["converged"] = True
        return sol, info
    U = [{r: torch.empty_like(rhs[r]) for r in P}]
    for r in P:
        if rhs_pre:
            U[0][r].copy_(rhs[r])
        else:
            ops[r].precond(rhs[r], U[0][r])
    unorm = math.sqrt(gdot(U[0], U[0]))
    info["res0"] = unorm
    epsnrm = tol * unorm
    H = np.zeros((kspace + 1, kspace))
    e = np.zeros(kspace + 1)
    rc, rs = np.zeros(kspace), np.zeros(kspace)
    e[0] = unorm
    for r in P:
        U[0][r] = U[0][r] * (1.0 / unorm) if tem else U[0][r] / unorm
    iks, ercheck = 0, 0.0
    for ik in range(1, kspace + 1):
        iks = ik
        if split:
            # ghost rows of w stay 0: no dot reads them, and the next halo
            # exchange overwrites them before any product does
            w = {r: torch.zeros_like(rhs[r]) for r in P}
            h = comm.halo_start(U[ik - 1])
            for r in P:
                ops[r].matvec_part(U[ik - 1][r], w[r], "interior")
            comm.halo_finish(h)
            for r in P:
                ops[r].matvec_part(U[ik - 1][r], w[r], "boundary")
        else:
            comm.halo(U[ik - 1])
            w = {r: torch.empty_like(rhs[r]) for r in P}
            for r in P:
                ops[r].matvec(U[ik - 1][r], w[r])
        U.append(w)
        if orthog == "mgs":
            # the k + 1 dots of the reference order stay on the device: each
            # projection uses the previous dot as a device scalar, the
            # all-reduces queue one after another, and the column of H comes
            # to the host once per step
            col = []
            beta_t = None
            for jk in range(1, ik + 2):
                if jk > 1:
                    for r in P:
                        w[r] = w[r] - beta_t.to(w[r].device) * U[jk - 2][r]
                    U[ik] = w
                other = U[jk - 1] if jk - 1 < ik else w
                beta_t = comm.allreduce_t([(w[r][:, ow[r]] * other[r][:, ow[r]]).sum() for r in P])
                col.append(beta_t)
            hcol = torch.stack([c.to(col[0].device) for c in col]).cpu().numpy()
            H[:ik + 1, ik - 1] = hcol
            beta = float(hcol[-1])
        else:
            for _ in range(2):
                loc = [np.array([float((U[j][r][:, ow[r]] * w[r][:, ow[r]]).sum()) for j in range(ik)]) for r in P]
                h = comm.allreduce_vec(loc)
                for r in P:
                    for j in range(ik):
                        w[r] = w[r] - float(h[j]) * U[j][r]
                H[:ik, ik - 1] += h
            U[ik] = w
            beta = gdot(w, w)
        unorm = math.sqrt(beta)
        H[ik, ik - 1] = unorm
        for r in P:
            w[r] = w[r] * (1.0 / unorm) if tem else w[r] / unorm
        U[ik] = w
        for jk in range(1, ik):
            t = rc[jk - 1] * H[jk - 1, ik - 1] + rs[jk - 1] * H[jk, ik - 1]
            H[jk, ik - 1] = -rs[jk - 1] * H[jk - 1, ik - 1] + rc[jk - 1] * H[jk, ik - 1]
            H[jk - 1, ik - 1] = t
        a, b = H[ik - 1, ik - 1], H[ik, ik - 1]
        t = math.sqrt(a * a + b * b)
        if tem:
            t1 = 1.0 / t
            rc[ik - 1], rs[ik - 1] = a * t1, b * t1
        else:
            rc[ik - 1], rs[ik - 1] = a / t, b / t
        H[ik - 1, ik - 1] = t
        H[ik, ik - 1] = 0.0
        t = rc[ik - 1] * e[ik - 1] + rs[ik - 1] * e[ik]
        e[ik] = -rs[ik - 1] * e[ik - 1] + rc[ik - 1] * e[ik]
        e[ik - 1] = t
        ercheck = abs(e[ik])
        if ercheck <= epsnrm and ik >= kspace_min:
            break
    y = np.zeros(iks)
    for jk in range(iks, 0, -1):
        y[jk - 1] = e[jk - 1] / H[jk - 1, jk - 1]
        for lk in range(1, jk):
            e[lk - 1] = e[lk - 1] - y[jk - 1] * H[lk - 1, jk - 1]
    for jk in range(1, iks + 1):
        for r in P:
            sol[r] = sol[r] + float(y[jk - 1]) * U[jk - 1][r]
    comm.halo(sol)   # commu 'out': ghosts take their owners' values
    info.update(iterations=iks, ercheck=ercheck, converged=bool(ercheck <= epsnrm))
    return sol, info


def solve_refined(comm, inner: dict, outer: dict, rhs: dict, rtol: float, kspace: int = 50,
                  max_cycles: int = 100, tem: bool = False, orthog: str = "mgs", floor_tol: float = 1e-6):
    """A x = b to a true relative residual ||b - A x||_2 <= rtol ||b||_2 over
    the partitions: `ovs_solve`'s refinement loop on distributed vectors.
    Each cycle solves the current residual with one GMRES cycle on the
    `inner` operators (P^-1 A and P^-1 of the FP32 system for mixed
    precision) to the relative tolerance rtol/rel, clamped to
    [floor_tol, 0.5], adds the correction, and forms r = b - A x with the
    `outer` operators' plain FP64 product (`apply`) after a halo update of x.
    Norms are global sums over owned rows.  Returns (x per part with ghosts
    filled, info: cycles, iterations, converged, rel_residual)."""
    import torch
    P = comm.parts()
    pl = comm.plan
    ow = {r: torch.as_tensor(pl.owned[r], dtype=torch.long, device=rhs[r].device) for r in P}

    def gnorm2(v):
        return comm.allreduce([float((v[r][:, ow[r]] ** 2).sum()) for r in P])

    x = {r: torch.zeros_like(rhs[r]) for r in P}
    res = {r: rhs[r].clone() for r in P}
    bnorm = math.sqrt(gnorm2(rhs))
    rel = 1.0 if bnorm > 0.0 else 0.0
    cycles = iters = 0
    while rel > rtol and cycles < max_cycles:
        tin = min(max(rtol / rel, floor_tol), 0.5)
        dx, info = gmres_cycle(comm, inner, res, tin, kspace, 1, tem=tem, orthog=orthog)
        iters += info["iterations"]
        cycles += 1
        for r in P:
            x[r] = x[r] + dx[r]
        comm.halo(x)
        for r in P:
            ax = torch.empty_like(x[r])
            outer[r].apply(x[r], ax)
            res[r] = rhs[r] - ax
        rel = math.sqrt(gnorm2(res)) / bnorm
        if rel != rel or info["iterations"] == 0:
            break
    return x, {"cycles": cycles, "iterations": iters, "converged": bool(rel <= rtol), "rel_residual": rel}


def solve_flexible(comm, inner: dict, outer: dict, rhs: dict, rtol: float, kspace: int = 50,
                   max_cycles: int = 100, m: int = 30, tem: bool = False, orthog: str = "mgs",
                   floor_tol: float = 1e-6):
    """A x = b to a true relative residual ||b - A x||_2 <= rtol ||b||_2 over
    the partitions: `ovs_solve`'s OVS_MIXED flexible outer on distributed
    vectors.  FGMRES(m) in FP64 on the `outer` operators (P^-1 A and P^-1 of
    the FP64 system) minimizes the preconditioned residual; each direction
    z_j is one GMRES cycle on the `inner` operators (the FP32 system) with
    the right-hand side v_j taken as preconditioned, rounded to FP32 before
    P^-1 A z_j is formed.  After m directions, or when the outer estimate
    reaches the reduction still needed, x is updated and r = b - A x formed
    with the outer operators' plain product (`apply`) after a halo update of
    x.  Dots are global sums over owned rows.  Returns (x per part with
    ghosts filled, info: cycles (inner cycles), iterations, converged,
    rel_residual)."""
    import torch
    P = comm.parts()
    pl = comm.plan
    ow = {r: torch.as_tensor(pl.owned[r], dtype=torch.long, device=rhs[r].device) for r in P}

    def gdot(a, b):
        return comm.allreduce([float((a[r][:, ow[r]] * b[r][:, ow[r]]).sum()) for r in P])

    x = {r: torch.zeros_like(rhs[r]) for r in P}
    res = {r: rhs[r].clone() for r in P}
    bnorm = math.sqrt(gdot(rhs, rhs))
    rel = 1.0 if bnorm > 0.0 else 0.0
    cycles = iters = 0
    while rel > rtol and cycles < max_cycles:
        v0 = {r: torch.empty_like(rhs[r]) for r in P}
        for r in P:
            outer[r].precond(res[r], v0[r])
        beta = math.sqrt(gdot(v0, v0))
        if not beta > 0.0:
            break
        V = [{r: v0[r] / beta for r in P}]
        Z = []
        target = 0.5 * beta * rtol / rel
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        cs, sn = np.zeros(m), np.zeros(m)
        g[0] = beta
        j = 0
        while j < m and cycles < max_cycles:
            tin = min(max(target / abs(g[j]), floor_tol), 0.5)
            z, info = gmres_cycle(comm, inner, V[j], tin, kspace, 1, tem=tem, orthog=orthog, rhs_pre=True)
            iters += info["iterations"]
            cycles += 1
            z = {r: z[r].float().double() for r in P}   # the stored direction, FP32
            w = {r: torch.empty_like(rhs[r]) for r in P}
            for r in P:
                outer[r].matvec(z[r], w[r])
            for i in range(j + 1):
                h = gdot(w, V[i])
                H[i, j] = h
                for r in P:
                    w[r] = w[r] - h * V[i][r]
            hn = math.sqrt(gdot(w, w))
            H[j + 1, j] = hn
            if hn > 0.0:
                for r in P:
                    w[r] = w[r] / hn
            V.append(w)
            Z.append(z)
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den = math.hypot(H[j, j], H[j + 1, j])
            if den == 0.0:   # a zero column: the directions so far span the solution
                Z.pop()
                break
            cs[j], sn[j] = H[j, j] / den, H[j + 1, j] / den
            H[j, j], H[j + 1, j] = den, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            j += 1
            if not hn > 0.0 or abs(g[j]) <= target:
                break
        k = len(Z)
        y = np.zeros(k)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:k] @ y[i + 1:k]) / H[i, i] if H[i, i] != 0.0 else 0.0
        for i in range(k):
            for r in P:
                x[r] = x[r] + float(y[i]) * Z[i][r]
        comm.halo(x)
        for r in P:
            ax = torch.empty_like(x[r])
            outer[r].apply(x[r], ax)
            res[r] = rhs[r] - ax
        rel = math.sqrt(gdot(res, res)) / bnorm
        if rel != rel or k == 0:
            break
    return x, {"cycles": cycles, "iterations": iters, "converged": bool(rel <= rtol), "rel_residual": rel}


# assembleQuenching field flags (commonpars, src/modules.f90:218-222)
FIELD_NS, FIELD_VOF, FIELD_TEM = 1, 2, 4
_KIND_SYS = {"nsvof": F.OVS_SYS_NSVOF, "tem": F.OVS_SYS_TEM}


class ContextPartition:
    """One partition's local system on its own context (`api.Context` of
    `partition.local_case`) for `quench_newton`: FP64 assembly, the sums of
    squares of its owned residual rows, the right-hand sides as FP64 device
    vectors (nf, N_local), the preconditioned operators, the Newton update
    with a solution from the partitioned GMRES (ovs_set_solution, then
    ovs_newton_update), and, for `quench_time_steps`, the driver's predictor
    and old-value copies (ovs_predictor, ovs_commit_old)."""

    def __init__(self, ctx, owned, device=None):
        import torch
        self.ctx = ctx
        self.owned = np.asarray(owned, dtype=np.int64)
        self.device = device if device is not None else f"cuda:{torch.cuda.current_device()}"

    def apply_bcs(self):
        self.ctx.apply_bcs(3)

    def assemble(self, tensor_flag: int, field_flag: int, precision: int = F.OVS_FP64):
        if field_flag & (FIELD_NS | FIELD_VOF):
            self.ctx.assemble(F.OVS_ASM_NSVOF, tensor_flag, precision)
        if field_flag & FIELD_TEM:
            self.ctx.assemble(F.OVS_ASM_TEM, tensor_flag, precision)

    def residual_sq(self, precision: int = F.OVS_FP64) -> np.ndarray:
        o = self.owned
        f = self.ctx.get_rhs(F.OVS_SYS_NSVOF, precision)[o]
        t = self.ctx.get_rhs(F.OVS_SYS_TEM, precision)[o]
        return np.array([np.sum(f[:, :3] ** 2), np.sum(f[:, 3] ** 2), np.sum(f[:, 4] ** 2), np.sum(t ** 2)])

    def rhs(self, kind: str, precision: int = F.OVS_FP64):
        import torch
        r = self.ctx.get_rhs(_KIND_SYS[kind], precision)
        return torch.as_tensor(np.ascontiguousarray(r.T), device=self.device)

    def operator(self, kind: str, precision: int = F.OVS_FP64):
        return DeviceOperator(self.ctx, _KIND_SYS[kind], precision)

    def round(self, kind: str):
        """The FP32 rounding of the part's FP64 matrix of `kind` (the inner
        operator of the OVS_MIXED refinement)."""
        self.ctx.round_matrix(_KIND_SYS[kind])

    def update(self, kind: str, sol):
        self.ctx.set_solution(_KIND_SYS[kind], sol.contiguous())
        self.ctx.newton_update(_KIND_SYS[kind])

    def predictor(self):
        self.ctx.predictor()

    def commit_old(self, update_vof_tem_old: bool):
        self.ctx.commit_old(update_vof_tem_old)


def quench_newton(comm, parts: dict, newton_max: int = 3, solve_tem: bool = True, kspace: int = 50,
                  kspace_min: int = 1, tol_ns: float = 1e-6, tol_tem: float = 1e-6, utol=(1e-3,) * 4,
                  atol=(1e-15,) * 4, orthog: str = "mgs", bcs: bool = False, mode: int = F.OVS_FP64,
                  max_cycles: int = 100, mixed_outer: int = 30) -> dict:
    """The Newton loop of one quench time step over owner-computes partitions:
    solmultiphasethermofluid_stag (src/solveFlow.f90:4-164) as the reference
    runs it on several ranks.  `parts[r]` is part r's local system
    (`ContextPartition`, or any object with the same methods).

    The steps, in the reference's order:

    * with `bcs`, the BC producers on every part (setBCs_NSVOF and
      setBCs_Tem, :34-36, :57-59);
    * the residual of all fields, then the NS+VOF matrix and residual and one
      GMRES cycle from zero over all parts (`gmres_cycle`);
    * the update (:99-104); with `solve_tem`, the temperature the same way
      (:109-140);
    * the residual of all fields again and check_convergence (:148-157,
      :192-215).

    Every part assembles only its local elements, and its owned rows are then
    complete.  Residuals are sums of squares over the owned rows, one global
    sum per evaluation, as calculate_residual's MPI_ALLREDUCE (:169-187).
    The loop body runs at least once.  The returned dict has iterations,
    converged, field_converged, residual0, residual and the Krylov
    iterations of both systems.

    mode OVS_FP32 is ovs_quench_newton's OVS_FP32 mode over the partitions:
    FP32 assembly, residuals from the FP32 right-hand sides, and each solve
    by `solve_refined` on the FP32 operators to the relative residual tol_ns
    / tol_tem (max_cycles refinement cycles) instead of one FP64 cycle.
    mode OVS_MIXED is its OVS_MIXED mode: FP64 assembly and residuals, and
    each solve with the FP64 operators outside and, inside, the FP32
    rounding of each part's FP64 matrix (the parts' `round`): by
    `solve_flexible` with an FGMRES(mixed_outer) outer (the default, as
    OVS_OPT_MIXED_OUTER = 30), or by `solve_refined` with mixed_outer = 0.
    The parts then take a precision argument in assemble, residual_sq, rhs
    and operator, and their operators provide `apply`."""
    P = comm.parts()
    mixed = mode in (F.OVS_FP32, F.OVS_MIXED)
    prec = F.OVS_FP32 if mode == F.OVS_FP32 else F.OVS_FP64
    pk = {"precision": prec} if mixed else {}

    def residual():
        return np.asarray(comm.allreduce_vec([np.asarray(parts[r].residual_sq(**pk), dtype=np.float64) for r in P]))

    def set_bcs():
        if bcs:
            for r in P:
                parts[r].apply_bcs()

    def solve(kind, tol):
        rhs = {r: parts[r].rhs(kind, **pk) for r in P}
        ops = {r: parts[r].operator(kind, **pk) for r in P}
        if mode == F.OVS_MIXED:
            for r in P:
                parts[r].round(kind)
            inner = {r: parts[r].operator(kind, precision=F.OVS_FP32) for r in P}
            if mixed_outer > 0:
                sol, info = solve_flexible(comm, inner, ops, rhs, tol, kspace, max_cycles, mixed_outer,
                                           tem=kind == "tem", orthog=orthog)
            else:
                sol, info = solve_refined(comm, inner, ops, rhs, tol, kspace, max_cycles, tem=kind == "tem",
                                          orthog=orthog)
        elif mixed:
            sol, info = solve_refined(comm, ops, ops, rhs, tol, kspace, max_cycles, tem=kind == "tem", orthog=orthog)
        else:
            sol, info = gmres_cycle(comm, ops, rhs, tol, kspace, kspace_min, tem=kind == "tem", orthog=orthog)
        for r in P:
            parts[r].update(kind, sol[r])
        return info["iterations"]

    def check(r, r0):   # check_convergence with all fields flagged, as the reference calls it
        return [bool(v) for v in check_convergence(r, r0, utol, FIELD_NS | FIELD_VOF | FIELD_TEM, atol)]

    set_bcs()
    for r in P:
        parts[r].assemble(F.OVS_TENSOR_VEC, FIELD_NS | FIELD_VOF | FIELD_TEM, **pk)
    r0 = residual()
    res = r0.copy()
    fc = check(res, r0)
    out = {"iterations": 0, "converged": all(fc), "field_converged": fc, "residual0": r0,
           "krylov_iterations_ns": 0, "krylov_iterations_tem": 0}
    for it in range(1, newton_max + 1):
        set_bcs()
        for r in P:
            parts[r].assemble(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, FIELD_NS | FIELD_VOF, **pk)
        out["krylov_iterations_ns"] += solve("nsvof", tol_ns)
        if solve_tem:
            for r in P:
                parts[r].assemble(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, FIELD_TEM, **pk)
            out["krylov_iterations_tem"] += solve("tem", tol_tem)
        for r in P:
            parts[r].assemble(F.OVS_TENSOR_VEC, FIELD_NS | FIELD_VOF | FIELD_TEM, **pk)
        res = residual()
        fc = check(res, r0)
        out.update(iterations=it, converged=all(fc), field_converged=fc)
        if out["converged"]:
            break
    out["residual"] = res
    return out


def quench_time_steps(comm, parts: dict, first_step: int, nsteps: int, update_vof_tem_old: bool = False,
                      newton_max: int = 3, solve_tem: bool = True, **newton):
    """`nsteps` steps of the reference driver's time loop (src/driver.f90:
    70-103) over the partitions.  Every step runs the predictor on every
    part (:83-85), then `quench_newton` (a single Newton iteration while
    istep <= 1, and no temperature solve at istep 0, src/solveFlow.f90:50-54,
    109), then the old-value copies (:98-103).  The parts also need
    predictor() and commit_old(flag).  Returns (the last step's Newton
    record, the Krylov iterations over all steps)."""
    P = comm.parts()
    last, kt = None, 0
    for k in range(nsteps):
        istep = first_step + k
        for r in P:
            parts[r].predictor()
        last = quench_newton(comm, parts, newton_max=1 if istep <= 1 else newton_max,
                             solve_tem=solve_tem and istep > 0, **newton)
        kt += last["krylov_iterations_ns"] + last["krylov_iterations_tem"]
        for r in P:
            parts[r].commit_old(update_vof_tem_old)
    return last, kt
