"""The reference's on-disk formats, so its meshes and restarts run through
this path: the partition mesh ``part.<id>.dat`` (read by input_mesh,
src/input.f90:15-120; written by genmesh_overset/mesh.f90:140-204), the
text restart ``restart.<step>.<rank+1>`` (readSol / writeSol,
src/iosol.f90:122-194, 377-454) and its ``step.dat`` (readStep, :82-117),
with the reference's file names (cname, src/cname.f90:4-37).  Both are Fortran list-directed text; this
module reads and writes them with numpy and builds the `mesh.Case` inputs
from them.  The overset boundary maps (``l2b.<id>.dat``) belong to the
overset coupling, which is outside this path, and are not read.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _ffi as F
from . import mesh as M


@dataclass
class Boundary:
    face_id: int
    face_ien: np.ndarray      # (NFACE, NSHLBmax) 1-based node ids
    f2e: np.ndarray           # (NFACE,) owning element, 1-based
    face_or: np.ndarray       # (NFACE,) face orientation code
    bnodes: np.ndarray        # (NNODE_b,) 1-based node ids
    nshlb: np.ndarray | None = None   # per-face node counts (non-FEM files only)


@dataclass
class PartMesh:
    nsd: int
    nshl: int
    nshlb_max: int
    xg: np.ndarray            # (N, NSD)
    node_id: np.ndarray       # (N,) NodeID (FEM files)
    elmnshl: np.ndarray       # (E,)
    ien: np.ndarray           # (E, NSHL) 1-based
    elm_id: np.ndarray        # (E,)
    bounds: list = field(default_factory=list)
    wg: np.ndarray | None = None      # NURBS weights (NPATCH > 0)
    epid: np.ndarray | None = None
    eijk: np.ndarray | None = None


class _Tokens:
    """Whitespace tokens of a list-directed file, one record per line."""

    def __init__(self, path):
        with open(path) as f:
            self.lines = [ln.split() for ln in f if ln.strip()]
        self.i = 0

    def record(self):
        t = self.lines[self.i]
        self.i += 1
        return t

    def block(self, nrec):
        rows = self.lines[self.i:self.i + nrec]
        self.i += nrec
        return rows


def _float(s: str) -> float:
    return float(s.replace("D", "E").replace("d", "e"))


def read_part(path, fem_flag: int = 1) -> PartMesh:
    """input_mesh (src/input.f90:31-120)."""
    tk = _Tokens(path)
    nsd, nshl, nshlb_max = (int(v) for v in tk.record()[:3])
    nnode, nelem, nbound, npatch = (int(v) for v in tk.record()[:4])
    rows = tk.block(nnode)
    xg = np.array([[_float(v) for v in r[:nsd]] for r in rows])
    node_id = np.array([int(r[nsd]) for r in rows], dtype=np.int32) if fem_flag == 1 else np.zeros(nnode, np.int32)
    rows = tk.block(nelem)
    elmnshl = np.array([int(r[0]) for r in rows], dtype=np.int32)
    ien = np.zeros((nelem, nshl), dtype=np.int32)
    elm_id = np.zeros(nelem, dtype=np.int32)
    for e, r in enumerate(rows):
        k = elmnshl[e]
        ien[e, :k] = [int(v) for v in r[1:1 + k]]
        if fem_flag == 1:
            elm_id[e] = int(r[1 + k])
    bounds = []
    for _ in range(nbound):
        face_id, nface, nbn = (int(v) for v in tk.record()[:3])
        rows = tk.block(nface)
        if fem_flag == 1:
            face_ien = np.array([[int(v) for v in r[:nshlb_max]] for r in rows], dtype=np.int32).reshape(nface, nshlb_max)
            nshlb = None
        else:
            nshlb = np.array([int(r[0]) for r in rows], dtype=np.int32)
            face_ien = np.array([[int(v) for v in r[1:1 + nshlb_max]] for r in rows], dtype=np.int32).reshape(nface, nshlb_max)
        rows = tk.block(nface)
        f2e = np.array([int(r[0]) for r in rows], dtype=np.int32)
        face_or = np.array([int(r[1]) for r in rows], dtype=np.int32)
        bnodes = np.array([int(r[0]) for r in tk.block(nbn)], dtype=np.int32)
        bounds.append(Boundary(face_id, face_ien, f2e, face_or, bnodes, nshlb))
    pm = PartMesh(nsd, nshl, nshlb_max, xg, node_id, elmnshl, ien, elm_id, bounds)
    if npatch > 0:
        pm.wg = np.array([_float(r[0]) for r in tk.block(nnode)])
        rows = tk.block(nelem)
        pm.epid = np.array([int(r[0]) for r in rows], dtype=np.int32)
        pm.eijk = np.array([[int(v) for v in r[1:1 + nsd]] for r in rows], dtype=np.int32)
    return pm


def write_part(path, pm: PartMesh, fem_flag: int = 1) -> None:
    """The same records in the order input_mesh reads them."""
    npatch = 1 if pm.wg is not None else 0
    with open(path, "w") as f:
        f.write(f"{pm.nsd} {pm.nshl} {pm.nshlb_max}\n")
        f.write(f"{pm.xg.shape[0]} {pm.ien.shape[0]} {len(pm.bounds)} {npatch}\n")
        for i in range(pm.xg.shape[0]):
            xs = " ".join(repr(float(v)) for v in pm.xg[i])
            f.write(f"{xs} {int(pm.node_id[i])}\n" if fem_flag == 1 else f"{xs}\n")
        for e in range(pm.ien.shape[0]):
            k = int(pm.elmnshl[e])
            ids = " ".join(str(int(v)) for v in pm.ien[e, :k])
            f.write(f"{k} {ids} {int(pm.elm_id[e])}\n" if fem_flag == 1 else f"{k} {ids}\n")
        for b in pm.bounds:
            f.write(f"{b.face_id} {b.face_ien.shape[0]} {b.bnodes.size}\n")
            for j in range(b.face_ien.shape[0]):
                ids = " ".join(str(int(v)) for v in b.face_ien[j])
                f.write(f"{ids}\n" if fem_flag == 1 else f"{int(b.nshlb[j])} {ids}\n")
            for j in range(b.face_ien.shape[0]):
                f.write(f"{int(b.f2e[j])} {int(b.face_or[j])}\n")
            for v in b.bnodes:
                f.write(f"{int(v)}\n")
        if npatch:
            for v in pm.wg:
                f.write(f"{repr(float(v))}\n")
            for e in range(pm.ien.shape[0]):
                f.write(f"{int(pm.epid[e])} " + " ".join(str(int(v)) for v in pm.eijk[e]) + "\n")


def part_from_mesh(m: "M.Mesh", face_ids=(1, 2, 3, 4, 5, 6)) -> PartMesh:
    """A PartMesh of one of this package's box meshes: node ids 0, one
    boundary per box face with its nodes and, for tets, its triangles
    (FACE_IEN, F2E, FACE_OR); hexahedral boundaries list nodes only."""
    N, E = m.nnode, m.nelem
    ien0 = np.asarray(m.ien, dtype=np.int32)
    if m.nshl == 4:
        tri = M.box_boundary_faces(m)
        fien = [ien0[f2e - 1][np.arange(f2e.size)[:, None], np.asarray(M.TET_FACE_NODES)[fo - 1]]
                for f2e, fo in tri]
    else:
        tri = [(np.zeros(0, np.int32), np.zeros(0, np.int32))] * len(m.faces)
        fien = [np.zeros((0, 4), np.int32)] * len(m.faces)
    bounds = [Boundary(int(fid), fi.astype(np.int32), f2e, fo, (np.asarray(nodes) + 1).astype(np.int32))
              for fid, nodes, (f2e, fo), fi in zip(face_ids, m.faces, tri, fien)]
    return PartMesh(3, m.nshl, 3 if m.nshl == 4 else 4, np.asarray(m.xg, dtype=np.float64),
                    np.zeros(N, np.int32), np.full(E, m.nshl, np.int32), np.asarray(m.ien, dtype=np.int32),
                    np.asarray(m.elm_id, dtype=np.int32), bounds)


def mesh_from_part(pm: PartMesh) -> "M.Mesh":
    """mesh.Mesh of a partition: the FE element block (one element type per
    partition, as this path assembles), 1-based ien, the boundary node sets
    in file order as faces."""
    if np.any(pm.elmnshl != pm.nshl):
        raise ValueError("mixed element types in one partition are not assembled by this path")
    lo, hi = pm.xg.min(axis=0), pm.xg.max(axis=0)
    faces = [np.sort(b.bnodes.astype(np.int64) - 1) for b in pm.bounds]
    return M.Mesh(np.asfortranarray(pm.xg[:, :3]), np.asfortranarray(pm.ien.astype(np.int32)),
                  pm.elm_id.astype(np.int32).copy(), faces, None, tuple(float(v) for v in (hi - lo)))


def faces_from_part(pm: PartMesh, weak=(), convective=None) -> "M.BoundaryFaces":
    """The face set of a partition for the face assemblies: the boundary
    faces (F2E, FACE_OR) in file order, as the reference's NBOUND loop visits
    them.  `weak`: FACE_IDs with BCugType == 2; `convective`: {FACE_ID:
    (h, T_inf)} for the convective heat term."""
    convective = convective or {}
    parts = []
    for b in pm.bounds:
        fl = (F.OVS_FACE_WEAK if b.face_id in weak else 0) | (F.OVS_FACE_CONVH if b.face_id in convective else 0)
        if not fl or b.f2e.size == 0:
            continue
        h, tinf = convective.get(b.face_id, (0.0, 0.0))
        n = b.f2e.size
        parts.append((b.f2e.astype(np.int32), b.face_or.astype(np.int32), np.full(n, fl, np.int32),
                      np.full(n, float(h)), np.full(n, float(tinf))))
    if not parts:
        z = np.zeros(0)
        return M.BoundaryFaces(z.astype(np.int32), z.astype(np.int32), z.astype(np.int32), z, z)
    return M.BoundaryFaces(*(np.concatenate(c) for c in zip(*parts)))


def bc_spec_from_part(pm: PartMesh, bcug_type, bcug_valu, bcphig_type, bcphig_valu, bctg_type, bctg_valu,
                      node_id=None) -> "M.BcSpec":
    """The input of setBCs_NSVOF / setBCs_Tem for a partition read from
    part.dat: per boundary in file order its FACE_ID and BNODES, with the
    tables of src/param.f90:296-340 as the reference holds them (the *Type
    tables read by FACE_ID, the *Valu tables by boundary number); NodeID from
    the file unless given."""
    nb = len(pm.bounds)
    fid = np.array([b.face_id for b in pm.bounds], dtype=np.int32)
    spec = M.BcSpec(fid, [np.asarray(b.bnodes, dtype=np.int32) for b in pm.bounds],
                    np.asarray(bcug_type, dtype=np.int32).reshape(-1, 3),
                    np.asarray(bcug_valu, dtype=np.float64).reshape(nb, 3),
                    np.asarray(bcphig_type, dtype=np.int32), np.asarray(bcphig_valu, dtype=np.float64),
                    np.asarray(bctg_type, dtype=np.int32), np.asarray(bctg_valu, dtype=np.float64),
                    np.asarray(pm.node_id if node_id is None else node_id, dtype=np.int32))
    nt = spec.bcug_type.shape[0]
    if fid.size and (fid.min() < 1 or fid.max() > nt):
        raise ValueError("a FACE_ID is outside the *Type tables (setBCs reads them by FACE_ID)")
    return spec


# the records of a restart, in file order, and the state arrays they fill
RESTART_READ = ("dgold", "ugold", "ugmold", "acgold", "acgmold", "phigold", "rphigold", "pgold", "tgold", "rtgold")
RESTART_WRITE = ("dg", "ug", "ugm", "acg", "acgm", "phig", "rphig", "pg", "tgold", "rtgold")


def cname(i: int) -> str:
    """cname (src/cname.f90:4-37): "." and the decimal digits of i without
    leading zeros, from the lowest nine digits the routine keeps
    (cname(0) = ".0", cname(1234567890) = ".234567890")."""
    if i < 0:
        raise ValueError("cname takes a non-negative integer")
    return "." + str(int(i) % 10 ** 9)


def part_name(part_id: int) -> str:
    """The partition mesh file input_mesh opens: 'part'//trim(cname(id))//'.dat'
    (src/input.f90:31)."""
    return "part" + cname(part_id) + ".dat"


def restart_name(step: int, rank: int) -> str:
    """The restart file of readSol / writeSol for 0-based MPI rank `rank`:
    trim('restart'//cname(step))//cname(myid + 1) (src/iosol.f90:137, 390)."""
    return "restart" + cname(step) + cname(rank + 1)


def read_step(path) -> tuple[int, float | None]:
    """readStep (src/iosol.f90:82-117): (Rstep, x_inflow) from step.dat;
    (0, None) when the file cannot be opened, as its iostat branch leaves
    Rstep = 0."""
    try:
        tk = _Tokens(path)
    except OSError:
        return 0, None
    head = tk.record()
    return int(head[0]), _float(head[1])


def write_step(path, istep: int, x_inflow: float) -> None:
    """The step.dat record writeSol leaves on the master rank
    (src/iosol.f90:447-452): istep and x_inflow."""
    with open(path, "w") as f:
        f.write(f"{int(istep)} {repr(float(x_inflow))}\n")


def read_restart(path, nnode: int) -> tuple[int, float, dict]:
    """readSol (src/iosol.f90:122-194): (step, time, arrays) with the arrays
    named as readSol fills them (the *old fields, pgold included)."""
    tk = _Tokens(path)
    head = tk.record()
    step, time = int(head[0]), _float(head[1])
    out = {}
    for name in RESTART_READ:
        rows = tk.block(nnode)
        a = np.array([[_float(v) for v in r] for r in rows])
        out[name] = a if a.shape[1] == 3 else a[:, 0].copy()
    return step, time, out


def write_restart(path, step: int, time: float, state: dict) -> None:
    """writeSol (src/iosol.f90:377-454): the current dg, ug, ugm, acg, acgm,
    phig, rphig, pg and, as the reference writes them, the OLD temperature
    arrays Tgold and rTgold."""
    with open(path, "w") as f:
        f.write(f"{step} {repr(float(time))}\n")
        for name in RESTART_WRITE:
            a = np.asarray(state[name])
            if a.ndim == 2:
                for row in a:
                    f.write(" ".join(repr(float(v)) for v in row) + "\n")
            else:
                for v in a:
                    f.write(repr(float(v)) + "\n")


def state_from_restart(arrays: dict, gami: float) -> dict:
    """The package state after readSol and the predictor of driver.f90:83-85
    (ug = ugold, acg = (gami - 1)/gami acgold, pg = pgold; the other current
    fields start from their old values)."""
    N = arrays["ugold"].shape[0]
    st = M.empty_state(N)
    for name in ("dgold", "ugold", "ugmold", "acgold", "acgmold", "phigold", "rphigold", "tgold", "rtgold"):
        st[name][:] = arrays[name]
    st["dg"][:] = arrays["dgold"]
    st["ug"][:] = arrays["ugold"]
    st["ugm"][:] = arrays["ugmold"]
    st["acg"][:] = (gami - 1.0) / gami * arrays["acgold"]
    st["acgm"][:] = arrays["acgmold"]
    st["pg"][:] = arrays["pgold"]
    st["phig"][:] = arrays["phigold"]
    st["rphig"][:] = arrays["rphigold"]
    st["tg"][:] = arrays["tgold"]
    st["rtg"][:] = arrays["rtgold"]
    return st


def load_rank(directory, rank: int, params: dict, initial_state: dict | None = None):
    """What the reference driver reads at start-up on MPI rank `rank`
    (src/driver.f90:39-60): the partition mesh part.<rank+1>.dat (input),
    step.dat (readStep), and for a step above 0 the restart
    restart.<step>.<rank+1> (readSol) with the predictor of the first step
    it resumes (driver.f90:83-85, applied by state_from_restart).  At step 0
    the reference generates its initial condition (generateIC, a harness of
    its own); here `initial_state` supplies it, zeros by default.  IBC starts
    at zero: the setBCs producers fill it.  Returns (mesh.Case, step, time,
    the PartMesh)."""
    from pathlib import Path
    d = Path(directory)
    pm = read_part(d / part_name(rank + 1))
    m = mesh_from_part(pm)
    N = m.nnode
    step, _x_inflow = read_step(d / "step.dat")
    time = 0.0
    if step > 0:
        _, time, arrays = read_restart(d / restart_name(step, rank), N)
        state = state_from_restart(arrays, params["gami"])
    else:
        state = M.empty_state(N)
        for k, v in (initial_state or {}).items():
            state[k][...] = v
    ibc = np.zeros((N, 8), dtype=np.int32, order="F")
    case = M.Case(f"part{rank + 1}", m, params, state, ibc, F.OVS_ASM_NSVOF)
    return case, step, time, pm
