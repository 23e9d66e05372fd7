"""Owner-computes partitions of a mesh for sharded assembly (one rank per GPU).

The reference partitions elements with METIS and sums the rows of shared
nodes across ranks after assembly (``commu 'in'``, src/commu.f90:118-185).
Here every rank owns a contiguous range of nodes and receives every element
that touches one of its nodes (one layer of overlap), in ascending global
element id.  The rows of owned nodes are then complete on their rank: the
row pass adds the same elements in the same order as on one GPU, so they
are bit-identical to the single-GPU rows, and assembly needs no data-path
collective at all (the elements of the overlap layer are computed on more
than one rank).  The Krylov solve on such partitions needs the owners'
values at the other local nodes before each SpMV and a sum of dot products
over ranks; that exchange is not built here.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import mesh as M


@dataclass
class Part:
    rank: int
    nodes: np.ndarray        # (n_local,) global node ids (0-based), ascending
    owned: np.ndarray        # (n_owned,) positions in `nodes` of the owned nodes
    elements: np.ndarray     # (e_local,) global element ids, ascending
    mesh: "M.Mesh"           # local mesh (1-based local ien, local coordinates)
    global_rows: np.ndarray  # (n_owned,) global ids of the owned rows


def owner_ranges(nnode: int, nparts: int) -> np.ndarray:
    """Contiguous node ranges: rank r owns [bounds[r], bounds[r+1])."""
    return np.linspace(0, nnode, nparts + 1).round().astype(np.int64)


def make_parts(m: "M.Mesh", nparts: int) -> list[Part]:
    if nparts < 1 or nparts > m.nnode:
        raise ValueError(f"need 1 <= nparts <= nnode ({m.nnode}): every part owns at least one node")
    ien0 = np.asarray(m.ien, dtype=np.int64) - 1
    bounds = owner_ranges(m.nnode, nparts)
    owner_of_node = np.searchsorted(bounds, np.arange(m.nnode), side="right") - 1
    parts = []
    for r in range(nparts):
        touches = np.any(owner_of_node[ien0] == r, axis=1)
        elems = np.nonzero(touches)[0]                       # ascending global ids
        nodes = np.unique(ien0[elems].ravel())               # ascending global ids
        loc = np.full(m.nnode, -1, dtype=np.int64)
        loc[nodes] = np.arange(nodes.size)
        lien = np.asfortranarray((loc[ien0[elems]] + 1).astype(np.int32))
        owned_glob = np.arange(bounds[r], bounds[r + 1])
        owned = loc[owned_glob]
        faces = [loc[f][loc[f] >= 0] for f in m.faces]
        lm = M.Mesh(np.asfortranarray(m.xg[nodes]), lien, np.asarray(m.elm_id)[elems].astype(np.int32).copy(),
                    faces, m.dims, m.lengths)
        parts.append(Part(r, nodes, owned, elems, lm, owned_glob))
    return parts


def local_faces(bf: "M.BoundaryFaces", part: Part) -> "M.BoundaryFaces":
    """The boundary faces whose element is in the partition, in the global
    loop order, with local element ids.  Every element touching an owned
    node is local, so the face terms of the owned rows are all there."""
    loc = np.full(int(part.elements.max()) + 2 if part.elements.size else 1, -1, dtype=np.int64)
    loc[part.elements] = np.arange(part.elements.size)
    e = np.asarray(bf.f2e, dtype=np.int64) - 1
    keep = (e < loc.size) & (loc[np.minimum(e, loc.size - 1)] >= 0)
    return M.BoundaryFaces((loc[e[keep]] + 1).astype(np.int32), np.asarray(bf.face_or)[keep],
                           np.asarray(bf.flags)[keep], np.asarray(bf.hconv)[keep], np.asarray(bf.tinf)[keep])


def local_bc_spec(spec: "M.BcSpec", part: Part) -> "M.BcSpec":
    """setBCs input of a partition: every boundary keeps its nodes that are
    local (1-based local ids, in the boundary's order), the FACE_ID and the
    tables as they are, NodeID restricted to the local nodes."""
    n = int(part.nodes.max()) + 1 if part.nodes.size else 0
    loc = np.full(max(n, int(max((int(b.max()) for b in spec.bnodes if len(b)), default=0))) + 1, -1,
                  dtype=np.int64)
    loc[part.nodes] = np.arange(part.nodes.size)
    bn = []
    for b in spec.bnodes:
        g = np.asarray(b, dtype=np.int64) - 1
        lg = loc[g]
        bn.append((lg[lg >= 0] + 1).astype(np.int32))
    nid = None if spec.node_id is None else np.asarray(spec.node_id)[part.nodes].astype(np.int32)
    return M.BcSpec(spec.face_id, bn, spec.bcug_type, spec.bcug_valu, spec.bcphig_type, spec.bcphig_valu,
                    spec.bctg_type, spec.bctg_valu, nid)


def local_case(case: "M.Case", part: Part) -> "M.Case":
    """The case restricted to a partition: local mesh, state, IBC and
    boundary faces."""
    st = {k: np.asfortranarray(np.asarray(v)[part.nodes]) for k, v in case.state.items()}
    ibc = np.asfortranarray(np.asarray(case.ibc)[part.nodes])
    lc = M.Case(f"{case.name}_p{part.rank}", part.mesh, dict(case.params), st, ibc, case.kernel,
                case.kspace, case.gmres_tol, case.newton_iters, dict(case.extra))
    if case.bfaces is not None:
        lc.bfaces = local_faces(case.bfaces, part)
    return lc


def owned_rows(col: np.ndarray, row: np.ndarray, vals: np.ndarray, part: Part):
    """The owned rows of a local CSR system (1-based `col` row pointer, `row`
    column indices) with global column ids: (rowptr 0-based over the owned
    rows, global column ids, values)."""
    col0 = np.asarray(col, dtype=np.int64) - 1
    starts, ends = col0[part.owned], col0[part.owned + 1]
    idx = np.concatenate([np.arange(a, b) for a, b in zip(starts, ends)]) if part.owned.size else np.zeros(0, np.int64)
    gcols = part.nodes[np.asarray(row, dtype=np.int64)[idx] - 1]
    rp = np.concatenate([[0], np.cumsum(ends - starts)])
    return rp, gcols, np.asarray(vals)[idx]
