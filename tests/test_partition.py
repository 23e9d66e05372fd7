"""Owner-computes partitions (oversetdevfort_b200.partition), CPU: the owned
rows assembled on each partition's local mesh (owned nodes plus every element
touching them) are bit-identical to the same rows of the global assembly,
checked with the oracle for the NS+VOF and temperature systems, and the
rows of two gloo ranks, gathered to rank 0, rebuild the global system."""
import os
import socket

import numpy as np
import pytest

from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200 import partition as P

BLOCKS = {"nsvof": ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS"), "tem": ("TEM",)}


def _assemble(oracle, case, kind):
    oc = oracle.OracleCase(case)
    oc.assemble_quenching(6, 3 if kind == "nsvof" else 4)
    return oc


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
@pytest.mark.parametrize("hexm", [False, True])
def test_owned_rows_match_global_assembly(oracle, kind, hexm):
    case = M.random_case(nx=5, ny=3, nz=3, seed=11, hex=hexm)
    og = _assemble(oracle, case, kind)
    gsys = og.system(kind)
    gcol = og.col.astype(np.int64) - 1
    for part in P.make_parts(case.mesh, 3):
        lc = P.local_case(case, part)
        ol = _assemble(oracle, lc, kind)
        lsys = ol.system(kind)
        for b in BLOCKS[kind]:
            rp, gcols, vals = P.owned_rows(ol.col, ol.row, lsys[b], part)
            for i, A in enumerate(part.global_rows):
                a, e = gcol[A], gcol[A + 1]
                np.testing.assert_array_equal(gcols[rp[i]:rp[i + 1]], og.row[a:e] - 1)
                np.testing.assert_array_equal(vals[rp[i]:rp[i + 1]], gsys[b][a:e])
        np.testing.assert_array_equal(lsys["rhs"][part.owned], gsys["rhs"][part.global_rows])


@pytest.mark.parametrize("kind", ["nsvof", "tem"])
def test_owned_rows_with_faces_match_global_assembly(oracle, kind):
    """With weak and convective boundary faces: each partition keeps the
    faces of its elements (global order), and its owned rows, face terms
    included, stay bit-identical to the global rows."""
    case = M.random_case(nx=5, ny=3, nz=3, seed=13)
    case.bfaces = M.face_set(case.mesh, weak=(1, 3, 6), convective={2: (20.0, 300.0), 5: (7.5, 350.0)})
    og = _assemble(oracle, case, kind)
    gsys = og.system(kind)
    gcol = og.col.astype(np.int64) - 1
    plain = case.bfaces
    case_nf = M.random_case(nx=5, ny=3, nz=3, seed=13)
    assert not np.array_equal(_assemble(oracle, case_nf, kind).system(kind)["rhs"], gsys["rhs"])  # faces act
    for part in P.make_parts(case.mesh, 3):
        lc = P.local_case(case, part)
        assert lc.bfaces is not None and 0 < len(lc.bfaces.f2e) <= len(plain.f2e)
        ol = _assemble(oracle, lc, kind)
        lsys = ol.system(kind)
        for b in BLOCKS[kind]:
            rp, gcols, vals = P.owned_rows(ol.col, ol.row, lsys[b], part)
            for i, A in enumerate(part.global_rows):
                a, e = gcol[A], gcol[A + 1]
                np.testing.assert_array_equal(vals[rp[i]:rp[i + 1]], gsys[b][a:e])
        np.testing.assert_array_equal(lsys["rhs"][part.owned], gsys["rhs"][part.global_rows])


def test_local_bc_spec_reproduces_global_setbcs(oracle):
    """setBCs on each partition (its boundary nodes and NodeID) gives, on
    every local node, the state and IBC of setBCs on the whole mesh."""
    case = M.random_case(nx=5, ny=3, nz=3, seed=17)
    m = case.mesh
    nid = np.zeros(m.nnode, np.int32)
    nid[::11] = 101
    spec = M.box_bc_spec(m, u={1: (0.0, 0.0, 0.0), 6: (1.0, None, 0.0)}, phi={5: 1.0}, T={2: 400.0, 5: 300.0},
                         node_id=nid, face_ids=(2, 1, 3, 4, 6, 5))
    og = oracle.OracleCase(case)
    og.set_bcs(spec, 3)
    for part in P.make_parts(m, 3):
        ol = oracle.OracleCase(P.local_case(case, part))
        ol.set_bcs(P.local_bc_spec(spec, part), 3)
        for k in ol.state_arrays:
            np.testing.assert_array_equal(ol.state_arrays[k], og.state_arrays[k][part.nodes])
        np.testing.assert_array_equal(ol.ibc, og.ibc[part.nodes])


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    from oracle import pyoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    case = M.random_case(nx=4, ny=3, nz=3, seed=12)
    part = P.make_parts(case.mesh, world)[rank]
    oc = pyoracle.OracleCase(P.local_case(case, part))
    oc.assemble_quenching(6, 4)
    rp, gcols, vals = P.owned_rows(oc.col, oc.row, oc.system("tem")["TEM"], part)
    rhs = oc.system("tem")["rhs"][part.owned, 0]
    payload = [part.global_rows, rp, gcols, vals, rhs]
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(payload, gathered, dst=0)
    if rank == 0:
        pyoracle.build()
        og = pyoracle.OracleCase(case)
        og.assemble_quenching(6, 4)
        g = og.system("tem")
        gcol = og.col.astype(np.int64) - 1
        ok = True
        covered = np.zeros(case.mesh.nnode, dtype=bool)
        for rows, rp, gc, v, r in gathered:
            for i, A in enumerate(rows):
                a, e = gcol[A], gcol[A + 1]
                ok &= np.array_equal(gc[rp[i]:rp[i + 1]], og.row[a:e] - 1)
                ok &= np.array_equal(v[rp[i]:rp[i + 1]], g["TEM"][a:e])
                ok &= r[i] == g["rhs"][A, 0]
                covered[A] = True
        q.put(bool(ok and covered.all()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_rebuild_global_system(oracle):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ok


def test_part_count_limits():
    """Every part owns at least one node: 1..N parts, the owned ranges cover
    the nodes once; more parts than nodes, or none, is an error."""
    import pytest
    m = M.box_tet(2, 2, 1)
    for n in (1, 5, m.nnode):
        parts = P.make_parts(m, n)
        owned = np.concatenate([p.nodes[p.owned] for p in parts])
        assert np.array_equal(np.sort(owned), np.arange(m.nnode)) and all(p.owned.size for p in parts)
    for n in (0, m.nnode + 1):
        with pytest.raises(ValueError):
            P.make_parts(m, n)
