"""Streaming time steps: fields staged on the upload stream while the
previous assembly runs, residuals read back on the download stream while the
next one runs, give the same residuals bit for bit as the synchronous
ovs_set_field / ovs_assemble / ovs_get_rhs sequence, over three steps with a
different state each; staging some fields swaps only those; a commit with
nothing staged is refused."""
import numpy as np
import pytest

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M
from oversetdevfort_b200.api import Context, PinnedArray

pytestmark = pytest.mark.gpu

FIELDS = ["dg", "dgold", "ug", "ugold", "acg", "acgold", "ugm", "ugmold", "pg", "phig", "phigold",
          "rphig", "rphigold", "tg", "tgold", "rtg", "rtgold"]


def _states(case, nsteps):
    rng = np.random.default_rng(9)
    out = []
    for i in range(nsteps):
        st = {}
        for f in FIELDS:
            a = PinnedArray(case.state[f].shape)
            a.array[...] = case.state[f] * (1.0 + 0.01 * i) + 1e-3 * rng.standard_normal(case.state[f].shape)
            st[f] = a
        out.append(st)
    return out


@pytest.mark.parametrize("prec", [F.OVS_FP32, F.OVS_FP64])
def test_streamed_steps_match_synchronous(prec):
    case = M.quench_case(M.box_tet(10, 10, 12, 1.0, 1.0, 1.25), "stream")
    N = case.mesh.nnode
    states = _states(case, 3)
    sync = Context.from_case(case)
    ref = []
    for st in states:
        for f in FIELDS:
            sync.set_field(f, st[f].array)
        sync.assemble(F.OVS_ASM_NSVOF, 6, prec)
        sync.assemble(F.OVS_ASM_TEM, 6, prec)
        ref.append((sync.get_rhs(F.OVS_SYS_NSVOF, prec), sync.get_rhs(F.OVS_SYS_TEM, prec)))
    sync.close()
    ctx = Context.from_case(case)
    outs = [(PinnedArray((N, 5)), PinnedArray((N, 1))) for _ in states]
    ctx.stage_fields({f: states[0][f].array for f in FIELDS})
    for i in range(len(states)):
        ctx.commit_staged()
        if i + 1 < len(states):
            ctx.stage_fields({f: states[i + 1][f].array for f in FIELDS})
        ctx.assemble(F.OVS_ASM_NSVOF, 6, prec)
        ctx.assemble(F.OVS_ASM_TEM, 6, prec)
        ctx.get_rhs_async(F.OVS_SYS_NSVOF, prec, outs[i][0].array)
        ctx.get_rhs_async(F.OVS_SYS_TEM, prec, outs[i][1].array)
    ctx.sync_copies()
    for (a, b), (ra, rb) in zip(outs, ref):
        np.testing.assert_array_equal(a.array, ra)
        np.testing.assert_array_equal(b.array, rb)
    ctx.close()


def test_partial_staging_and_empty_commit():
    case = M.quench_case(M.box_tet(6, 6, 8, 1.0, 1.0, 1.25), "stream2")
    ctx = Context.from_case(case)
    assert ctx.lib.ovs_commit_staged(ctx.h) == F.OVS_ERR_STATE
    tg0 = ctx.get_field("tg")
    ug = PinnedArray(case.state["ug"].shape)
    ug.array[...] = 3.25
    ctx.stage_fields({"ug": ug.array})
    ctx.commit_staged()
    np.testing.assert_array_equal(ctx.get_field("ug"), ug.array)
    np.testing.assert_array_equal(ctx.get_field("tg"), tg0)
    ug2 = PinnedArray(case.state["ug"].shape)
    ug2.array[...] = -1.5
    ctx.stage_fields({"ug": ug2.array})     # into the buffer retired by the first commit
    ctx.commit_staged()
    np.testing.assert_array_equal(ctx.get_field("ug"), ug2.array)
    ctx.sync_copies()
    ctx.close()


@pytest.mark.parametrize("prec", [F.OVS_FP32, F.OVS_FP64])
def test_streamed_async_quench_steady_state_matches_synchronous(prec):
    """The steady-state loop of a time loop: one OVS_ASM_QUENCH pass per step
    queued with ovs_assemble_async, every step staging the next step's
    fields (the last one the fields of a step after the loop), both
    residuals read back on the download stream per step into their own
    host buffers (the read-backs of the two systems do not wait for each
    other), the status read once per step."""
    case = M.quench_case(M.box_tet(10, 10, 12, 1.0, 1.0, 1.25), "stream3")
    N = case.mesh.nnode
    states = _states(case, 4)
    sync = Context.from_case(case)
    ref = []
    for st in states[:3]:
        for f in FIELDS:
            sync.set_field(f, st[f].array)
        sync.assemble(F.OVS_ASM_NSVOF, 6, prec)
        sync.assemble(F.OVS_ASM_TEM, 6, prec)
        ref.append((sync.get_rhs(F.OVS_SYS_NSVOF, prec), sync.get_rhs(F.OVS_SYS_TEM, prec)))
    sync.close()
    ctx = Context.from_case(case)
    outs = [(PinnedArray((N, 5)), PinnedArray((N, 1))) for _ in range(3)]
    ctx.stage_fields({f: states[0][f].array for f in FIELDS})
    ctx.sync_copies()
    for i in range(3):
        ctx.commit_staged()
        ctx.stage_fields({f: states[i + 1][f].array for f in FIELDS})
        ctx.assemble_async(F.OVS_ASM_QUENCH, 6, prec)
        ctx.get_rhs_async(F.OVS_SYS_NSVOF, prec, outs[i][0].array)
        ctx.get_rhs_async(F.OVS_SYS_TEM, prec, outs[i][1].array)
        ctx.assemble_wait()
    ctx.sync_copies()
    for (a, b), (ra, rb) in zip(outs, ref):
        np.testing.assert_array_equal(a.array, ra)
        np.testing.assert_array_equal(b.array, rb)
    # the fields staged by the last step are the fourth state's
    ctx.commit_staged()
    np.testing.assert_array_equal(ctx.get_field("ug"), states[3]["ug"].array)
    np.testing.assert_array_equal(ctx.get_field("tg"), states[3]["tg"].array)
    ctx.close()
