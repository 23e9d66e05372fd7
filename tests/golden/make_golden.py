"""Generate tests/golden/quench_small.npz with the CPU oracle.

    python tests/golden/make_golden.py

The reference ships no golden vectors and cannot be compiled here, so these
fixtures come from the oracle (a literal restatement of the reference); they
freeze its output on small seeded cases (every code path switched on) so that
the GPU tests can compare against committed numbers and any change of the
oracle shows up.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "quench_small.npz"


def compute() -> dict:
    from oversetdevfort_b200 import mesh as M
    from oversetdevfort_b200 import _ffi as F
    from oracle import pyoracle as O

    out = {}
    # NS+VOF + temperature on a small random case
    c = M.random_case(nx=3, ny=2, nz=2, seed=11)
    oc = O.OracleCase(c)
    out["q_col"], out["q_row"] = oc.col.copy(), oc.row.copy()
    out["q_cfl"] = np.array([oc.assemble_quenching(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC, 7)])
    for k in ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS", "TEM", "rhsu", "rhsp", "rhsls", "rhstem"):
        out["q_" + k] = oc.sys[k].copy()
    s, it, er, r0 = oc.gmres("nsvof", 1e-8, 20, 1)
    out["q_sol_nsvof"], out["q_it_nsvof"] = s, np.array([it])
    s, it, er, r0 = oc.gmres("tem", 1e-8, 20, 1)
    out["q_sol_tem"], out["q_it_tem"] = s, np.array([it])
    # NS-only lid-driven cavity on 3^3 cells
    c1 = M.config1(n=3)
    o1 = O.OracleCase(c1)
    out["n_cfl"] = np.array([o1.assemble_navsto(F.OVS_TENSOR_MAT | F.OVS_TENSOR_VEC)])
    for k in ("K11", "G", "D1", "M", "rhsu", "rhsp"):
        out["n_" + k] = o1.sys[k].copy()
    s, it, er, r0 = o1.gmres("ns", 1e-6, 30, 1)
    out["n_sol"], out["n_it"] = s, np.array([it])
    return out


if __name__ == "__main__":
    d = compute()
    np.savez_compressed(OUT, **d)
    print(OUT, {k: v.shape for k, v in d.items()})
