"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, the smoke check and the CPU-baseline leg of bench.py import
this module, as the checker.  The oracle is a literal FP64 restatement of the
reference (see ovs_oracle.h); PARITY UNPINNED: the reference has no golden
vectors and cannot be compiled here, so analytic known-answer tests pin it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# OVS_ORACLE_LIB selects another build of the same source, e.g. the
# sanitizer build of `make -C oracle asan` (run with the sanitizer runtimes
# in LD_PRELOAD); that build is made by its own make target, not here.
_OVERRIDE = os.environ.get("OVS_ORACLE_LIB")
LIB = Path(_OVERRIDE) if _OVERRIDE else HERE / "_build" / "libovs_oracle.so"

_dp = C.POINTER(C.c_double)
OVS_SYS_NSVOF, OVS_SYS_TEM = 2, 3   # system ids of include/ovs.h
_ip = C.POINTER(C.c_int)


def build() -> Path:
    if not _OVERRIDE:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


class OrcMesh(C.Structure):
    _fields_ = [("nnode", C.c_int), ("nelem", C.c_int), ("nshl", C.c_int), ("nibc", C.c_int),
                ("xg", _dp), ("ien", _ip), ("elm_id", _ip), ("ibc", _ip), ("col", _ip),
                ("row", _ip), ("icnt", C.c_int), ("quench_literal", C.c_int),
                ("nface", C.c_int), ("f2e", _ip), ("face_or", _ip), ("fflag", _ip), ("hconv", _dp),
                ("tinf", _dp)]


_STATE = ["dg", "dgold", "ug", "ugold", "acg", "acgold", "ugm", "ugmold", "acgm", "acgmold",
          "pg", "phig", "phigold", "rphig", "rphigold", "tg", "tgold", "rtg", "rtgold"]


class OrcState(C.Structure):
    _fields_ = [(n, _dp) for n in _STATE]


_SYS = ["K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS", "TEM", "rhsu", "rhsp", "rhsls", "rhstem"]


class OrcSystem(C.Structure):
    _fields_ = [(n, _dp) for n in _SYS]


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    from oversetdevfort_b200._ffi import OvsParams
    pp = C.POINTER(OvsParams)
    lib.orc_gen_spar_struc.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip]
    lib.orc_eval_shape.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.orc_eval_shape.restype = C.c_double
    lib.orc_sparse_mat_loc.argtypes = [_ip, C.c_int, C.c_int]
    lib.orc_slot_map.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip, _ip]
    lib.orc_slot_map.restype = None
    for fn in ("orc_assemble_navsto",):
        getattr(lib, fn).argtypes = [C.POINTER(OrcMesh), pp, C.POINTER(OrcState), C.POINTER(OrcSystem), C.c_int]
        getattr(lib, fn).restype = C.c_double
    lib.orc_assemble_quenching.argtypes = [C.POINTER(OrcMesh), pp, C.POINTER(OrcState),
                                           C.POINTER(OrcSystem), C.c_int, C.c_int]
    lib.orc_assemble_quenching.restype = C.c_double
    for fn in ("orc_elmloop_ns", "orc_elmloop_nsvof", "orc_elmloop_tem"):
        getattr(lib, fn).argtypes = [C.POINTER(OrcMesh), pp, C.POINTER(OrcState), C.POINTER(OrcSystem),
                                     C.c_int, C.c_int, C.c_int]
        getattr(lib, fn).restype = C.c_double
    from oversetdevfort_b200._ffi import OvsBcSpec
    lib.orc_set_bcs.argtypes = [C.c_int, C.c_int, _ip, pp, C.POINTER(OrcState), C.POINTER(OvsBcSpec), C.c_int]
    lib.orc_alpha_stage.argtypes = [C.c_int, pp, C.POINTER(OrcState), C.POINTER(OrcState)]
    lib.orc_sparse_prod_up_3d.argtypes = [C.c_int, _ip, _ip, C.POINTER(OrcSystem), _dp, _dp, _dp, _dp]
    lib.orc_sparse_prod_ns_conv.argtypes = [C.c_int, _ip, _ip, C.POINTER(OrcSystem), _dp, _dp, _dp,
                                            _dp, _dp, _dp]
    lib.orc_sparse_prod_ls.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp]
    lib.orc_gmres_up.argtypes = [C.c_int, _ip, _ip, C.POINTER(OrcSystem), C.c_double, C.c_int, C.c_int,
                                 _dp, _dp, _ip, _dp, _dp]
    lib.orc_gmres_ns_conv.argtypes = [C.c_int, _ip, _ip, C.POINTER(OrcSystem), C.c_double, C.c_int,
                                      C.c_int, _dp, _dp, _dp, _ip, _dp, _dp]
    lib.orc_gmres_tem.argtypes = [C.c_int, _ip, _ip, _dp, _dp, C.c_double, C.c_int, C.c_int, _dp, _ip,
                                  _dp, _dp]
    lib.orc_newton_update.argtypes = [C.c_int, C.c_int, pp, C.POINTER(OrcState), _dp]
    lib.orc_calculate_residual.argtypes = [C.c_int, C.POINTER(OrcSystem), _dp]
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def gen_spar_struc(ien: np.ndarray, nnode: int):
    lib = load()
    ien = np.asfortranarray(ien, dtype=np.int32)
    E, nshl = ien.shape
    col = np.zeros(nnode + 1, dtype=np.int32)
    icnt = C.c_int(0)
    st = lib.orc_gen_spar_struc(nnode, E, nshl, _i(ien), _i(col), None, C.byref(icnt))
    assert st == 0, st
    row = np.zeros(max(icnt.value, 1), dtype=np.int32)
    st = lib.orc_gen_spar_struc(nnode, E, nshl, _i(ien), _i(col), _i(row), C.byref(icnt))
    assert st == 0, st
    return col, row[: icnt.value]


def slot_map(ien: np.ndarray, col: np.ndarray, row: np.ndarray) -> np.ndarray:
    """k(e, a, b) of FillSparseMat_3D (src/FillSparseMat.f90:47-57) for
    every element entry: (E, nshl, nshl) Fortran-order int32, 1-based."""
    lib = load()
    ien = np.asfortranarray(ien, dtype=np.int32)
    E, nshl = ien.shape
    col = np.ascontiguousarray(col, dtype=np.int32)
    row = np.ascontiguousarray(row, dtype=np.int32)
    out = np.zeros((E, nshl, nshl), dtype=np.int32, order="F")
    lib.orc_slot_map(E, nshl, _i(ien), _i(col), _i(row), _i(out))
    return out


def eval_shape(nshl: int, igp: int, xl: np.ndarray, dl: np.ndarray | None = None):
    """eval_shape_fem at point igp of the element's rule: (DetJ, N (nshl),
    grad N (nshl, 3), G (3, 3), weight).  xl, dl: (nshl, 3)."""
    lib = load()
    x = np.ascontiguousarray(xl, dtype=np.float64)
    d = None if dl is None else np.ascontiguousarray(dl, dtype=np.float64)
    shl, shg, gij, gw = np.zeros(nshl), np.zeros((nshl, 3)), np.zeros((3, 3)), C.c_double(0)
    detj = lib.orc_eval_shape(nshl, igp, _d(x), None if d is None else _d(d), _d(shl), _d(shg), _d(gij),
                              C.byref(gw))
    return detj, shl, shg, gij, gw.value


class OracleCase:
    """Holds a case's arrays in the layout the oracle expects and keeps
    them alive while the C structures point at them."""

    def __init__(self, case, col=None, row=None, literal=False):
        from oversetdevfort_b200.mesh import to_ovs_params
        self.case = case
        m = case.mesh
        self.N, self.E, self.nshl = m.nnode, m.nelem, m.nshl
        self.xg = np.asfortranarray(m.xg, dtype=np.float64)
        self.ien = np.asfortranarray(m.ien, dtype=np.int32)
        self.elm = np.ascontiguousarray(m.elm_id, dtype=np.int32)
        self.ibc = np.asfortranarray(case.ibc, dtype=np.int32)
        if col is None:
            col, row = gen_spar_struc(self.ien, self.N)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.row = np.ascontiguousarray(row, dtype=np.int32)
        self.icnt = len(self.row)
        self.mesh = OrcMesh(self.N, self.E, self.nshl, self.ibc.shape[1], _d(self.xg), _i(self.ien),
                            _i(self.elm), _i(self.ibc), _i(self.col), _i(self.row), self.icnt,
                            1 if literal else 0)
        bf = getattr(case, "bfaces", None)
        if bf is not None and len(bf.f2e):
            self._faces = (np.ascontiguousarray(bf.f2e, dtype=np.int32),
                           np.ascontiguousarray(bf.face_or, dtype=np.int32),
                           np.ascontiguousarray(bf.flags, dtype=np.int32),
                           np.ascontiguousarray(bf.hconv, dtype=np.float64),
                           np.ascontiguousarray(bf.tinf, dtype=np.float64))
            f2e, fo, fl, hc, ti = self._faces
            self.mesh.nface = len(f2e)
            self.mesh.f2e, self.mesh.face_or, self.mesh.fflag = _i(f2e), _i(fo), _i(fl)
            self.mesh.hconv, self.mesh.tinf = _d(hc), _d(ti)
        self.params = to_ovs_params(case.params)
        self.state_arrays = {n: np.asfortranarray(case.state[n], dtype=np.float64).copy(order="F")
                             for n in _STATE}
        self.state = OrcState(*[_d(self.state_arrays[n]) for n in _STATE])
        K, N = self.icnt, self.N
        self.sys = {"K11": np.zeros((K, 9)), "G": np.zeros((K, 3)), "D1": np.zeros((K, 3)),
                    "M": np.zeros(K), "LS": np.zeros(K), "LSU": np.zeros((K, 3)), "ULS": np.zeros((K, 3)),
                    "PLS": np.zeros(K), "TEM": np.zeros(K), "rhsu": np.zeros((N, 3), order="F"),
                    "rhsp": np.zeros(N), "rhsls": np.zeros(N), "rhstem": np.zeros(N)}
        self.csys = OrcSystem(*[_d(self.sys[n]) for n in _SYS])

    # ------------------------------------------------------- BC producers
    def set_bcs(self, spec, which: int):
        """setBCs_NSVOF (which & 1) / setBCs_Tem (which & 2) on this case's
        state and IBC arrays."""
        keep, cs = spec.to_c()
        load().orc_set_bcs(self.N, self.ibc.shape[1], _i(self.ibc), C.byref(self.params), C.byref(self.state),
                           C.byref(cs), which)

    # ----------------------------------------------------------- assembly
    def assemble_navsto(self, tensor_flag: int) -> float:
        return load().orc_assemble_navsto(C.byref(self.mesh), C.byref(self.params),
                                          C.byref(self.state), C.byref(self.csys), tensor_flag)

    def assemble_quenching(self, tensor_flag: int, field_flag: int) -> float:
        return load().orc_assemble_quenching(C.byref(self.mesh), C.byref(self.params),
                                             C.byref(self.state), C.byref(self.csys), tensor_flag,
                                             field_flag)

    def system(self, kind: str) -> dict:
        """Copy of the assembled system in the GPU API's block naming."""
        s = self.sys
        if kind == "ns":
            d = {k: s[k].copy() for k in ("K11", "G", "D1", "M")}
            d["rhs"] = np.concatenate([s["rhsu"], s["rhsp"][:, None]], axis=1)
        elif kind == "nsvof":
            d = {k: s[k].copy() for k in ("K11", "G", "D1", "M", "LS", "LSU", "ULS", "PLS")}
            d["rhs"] = np.concatenate([s["rhsu"], s["rhsp"][:, None], s["rhsls"][:, None]], axis=1)
        else:
            d = {"TEM": s["TEM"].copy(), "rhs": s["rhstem"][:, None].copy()}
        return d

    def load_system(self, kind: str, d: dict):
        for k, v in d.items():
            if k == "rhs":
                continue
            self.sys[k][...] = v
        r = d["rhs"]
        if kind == "tem":
            self.sys["rhstem"][:] = r[:, 0]
        else:
            self.sys["rhsu"][:] = r[:, :3]
            self.sys["rhsp"][:] = r[:, 3]
            if kind == "nsvof":
                self.sys["rhsls"][:] = r[:, 4]

    # --------------------------------------------------------------- spmv
    def spmv(self, kind: str, x: np.ndarray) -> np.ndarray:
        lib = load()
        N = self.N
        x = np.asfortranarray(x, dtype=np.float64)
        y = np.zeros_like(x, order="F")
        if kind == "ns":
            xu, xp = np.asfortranarray(x[:, :3]), np.ascontiguousarray(x[:, 3])
            yu, yp = np.zeros((N, 3), order="F"), np.zeros(N)
            lib.orc_sparse_prod_up_3d(N, _i(self.col), _i(self.row), C.byref(self.csys), _d(xu), _d(xp),
                                      _d(yu), _d(yp))
            y[:, :3], y[:, 3] = yu, yp
        elif kind == "nsvof":
            xu = np.asfortranarray(x[:, :3])
            xp, xl = np.ascontiguousarray(x[:, 3]), np.ascontiguousarray(x[:, 4])
            yu, yp, yl = np.zeros((N, 3), order="F"), np.zeros(N), np.zeros(N)
            lib.orc_sparse_prod_ns_conv(N, _i(self.col), _i(self.row), C.byref(self.csys), _d(xu),
                                        _d(xp), _d(xl), _d(yu), _d(yp), _d(yl))
            y[:, :3], y[:, 3], y[:, 4] = yu, yp, yl
        else:
            xt = np.ascontiguousarray(x[:, 0])
            yt = np.zeros(N)
            lib.orc_sparse_prod_ls(N, _i(self.col), _i(self.row), _d(self.sys["TEM"]), _d(xt), _d(yt))
            y[:, 0] = yt
        return y

    # -------------------------------------------------------------- gmres
    def gmres(self, kind: str, tol: float, kspace: int, kmin: int, sol=None):
        lib = load()
        N = self.N
        nf = {"ns": 4, "nsvof": 5, "tem": 1}[kind]
        s = np.zeros((N, nf), order="F") if sol is None else np.asfortranarray(sol, dtype=np.float64).copy(order="F")
        it, er, r0 = C.c_int(0), C.c_double(0), C.c_double(0)
        if kind == "ns":
            su, sp = np.asfortranarray(s[:, :3]), np.ascontiguousarray(s[:, 3])
            st = lib.orc_gmres_up(N, _i(self.col), _i(self.row), C.byref(self.csys), tol, kspace, kmin,
                                  _d(su), _d(sp), C.byref(it), C.byref(er), C.byref(r0))
            s[:, :3], s[:, 3] = su, sp
        elif kind == "nsvof":
            su = np.asfortranarray(s[:, :3])
            sp, sl = np.ascontiguousarray(s[:, 3]), np.ascontiguousarray(s[:, 4])
            st = lib.orc_gmres_ns_conv(N, _i(self.col), _i(self.row), C.byref(self.csys), tol, kspace, kmin,
                                       _d(su), _d(sp), _d(sl), C.byref(it), C.byref(er), C.byref(r0))
            s[:, :3], s[:, 3], s[:, 4] = su, sp, sl
        else:
            st_ = np.ascontiguousarray(s[:, 0])
            st = lib.orc_gmres_tem(N, _i(self.col), _i(self.row), _d(self.sys["TEM"]),
                                   _d(self.sys["rhstem"]), tol, kspace, kmin, _d(st_), C.byref(it),
                                   C.byref(er), C.byref(r0))
            s[:, 0] = st_
        assert st == 0, st
        return s, it.value, er.value, r0.value

    def newton_update(self, system: int, sol: np.ndarray):
        s = np.asfortranarray(sol, dtype=np.float64)
        load().orc_newton_update(self.N, system, C.byref(self.params), C.byref(self.state), _d(s))

    def quench_newton(self, newton_max: int, solve_tem: bool, kspace: int, kspace_min: int, tol_ns: float,
                      tol_tem: float, utol, atol):
        """The Newton loop of solmultiphasethermofluid_stag
        (src/solveFlow.f90:4-164) on this case's state: the residual of all
        fields first (:39-46), then per Newton iteration the NS+VOF matrix and
        residual, one reference GMRES cycle from zero (SparseGMRES_ns_conv),
        its update (:99-104); the temperature likewise when solve_tem
        (:116-140); the residual of all fields again and check_convergence
        (:190-215: r < utol r0 or r < atol per field group, all groups).
        Returns a dict with iterations, converged, residual0, residual and
        the Krylov iterations."""
        def vec_all():   # one call for all fields, as :39-40 and :148-149 (a call zeroes every RHS)
            self.assemble_quenching(2, 7)
            return self.calculate_residual()

        r0 = vec_all()
        r = r0.copy()
        conv = lambda rr: all(rr[k] < utol[k] * r0[k] or rr[k] < atol[k] for k in range(4))
        out = {"iterations": 0, "converged": conv(r), "residual0": r0, "krylov_ns": 0, "krylov_tem": 0}
        for it in range(1, newton_max + 1):
            self.assemble_quenching(6, 3)
            s, k, _, _ = self.gmres("nsvof", tol_ns, kspace, kspace_min)
            out["krylov_ns"] += k
            self.newton_update(OVS_SYS_NSVOF, s)
            if solve_tem:
                self.assemble_quenching(6, 4)
                s, k, _, _ = self.gmres("tem", tol_tem, kspace, kspace_min)
                out["krylov_tem"] += k
                self.newton_update(OVS_SYS_TEM, s)
            r = vec_all()
            out["iterations"] = it
            out["converged"] = conv(r)
            if out["converged"]:
                break
        out["residual"] = r
        return out

    def quench_time_steps(self, first_step: int, nsteps: int, newton_max: int, solve_tem: bool, kspace: int,
                          kspace_min: int, tol_ns: float, tol_tem: float, utol, atol):
        """The driver's time loop around the Newton routine (src/driver.f90:
        70-100): per step the predictor ug = ugold, acg = (gami - 1)/gami
        acgold (:83-85), the Newton loop with NL_max = 1 while istep <= 1
        (src/solveFlow.f90:50-54) and no temperature solve at istep 0
        (:109), then the old values the driver updates (ug, acg, dg, ugm,
        acgm).  Returns the last step's Newton record."""
        st = self.state_arrays
        g = self.params.gami
        out = None
        for k in range(nsteps):
            istep = first_step + k
            st["ug"][...] = st["ugold"]
            st["acg"][...] = (g - 1.0) / g * st["acgold"]
            out = self.quench_newton(1 if istep <= 1 else newton_max, solve_tem and istep > 0, kspace,
                                     kspace_min, tol_ns, tol_tem, utol, atol)
            for cur, old in (("ug", "ugold"), ("acg", "acgold"), ("dg", "dgold"), ("ugm", "ugmold"),
                             ("acgm", "acgmold")):
                st[old][...] = st[cur]
        return out

    def calculate_residual(self) -> np.ndarray:
        r = np.zeros(4)
        load().orc_calculate_residual(self.N, C.byref(self.csys), _d(r))
        return r

    # ------------------------------------------------- timed element loop
    def time_element_loop(self, kind: str, tensor_flag: int, e0: int, e1: int) -> float:
        """Seconds spent by the element loop (alpha stage done beforehand)
        on elements [e0, e1)."""
        import time
        lib = load()
        if not hasattr(self, "_alpha"):
            self._alpha_arrays = {n: np.zeros_like(self.state_arrays[n]) for n in _STATE}
            self._alpha = OrcState(*[_d(self._alpha_arrays[n]) for n in _STATE])
            lib.orc_alpha_stage(self.N, C.byref(self.params), C.byref(self.state), C.byref(self._alpha))
        fn = {"ns": lib.orc_elmloop_ns, "nsvof": lib.orc_elmloop_nsvof, "tem": lib.orc_elmloop_tem}[kind]
        t0 = time.perf_counter()
        fn(C.byref(self.mesh), C.byref(self.params), C.byref(self._alpha), C.byref(self.csys), tensor_flag,
           e0, e1)
        return time.perf_counter() - t0

    def time_alpha_stage(self) -> float:
        import time
        lib = load()
        if not hasattr(self, "_alpha"):
            self._alpha_arrays = {n: np.zeros_like(self.state_arrays[n]) for n in _STATE}
            self._alpha = OrcState(*[_d(self._alpha_arrays[n]) for n in _STATE])
        t0 = time.perf_counter()
        lib.orc_alpha_stage(self.N, C.byref(self.params), C.byref(self.state), C.byref(self._alpha))
        return time.perf_counter() - t0
