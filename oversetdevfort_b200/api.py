"""Host-side mirror of the reference's hot-path interface.

The reference calls these Fortran routines from its Newton drivers
(src/solveFlow.f90, src/solveOverset.f90):

    genSparStruc()                                   src/genSparStruc.f90:4
    assembleNavSto(tensor_flag, subdomain_flag)      src/assembleNavSto.f90:4
    assembleQuenching(tensor_flag, field_flag)       src/solveQuenching.f90:4
    SparseGMRES_up(..., Utol, Kspaceu, Kspaceu_mn)   src/SparseGMRES_NS.f90:4
    SparseGMRES_ns_conv(...)                         src/SparseGMRES_NS_conv.f:1
    SparseGMRES_tem(...)                             src/SparseGMRES_tem.f90:1
    calculate_residual(...)                          src/solveFlow.f90:169

The functions of the same names below take a :class:`Context` (the device
resident replacement of the module globals) and keep the argument meaning,
flag values and in/out behaviour: assembly overwrites the LHS/RHS of the
fields it assembles, GMRES accumulates into ``sol``.  Everything runs in the
CUDA library (``_lib/libovs_b200.so``); there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi as F
from .mesh import Case, Mesh, to_ovs_params

ASSEMBLE_FIELD_NS, ASSEMBLE_FIELD_VOF, ASSEMBLE_FIELD_TEM = 1, 2, 4
ASSEMBLE_TENSOR_VEC, ASSEMBLE_TENSOR_MAT = F.OVS_TENSOR_VEC, F.OVS_TENSOR_MAT

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def _f64(a) -> np.ndarray:
    return np.asfortranarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.asfortranarray(a, dtype=np.int32)


NF = {F.OVS_SYS_NS: 4, F.OVS_SYS_NSVOF: 5, F.OVS_SYS_TEM: 1}
BLOCK_W = {F.OVS_BLK_K11: 9, F.OVS_BLK_G: 3, F.OVS_BLK_D1: 3, F.OVS_BLK_M: 1, F.OVS_BLK_LS: 1,
           F.OVS_BLK_LSU: 3, F.OVS_BLK_ULS: 3, F.OVS_BLK_PLS: 1, F.OVS_BLK_TEM: 1}
BLOCK_NAME = {F.OVS_BLK_K11: "K11", F.OVS_BLK_G: "G", F.OVS_BLK_D1: "D1", F.OVS_BLK_M: "M",
              F.OVS_BLK_LS: "LS", F.OVS_BLK_LSU: "LSU", F.OVS_BLK_ULS: "ULS", F.OVS_BLK_PLS: "PLS",
              F.OVS_BLK_TEM: "TEM"}
SYS_BLOCKS = {F.OVS_SYS_NS: [F.OVS_BLK_K11, F.OVS_BLK_G, F.OVS_BLK_D1, F.OVS_BLK_M],
              F.OVS_SYS_NSVOF: [F.OVS_BLK_K11, F.OVS_BLK_G, F.OVS_BLK_D1, F.OVS_BLK_M, F.OVS_BLK_LS,
                                F.OVS_BLK_LSU, F.OVS_BLK_ULS, F.OVS_BLK_PLS],
              F.OVS_SYS_TEM: [F.OVS_BLK_TEM]}


class Context:
    """Device-resident mesh, pattern, state and assembled systems (one CUDA
    stream).  Wraps ``ovs_ctx`` of include/ovs.h."""

    def __init__(self, nnode: int, nelem: int, nshl: int = 4, device: int = -1):
        self.lib = F.load()
        self.N, self.E, self.nshl = int(nnode), int(nelem), int(nshl)
        self.h = C.c_void_p()
        d = F.OvsDims(self.N, self.E, self.nshl, int(device))
        F.check(self.lib.ovs_create(C.byref(self.h), C.byref(d)), "ovs_create")
        self.icnt = 0
        self.last_status = 0

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if self.h:
            self.lib.ovs_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @classmethod
    def from_case(cls, case: Case, build: bool = True, device: int = -1) -> "Context":
        m = case.mesh
        ctx = cls(m.nnode, m.nelem, m.nshl, device)
        ctx.upload_mesh(m)
        if build:
            ctx.build_pattern()
        ctx.set_params(case.params)
        ctx.set_ibc(case.ibc)
        ctx.set_state(case.state)
        if case.bfaces is not None:
            ctx.set_faces(case.bfaces)
        return ctx

    # ----------------------------------------------------------------- mesh
    def upload_mesh(self, m: Mesh):
        self._xg = _f64(m.xg)
        ien = _i32(m.ien)
        elm = np.ascontiguousarray(m.elm_id, dtype=np.int32)
        F.check(self.lib.ovs_upload_mesh(self.h, _dptr(self._xg), _iptr(ien), _iptr(elm)),
                "ovs_upload_mesh")
        self.xg = self._xg

    def build_pattern(self) -> int:
        icnt = C.c_int(0)
        F.check(self.lib.ovs_build_pattern(self.h, C.byref(icnt)), "ovs_build_pattern")
        self.icnt = icnt.value
        return self.icnt

    def get_pattern(self):
        col = np.zeros(self.N + 1, dtype=np.int32)
        row = np.zeros(max(self.icnt, 1), dtype=np.int32)
        F.check(self.lib.ovs_get_pattern(self.h, _iptr(col), _iptr(row)), "ovs_get_pattern")
        return col, row[: self.icnt]

    def get_slot_map(self) -> np.ndarray:
        """k(e, a, b) of FillSparseMat_3D for every element entry: (E, nshl,
        nshl) Fortran-order int32, 1-based CSR slots (ovs_get_slot_map)."""
        out = np.zeros((self.E, self.nshl, self.nshl), dtype=np.int32, order="F")
        F.check(self.lib.ovs_get_slot_map(self.h, _iptr(out)), "ovs_get_slot_map")
        return out

    # ---------------------------------------------------------- parameters
    def set_params(self, p: dict):
        self.params = dict(p)
        op = to_ovs_params(p)
        F.check(self.lib.ovs_set_params(self.h, C.byref(op)), "ovs_set_params")

    def set_ibc(self, ibc: np.ndarray):
        a = _i32(ibc)
        F.check(self.lib.ovs_set_ibc(self.h, _iptr(a), a.shape[1]), "ovs_set_ibc")

    def set_option(self, option: int, value: int):
        """A kernel-variant option of this context (OVS_OPT_*: HEX_TC,
        ARNOLDI_FUSED, ROWS_STAGED, ELEM_SMEM, ROWS_GATHER, ROWS_TILED,
        TILE_ELEMS); see include/ovs.h for the values."""
        F.check(self.lib.ovs_set_option(self.h, option, int(value)), "ovs_set_option")

    def set_faces(self, bf):
        """Boundary faces for the face assemblies (mesh.BoundaryFaces, or None
        to clear): FaceAssembly_NS_weak / _outflow on OVS_FACE_WEAK faces and
        the convective heat term on OVS_FACE_CONVH faces."""
        if bf is None or len(bf.f2e) == 0:
            F.check(self.lib.ovs_set_faces(self.h, 0, None, None, None, None, None), "ovs_set_faces")
            return
        f2e, fo, fl = _i32(bf.f2e), _i32(bf.face_or), _i32(bf.flags)
        hc = np.ascontiguousarray(bf.hconv, dtype=np.float64)
        ti = np.ascontiguousarray(bf.tinf, dtype=np.float64)
        F.check(self.lib.ovs_set_faces(self.h, len(f2e), _iptr(f2e), _iptr(fo), _iptr(fl), _dptr(hc), _dptr(ti)),
                "ovs_set_faces")

    def set_bc_spec(self, spec):
        """Boundary data of setBCs_NSVOF / setBCs_Tem (mesh.BcSpec, or None to
        clear); applied by quench_newton where the reference calls them."""
        if spec is None:
            F.check(self.lib.ovs_set_bc_spec(self.h, None), "ovs_set_bc_spec")
            return
        keep, cs = spec.to_c()
        F.check(self.lib.ovs_set_bc_spec(self.h, C.byref(cs)), "ovs_set_bc_spec")

    def apply_bcs(self, which: int = 3):
        """setBCs_NSVOF (which & 1) and setBCs_Tem (which & 2) on the device."""
        F.check(self.lib.ovs_apply_bcs(self.h, which), "ovs_apply_bcs")

    def get_ibc(self, nibc: int = 8) -> np.ndarray:
        out = np.zeros((self.N, nibc), dtype=np.int32, order="F")
        F.check(self.lib.ovs_get_ibc(self.h, _iptr(out), nibc), "ovs_get_ibc")
        return out

    # ------------------------------------------------ streaming time steps
    def stage_fields(self, arrays: dict):
        """Copies {field name: host array (reference layout; page-locked for
        asynchronous copies, e.g. PinnedArray.array)} into the staging buffers
        on the upload streams; returns at once.  The arrays must stay alive
        and unchanged until, after the commit that consumes them, a call that
        waits for the compute stream (assemble, sync_copies) has returned."""
        names = list(arrays)
        ids = (C.c_int * len(names))(*[F.FIELD_ID[n] for n in names])
        self._staged_keep = [np.asarray(arrays[n]) for n in names]
        for a in self._staged_keep:
            if a.dtype != np.float64 or not (a.flags.f_contiguous or a.ndim == 1):
                raise ValueError("stage_fields wants float64 arrays in reference (column-major) layout")
        ptrs = (C.POINTER(C.c_double) * len(names))(*[_dptr(a) for a in self._staged_keep])
        F.check(self.lib.ovs_stage_fields(self.h, len(names), ids, ptrs), "ovs_stage_fields")

    def commit_staged(self):
        F.check(self.lib.ovs_commit_staged(self.h), "ovs_commit_staged")

    def get_rhs_async(self, system: int, precision: int, out: np.ndarray):
        """Queues the read-back of the right-hand side into `out` ((N, nf)
        float64, column-major; page-locked for an asynchronous copy); valid
        after sync_copies."""
        if out.dtype != np.float64 or out.shape != (self.N, NF[system]) or not out.flags.f_contiguous:
            raise ValueError("out must be a column-major float64 (N, nf) array")
        F.check(self.lib.ovs_get_rhs_async(self.h, system, precision, _dptr(out)), "ovs_get_rhs_async")

    def sync_copies(self):
        F.check(self.lib.ovs_sync_copies(self.h), "ovs_sync_copies")

    def set_field(self, name: str, arr: np.ndarray):
        a = _f64(arr)
        F.check(self.lib.ovs_set_field(self.h, F.FIELD_ID[name], _dptr(a)), f"ovs_set_field({name})")

    def get_field(self, name: str) -> np.ndarray:
        shape = (self.N, 3) if F.FIELD_WIDTH[name] == 3 else (self.N,)
        a = np.zeros(shape, order="F")
        F.check(self.lib.ovs_get_field(self.h, F.FIELD_ID[name], _dptr(a)), f"ovs_get_field({name})")
        return a

    def set_state(self, st: dict):
        for n, v in st.items():
            if n != "xg":
                self.set_field(n, v)

    # ------------------------------------------------------------- assembly
    def assemble(self, kernel: int, tensor_flag: int, precision: int = F.OVS_FP64) -> float:
        cfl = C.c_double(0.0)
        st = self.lib.ovs_assemble(self.h, kernel, tensor_flag, precision, C.byref(cfl))
        self.last_status = F.check(st, "ovs_assemble")
        return cfl.value

    def assemble_async(self, kernel: int, tensor_flag: int, precision: int = F.OVS_FP64):
        """ovs_assemble_async: queue the pass and return at once."""
        F.check(self.lib.ovs_assemble_async(self.h, kernel, tensor_flag, precision), "ovs_assemble_async")

    def assemble_wait(self) -> float:
        """ovs_assemble_wait: wait for the queued passes; raises on an error,
        keeps a warning in last_status; returns the largest CFL number."""
        cfl = C.c_double(0.0)
        self.last_status = F.check(self.lib.ovs_assemble_wait(self.h, C.byref(cfl)), "ovs_assemble_wait")
        return cfl.value

    def get_rhs(self, system: int, precision: int = F.OVS_FP64) -> np.ndarray:
        a = np.zeros((self.N, NF[system]), order="F")
        F.check(self.lib.ovs_get_rhs(self.h, system, precision, _dptr(a)), "ovs_get_rhs")
        return a

    def set_rhs(self, system: int, precision: int, rhs: np.ndarray):
        a = _f64(np.reshape(rhs, (self.N, NF[system]), order="F"))
        F.check(self.lib.ovs_set_rhs(self.h, system, precision, _dptr(a)), "ovs_set_rhs")

    def get_lhs(self, system: int, precision: int, block: int) -> np.ndarray:
        w = BLOCK_W[block]
        a = np.zeros((self.icnt, w))
        F.check(self.lib.ovs_get_lhs_block(self.h, system, precision, block, _dptr(a)),
                "ovs_get_lhs_block")
        return a if w > 1 else a[:, 0]

    def set_lhs(self, system: int, precision: int, block: int, vals: np.ndarray):
        w = BLOCK_W[block]
        a = np.ascontiguousarray(np.reshape(vals, (self.icnt, w)), dtype=np.float64)
        F.check(self.lib.ovs_set_lhs_block(self.h, system, precision, block, _dptr(a)),
                "ovs_set_lhs_block")

    def get_system(self, system: int, precision: int = F.OVS_FP64) -> dict:
        out = {BLOCK_NAME[b]: self.get_lhs(system, precision, b) for b in SYS_BLOCKS[system]}
        out["rhs"] = self.get_rhs(system, precision)
        return out

    def set_system(self, system: int, precision: int, blocks: dict, rhs: np.ndarray):
        for b in SYS_BLOCKS[system]:
            self.set_lhs(system, precision, b, blocks[BLOCK_NAME[b]])
        self.set_rhs(system, precision, rhs)

    # ---------------------------------------------------------------- solve
    def spmv(self, system: int, precision: int, x: np.ndarray) -> np.ndarray:
        xa = _f64(np.reshape(x, (self.N, NF[system]), order="F"))
        y = np.zeros_like(xa, order="F")
        F.check(self.lib.ovs_spmv(self.h, system, precision, _dptr(xa), _dptr(y)), "ovs_spmv")
        return y

    def gmres(self, system: int, tol: float, kspace: int, kspace_min: int, sol: np.ndarray):
        s = _f64(np.reshape(sol, (self.N, NF[system]), order="F")).copy(order="F")
        info = F.OvsGmresInfo()
        F.check(self.lib.ovs_gmres(self.h, system, tol, kspace, kspace_min, _dptr(s), C.byref(info)),
                "ovs_gmres")
        return s, info

    def solve(self, system: int, mode: int, rtol: float, kspace: int = 50, max_cycles: int = 100,
              want_solution: bool = True):
        """ovs_solve: drive ||b - A x|| / ||b|| to rtol.  mode OVS_FP64
        (restarted FP64 GMRES), OVS_MIXED (the FP64 system refined with FP32
        inner cycles on the rounded FP64 matrix) or OVS_FP32 (the
        FP32-assembled system).  Returns (solution or None, OvsSolveInfo)."""
        info = F.OvsSolveInfo()
        s = np.zeros((self.N, NF[system]), order="F") if want_solution else None
        F.check(self.lib.ovs_solve(self.h, system, mode, rtol, kspace, max_cycles,
                                   _dptr(s) if s is not None else None, C.byref(info)), "ovs_solve")
        return s, info

    def residual_vjp(self, kernel: int, cot: np.ndarray) -> np.ndarray:
        """(d RHS / d state)^T cot for the FP64 RHS of `kernel` (OVS_ASM_NSVOF:
        cot (N,5); OVS_ASM_TEM: cot (N,) or (N,1)); returns (N, OVS_VJP_COUNT)
        with the columns OVS_VJP_* (coordinates, u, p, phi, T, a, phidot,
        Tdot)."""
        nf = 1 if kernel == F.OVS_ASM_TEM else 5
        c = _f64(np.reshape(cot, (self.N, nf), order="F"))
        g = np.zeros((self.N, F.OVS_VJP_COUNT), order="F")
        F.check(self.lib.ovs_residual_vjp(self.h, kernel, _dptr(c), _dptr(g)), "ovs_residual_vjp")
        return g

    def gmres_transposed(self, system: int, rhs: np.ndarray, tol: float, kspace: int, kspace_min: int = 1):
        """A^T x = rhs for the assembled FP64 temperature matrix (zero start)."""
        b = _f64(np.reshape(rhs, (self.N,)))
        x = np.zeros(self.N)
        info = F.OvsGmresInfo()
        F.check(self.lib.ovs_gmres_transposed(self.h, system, _dptr(b), tol, kspace, kspace_min, _dptr(x),
                                              C.byref(info)), "ovs_gmres_transposed")
        return x, info

    def quench_newton(self, mode: int = F.OVS_FP64, newton_max: int = 3, solve_tem: bool = True,
                      kspace: int = 50, kspace_min: int = 1, max_cycles: int = 100, tol_ns: float = 1e-6,
                      tol_tem: float = 1e-6, utol=(1e-3, 1e-3, 1e-3, 1e-3), atol=(1e-15, 1e-15, 1e-15, 1e-15)):
        """The Newton loop of one quench time step on the device
        (solmultiphasethermofluid_stag): returns the OvsNewtonInfo."""
        o = F.OvsNewtonOpts(mode, newton_max, int(solve_tem), kspace, kspace_min, max_cycles, tol_ns, tol_tem,
                            (C.c_double * 4)(*utol), (C.c_double * 4)(*atol))
        info = F.OvsNewtonInfo()
        F.check(self.lib.ovs_quench_newton(self.h, C.byref(o), C.byref(info)), "ovs_quench_newton")
        return info

    def quench_time_steps(self, first_step: int, nsteps: int, update_vof_tem_old: bool = False, **newton):
        """nsteps time steps of the reference driver on the device (predictor,
        Newton loop, old-value update); returns (last step's OvsNewtonInfo,
        Krylov iterations over all steps).  Keyword arguments as quench_newton."""
        d = dict(mode=F.OVS_FP64, newton_max=3, solve_tem=True, kspace=50, kspace_min=1, max_cycles=100,
                 tol_ns=1e-6, tol_tem=1e-6, utol=(1e-3,) * 4, atol=(1e-15,) * 4)
        d.update(newton)
        o = F.OvsNewtonOpts(d["mode"], d["newton_max"], int(d["solve_tem"]), d["kspace"], d["kspace_min"],
                            d["max_cycles"], d["tol_ns"], d["tol_tem"], (C.c_double * 4)(*d["utol"]),
                            (C.c_double * 4)(*d["atol"]))
        info = F.OvsNewtonInfo()
        kt = C.c_int(0)
        F.check(self.lib.ovs_quench_time_steps(self.h, first_step, nsteps, C.byref(o), int(update_vof_tem_old),
                                               C.byref(info), C.byref(kt)), "ovs_quench_time_steps")
        return info, kt.value

    def round_matrix(self, system: int):
        """ovs_round_matrix: the FP32 matrix of `system` := the FP32 rounding
        of its FP64 matrix (the inner operator of the OVS_MIXED refinement)."""
        F.check(self.lib.ovs_round_matrix(self.h, system), "ovs_round_matrix")

    def newton_update(self, system: int):
        F.check(self.lib.ovs_newton_update(self.h, system), "ovs_newton_update")

    def predictor(self):
        """ovs_predictor: ug = ugold, acg = (gami - 1)/gami acgold
        (src/driver.f90:83-85)."""
        F.check(self.lib.ovs_predictor(self.h), "ovs_predictor")

    def commit_old(self, update_vof_tem_old: bool = False):
        """ovs_commit_old: the old values the driver updates after a step
        (src/driver.f90:98-103)."""
        F.check(self.lib.ovs_commit_old(self.h, int(update_vof_tem_old)), "ovs_commit_old")

    def set_solution(self, system: int, sol):
        """ovs_set_solution: the solution the next `newton_update` of `system`
        applies.  `sol` is a host array (N, nf) or a contiguous FP64 CUDA
        tensor (nf, N) on this context's device (the same field-major
        layout)."""
        nf = {F.OVS_SYS_NS: 4, F.OVS_SYS_NSVOF: 5, F.OVS_SYS_TEM: 1}[system]
        if hasattr(sol, "data_ptr"):
            import torch
            if sol.dtype != torch.float64 or not sol.is_cuda or not sol.is_contiguous() \
                    or tuple(sol.shape) != (nf, self.N):
                raise ValueError(f"expected a contiguous float64 CUDA tensor of shape ({nf}, {self.N})")
            torch.cuda.current_stream(sol.device).synchronize()
            ptr = C.c_void_p(sol.data_ptr())
        else:
            a = np.asfortranarray(sol, dtype=np.float64).reshape(self.N, nf, order="F")
            self._sol_keep = a
            ptr = a.ctypes.data_as(C.c_void_p)
        F.check(self.lib.ovs_set_solution(self.h, system, ptr), "ovs_set_solution")

    def residual_norms(self, precision: int = F.OVS_FP64) -> np.ndarray:
        r = np.zeros(4)
        F.check(self.lib.ovs_residual_norms(self.h, precision, _dptr(r)), "ovs_residual_norms")
        return r

    def synchronize(self):
        F.check(self.lib.ovs_synchronize(self.h), "ovs_synchronize")

    # ---------------------------------------------------------- measurement
    def profile(self, what: int, system: int, precision: int, reps: int = 10) -> float:
        """Average device ms of one internal kernel (see ovs_profile)."""
        ms = C.c_double(0.0)
        F.check(self.lib.ovs_profile(self.h, what, system, precision, reps, C.byref(ms)), "ovs_profile")
        return ms.value

    def measure_fp32_peak(self) -> float:
        """Measured FP32 FMA throughput of the device, TFLOP/s."""
        t = C.c_double(0.0)
        F.check(self.lib.ovs_measure_fp32_peak(self.h, C.byref(t)), "ovs_measure_fp32_peak")
        return t.value

    def measure_fp64_peak(self) -> float:
        """Measured FP64 FMA throughput of the device, TFLOP/s."""
        t = C.c_double(0.0)
        F.check(self.lib.ovs_measure_fp64_peak(self.h, C.byref(t)), "ovs_measure_fp64_peak")
        return t.value

    def launch_count(self) -> int:
        n = C.c_longlong(0)
        F.check(self.lib.ovs_launch_count(self.h, C.byref(n)), "ovs_launch_count")
        return n.value

    def last_device_ms(self) -> float:
        ms = C.c_double(0.0)
        F.check(self.lib.ovs_last_device_ms(self.h, C.byref(ms)), "ovs_last_device_ms")
        return ms.value


class PinnedArray:
    """numpy view of a page-locked host buffer (ovs_host_alloc)."""

    def __init__(self, shape, dtype=np.float64, order="F"):
        self.lib = F.load()
        dt = np.dtype(dtype)
        n = int(np.prod(shape)) * dt.itemsize
        self.ptr = C.c_void_p()
        F.check(self.lib.ovs_host_alloc(C.byref(self.ptr), n), "ovs_host_alloc")
        buf = (C.c_char * n).from_address(self.ptr.value)
        self.array = np.ndarray(shape, dtype=dt, buffer=buf, order=order)

    def free(self):
        if self.ptr:
            self.array = None
            self.lib.ovs_host_free(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# --------------------------------------------------- reference-named routines
def genSparStruc(ien: np.ndarray, nnode: int):
    """CSR pattern of IEN(E,nshl) (1-based): returns (col(N+1), row(icnt)),
    col = row pointer, row = column indices, 1-based, rows ascending
    (src/genSparStruc.f90:4-47)."""
    lib = F.load()
    ien = _i32(ien)
    E, nshl = ien.shape
    col = np.zeros(nnode + 1, dtype=np.int32)
    icnt = C.c_int(0)
    F.check(lib.ovs_gen_spar_struc(nnode, E, nshl, _iptr(ien), _iptr(col), None, C.byref(icnt)),
            "genSparStruc")
    row = np.zeros(max(icnt.value, 1), dtype=np.int32)
    F.check(lib.ovs_gen_spar_struc(nnode, E, nshl, _iptr(ien), _iptr(col), _iptr(row),
                                   C.byref(icnt)), "genSparStruc")
    return col, row[: icnt.value]


def assembleNavSto(ctx: Context, assemble_tensor_flag: int, precision: int = F.OVS_FP64) -> float:
    """src/assembleNavSto.f90:4-72 (NS-only; the subdomain flag lives in the
    parameters).  Returns the CFL number the reference prints."""
    return ctx.assemble(F.OVS_ASM_NS, assemble_tensor_flag, precision)


def assembleQuenching(ctx: Context, assemble_tensor_flag: int, assemble_field_flag: int,
                      precision: int = F.OVS_FP64) -> float:
    """src/solveQuenching.f90:4-117: NS+VOF when NS or VOF is flagged, then
    the temperature pass when TEM is flagged (both flagged: one
    OVS_ASM_QUENCH call; its CFL number is the larger of the two passes',
    which evaluate the same advection speed)."""
    cfl = 0.0
    if assemble_field_flag & ASSEMBLE_FIELD_TEM and assemble_field_flag & (ASSEMBLE_FIELD_NS | ASSEMBLE_FIELD_VOF):
        return ctx.assemble(F.OVS_ASM_QUENCH, assemble_tensor_flag, precision)
    if assemble_field_flag & (ASSEMBLE_FIELD_NS | ASSEMBLE_FIELD_VOF):
        cfl = ctx.assemble(F.OVS_ASM_NSVOF, assemble_tensor_flag, precision)
    if assemble_field_flag & ASSEMBLE_FIELD_TEM:
        c2 = ctx.assemble(F.OVS_ASM_TEM, assemble_tensor_flag, precision)
        if not assemble_field_flag & (ASSEMBLE_FIELD_NS | ASSEMBLE_FIELD_VOF):
            cfl = c2
    return cfl


def SparseGMRES_up(ctx: Context, Utol: float, Kspaceu: int, Kspaceu_mn: int,
                   solu: np.ndarray, solp: np.ndarray):
    """src/SparseGMRES_NS.f90:4-369 on the resident FP64 (u,p) system; solu
    (N,3) and solp (N) are accumulated into and returned with the info."""
    sol = np.concatenate([_f64(solu).reshape(-1, 3, order="F"), _f64(solp).reshape(-1, 1)], axis=1)
    s, info = ctx.gmres(F.OVS_SYS_NS, Utol, Kspaceu, Kspaceu_mn, sol)
    return np.asfortranarray(s[:, :3]), s[:, 3].copy(), info


def SparseGMRES_ns_conv(ctx: Context, Utol: float, Kspaceu: int, Kspaceu_mn: int,
                        solu: np.ndarray, solp: np.ndarray, solls: np.ndarray):
    """src/SparseGMRES_NS_conv.f:1-406 on the resident FP64 (u,p,phi) system."""
    sol = np.concatenate([_f64(solu).reshape(-1, 3, order="F"), _f64(solp).reshape(-1, 1),
                          _f64(solls).reshape(-1, 1)], axis=1)
    s, info = ctx.gmres(F.OVS_SYS_NSVOF, Utol, Kspaceu, Kspaceu_mn, sol)
    return np.asfortranarray(s[:, :3]), s[:, 3].copy(), s[:, 4].copy(), info


def SparseGMRES_tem(ctx: Context, Utol: float, Kspaceu: int, Kspaceu_mn: int, sol: np.ndarray):
    """src/SparseGMRES_tem.f90:1-256 on the resident FP64 temperature system."""
    s, info = ctx.gmres(F.OVS_SYS_TEM, Utol, Kspaceu, Kspaceu_mn, _f64(sol).reshape(-1, 1))
    return s[:, 0].copy(), info


def calculate_residual(ctx: Context, precision: int = F.OVS_FP64) -> np.ndarray:
    """src/solveFlow.f90:169-187: sums of squares (no square root) of the
    momentum, continuity, VOF and temperature residuals."""
    return ctx.residual_norms(precision)


def check_convergence(residual, residual0, tol, assemble_field_flag: int, atol) -> np.ndarray:
    """src/solveFlow.f90:192-222: converged(4) as 0/1 ints.  Momentum and
    continuity (entries 1, 2) when NS is flagged, VOF (3) when VOF is,
    temperature (4) when TEM is; a field converges when residual < tol *
    residual0 or residual < its absolute tolerance (strict comparisons;
    the reference uses NS_GMRES_atol for both NS entries, LSC_GMRES_atol and
    TEM_GMRES_atol for the others: atol holds the four in that order).
    Fields outside the flag stay 0, as the reference leaves them."""
    r, r0 = np.asarray(residual, dtype=np.float64), np.asarray(residual0, dtype=np.float64)
    out = np.zeros(4, dtype=np.int32)
    groups = ((ASSEMBLE_FIELD_NS, (0, 1)), (ASSEMBLE_FIELD_VOF, (2,)), (ASSEMBLE_FIELD_TEM, (3,)))
    for bit, ks in groups:
        if assemble_field_flag & bit:
            for k in ks:
                out[k] = int(r[k] < tol[k] * r0[k] or r[k] < atol[k])
    return out


def setBCs_NSVOF(ctx: Context):
    """src/setBCs.f90:172-244 on the registered BC spec (Context.set_bc_spec):
    IBC columns 1-5 reset and set, Dirichlet velocity and VOF values with
    their rates."""
    ctx.apply_bcs(1)


def setBCs_Tem(ctx: Context):
    """src/setBCs.f90:248-278: Dirichlet temperature and its rate."""
    ctx.apply_bcs(2)


def solmultiphasethermofluid_stag(ctx: Context, istep: int, **newton):
    """The Newton routine of one quench time step (src/solveFlow.f90:4-164)
    as the driver calls it with istep: a single Newton iteration while
    istep <= 1 (:50-54) and no temperature solve at istep 0 (:109); the
    other keyword arguments as Context.quench_newton.  Returns its
    OvsNewtonInfo."""
    nm = newton.pop("newton_max", 3)
    tem = newton.pop("solve_tem", True)
    return ctx.quench_newton(newton_max=1 if istep <= 1 else nm, solve_tem=bool(tem and istep > 0), **newton)


def check_bc_spec(spec, nnode: int) -> int:
    """ovs_check_bc_spec: the checks of Context.set_bc_spec for a mesh of
    nnode nodes, without a device.  Returns the status (OVS_OK or
    OVS_ERR_ARG)."""
    keep, cs = spec.to_c()
    return int(F.load().ovs_check_bc_spec(C.byref(cs), int(nnode)))


def check_faces(bf, nelem: int) -> int:
    """ovs_check_faces: the checks of Context.set_faces for a face set
    (mesh.BoundaryFaces) on a tet mesh of nelem elements, without a device.
    Returns the status (OVS_OK or OVS_ERR_ARG)."""
    f2e, fo, fl = (np.ascontiguousarray(a, dtype=np.int32) for a in (bf.f2e, bf.face_or, bf.flags))
    hc, ti = (np.ascontiguousarray(a, dtype=np.float64) for a in (bf.hconv, bf.tinf))
    n = int(f2e.size)
    return int(F.load().ovs_check_faces(int(nelem), n, _iptr(f2e), _iptr(fo), _iptr(fl),
                                        _dptr(hc) if hc.size else None, _dptr(ti) if ti.size else None))
