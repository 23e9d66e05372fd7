"""ctypes declarations of the C ABI in ``include/ovs.h``.

The shared library is the in-tree ``_lib/libovs_b200.so`` built by
``oversetdevfort_b200.build``.  There is no fallback: if the library is
missing or fails to load, importing the API raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libovs_b200.so"

# status codes
OVS_OK = 0
OVS_WARN_NEG_DETJ = 1
OVS_ERR_ARG = -1
OVS_ERR_CUDA = -2
OVS_ERR_NOMEM = -3
OVS_ERR_STATE = -4
OVS_ERR_NONFINITE = -5
OVS_ERR_PATTERN = -6
OVS_ERR_NODEVICE = -7
OVS_ERR_TIMEOUT = -8

OVS_FP64, OVS_FP32, OVS_MIXED = 0, 1, 2
OVS_ASM_NS, OVS_ASM_NSVOF, OVS_ASM_TEM, OVS_ASM_QUENCH = 1, 2, 3, 4
OVS_SYS_NS, OVS_SYS_NSVOF, OVS_SYS_TEM = 1, 2, 3
OVS_TENSOR_VEC, OVS_TENSOR_MAT = 2, 4
OVS_PROF_SPMV, OVS_PROF_ASSEMBLE, OVS_PROF_ARNOLDI, OVS_PROF_ARNOLDI_FUSED = 1, 2, 3, 4
OVS_PROF_ASSEMBLE_ELEMENTS, OVS_PROF_ASSEMBLE_ROWS = 5, 6
# fields of the residual VJP (ovs_residual_vjp), N values each
OVS_VJP_XG, OVS_VJP_UG, OVS_VJP_PG, OVS_VJP_PHIG, OVS_VJP_TG = 0, 3, 6, 7, 8
OVS_VJP_ACG, OVS_VJP_RPHIG, OVS_VJP_RTG, OVS_VJP_COUNT = 9, 12, 13, 14
OVS_NOALLOC_MAX_N, OVS_NOALLOC_MAX_KSPACE = 16384, 40
OVS_FACE_WEAK, OVS_FACE_CONVH = 1, 2
OVS_OPT_HEX_TC, OVS_OPT_ARNOLDI_FUSED, OVS_OPT_ROWS_STAGED, OVS_OPT_ELEM_SMEM = 1, 2, 3, 4
OVS_OPT_ROWS_GATHER, OVS_OPT_ROWS_TILED, OVS_OPT_TILE_ELEMS, OVS_OPT_MIXED_OUTER = 5, 6, 7, 8
OVS_SPMV_PRECOND = 1
(OVS_BLK_K11, OVS_BLK_G, OVS_BLK_D1, OVS_BLK_M, OVS_BLK_LS, OVS_BLK_LSU,
 OVS_BLK_ULS, OVS_BLK_PLS, OVS_BLK_TEM) = range(9)
FIELDS = ["xg", "dg", "dgold", "ug", "ugold", "acg", "acgold", "ugm", "ugmold",
          "acgm", "acgmold", "pg", "phig", "phigold", "rphig", "rphigold", "tg",
          "tgold", "rtg", "rtgold"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
FIELD_WIDTH = {n: (3 if i <= FIELD_ID["acgmold"] else 1) for n, i in FIELD_ID.items()}

# exported symbols (every entry point declared in include/ovs.h)
EXPORTS = [
    "ovs_params_genalpha", "ovs_version", "ovs_status_string", "ovs_gen_spar_struc",
    "ovs_create", "ovs_destroy", "ovs_synchronize", "ovs_get_stream", "ovs_upload_mesh",
    "ovs_build_pattern", "ovs_get_pattern", "ovs_get_slot_map", "ovs_set_params", "ovs_set_ibc", "ovs_set_field",
    "ovs_get_field", "ovs_assemble", "ovs_get_rhs", "ovs_set_rhs", "ovs_get_lhs_block",
    "ovs_set_lhs_block", "ovs_spmv", "ovs_gmres", "ovs_solve", "ovs_round_matrix", "ovs_newton_update", "ovs_set_solution", "ovs_predictor", "ovs_commit_old",
    "ovs_residual_norms", "ovs_profile", "ovs_launch_count", "ovs_last_device_ms",
    "ovs_host_alloc", "ovs_host_free", "ovs_residual_vjp", "ovs_gmres_transposed", "ovs_quench_newton",
    "ovs_quench_time_steps", "ovs_stage_fields", "ovs_commit_staged", "ovs_get_rhs_async", "ovs_sync_copies",
    "ovs_build_precond", "ovs_spmv_device", "ovs_spmv_device_rows", "ovs_precond_device", "ovs_measure_fp32_peak", "ovs_measure_fp64_peak", "ovs_set_option", "ovs_set_faces", "ovs_check_faces", "ovs_set_bc_spec", "ovs_check_bc_spec", "ovs_assemble_async", "ovs_assemble_wait", "ovs_apply_bcs", "ovs_get_ibc",
    "ovs_gmres_tem_noalloc",
]


class OvsDims(C.Structure):
    _fields_ = [("nnode", C.c_int), ("nelem", C.c_int), ("nshl", C.c_int), ("device", C.c_int)]


PARAM_DOUBLES = ["almi", "alfi", "gami", "beti", "delt", "rhow", "rhoa", "rhos", "muw", "mua",
                 "mus", "cpw", "cpa", "cps", "kappaw", "kappaa", "kappas", "ts", "lh", "c_evap",
                 "c_cond", "c_dmdot", "ns_kdc_w", "ns_kdc_a", "lsc_kdc", "tem_kdc", "tref"]


class OvsParams(C.Structure):
    _fields_ = ([(n, C.c_double) for n in PARAM_DOUBLES] +
                [("gravvec", C.c_double * 3), ("fluid_elm_id", C.c_int),
                 ("subdomain_flag", C.c_int), ("elm_id_set", C.c_int * 2)])


class OvsBcSpec(C.Structure):
    _fields_ = [("nbound", C.c_int), ("ntype", C.c_int), ("face_id", C.POINTER(C.c_int)),
                ("bnode_ptr", C.POINTER(C.c_int)), ("bnodes", C.POINTER(C.c_int)),
                ("node_id", C.POINTER(C.c_int)), ("bcug_type", C.POINTER(C.c_int)),
                ("bcug_valu", C.POINTER(C.c_double)), ("bcphig_type", C.POINTER(C.c_int)),
                ("bcphig_valu", C.POINTER(C.c_double)), ("bctg_type", C.POINTER(C.c_int)),
                ("bctg_valu", C.POINTER(C.c_double))]


class OvsNewtonOpts(C.Structure):
    _fields_ = [("mode", C.c_int), ("newton_max", C.c_int), ("solve_tem", C.c_int), ("kspace", C.c_int),
                ("kspace_min", C.c_int), ("max_cycles", C.c_int), ("tol_ns", C.c_double),
                ("tol_tem", C.c_double), ("utol", C.c_double * 4), ("atol", C.c_double * 4)]


class OvsNewtonInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("field_converged", C.c_int * 4),
                ("residual0", C.c_double * 4), ("residual", C.c_double * 4),
                ("krylov_iterations_ns", C.c_int), ("krylov_iterations_tem", C.c_int), ("seconds", C.c_double)]


class OvsGmresInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("breakdown", C.c_int),
                ("reserved", C.c_int), ("res0", C.c_double), ("ercheck", C.c_double)]


class OvsSolveInfo(C.Structure):
    _fields_ = [("cycles", C.c_int), ("iterations", C.c_int), ("converged", C.c_int),
                ("reserved", C.c_int), ("rel_residual", C.c_double), ("seconds", C.c_double)]


_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the CUDA library (raises if it is absent: there is no CPU path)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise OSError(f"{p} not found: build it with `python -m oversetdevfort_b200.build`")
    lib = C.CDLL(str(p))
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    sig = {
        "ovs_params_genalpha": ([C.c_double, C.POINTER(OvsParams)], C.c_int),
        "ovs_version": ([], C.c_int),
        "ovs_status_string": ([C.c_int], C.c_char_p),
        "ovs_gen_spar_struc": ([C.c_int, C.c_int, C.c_int, ip, ip, ip, ip], C.c_int),
        "ovs_create": ([C.POINTER(vp), C.POINTER(OvsDims)], C.c_int),
        "ovs_destroy": ([vp], C.c_int),
        "ovs_synchronize": ([vp], C.c_int),
        "ovs_get_stream": ([vp, C.POINTER(vp)], C.c_int),
        "ovs_upload_mesh": ([vp, dp, ip, ip], C.c_int),
        "ovs_build_pattern": ([vp, ip], C.c_int),
        "ovs_get_pattern": ([vp, ip, ip], C.c_int),
        "ovs_get_slot_map": ([vp, ip], C.c_int),
        "ovs_set_params": ([vp, C.POINTER(OvsParams)], C.c_int),
        "ovs_set_ibc": ([vp, ip, C.c_int], C.c_int),
        "ovs_set_faces": ([vp, C.c_int, ip, ip, ip, dp, dp], C.c_int),
        "ovs_check_faces": ([C.c_int, C.c_int, ip, ip, ip, dp, dp], C.c_int),
        "ovs_set_option": ([vp, C.c_int, C.c_int], C.c_int),
        "ovs_stage_fields": ([vp, C.c_int, ip, C.POINTER(dp)], C.c_int),
        "ovs_commit_staged": ([vp], C.c_int),
        "ovs_get_rhs_async": ([vp, C.c_int, C.c_int, dp], C.c_int),
        "ovs_sync_copies": ([vp], C.c_int),
        "ovs_build_precond": ([vp, C.c_int, C.c_int], C.c_int),
        "ovs_spmv_device": ([vp, C.c_int, C.c_int, C.c_int, vp, vp], C.c_int),
        "ovs_precond_device": ([vp, C.c_int, C.c_int, vp, vp], C.c_int),
        "ovs_spmv_device_rows": ([vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int], C.c_int),
        "ovs_measure_fp32_peak": ([vp, dp], C.c_int),
        "ovs_measure_fp64_peak": ([vp, dp], C.c_int),
        "ovs_set_bc_spec": ([vp, C.POINTER(OvsBcSpec)], C.c_int),
        "ovs_check_bc_spec": ([C.POINTER(OvsBcSpec), C.c_int], C.c_int),
        "ovs_apply_bcs": ([vp, C.c_int], C.c_int),
        "ovs_get_ibc": ([vp, ip, C.c_int], C.c_int),
        "ovs_set_field": ([vp, C.c_int, dp], C.c_int),
        "ovs_get_field": ([vp, C.c_int, dp], C.c_int),
        "ovs_assemble": ([vp, C.c_int, C.c_int, C.c_int, dp], C.c_int),
        "ovs_assemble_async": ([vp, C.c_int, C.c_int, C.c_int], C.c_int),
        "ovs_assemble_wait": ([vp, dp], C.c_int),
        "ovs_get_rhs": ([vp, C.c_int, C.c_int, dp], C.c_int),
        "ovs_set_rhs": ([vp, C.c_int, C.c_int, dp], C.c_int),
        "ovs_get_lhs_block": ([vp, C.c_int, C.c_int, C.c_int, dp], C.c_int),
        "ovs_set_lhs_block": ([vp, C.c_int, C.c_int, C.c_int, dp], C.c_int),
        "ovs_spmv": ([vp, C.c_int, C.c_int, dp, dp], C.c_int),
        "ovs_gmres": ([vp, C.c_int, C.c_double, C.c_int, C.c_int, dp, C.POINTER(OvsGmresInfo)], C.c_int),
        "ovs_solve": ([vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, dp,
                       C.POINTER(OvsSolveInfo)], C.c_int),
        "ovs_round_matrix": ([vp, C.c_int], C.c_int),
        "ovs_newton_update": ([vp, C.c_int], C.c_int),
        "ovs_set_solution": ([vp, C.c_int, vp], C.c_int),
        "ovs_predictor": ([vp], C.c_int),
        "ovs_commit_old": ([vp, C.c_int], C.c_int),
        "ovs_residual_norms": ([vp, C.c_int, dp], C.c_int),
        "ovs_profile": ([vp, C.c_int, C.c_int, C.c_int, C.c_int, dp], C.c_int),
        "ovs_launch_count": ([vp, C.POINTER(C.c_longlong)], C.c_int),
        "ovs_last_device_ms": ([vp, dp], C.c_int),
        "ovs_host_alloc": ([C.POINTER(vp), C.c_size_t], C.c_int),
        "ovs_host_free": ([vp], C.c_int),
        "ovs_residual_vjp": ([vp, C.c_int, dp, dp], C.c_int),
        "ovs_quench_newton": ([vp, C.POINTER(OvsNewtonOpts), C.POINTER(OvsNewtonInfo)], C.c_int),
        "ovs_quench_time_steps": ([vp, C.c_int, C.c_int, C.POINTER(OvsNewtonOpts), C.c_int,
                                   C.POINTER(OvsNewtonInfo), C.POINTER(C.c_int)], C.c_int),
        "ovs_gmres_transposed": ([vp, C.c_int, dp, C.c_double, C.c_int, C.c_int, dp, C.POINTER(OvsGmresInfo)],
                                 C.c_int),
        "ovs_gmres_tem_noalloc": ([C.c_int, vp, vp, vp, vp, vp, C.c_double, C.c_int, C.c_int, vp,
                                   C.POINTER(OvsGmresInfo)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


class OvsError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.ovs_status_string(status).decode()
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def check(status: int, where: str) -> int:
    if status < 0:
        raise OvsError(status, where)
    return status
