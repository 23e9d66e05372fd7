/*
 * ovs.h - C ABI of the B200 (sm_100a) implementation of the OversetDevFort
 * per-timestep hot path: finite-element assembly of the VMS Navier-Stokes,
 * VOF and temperature equations into the node-block CSR system, and the
 * diagonally preconditioned GMRES solve of that system.
 *
 * Conventions (identical to the Fortran reference so that its arrays can be
 * passed straight through):
 *   - every array is column-major, "(N,3)" means three contiguous length-N
 *     columns; element connectivity IEN(E,nshl) is 1-based;
 *   - the CSR pattern uses the reference names: col(N+1) is the ROW POINTER,
 *     row(icnt) holds the COLUMN indices, both 1-based, rows sorted ascending
 *     (src/genSparStruc.f90:27-45);
 *   - block values of slot k are stored the reference way: LHSK11(9,icnt)
 *     with index (i-1)*3+j = (row component i, column component j),
 *     LHSG(3,icnt), LHSD1(3,icnt), LHSM(icnt), LHSLS(icnt), LHSLSU(3,icnt),
 *     LHSULS(3,icnt), LHSPLS(icnt), LHSTem(icnt) (src/alloc.f90:47-57).
 *
 * Every entry point returns an int status (OVS_OK = 0, negative = error,
 * positive = warning, results valid).  All calls on one context are
 * synchronous at return and must not be made concurrently from several host
 * threads.  Device state stays resident in the context between calls.
 */
#ifndef OVS_H
#define OVS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  OVS_OK = 0,
  OVS_WARN_NEG_DETJ = 1,      /* some element had DetJ <= 0 (the reference
                                 prints a warning and carries on:
                                 src/eval_shape_FEM.f90:54-60) */
  OVS_ERR_ARG = -1,           /* bad argument / size */
  OVS_ERR_CUDA = -2,          /* CUDA runtime error */
  OVS_ERR_NOMEM = -3,         /* device allocation failed */
  OVS_ERR_STATE = -4,         /* call order (e.g. assemble before pattern) */
  OVS_ERR_NONFINITE = -5,     /* NaN/Inf in an assembled residual */
  OVS_ERR_PATTERN = -6,       /* a node's CSR row would exceed 128 entries
                                 (the reference stops at 27*nshl: 108 for
                                 tets, 216 for hexes; src/genSparStruc.f90:93) */
  OVS_ERR_NODEVICE = -7,      /* no CUDA device */
  OVS_ERR_TIMEOUT = -8        /* a bounded host wait on the device expired */
};

/* ------------------------------------------------------------- selectors */
/* Storage precisions of the assembled systems (and of an assembly pass).
 * OVS_MIXED is a solve mode only (ovs_solve, ovs_newton_opts.mode): the FP64
 * system solved with an FP32 inner Krylov method, see ovs_solve. */
enum { OVS_FP64 = 0, OVS_FP32 = 1, OVS_MIXED = 2 };

/* assembly kernels (the reference element routines they replace) */
enum {
  OVS_ASM_NS = 1,     /* IntElmAss_NS_overset, src/assembleNavSto.f90:76-336 */
  OVS_ASM_NSVOF = 2,  /* IntElmAss_NSVOF_Quenching_STAB, src/solveQuenching.f90:122-573 */
  OVS_ASM_TEM = 3,    /* IntElmAss_Tem_Quenching_STAB, src/solveQuenching.f90:579-882 */
  OVS_ASM_QUENCH = 4  /* both quench passes, NS+VOF then T: assembleQuenching with ASSEMBLE_FIELD_NS, _VOF
                         and _TEM (src/solveQuenching.f90:4-117), one status (cfl: the larger of the two
                         passes', which evaluate the same advection speed) */
};

/* linear systems (dofs per node) */
enum {
  OVS_SYS_NS = 1,     /* u,v,w,p   : SparseGMRES_up / SparseProdUP_3D         */
  OVS_SYS_NSVOF = 2,  /* u,v,w,p,phi: SparseGMRES_ns_conv / SparseProd_NS_conv */
  OVS_SYS_TEM = 3     /* T          : SparseGMRES_tem / SparseProd_LS           */
};

/* tensor flags, same values as commonpars (src/modules.f90:218-228) */
enum { OVS_TENSOR_VEC = 2, OVS_TENSOR_MAT = 4 };

/* matrix blocks for ovs_get_lhs_block / ovs_set_lhs_block */
enum {
  OVS_BLK_K11 = 0,  /* (9,icnt) */
  OVS_BLK_G = 1,    /* (3,icnt) */
  OVS_BLK_D1 = 2,   /* (3,icnt) */
  OVS_BLK_M = 3,    /* (icnt)   */
  OVS_BLK_LS = 4,   /* (icnt)   */
  OVS_BLK_LSU = 5,  /* (3,icnt) row phi, column u_i   */
  OVS_BLK_ULS = 6,  /* (3,icnt) row u_i, column phi   */
  OVS_BLK_PLS = 7,  /* (icnt)   row p,   column phi   */
  OVS_BLK_TEM = 8   /* (icnt)   */
};

/* nodal state arrays (module aAdjKeep, src/modules.f90:235-320) */
enum {
  OVS_F_XG = 0,                     /* (N,3) reference coordinates   */
  OVS_F_DG, OVS_F_DGOLD,            /* (N,3) displacement            */
  OVS_F_UG, OVS_F_UGOLD,            /* (N,3) velocity                */
  OVS_F_ACG, OVS_F_ACGOLD,          /* (N,3) acceleration            */
  OVS_F_UGM, OVS_F_UGMOLD,          /* (N,3) mesh velocity           */
  OVS_F_ACGM, OVS_F_ACGMOLD,        /* (N,3) mesh acceleration       */
  OVS_F_PG,                         /* (N)   pressure                */
  OVS_F_PHIG, OVS_F_PHIGOLD,        /* (N)   VOF                     */
  OVS_F_RPHIG, OVS_F_RPHIGOLD,      /* (N)   VOF rate                */
  OVS_F_TG, OVS_F_TGOLD,            /* (N)   temperature             */
  OVS_F_RTG, OVS_F_RTGOLD,          /* (N)   temperature rate        */
  OVS_F_COUNT
};

/* per-context options (ovs_set_option) */
enum {
  OVS_OPT_HEX_TC = 1,          /* 1: FP32 NS+VOF hexahedra take the tcgen05 element-matrix pass (3xTF32);
                                  0 (default, the faster one measured; env OVS_HEX_TC=1 sets 1): the
                                  CUDA-core row expansion */
  OVS_OPT_ARNOLDI_FUSED = 2,   /* 1: one-launch Arnoldi variant (default 0; env OVS_ARNOLDI_FUSED=1) */
  OVS_OPT_ROWS_STAGED = 3,     /* chunked tet row pass (OVS_OPT_ROWS_GATHER = 0), NS and NS+VOF kernels: 1
                                  (default) stages each chunk's element summaries in shared memory with
                                  asynchronous copies; 0 (env OVS_ROWS_STAGED=0) reads them from global memory
                                  lane by lane */
  OVS_OPT_ELEM_SMEM = 4,       /* FP64 tet element pass: 0 (env OVS_ELEM_SMEM=0) holds the node records in
                                  registers, 1 (env OVS_ELEM_SMEM=1) in shared memory; -1 (default) shared
                                  memory for NS+VOF and registers for NS and T, the faster of the two
                                  measured for each */
  OVS_OPT_ROWS_GATHER = 5,     /* tet row pass without tiles (OVS_OPT_ROWS_TILED = 0): 1 (default) every lane
                                  gathers whole blocks of the row by the contribution lists built with the
                                  pattern, reading the summaries from global memory; 0 (env
                                  OVS_ROWS_GATHER=0) the chunked pass, element blocks reduced through shared
                                  memory */
  OVS_OPT_ROWS_TILED = 6,      /* tet row pass: 1 (env OVS_ROWS_TILED=1) one CTA per tile of rows, the tile's
                                  element summaries staged in shared memory by bulk copies, then gathered as
                                  above; 0 (default, the faster one measured) the untiled passes */
  OVS_OPT_TILE_ELEMS = 7,      /* element budget of a row tile (default 96, env OVS_TILE_ELEMS; 4..4000);
                                  rows with more elements take the untiled gather pass */
  OVS_OPT_MIXED_OUTER = 8      /* OVS_MIXED solves: m > 0 (default 30, env OVS_MIXED_OUTER; up to 200) a
                                  flexible GMRES(m) outer in FP64 whose directions are preconditioned by one
                                  FP32 GMRES cycle each; 0 the restarted refinement (one FP32 cycle on the
                                  true FP64 residual per step) */
};

/* boundary-face flags (ovs_set_faces) */
enum {
  OVS_FACE_WEAK = 1,   /* face of a boundary with BCugType(b,d) == 2: the weak Dirichlet
                          (Nitsche) and outflow face terms, src/FaceAssembly_weak.f90 */
  OVS_FACE_CONVH = 2   /* convective heat flux h (T - T_inf) on the temperature system */
};

/* ---------------------------------------------------------------- types */
typedef struct ovs_ctx ovs_ctx;

typedef struct ovs_dims {
  int nnode;   /* NNODE */
  int nelem;   /* NELEM */
  int nshl;    /* nodes per element: 4 (linear tet) or 8 (trilinear hex) */
  int device;  /* CUDA device ordinal, or -1 for the calling thread's current one */
} ovs_dims;

/* Scalars of module commonvars the element routines read
 * (src/modules.f90:325-455, src/param.f90:205-490). */
typedef struct ovs_params {
  double almi, alfi, gami, beti;   /* generalized-alpha (src/param.f90:469-480) */
  double delt;                     /* time step Delt                        */
  double rhow, rhoa, rhos;         /* density: liquid (phi=0), gas (phi=1), solid */
  double muw, mua, mus;            /* viscosity                               */
  double cpw, cpa, cps;            /* heat capacity                           */
  double kappaw, kappaa, kappas;   /* conductivity                            */
  double ts;                       /* saturation temperature Ts               */
  double lh;                       /* latent heat Lh                          */
  double c_evap, c_cond, c_dmdot;  /* phase-change model constants            */
  double ns_kdc_w, ns_kdc_a;       /* NS discontinuity capturing              */
  double lsc_kdc, tem_kdc, tref;   /* VOF / temperature discontinuity capturing */
  double gravvec[3];               /* body force per unit mass (0,0,-9.81)    */
  int fluid_elm_id;                /* ELM_ID of fluid elements (102)          */
  int subdomain_flag;              /* assembleNavSto subdomain bit flags       */
  int elm_id_set[2];               /* ELM_ID_SET(1:2)                          */
} ovs_params;

typedef struct ovs_gmres_info {
  int iterations;      /* iKs on exit                                   */
  int converged;       /* |e(iKs+1)| <= tol*|P^-1 b| and iKs >= kspace_min */
  int breakdown;       /* H(k+1,k) == 0 met (exact solution reached)     */
  int reserved;
  double res0;         /* |P^-1 b| (unorm at entry)                      */
  double ercheck;      /* |e(iKs+1)| on exit                             */
} ovs_gmres_info;

typedef struct ovs_solve_info {
  int cycles;          /* outer refinement / restart cycles              */
  int iterations;      /* total inner Krylov iterations                  */
  int converged;       /* true relative residual <= rtol                  */
  int reserved;
  double rel_residual; /* ||b - A x||_2 / ||b||_2 in FP64 on exit        */
  double seconds;      /* device time of the solve (CUDA events)          */
} ovs_solve_info;

/* ------------------------------------------------------- generalized-alpha */
/* almi, alfi, gami, beti from rho_inf exactly as src/param.f90:469-480
 * (backward Euler when rho_inf is outside [0,1]). */
int ovs_params_genalpha(double rhoinf, ovs_params* p);

/* ------------------------------------------------------------ stateless */
int ovs_version(void);
const char* ovs_status_string(int status);

/* genSparStruc drop-in (src/genSparStruc.f90:4-105): builds the sorted,
 * unique node-adjacency CSR of IEN on the GPU.  On entry *icnt is the
 * capacity of `row`; on exit it is the number of entries.  Pass row=NULL to
 * query icnt only.  col has N+1 entries.  All indices 1-based. */
int ovs_gen_spar_struc(int nnode, int nelem, int nshl, const int* ien,
                       int* col, int* row, int* icnt);

/* -------------------------------------------------------------- context */
int ovs_create(ovs_ctx** out, const ovs_dims* dims);
int ovs_destroy(ovs_ctx* ctx);
int ovs_synchronize(ovs_ctx* ctx);
/* the cudaStream_t every call of this context is issued on */
int ovs_get_stream(ovs_ctx* ctx, void** stream);

/* mesh: xg(N,3), IEN(E,nshl) 1-based, ELM_ID(E) (may be NULL: all 102) */
int ovs_upload_mesh(ovs_ctx* ctx, const double* xg, const int* ien,
                    const int* elm_id);
/* genSparStruc on the resident mesh; *icnt receives the entry count */
int ovs_build_pattern(ovs_ctx* ctx, int* icnt);
/* copy the pattern out (1-based, reference layout), col(N+1), row(icnt) */
int ovs_get_pattern(ovs_ctx* ctx, int* col, int* row);
/* The element-slot -> CSR-slot map the assembly scatters through: lmap is
 * (NELEM, nshl, nshl) column-major, lmap(e,a,b) = the 1-based slot k that
 * FillSparseMat_3D adds element entry (a, b) of element e to,
 * k = SparseMatLoc_3D(row(c:c+n-1), n, IEN(e,b)) + c - 1 with
 * c = col(IEN(e,a)), n = col(IEN(e,a)+1) - c (src/FillSparseMat.f90:4-28,
 * 47-57).  Computed once by ovs_build_pattern. */
int ovs_get_slot_map(ovs_ctx* ctx, int* lmap);

int ovs_set_params(ovs_ctx* ctx, const ovs_params* p);
/* IBC(N,nibc) column-major, entries 0/1 (src/setBCs.f90:183-187: columns
 * 1-3 velocity, 4 pressure, 5 VOF, 6 temperature) */
int ovs_set_ibc(ovs_ctx* ctx, const int* ibc, int nibc);
/* Sets a per-context option (OVS_OPT_*); OVS_ERR_ARG for an unknown one. */
int ovs_set_option(ovs_ctx* ctx, int option, int value);

/* Boundary faces for the face assemblies, in the reference's loop order
 * (boundary b = 1..NBOUND, then the faces of bound(b)): f2e = bound(b)%F2E
 * (1-based owning element), face_or = bound(b)%FACE_OR (1..4), flags
 * OVS_FACE_*; hconv / tinf (may be NULL without OVS_FACE_CONVH) give h and
 * T_inf per face.  Every later ovs_assemble adds, after the element pass:
 *   OVS_ASM_NS:    FaceAssembly_NS_weak, then FaceAssembly_NS_outflow, on the
 *                  OVS_FACE_WEAK faces (src/FaceAssembly_weak.f90:4-409,
 *                  called at src/assembleNavSto.f90:55-61);
 *   OVS_ASM_NSVOF: the same two routines on the velocity/pressure blocks, every
 *                  element a target (the quench driver's face calls,
 *                  src/solveQuenching.f90:75-83, name an undefined routine and
 *                  pass 11 arguments to the 8-argument outflow routine);
 *   OVS_ASM_TEM:   the convective heat flux h (T - T_inf) on OVS_FACE_CONVH
 *                  faces (FaceAssembly_ConvectiveH, called at
 *                  src/solveQuenching.f90:92, is not defined by the reference).
 * Each face's arrays pass through BCLhs_3D / BCLhs_tem before the scatter, as
 * in the reference.  Linear tets only (OVS_ERR_ARG otherwise); nface = 0
 * clears the set.  ovs_residual_vjp returns OVS_ERR_STATE while a face set is
 * active (face terms are not differentiated). */
int ovs_set_faces(ovs_ctx* ctx, int nface, const int* f2e, const int* face_or,
                  const int* flags, const double* hconv, const double* tinf);
/* The checks ovs_set_faces makes, without a context or a device, for a tet
 * mesh of nelem elements: OVS_OK, or OVS_ERR_ARG for an owning element
 * outside 1..nelem, a FACE_OR outside 1..4, an unknown flag bit, or a
 * convective face without the hconv / tinf tables. */
int ovs_check_faces(int nelem, int nface, const int* f2e, const int* face_or, const int* flags,
                    const double* hconv, const double* tinf);

/* Boundary data of setBCs_NSVOF / setBCs_Tem (src/setBCs.f90:172-278) as the
 * reference holds it: the node sets of the boundaries and the tables read by
 * src/param.f90:296-340.  setBCs reads the *Type tables by FACE_ID and the
 * *Valu tables by boundary number; both are kept. */
typedef struct ovs_bc_spec {
  int nbound;                 /* NBOUND                                          */
  int ntype;                  /* rows of the *Type tables (NBOUND in the reference) */
  const int* face_id;         /* bound(b)%FACE_ID, nbound values in 1..ntype     */
  const int* bnode_ptr;       /* nbound + 1 offsets into bnodes, bnode_ptr[0] = 0 */
  const int* bnodes;          /* bound(b)%BNODES concatenated, 1-based node ids  */
  const int* node_id;         /* NodeID (N values), or NULL when no node is 101  */
  const int* bcug_type;       /* BCugType, column-major (ntype, 3)              */
  const double* bcug_valu;    /* BCugValu, column-major (nbound, 3)             */
  const int* bcphig_type;     /* BCphigType (ntype)                             */
  const double* bcphig_valu;  /* BCphigValu (nbound)                            */
  const int* bctg_type;       /* BCTgType (ntype)                               */
  const double* bctg_valu;    /* BCTgValu (nbound)                              */
} ovs_bc_spec;

/* Registers the boundary data (NULL clears it).  While it is set,
 * ovs_quench_newton applies setBCs_NSVOF and setBCs_Tem where the
 * reference's Newton routine calls them (src/solveFlow.f90:35-36 before the
 * first residual, :58-60 at the top of every Newton iteration). */
int ovs_set_bc_spec(ovs_ctx* ctx, const ovs_bc_spec* spec);
/* The checks ovs_set_bc_spec makes, without a context or a device, for a
 * mesh of nnode nodes: OVS_OK, or OVS_ERR_ARG for a FACE_ID outside
 * 1..ntype, offsets that do not ascend from 0, a node id outside 1..nnode,
 * a node listed twice in one boundary, or a missing table. */
int ovs_check_bc_spec(const ovs_bc_spec* spec, int nnode);

/* which & 1: setBCs_NSVOF (IBC = 0; NodeID 101 -> IBC(1:5) = 1; Dirichlet
 * velocity / VOF values with acg, rphig = ((v - vold) Dtgl + (gami - 1)
 * rate_old) / gami); which & 2: setBCs_Tem (IBC(:,6) = 0; Dirichlet T, rTg).
 * On the device state and IBC of the context. */
int ovs_apply_bcs(ovs_ctx* ctx, int which);

/* The context's IBC as an (N, nibc) column-major array of 0/1. */
int ovs_get_ibc(ovs_ctx* ctx, int* ibc, int nibc);
int ovs_set_field(ovs_ctx* ctx, int field, const double* host);
int ovs_get_field(ovs_ctx* ctx, int field, double* host);

/* Assembly.  Replaces assembleNavSto (kernel OVS_ASM_NS,
 * src/assembleNavSto.f90:4-72) and assembleQuenching with
 * ASSEMBLE_FIELD_NS+VOF (OVS_ASM_NSVOF), ASSEMBLE_FIELD_TEM (OVS_ASM_TEM) or
 * all three (OVS_ASM_QUENCH) (src/solveQuenching.f90:4-117): alpha-stage
 * blend, zeroing, element loop, element Dirichlet BCs and the scatter into
 * CSR/RHS, in `precision`.  cfl (may be NULL) receives the largest element
 * CFL number. */
int ovs_assemble(ovs_ctx* ctx, int kernel, int tensor_flag, int precision,
                 double* cfl);
/* ovs_assemble without the wait: the pass is queued on the context stream
 * and the call returns; its status and CFL number are read by
 * ovs_assemble_wait, which waits for every pass queued since the last wait
 * and returns the status ovs_assemble would have (the first error in queue
 * order, else OVS_WARN_NEG_DETJ if any pass warned) and the largest CFL.
 * At most 16 passes between waits (OVS_ERR_STATE beyond).  Lets a caller
 * queue the next step's copies (ovs_stage_fields) while a pass runs. */
int ovs_assemble_async(ovs_ctx* ctx, int kernel, int tensor_flag, int precision);
int ovs_assemble_wait(ovs_ctx* ctx, double* cfl);

/* RHS of `system` in reference layout: NS -> RHSGu(N,3),RHSGp(N);
 * NSVOF -> additionally RHSGls(N); TEM -> RHSGtem(N).  Concatenated. */
int ovs_get_rhs(ovs_ctx* ctx, int system, int precision, double* rhs);
int ovs_set_rhs(ovs_ctx* ctx, int system, int precision, const double* rhs);
/* one matrix block in reference layout (see OVS_BLK_*) */
int ovs_get_lhs_block(ovs_ctx* ctx, int system, int precision, int block,
                      double* out);
int ovs_set_lhs_block(ovs_ctx* ctx, int system, int precision, int block,
                      const double* in);

/* y = A x without preconditioning (SparseProdUP_3D / SparseProd_NS_conv /
 * SparseProd_LS, src/SparseProd.f90:4-60,128-242) on host vectors in
 * reference layout. */
int ovs_spmv(ovs_ctx* ctx, int system, int precision, const double* x,
             double* y);

/* Device-vector building blocks of a distributed Krylov solve over
 * owner-computes partitions (the reference's SparseGMRES_* with their commu
 * and MPI_ALLREDUCE steps, src/SparseGMRES_NS_conv.f:65-76,169-176,210-251,
 * 287-308,391-395): dx, dy are FP64 device vectors on this context's device
 * in the reference layout (field-major, N x nf); each call synchronizes the
 * context's stream before returning.
 * ovs_build_precond: the block-diagonal preconditioner of SparseGMRES_*
 * (3x3 velocity blocks, 1/M, 1/LS; 1/M for the temperature system) from the
 * assembled `system`/`precision`, rebuilt on every call.
 * ovs_spmv_device: y = A x, or y = P^-1 A x with OVS_SPMV_PRECOND.
 * ovs_precond_device: y = P^-1 x. */
#define OVS_SPMV_PRECOND 1
int ovs_build_precond(ovs_ctx* ctx, int system, int precision);
int ovs_spmv_device(ovs_ctx* ctx, int system, int precision, int flags,
                    const double* dx, double* dy);
int ovs_precond_device(ovs_ctx* ctx, int system, int precision,
                       const double* dx, double* dy);
/* ovs_spmv_device_rows: ovs_spmv_device on the rows drows[0..nrows) only
 * (drows: a device int array of 0-based local rows, each in [0, N); an
 * index outside that range is skipped); the other rows of dy are left as
 * they are, and every listed row equals the full product's bit for bit.
 * A partition computes the rows that read no ghost entry of dx while the
 * halo exchange is in flight, then the others (src/SparseGMRES_NS_conv.f
 * :169-176 exchanges before the whole product).  nrows = 0 does nothing. */
int ovs_spmv_device_rows(ovs_ctx* ctx, int system, int precision, int flags,
                         const double* dx, double* dy, const int* drows, int nrows);

/* Streaming time steps (the Newton drivers push the state and read the
 * residual back every iteration, src/solveFlow.f90:39-40, 71-72, 116-117,
 * 148-149): copies that overlap the assembly instead of preceding it.
 * ovs_stage_fields: copies host fields (ids OVS_F_*, reference layout;
 *   page-locked host memory lets the copies run asynchronously) into a second
 *   device buffer per field on an upload stream, after the work committed
 *   so far has stopped reading those buffers; returns at once; the host
 *   arrays must stay unchanged until, after the commit that consumes them, a
 *   call that waits for the compute stream (ovs_assemble, ovs_sync_copies)
 *   has returned.
 * ovs_commit_staged: work issued afterwards waits for the staged copies and
 *   reads the staged fields (the swap covers only the fields staged since the
 *   last commit); OVS_ERR_STATE when nothing is staged.
 * ovs_get_rhs_async: the right-hand side of `system` as FP64 into `host`
 *   through a download stream, after the work issued so far; `host` is valid
 *   after ovs_sync_copies.  Each system has its own read-back buffer: a
 *   read-back waits only for the previous read-back of the same system.
 * ovs_sync_copies: waits for both copy streams. */
int ovs_stage_fields(ovs_ctx* ctx, int nfields, const int* ids, const double* const* host);
int ovs_commit_staged(ovs_ctx* ctx);
int ovs_get_rhs_async(ovs_ctx* ctx, int system, int precision, double* host);
int ovs_sync_copies(ovs_ctx* ctx);

/* One GMRES cycle with the reference's exact semantics, in FP64 on the FP64
 * system: SparseGMRES_up (src/SparseGMRES_NS.f90:4-369),
 * SparseGMRES_ns_conv (src/SparseGMRES_NS_conv.f:1-406),
 * SparseGMRES_tem (src/SparseGMRES_tem.f90:1-256).  sol (host, reference
 * layout) is accumulated into: sol += sum_j y_j v_j. */
int ovs_gmres(ovs_ctx* ctx, int system, double tol, int kspace,
              int kspace_min, double* sol, ovs_gmres_info* info);

/* Solve A x = b to ||b - A x||_2 <= rtol ||b||_2 (true residual, FP64).
 * mode OVS_FP64: restarted FP64 GMRES(kspace) on the FP64 system.
 * mode OVS_MIXED: the FP64 system (needs an FP64 assembly of `system`).
 *   Default (OVS_OPT_MIXED_OUTER = m > 0): a flexible GMRES(m) outer in FP64
 *   arithmetic on the FP64 matrix, minimizing the block-Jacobi-preconditioned
 *   residual, each of whose directions is one GMRES(kspace) cycle on the FP32
 *   rounding of that matrix (FP32 values, preconditioner, SpMV and Krylov
 *   basis; FP64 Gram-Schmidt dots, Givens rotations and back-substitution);
 *   after m directions, or when the outer estimate is reached, the true
 *   residual b - A x is formed with the FP64 matrix and the outer restarts
 *   from it.  OVS_OPT_MIXED_OUTER = 0: iterative refinement, one FP32 cycle
 *   on the true FP64 residual per step.  max_cycles bounds the FP32 cycles.
 *   The rounding is written into the FP32 matrix of `system` (overwriting an
 *   FP32 assembly) inside the timed solve.  The solution converges to the
 *   FP64 system's, not to an FP32-assembled one.
 * mode OVS_FP32: the same scheme on the FP32-assembled system alone (matrix
 *   and right-hand side assembled in FP32; the refinement residual in FP64
 *   arithmetic on those FP32 values): it converges to the solution of the
 *   FP32-assembled system, which differs from the FP64 system's by the
 *   FP32 assembly's rounding times the condition number.
 * The solution stays on the device (ovs_newton_update applies it); sol
 * (host, may be NULL) receives a copy. */
int ovs_solve(ovs_ctx* ctx, int system, int mode, double rtol, int kspace,
              int max_cycles, double* sol, ovs_solve_info* info);

/* The FP32 matrix of `system` := the FP32 rounding of its FP64 matrix (needs
 * an FP64 assembly of `system`): the inner operator of the OVS_MIXED
 * refinement, for a solve driven from outside (the partitioned Newton loop);
 * ovs_solve(OVS_MIXED) does the same itself.  No reference counterpart (a
 * part of the mixed-precision extension). */
int ovs_round_matrix(ovs_ctx* ctx, int system);

/* Newton update with the last solution of `system` (src/solveFlow.f90:99-104,
 * 139-140; src/solveOverset.f90:76-78):
 *   NS/NSVOF: acg += du; ug += gami*Delt*du; pg += alfi*gami*Delt*dp;
 *   NSVOF:    rphig += dphi; phig += gami*Delt*dphi;
 *   TEM:      rTg += dT; Tg += gami*Delt*dT. */
int ovs_newton_update(ovs_ctx* ctx, int system);
/* The solution the next ovs_newton_update of `system` applies, from `sol`
 * (reference layout, N x nf FP64, in host memory or in this context's
 * device memory): for a solution computed outside the context, such as the
 * partitioned GMRES over several contexts, whose per-rank solutions the
 * reference applies as the same update after SparseGMRES_* returns
 * (src/solveFlow.f90:99-104, 139-140). */
int ovs_set_solution(ovs_ctx* ctx, int system, const double* sol);

/* calculate_residual (src/solveFlow.f90:169-187): sums of squares (no sqrt)
 * of RHSGu, RHSGp, RHSGls, RHSGtem of the given precision. */
int ovs_residual_norms(ovs_ctx* ctx, int precision, double r[4]);

/* The Newton loop of one quench time step, on the device:
 * solmultiphasethermofluid_stag (src/solveFlow.f90:4-164).  residual0 from a
 * vector assembly of all fields; then up to newton_max times: assemble the
 * NS+VOF system, solve, Newton update (acg, ug, pg, rphig, phig); if
 * solve_tem, the same for the temperature (rTg, Tg); assemble the vectors
 * of all fields and stop when every field passes check_convergence (:190-215:
 * residual < utol * residual0 or residual < atol, sums of squares as
 * calculate_residual).  mode OVS_FP64: FP64 assembly and the reference GMRES
 * cycle (tol, kspace, kspace_min, zero start); OVS_MIXED: FP64 assembly and
 * residuals, every solve by ovs_solve's OVS_MIXED refinement to relative
 * residual tol (max_cycles); OVS_FP32: FP32 assembly and residuals, every
 * solve by ovs_solve's OVS_FP32 refinement.
 * The predictor of driver.f90:83-85 and the BC producers stay with the
 * caller (set the fields and IBC before the call).  Only the 4 residual
 * norms per iteration travel to the host. */
typedef struct ovs_newton_opts {
  int mode, newton_max, solve_tem;
  int kspace, kspace_min, max_cycles;
  double tol_ns, tol_tem;
  double utol[4];    /* NS_NL_UTOL, NS_NL_PTOL, LSC_NL_TOL, TEM_NL_TOL */
  double atol[4];    /* NS_GMRES_atol (u, p), LSC_GMRES_atol, TEM_GMRES_atol */
} ovs_newton_opts;
typedef struct ovs_newton_info {
  int iterations, converged;
  int field_converged[4];
  double residual0[4], residual[4];
  int krylov_iterations_ns, krylov_iterations_tem;
  double seconds;    /* wall time of the call */
} ovs_newton_info;
int ovs_quench_newton(ovs_ctx* ctx, const ovs_newton_opts* opts, ovs_newton_info* info);
/* nsteps time steps of the reference driver (src/driver.f90:70-100) from
 * step first_step: predictor (ug = ugold, acg = (gami-1)/gami acgold), the
 * Newton loop above (a single Newton iteration while istep <= 1 and no
 * temperature solve at istep 0, src/solveFlow.f90:50-54,109), then the old
 * values the driver updates: ugold, acgold, dgold, ugmold, acgmold (the
 * driver leaves phigold, rphigold, Tgold, rTgold alone; update_vof_tem_old
 * = 1 copies them too).  last: the Newton info of the last step;
 * krylov_total: Krylov iterations over all steps (either may be NULL). */
int ovs_quench_time_steps(ovs_ctx* ctx, int first_step, int nsteps, const ovs_newton_opts* opts,
                          int update_vof_tem_old, ovs_newton_info* last, int* krylov_total);
/* The two halves of a driver step around the Newton loop, for a time loop
 * driven from outside (over partitions, say).  ovs_predictor is
 * src/driver.f90:83-85: ug = ugold, acg = (gami-1)/gami acgold
 * (OVS_ERR_STATE before ovs_set_params).  ovs_commit_old copies the old
 * values of :98-103: ugold, acgold, dgold, ugmold, acgmold, and with
 * update_vof_tem_old = 1 also phigold, rphigold, Tgold, rTgold.  The
 * pg = pgold / pgold = pg pair of the driver is the identity here. */
int ovs_predictor(ovs_ctx* ctx);
int ovs_commit_old(ovs_ctx* ctx, int update_vof_tem_old);

/* ----------------------------------------------------------- measurement
 * Hooks for benchmarking; they have no counterpart in the reference. */
/* Measured FP32 FMA throughput of the context's device in TFLOP/s (the
 * compute-side roofline denominator of the CUDA-core assembly kernels);
 * no reference counterpart (a measurement helper). */
int ovs_measure_fp32_peak(ovs_ctx* ctx, double* tflops);
/* The same for FP64 FMAs (the FP64 assembly kernels' compute-side
 * denominator); no reference counterpart (a measurement helper). */
int ovs_measure_fp64_peak(ovs_ctx* ctx, double* tflops);

enum { OVS_PROF_SPMV = 1, OVS_PROF_ASSEMBLE = 2, OVS_PROF_ARNOLDI = 3, OVS_PROF_ARNOLDI_FUSED = 4,
       OVS_PROF_ASSEMBLE_ELEMENTS = 5, OVS_PROF_ASSEMBLE_ROWS = 6 };
/* Average device time in ms (CUDA events on the context stream) of `reps`
 * back-to-back launches of one internal kernel on the resident data:
 *   OVS_PROF_SPMV      preconditioned SpMV y = P^-1 A x of `system`, matrix
 *                      and vectors in `precision` (needs the matrix);
 *   OVS_PROF_ASSEMBLE  the element and row passes of assembly kernel
 *                      `system` (an OVS_ASM_* value), MAT+VEC, on the node
 *                      records of the last ovs_assemble of that kernel and
 *                      precision; OVS_PROF_ASSEMBLE_ELEMENTS and
 *                      OVS_PROF_ASSEMBLE_ROWS time each pass alone;
 *   OVS_PROF_ARNOLDI   one Arnoldi iteration (preconditioned SpMV, k+1
 *                      Gram-Schmidt steps, normalization, Givens) at k = 25
 *                      of a 50-vector cycle, `system` in `precision`, as
 *                      the solvers run it (SpMV launch, then Gram-Schmidt
 *                      with the new vector held on chip);
 *   OVS_PROF_ARNOLDI_FUSED  the same iteration as one cooperative launch
 *                      (the variant selected by OVS_ARNOLDI_FUSED=1). */
int ovs_profile(ovs_ctx* ctx, int what, int system, int precision, int reps,
                double* avg_ms);
/* number of CUDA kernels this context has launched so far */
int ovs_launch_count(ovs_ctx* ctx, long long* n);
/* device time in ms (CUDA events) of the most recent ovs_assemble,
 * ovs_solve or ovs_gmres call of this context */
int ovs_last_device_ms(ovs_ctx* ctx, double* ms);
/* page-locked host buffers for fast transfers of state and results */
int ovs_host_alloc(void** p, size_t bytes);
int ovs_host_free(void* p);

/* ------------------------------------------------------------- adjoint
 * No counterpart in the reference (the reference has no adjoint): the
 * vector-Jacobian product of the assembled residual and a GMRES on the
 * transposed temperature matrix, for sensitivities of functionals. */
/* fields of the VJP result, N values each (field-major): node coordinates
 * xg (3), velocity ug (3), pressure pg, VOF phig, temperature Tg,
 * acceleration acg (3), VOF rate rphig, temperature rate rTg */
enum { OVS_VJP_XG = 0, OVS_VJP_UG = 3, OVS_VJP_PG = 6, OVS_VJP_PHIG = 7, OVS_VJP_TG = 8,
       OVS_VJP_ACG = 9, OVS_VJP_RPHIG = 12, OVS_VJP_RTG = 13, OVS_VJP_COUNT = 14 };
/* grad = (d RHS / d state)^T cot: RHS is the FP64 right-hand side that
 * ovs_assemble(kernel, OVS_TENSOR_VEC, OVS_FP64) would write for the current
 * state, parameters and IBC (kernel OVS_ASM_NSVOF: cot is N x 5 field-major
 * u1 u2 u3 p phi; OVS_ASM_TEM: N x 1), the state the nodal fields above.
 * Each element's Gauss-point quantities are recomputed in forward-mode
 * dual arithmetic per nodal input (nothing is stored between assembly and
 * adjoint); the node sums run in ascending element id, so the result is
 * deterministic.  grad is N x OVS_VJP_COUNT (fields the kernel does not
 * depend on come back 0).  Host arrays; synchronous. */
int ovs_residual_vjp(ovs_ctx* ctx, int kernel, const double* cot, double* grad);
/* Solve A^T x = rhs by GMRES (the reference-semantics cycle of ovs_gmres,
 * diagonal preconditioner, zero initial guess), A the assembled FP64
 * temperature matrix (system OVS_SYS_TEM), through a transposed copy of its
 * values on the same (symmetric) pattern.  rhs and sol: N values (host). */
int ovs_gmres_transposed(ovs_ctx* ctx, int system, const double* rhs, double tol, int kspace,
                         int kspace_min, double* sol, ovs_gmres_info* info);

/* ------------------------------------------------- allocation-free solve
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory at solve time - code inside a framework whose
 * memory pool owns the device memory, time-critical loops that cannot take
 * the device-wide synchronization of cudaMalloc/cudaFree, plug-in hosts that
 * only allow allocation at initialization.
 *
 * One GMRES cycle with SparseGMRES_tem semantics (as ovs_gmres with
 * OVS_SYS_TEM) on a caller-owned scalar CSR system in DEVICE memory:
 * rowptr[n+1], colidx[nnz] (0-based, rows sorted), vals[nnz], rhs[n] (FP64),
 * sol[n] accumulated into.  It calls no cudaMalloc/cudaFree and no allocating
 * library routine: all its temporaries live in one fixed __device__ array of
 * OVS_NOALLOC_SCRATCH_BYTES inside the library (held by every GPU that loads
 * the library until the process exits).  Limits: n <= OVS_NOALLOC_MAX_N and
 * kspace <= OVS_NOALLOC_MAX_KSPACE; larger requests return OVS_ERR_ARG.
 * Set-up on first use: the first call on a device looks up the device
 * address of that array (cudaGetSymbolAddress), and under CUDA's default
 * lazy module loading it is also the call that loads the library's module
 * onto the device, which is when the array itself is allocated.  Make that
 * first call (a warm-up call will do) before any stream capture and before
 * any phase in which nothing may be allocated; later calls allocate nothing.
 * All calls share the array, which keeps the last call's contents: serialize
 * them (one stream, one host thread at a time); calls that overlap on the
 * GPU (other streams, other host threads) race, their info read-back
 * included.  `stream` is a cudaStream_t (NULL: default stream); the call is
 * synchronous and returns after the solve.  Results follow SparseGMRES_tem's
 * arithmetic (reciprocal scaling of the Krylov vectors and rotations); a
 * zero Hessenberg column, where the reference's rotation is 0/0, ends the
 * cycle with the previous columns' solution and breakdown = 1. */
#define OVS_NOALLOC_MAX_N 16384
#define OVS_NOALLOC_MAX_KSPACE 40
#define OVS_NOALLOC_SCRATCH_BYTES 5537792
int ovs_gmres_tem_noalloc(int n, const int* rowptr, const int* colidx,
                          const double* vals, const double* rhs, double* sol,
                          double tol, int kspace, int kspace_min, void* stream,
                          ovs_gmres_info* info);

#ifdef __cplusplus
}
#endif
#endif /* OVS_H */
