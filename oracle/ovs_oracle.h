/*
 * ORACLE - TEST INFRASTRUCTURE ONLY.  Nothing in the product library links,
 * loads or calls this code; only tests/, the smoke check and the CPU
 * baseline leg of bench.py do, as the checker.
 *
 * A single-threaded FP64 CPU restatement, in C, of the reference's
 * (zexxzhao/OversetDevFort, Fortran) per-timestep hot path.  Every function
 * cites the reference file:line it follows and keeps the reference's loop
 * order, argument meaning and quirks.
 *
 * PARITY UNPINNED: the reference ships no tests, golden vectors or sample
 * outputs, and it cannot be compiled here (no Fortran compiler).  This
 * restatement is pinned instead by analytic known-answer tests (volumes,
 * partition of unity, closed-form pattern counts, Galerkin mass blocks,
 * dense-LU GMRES checks) in tests/test_oracle_kat.py.
 */
#ifndef OVS_ORACLE_H
#define OVS_ORACLE_H
#include "../include/ovs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* mesh + pattern (reference layout: column-major, 1-based indices) */
typedef struct orc_mesh {
  int nnode, nelem, nshl, nibc;
  const double* xg;   /* (N,3)     */
  const int* ien;     /* (E,nshl)  */
  const int* elm_id;  /* (E)       */
  const int* ibc;     /* (N,nibc)  */
  const int* col;     /* (N+1)     */
  const int* row;     /* (icnt)    */
  int icnt;
  int quench_literal; /* 1: literal signature-mismatch semantics (VOF frozen) */
  /* boundary faces in the reference's loop order (boundary b = 1..NBOUND,
   * then the faces of bound(b)); nface = 0: no face assembly */
  int nface;
  const int* f2e;      /* owning element, 1-based (bound(b)%F2E)   */
  const int* face_or;  /* face orientation 1..4 (bound(b)%FACE_OR) */
  const int* fflag;    /* OVS_FACE_WEAK | OVS_FACE_CONVH           */
  const double* hconv; /* heat transfer coefficient per face       */
  const double* tinf;  /* ambient temperature per face             */
} orc_mesh;

/* nodal state, module aAdjKeep (src/modules.f90:235-320) */
typedef struct orc_state {
  double *dg, *dgold, *ug, *ugold, *acg, *acgold, *ugm, *ugmold, *acgm,
      *acgmold;                                      /* (N,3) */
  double *pg, *phig, *phigold, *rphig, *rphigold, *tg, *tgold, *rtg,
      *rtgold;                                       /* (N)   */
} orc_state;

/* assembled system (src/alloc.f90:43-57) */
typedef struct orc_system {
  double *K11, *G, *D1, *M, *LS, *LSU, *ULS, *PLS, *TEM;  /* per slot */
  double *rhsu, *rhsp, *rhsls, *rhstem;                   /* (N,3),(N)... */
} orc_system;

int orc_gen_spar_struc(int nnode, int nelem, int nshl, const int* ien,
                       int* col, int* row, int* icnt);
int orc_sparse_mat_loc(const int* list, int n, int goal);
/* k(e,a,b) of FillSparseMat_3D for every element entry: (nelem,nshl,nshl)
 * column-major, 1-based global CSR slots */
void orc_slot_map(int nelem, int nshl, const int* ien, const int* col, const int* row, int* lmap);

/* full assembly drivers (alpha stage + zeroing + element loop) */
double orc_assemble_navsto(const orc_mesh* m, const ovs_params* p,
                           const orc_state* s, orc_system* sys,
                           int tensor_flag);
double orc_assemble_quenching(const orc_mesh* m, const ovs_params* p,
                              const orc_state* s, orc_system* sys,
                              int tensor_flag, int field_flag);
/* element-loop range versions for the bounded CPU baseline: the caller
 * passes the alpha-stage arrays in `a` (already blended) */
double orc_elmloop_ns(const orc_mesh* m, const ovs_params* p,
                      const orc_state* a, orc_system* sys, int tensor_flag,
                      int e0, int e1);
double orc_elmloop_nsvof(const orc_mesh* m, const ovs_params* p,
                         const orc_state* a, orc_system* sys, int tensor_flag,
                         int e0, int e1);
double orc_elmloop_tem(const orc_mesh* m, const ovs_params* p,
                       const orc_state* a, orc_system* sys, int tensor_flag,
                       int e0, int e1);
/* face assemblies on the alpha-stage arrays `a` (FaceAssembly_NS_weak then
 * FaceAssembly_NS_outflow, src/FaceAssembly_weak.f90:4-409; the convective
 * heat term on the temperature system) */
void orc_face_ns(const orc_mesh* m, const ovs_params* p, const orc_state* a,
                 orc_system* sys, int tensor_flag, int use_subdomain);
void orc_face_convh(const orc_mesh* m, const ovs_params* p, const orc_state* a,
                    orc_system* sys, int tensor_flag);
/* setBCs_NSVOF (which & 1) and setBCs_Tem (which & 2), src/setBCs.f90:
 * 172-278, on the state and on IBC (nnode, nibc) column-major */
void orc_set_bcs(int nnode, int nibc, int* ibc, const ovs_params* p,
                 orc_state* s, const ovs_bc_spec* sp, int which);
void orc_alpha_stage(int nnode, const ovs_params* p, const orc_state* s,
                     orc_state* a);

void orc_sparse_prod_up_3d(int nnode, const int* col, const int* row,
                           const orc_system* sys, const double* xu,
                           const double* xp, double* yu, double* yp);
void orc_sparse_prod_ns_conv(int nnode, const int* col, const int* row,
                             const orc_system* sys, const double* xu,
                             const double* xp, const double* xls, double* yu,
                             double* yp, double* yls);
void orc_sparse_prod_ls(int nnode, const int* col, const int* row,
                        const double* lhs, const double* x, double* y);

int orc_gmres_up(int nnode, const int* col, const int* row,
                 const orc_system* sys, double tol, int kspace,
                 int kspace_min, double* solu, double* solp, int* iters,
                 double* ercheck_out, double* res0_out);
int orc_gmres_ns_conv(int nnode, const int* col, const int* row,
                      const orc_system* sys, double tol, int kspace,
                      int kspace_min, double* solu, double* solp,
                      double* solls, int* iters, double* ercheck_out,
                      double* res0_out);
int orc_gmres_tem(int nnode, const int* col, const int* row,
                  const double* lhs, const double* rhs, double tol,
                  int kspace, int kspace_min, double* sol, int* iters,
                  double* ercheck_out, double* res0_out);

void orc_newton_update(int nnode, int system, const ovs_params* p,
                       orc_state* s, const double* sol);
void orc_calculate_residual(int nnode, const orc_system* sys, double r[4]);
/* test hook: eval_shape_fem at point igp of the element's rule */
double orc_eval_shape(int nshl, int igp, const double* xl, const double* dl, double* shl,
                      double* shg, double* gij, double* gw_out);

#ifdef __cplusplus
}
#endif
#endif
