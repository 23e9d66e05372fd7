/*
 * ORACLE - TEST INFRASTRUCTURE ONLY (see ovs_oracle.h).  PARITY UNPINNED:
 * no reference golden vectors exist and the Fortran reference cannot be
 * compiled here; pinned by analytic known-answer tests instead.
 *
 * Literal FP64 restatement of the reference hot path.  Array conventions
 * follow the reference: column-major, so X(i,d) of an (N,3) array is
 * x[i + N*d]; connectivity IEN(e,a) = ien[e + E*a] holds 1-based node ids.
 * Loop nests and the order of the += updates follow the cited Fortran.
 */
#include "ovs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NSD 3
#define NSHL_MAX 8
#define NGP_MAX 8

static inline size_t cm(size_t i, size_t n, size_t d) { return i + n * d; }

/* ----------------------------------------------------------------------
 * genSparStruc + Asadj: src/genSparStruc.f90:4-105.  Per node the list of
 * nodes sharing an element, in element-visit order (Asadj :65-103), then
 * col(1)=1, col(i+1)=col(i)+adjcnt(i) (:27-30) and each row sorted by
 * repeated minval/minloc (:33-45).
 * -------------------------------------------------------------------- */
int orc_gen_spar_struc(int nnode, int nelem, int nshl, const int* ien,
                       int* col, int* row, int* icnt) {
  const int maxlen = 27 * nshl;
  int* fill = (int*)calloc((size_t)nnode * maxlen, sizeof(int));
  int* adjcnt = (int*)calloc((size_t)nnode, sizeof(int));
  int* tmpr = (int*)malloc(sizeof(int) * (size_t)maxlen);
  if (!fill || !adjcnt || !tmpr) { free(fill); free(adjcnt); free(tmpr); return OVS_ERR_NOMEM; }
  int overflow = 0;
  for (int e = 0; e < nelem; ++e) {
    int ndlist[NSHL_MAX];
    for (int j = 0; j < nshl; ++j) ndlist[j] = ien[cm(e, nelem, j)];
    for (int j = 0; j < nshl; ++j) {
      int jnd = ndlist[j] - 1;
      int jl = adjcnt[jnd];
      for (int k = 0; k < nshl; ++k) {
        int knd = ndlist[k];
        int broke = 0;
        for (int l = 0; l < jl; ++l)
          if (fill[(size_t)jnd * maxlen + l] == knd) { broke = 1; break; }
        if (!broke) {
          if (jl >= maxlen) { overflow = 1; continue; }  /* "Stop the Music!!!" */
          fill[(size_t)jnd * maxlen + jl] = knd;
          ++jl;
        }
      }
      adjcnt[jnd] = jl;
    }
  }
  long total = 0;
  for (int i = 0; i < nnode; ++i) total += adjcnt[i];
  if (row != NULL && total > *icnt) { free(fill); free(adjcnt); free(tmpr); return OVS_ERR_ARG; }
  *icnt = (int)total;
  col[0] = 1;
  for (int i = 0; i < nnode; ++i) col[i + 1] = col[i] + adjcnt[i];
  if (row != NULL) {
    const int ibig = 10 * nnode;
    int k = 0;
    for (int i = 0; i < nnode; ++i) {
      int ncol = adjcnt[i];
      memcpy(tmpr, fill + (size_t)i * maxlen, sizeof(int) * (size_t)ncol);
      for (int j = 0; j < ncol; ++j) {
        int imin = tmpr[0], mloc = 0;  /* minval / first minloc */
        for (int t = 1; t < ncol; ++t)
          if (tmpr[t] < imin) { imin = tmpr[t]; mloc = t; }
        row[k++] = imin;
        tmpr[mloc] = ibig;
      }
    }
  }
  free(fill); free(adjcnt); free(tmpr);
  return overflow ? OVS_ERR_PATTERN : OVS_OK;
}

/* SparseMatLoc_3D: src/FillSparseMat.f90:4-28 - binary search returning the
 * LAST 1-based index idx with list(idx) <= goal (no not-found check). */
int orc_sparse_mat_loc(const int* list, int n, int goal) {
  int lo = 1, hi = n + 1;
  while (hi - lo > 1) {
    int mid = (hi + lo) / 2;
    if (list[mid - 1] > goal) hi = mid; else lo = mid;
  }
  return lo;
}

/* The global slots FillSparseMat_3D scatters element entry (a, b) to
 * (src/FillSparseMat.f90:47-57): i = IEN(e,a), c = col(i), n = col(i+1) - c,
 * locn = SparseMatLoc_3D(row(c:c+n-1), n, IEN(e,b)), k = locn + c - 1.
 * lmap is (nelem, nshl, nshl) column-major, 1-based k. */
void orc_slot_map(int nelem, int nshl, const int* ien, const int* col, const int* row, int* lmap) {
  for (int e = 0; e < nelem; ++e)
    for (int a = 0; a < nshl; ++a) {
      const int i = ien[cm(e, nelem, a)];
      const int c = col[i - 1], n = col[i] - c;
      for (int b = 0; b < nshl; ++b) {
        const int locn = orc_sparse_mat_loc(row + (c - 1), n, ien[cm(e, nelem, b)]);
        lmap[(size_t)e + (size_t)nelem * ((size_t)a + (size_t)nshl * b)] = locn + c - 1;
      }
    }
}

/* ----------------------------------------------------------------------
 * Quadrature: genGPandGWtetpri src/genGP_GW.f90:317-431 (tet 4-pt, hex 8-pt)
 * -------------------------------------------------------------------- */
static void gen_gp_gw(int ngp, double gp[][3], double* gw) {
  if (ngp == 4) {
    const double a = 0.5854101966249685, b = 0.1381966011250105;
    double pts[4][3] = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    for (int g = 0; g < 4; ++g) {
      for (int d = 0; d < 3; ++d) gp[g][d] = pts[g][d];
      gw[g] = 0.25 / 6.0;
    }
  } else if (ngp == 8) {
    const double q = 0.57735026918963;
    const double s[8][3] = {{-q, -q, -q}, {q, -q, -q}, {-q, q, -q}, {q, q, -q},
                            {-q, -q, q},  {q, -q, q},  {-q, q, q},  {q, q, q}};
    for (int g = 0; g < 8; ++g) {
      for (int d = 0; d < 3; ++d) gp[g][d] = s[g][d];
      gw[g] = 1.0;
    }
  } else {
    gp[0][0] = gp[0][1] = gp[0][2] = 0.25;
    gw[0] = 1.0 / 6.0;
  }
}

/* lintetshl src/eval_shape_FEM.f90:201-225 */
static void lintetshl(const double* gp, double* shl, double shgradl[][3]) {
  shl[0] = gp[0]; shl[1] = gp[1]; shl[2] = gp[2];
  shl[3] = 1.0 - gp[0] - gp[1] - gp[2];
  for (int a = 0; a < 4; ++a) for (int d = 0; d < 3; ++d) shgradl[a][d] = 0.0;
  shgradl[0][0] = 1.0; shgradl[1][1] = 1.0; shgradl[2][2] = 1.0;
  shgradl[3][0] = -1.0; shgradl[3][1] = -1.0; shgradl[3][2] = -1.0;
}

/* linhexshl src/eval_shape_FEM.f90:148-196 (not wired in the reference;
 * used by the hex extension) */
static void linhexshl(const double* gp, double* shl, double shgradl[][3]) {
  const double zi = gp[0], eta = gp[1], zeta = gp[2], e = 0.125;
  shl[0] = (zi - 1) * (eta + 1) * (zeta - 1) * e;
  shl[1] = -(zi + 1) * (eta + 1) * (zeta - 1) * e;
  shl[2] = (zi + 1) * (eta + 1) * (zeta + 1) * e;
  shl[3] = -(zi - 1) * (eta + 1) * (zeta + 1) * e;
  shl[4] = -(zi - 1) * (eta - 1) * (zeta - 1) * e;
  shl[5] = (zi + 1) * (eta - 1) * (zeta - 1) * e;
  shl[6] = -(zi + 1) * (eta - 1) * (zeta + 1) * e;
  shl[7] = (zi - 1) * (eta - 1) * (zeta + 1) * e;
  shgradl[0][0] = (eta + 1) * (zeta - 1) * e;  shgradl[1][0] = -(eta + 1) * (zeta - 1) * e;
  shgradl[2][0] = (eta + 1) * (zeta + 1) * e;  shgradl[3][0] = -(eta + 1) * (zeta + 1) * e;
  shgradl[4][0] = -(eta - 1) * (zeta - 1) * e; shgradl[5][0] = (eta - 1) * (zeta - 1) * e;
  shgradl[6][0] = -(eta - 1) * (zeta + 1) * e; shgradl[7][0] = (eta - 1) * (zeta + 1) * e;
  shgradl[0][1] = (zi - 1) * (zeta - 1) * e;   shgradl[1][1] = -(zi + 1) * (zeta - 1) * e;
  shgradl[2][1] = (zi + 1) * (zeta + 1) * e;   shgradl[3][1] = -(zi - 1) * (zeta + 1) * e;
  shgradl[4][1] = -(zi - 1) * (zeta - 1) * e;  shgradl[5][1] = (zi + 1) * (zeta - 1) * e;
  shgradl[6][1] = -(zi + 1) * (zeta + 1) * e;  shgradl[7][1] = (zi - 1) * (zeta + 1) * e;
  shgradl[0][2] = (zi - 1) * (eta + 1) * e;    shgradl[1][2] = -(zi + 1) * (eta + 1) * e;
  shgradl[2][2] = (zi + 1) * (eta + 1) * e;    shgradl[3][2] = -(zi - 1) * (eta + 1) * e;
  shgradl[4][2] = -(zi - 1) * (eta - 1) * e;   shgradl[5][2] = (zi + 1) * (eta - 1) * e;
  shgradl[6][2] = -(zi + 1) * (eta - 1) * e;   shgradl[7][2] = (zi - 1) * (eta - 1) * e;
}

/* get_inverse_3x3 src/eval_shape.f90:85-112 (A, Ainv indexed [row][col]) */
static double get_inverse_3x3(double A[3][3], double Ai[3][3]) {
  Ai[0][0] = A[1][1] * A[2][2] - A[2][1] * A[1][2];
  Ai[0][1] = A[2][1] * A[0][2] - A[0][1] * A[2][2];
  Ai[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  double tmp = 1.0 / (Ai[0][0] * A[0][0] + Ai[0][1] * A[1][0] + Ai[0][2] * A[2][0]);
  Ai[0][0] *= tmp; Ai[0][1] *= tmp; Ai[0][2] *= tmp;
  Ai[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * tmp;
  Ai[1][1] = (A[0][0] * A[2][2] - A[2][0] * A[0][2]) * tmp;
  Ai[1][2] = (A[1][0] * A[0][2] - A[0][0] * A[1][2]) * tmp;
  Ai[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * tmp;
  Ai[2][1] = (A[2][0] * A[0][1] - A[0][0] * A[2][1]) * tmp;
  Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * tmp;
  return 1.0 / tmp;
}

/* eval_shape_fem src/eval_shape_FEM.f90:4-61: basis, dx/dxi on the CURRENT
 * configuration x+d (:31-36), inverse, global gradients (:41-45) and the
 * metric G_ij = sum_k dxi_k/dx_i dxi_k/dx_j (:47-52).  Returns DetJ. */
static double eval_shape_fem_dx(int nshl, const double* gp, double xl[][3],
                                double dl[][3], double* shl, double shg[][3],
                                double Gij[3][3], double dxidx[3][3]) {
  double shgl[NSHL_MAX][3], dxdxi[3][3];
  if (nshl == 4) lintetshl(gp, shl, shgl); else linhexshl(gp, shl, shgl);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int a = 0; a < nshl; ++a) s += (xl[a][i] + dl[a][i]) * shgl[a][j];
      dxdxi[i][j] = s;
    }
  double detj = get_inverse_3x3(dxdxi, dxidx);
  for (int a = 0; a < nshl; ++a)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += shgl[a][k] * dxidx[k][j];
      shg[a][j] = s;
    }
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += dxidx[k][i] * dxidx[k][j];
      Gij[i][j] = s;
    }
  return detj;
}

static double eval_shape_fem(int nshl, const double* gp, double xl[][3],
                             double dl[][3], double* shl, double shg[][3],
                             double Gij[3][3]) {
  double dxidx[3][3];
  return eval_shape_fem_dx(nshl, gp, xl, dl, shl, shg, Gij, dxidx);
}

/* Test hook, no reference counterpart: point igp of the element's rule
 * (gen_gp_gw with NGAUSS = NSHL, src/input.f90:158) and eval_shape_fem
 * there, for nodal coordinates xl and displacements dl (node a at
 * [3a..3a+2]; dl may be NULL): N_a, grad N_a (shg[3a+i]), G_ij
 * (gij[3i+j]) and the weight; returns DetJ. */
double orc_eval_shape(int nshl, int igp, const double* xl, const double* dl, double* shl,
                      double* shg, double* gij, double* gw_out) {
  double gp[8][3], gw[8], x[NSHL_MAX][3], d[NSHL_MAX][3], sg[NSHL_MAX][3], G[3][3];
  if ((nshl != 4 && nshl != 8) || igp < 0 || igp >= nshl) return 0.0;
  gen_gp_gw(nshl, gp, gw);
  for (int a = 0; a < nshl; ++a)
    for (int k = 0; k < 3; ++k) {
      x[a][k] = xl[3 * a + k];
      d[a][k] = dl ? dl[3 * a + k] : 0.0;
    }
  const double detj = eval_shape_fem(nshl, gp[igp], x, d, shl, sg, G);
  for (int a = 0; a < nshl; ++a)
    for (int k = 0; k < 3; ++k) shg[3 * a + k] = sg[a][k];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) gij[3 * i + j] = G[i][j];
  *gw_out = gw[igp];
  return detj;
}

/* prop_interp src/e3int.f90:4-13 */
static double prop_interp(double a, double b, double phi) {
  double pc = fmax(0.0, fmin(1.0, phi));
  return a * (1.0 - pc) + b * pc;
}

static double uGu(const double* u, double G[3][3]) {
  double t = 0.0;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) t += u[i] * G[i][j] * u[j];
  return t;
}
static double GG(double G[3][3]) {
  double s = 0.0;
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) s += G[i][j] * G[i][j];
  return s;
}

/* e3STAB_3D src/e3STAB.f90:4-44 */
static void e3stab_3d(double G[3][3], double dt, const double* u, double rho,
                      double mu, double* tauM, double* tauP, double* tauC) {
  double taua = uGu(u, G), nu = mu / rho;
  double taud = nu * nu * 12.0 * GG(G), taut = 4.0 / (dt * dt);
  *tauM = 1.0 / (rho * sqrt(taut + taua + taud));
  *tauP = *tauM;
  *tauC = rho * sqrt(taua + taud) / (G[0][0] + G[1][1] + G[2][2]);
}

/* e3STAB_3D_NSVOF src/e3STAB.f90:292-333 */
static void e3stab_3d_nsvof(double G[3][3], double dt, const double* u,
                            double rho, double mu, double* tauM, double* tauP,
                            double* tauC, double* tauLS) {
  double taua = uGu(u, G), nu = mu / rho;
  double taud = nu * nu * 12.0 * GG(G), taut = 4.0 / (dt * dt);
  *tauM = 1.0 / (rho * sqrt(taut + taua + taud));
  *tauLS = 1.0 / sqrt(taut + taua);
  *tauP = *tauM;
  *tauC = rho * sqrt(taua + taud) / (G[0][0] + G[1][1] + G[2][2]);
}

/* e3STAB_3D_TEM src/e3STAB.f90:338-367 */
static double e3stab_3d_tem(double G[3][3], const double* u, double dt,
                            double rho, double cp, double hk) {
  double t = uGu(u, G) + 4.0 / (dt * dt);
  double k = hk / (rho * cp);
  t = t + k * k * 12.0 * GG(G);
  return 1.0 / (rho * cp * sqrt(t));
}

/* e3DC_beta2 src/e3STAB.f90:175-189.  Its dummy ns_kdc is declared INTEGER
 * but every caller passes a real(8) (src/assembleNavSto.f90:270,
 * src/solveQuenching.f90:415-416): under the gfortran by-reference ABI the
 * callee reads the first 4 bytes of the double.  Reproduced here. */
static double e3dc_beta2(double ns_kdc_real, double G[3][3], const double* res) {
  int ns_kdc;
  memcpy(&ns_kdc, &ns_kdc_real, sizeof(int));
  double rr = res[0] * res[0] + res[1] * res[1] + res[2] * res[2];
  return ns_kdc * sqrt(rr / GG(G));
}

/* e3CFL src/e3STAB.f90:394-412 */
static double e3cfl(const double* u, double G[3][3], double dt) {
  double c = 0.0;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) c += u[i] * G[i][j] * u[j];
  return dt * sqrt(c);
}

/* ---------------------------------------------------------------------- */
/* element-local storage, indices [a][b] = (aa,bb) of the Fortran arrays  */
typedef struct elm_arrays {
  double K[9][NSHL_MAX][NSHL_MAX], G[3][NSHL_MAX][NSHL_MAX], D[3][NSHL_MAX][NSHL_MAX];
  double M[NSHL_MAX][NSHL_MAX], LS[NSHL_MAX][NSHL_MAX], LSU[3][NSHL_MAX][NSHL_MAX];
  double ULS[3][NSHL_MAX][NSHL_MAX], PLS[NSHL_MAX][NSHL_MAX];
  double Ru[3][NSHL_MAX], Rp[NSHL_MAX], Rphi[NSHL_MAX];
} elm_arrays;

static int IBC(const orc_mesh* m, int node0, int c1) {
  if (c1 > m->nibc) return 0;
  return m->ibc[cm(node0, m->nnode, c1 - 1)];
}

/* BCLhs_3D src/BCLhs_3D.f90:4-122 (element Dirichlet: zero rows and
 * columns, element diagonal set to 1, RHS zeroed) */
static void bclhs_3d(const orc_mesh* m, int e, int nshl, elm_arrays* L) {
  for (int aa = 0; aa < nshl; ++aa) {
    int cc = m->ien[cm(e, m->nelem, aa)] - 1;
    for (int d = 0; d < 3; ++d) {
      if (IBC(m, cc, d + 1) == 1) {
        for (int bb = 0; bb < nshl; ++bb) {
          L->K[3 * d + 0][aa][bb] = 0.0; L->K[3 * d + 1][aa][bb] = 0.0;
          L->K[3 * d + 2][aa][bb] = 0.0; L->G[d][aa][bb] = 0.0;
        }
        for (int bb = 0; bb < nshl; ++bb) {
          L->K[d][bb][aa] = 0.0; L->K[3 + d][bb][aa] = 0.0;
          L->K[6 + d][bb][aa] = 0.0; L->D[d][bb][aa] = 0.0;
        }
        L->K[4 * d][aa][aa] = 1.0;
        L->Ru[d][aa] = 0.0;
      }
    }
    if (IBC(m, cc, 4) == 1) {
      for (int bb = 0; bb < nshl; ++bb) {
        L->M[aa][bb] = 0.0;
        for (int d = 0; d < 3; ++d) { L->D[d][aa][bb] = 0.0; L->G[d][bb][aa] = 0.0; }
      }
      L->M[aa][aa] = 1.0;
      L->Rp[aa] = 0.0;
    }
  }
}

/* BCLhs_NS_conv src/BCLhs_3D.f90:278-428 with the setBCs_NSVOF column
 * layout (pressure IBC col 4, VOF col 5; src/setBCs.f90:183-187) - the
 * semantics chosen for the quench path, whose call to the 8-argument
 * BCLhs_3D with 13 arguments (src/solveQuenching.f90:526-528) cannot be
 * honoured literally.  xDebe2 does not exist on this path and is skipped. */
static void bclhs_ns_conv(const orc_mesh* m, int e, int nshl, elm_arrays* L) {
  for (int aa = 0; aa < nshl; ++aa) {
    int cc = m->ien[cm(e, m->nelem, aa)] - 1;
    for (int d = 0; d < 3; ++d) {
      if (IBC(m, cc, d + 1) == 1) {
        for (int bb = 0; bb < nshl; ++bb) {
          L->K[3 * d + 0][aa][bb] = 0.0; L->K[3 * d + 1][aa][bb] = 0.0;
          L->K[3 * d + 2][aa][bb] = 0.0; L->G[d][aa][bb] = 0.0;
          L->LSU[d][aa][bb] = 0.0;
        }
        for (int bb = 0; bb < nshl; ++bb) {
          L->K[d][bb][aa] = 0.0; L->K[3 + d][bb][aa] = 0.0;
          L->K[6 + d][bb][aa] = 0.0; L->D[d][bb][aa] = 0.0;
          L->LSU[d][bb][aa] = 0.0;
        }
        L->K[4 * d][aa][aa] = 1.0;
        L->Ru[d][aa] = 0.0;
      }
    }
    if (IBC(m, cc, 4) == 1) {
      for (int bb = 0; bb < nshl; ++bb) {
        L->M[aa][bb] = 0.0;
        for (int d = 0; d < 3; ++d) { L->D[d][aa][bb] = 0.0; L->G[d][bb][aa] = 0.0; }
        for (int t = 0; t < nshl; ++t) L->PLS[aa][t] = 0.0;
      }
      L->M[aa][aa] = 1.0;
      L->Rp[aa] = 0.0;
    }
    if (IBC(m, cc, 5) == 1) {
      for (int t = 0; t < nshl; ++t) { L->LS[aa][t] = 0.0; L->LS[t][aa] = 0.0; }
      for (int d = 0; d < 3; ++d)
        for (int t = 0; t < nshl; ++t) L->LSU[d][aa][t] = 0.0;
      for (int t = 0; t < nshl; ++t) L->PLS[t][aa] = 0.0;
      for (int d = 0; d < 3; ++d)
        for (int t = 0; t < nshl; ++t) L->ULS[d][t][aa] = 0.0;
      L->LS[aa][aa] = 1.0;
      L->Rphi[aa] = 0.0;
    }
  }
}

/* FillSparseMat_3D / FillSparseMat_NS_conv src/FillSparseMat.f90:33-67,
 * 237-288: slot by SparseMatLoc_3D, += element block */
static void fill_sparse(const orc_mesh* m, int e, int nshl,
                        const elm_arrays* L, orc_system* S, int with_vof) {
  for (int a = 0; a < nshl; ++a) {
    int i = m->ien[cm(e, m->nelem, a)] - 1;
    int c = m->col[i];
    int n = m->col[i + 1] - c;
    for (int b = 0; b < nshl; ++b) {
      int locn = orc_sparse_mat_loc(m->row + (c - 1), n, m->ien[cm(e, m->nelem, b)]);
      size_t k = (size_t)(locn + c - 1) - 1;
      for (int t = 0; t < 9; ++t) S->K11[k * 9 + t] += L->K[t][a][b];
      for (int t = 0; t < 3; ++t) S->G[k * 3 + t] += L->G[t][a][b];
      for (int t = 0; t < 3; ++t) S->D1[k * 3 + t] += L->D[t][a][b];
      S->M[k] += L->M[a][b];
      if (with_vof) {
        S->LS[k] += L->LS[a][b];
        for (int t = 0; t < 3; ++t) S->LSU[k * 3 + t] += L->LSU[t][a][b];
        S->PLS[k] += L->PLS[a][b];
        for (int t = 0; t < 3; ++t) S->ULS[k * 3 + t] += L->ULS[t][a][b];
      }
    }
  }
}

static void gather3(const double* g, int n, int node0, double* out) {
  for (int d = 0; d < 3; ++d) out[d] = g[cm(node0, n, d)];
}

/* ----------------------------------------------------------------------
 * e3LHS_3D_fluid_Old src/e3LHS.f90:4-161
 * -------------------------------------------------------------------- */
static void e3lhs_3d_fluid_old(const ovs_params* p, int nshl, double rhoi,
                               double mui, const double* ui, const double* umi,
                               const double* rLi, double tauM, double tauP,
                               double tauC, double tauBar, double kap_dc,
                               double gwt, const double* shgu,
                               double shgradgu[][3], double DetJ,
                               elm_arrays* L) {
  double fact1 = p->almi, fact2 = p->alfi * p->gami * p->delt;
  double mupkdc = mui + kap_dc;
  double tmp1[NSHL_MAX], tmp2[NSHL_MAX], tmp4[NSHL_MAX][NSHL_MAX];
  double advu1[3], advu2[3];
  for (int d = 0; d < 3; ++d) { advu1[d] = ui[d] - umi[d]; advu2[d] = -tauM * rLi[d]; }
  for (int a = 0; a < nshl; ++a) {
    tmp1[a] = rhoi * (advu1[0] * shgradgu[a][0] + advu1[1] * shgradgu[a][1] +
                      advu1[2] * shgradgu[a][2]);
    tmp2[a] = advu2[0] * shgradgu[a][0] + advu2[1] * shgradgu[a][1] +
              advu2[2] * shgradgu[a][2];
  }
  for (int bb = 0; bb < nshl; ++bb)
    for (int aa = 0; aa < nshl; ++aa)
      tmp4[aa][bb] = fact1 * (shgu[aa] * rhoi * shgu[bb] + tmp1[aa] * tauM * rhoi * shgu[bb]) +
                     fact2 * (shgu[aa] * tmp1[bb] + tmp1[aa] * tauM * tmp1[bb] +
                              mupkdc * (shgradgu[aa][0] * shgradgu[bb][0] +
                                        shgradgu[aa][1] * shgradgu[bb][1] +
                                        shgradgu[aa][2] * shgradgu[bb][2]) +
                              tmp2[aa] * rhoi * tauBar * tmp2[bb]);
  const double w = DetJ * gwt;
  for (int bb = 0; bb < nshl; ++bb)
    for (int aa = 0; aa < nshl; ++aa) {
      const double* ga = shgradgu[aa];
      const double* gb = shgradgu[bb];
      L->K[0][aa][bb] += (tmp4[aa][bb] + fact2 * (ga[0] * mupkdc * gb[0] + ga[0] * tauC * gb[0])) * w;
      L->K[4][aa][bb] += (tmp4[aa][bb] + fact2 * (ga[1] * mupkdc * gb[1] + ga[1] * tauC * gb[1])) * w;
      L->K[8][aa][bb] += (tmp4[aa][bb] + fact2 * (ga[2] * mupkdc * gb[2] + ga[2] * tauC * gb[2])) * w;
      L->K[1][aa][bb] += fact2 * (ga[1] * mupkdc * gb[0] + ga[0] * tauC * gb[1]) * w;
      L->K[3][aa][bb] += fact2 * (ga[0] * mupkdc * gb[1] + ga[1] * tauC * gb[0]) * w;
      L->K[2][aa][bb] += fact2 * (ga[2] * mupkdc * gb[0] + ga[0] * tauC * gb[2]) * w;
      L->K[6][aa][bb] += fact2 * (ga[0] * mupkdc * gb[2] + ga[2] * tauC * gb[0]) * w;
      L->K[5][aa][bb] += fact2 * (ga[2] * mupkdc * gb[1] + ga[1] * tauC * gb[2]) * w;
      L->K[7][aa][bb] += fact2 * (ga[1] * mupkdc * gb[2] + ga[2] * tauC * gb[1]) * w;
    }
  for (int bb = 0; bb < nshl; ++bb)
    for (int aa = 0; aa < nshl; ++aa)
      for (int d = 0; d < 3; ++d)
        L->G[d][aa][bb] += fact2 * (-shgradgu[aa][d] * shgu[bb] + tmp1[aa] * tauM * shgradgu[bb][d]) * w;
  for (int bb = 0; bb < nshl; ++bb)
    for (int aa = 0; aa < nshl; ++aa)
      for (int d = 0; d < 3; ++d)
        L->D[d][aa][bb] += (fact2 * (shgu[aa] * shgradgu[bb][d] + shgradgu[aa][d] * tauP * tmp1[bb]) +
                            fact1 * (shgradgu[aa][d] * tauP * rhoi * shgu[bb])) * w;
  for (int bb = 0; bb < nshl; ++bb)
    for (int aa = 0; aa < nshl; ++aa)
      L->M[aa][bb] += fact2 * tauP *
                      (shgradgu[aa][0] * shgradgu[bb][0] + shgradgu[aa][1] * shgradgu[bb][1] +
                       shgradgu[aa][2] * shgradgu[bb][2]) * w;
}

/* e3Rhs_3D_fluid src/e3RHS.f90:4-97 */
static void e3rhs_3d_fluid(int nshl, double rhoi, double mui, const double* aci,
                           const double* uadvi, double pri, const double* fi,
                           double du[3][3], double tauC, double tauBar,
                           double kap_dc, double gwt, const double* shgu,
                           double shgradgu[][3], const double* uprime,
                           double DetJ, elm_arrays* L) {
  double mupkdc = mui + kap_dc;
  double divu = du[0][0] + du[1][1] + du[2][2];
  double advu[3], tmp1[3], tmp4[3], tmp2[3][3];
  for (int d = 0; d < 3; ++d) advu[d] = uadvi[d] + uprime[d];
  double ptot = pri - tauC * divu;
  for (int i = 0; i < 3; ++i) {
    tmp1[i] = rhoi * (aci[i] + advu[0] * du[i][0] + advu[1] * du[i][1] + advu[2] * du[i][2]) - fi[i];
    tmp4[i] = uprime[0] * du[i][0] + uprime[1] * du[i][1] + uprime[2] * du[i][2];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = (i == j) ? (-ptot + 2.0 * mupkdc * du[i][i]) : mupkdc * (du[i][j] + du[j][i]);
      tmp2[i][j] = v - rhoi * (uadvi[j] + uprime[j]) * uprime[i] + rhoi * uprime[j] * tauBar * tmp4[i];
    }
  const double w = DetJ * gwt;
  for (int aa = 0; aa < nshl; ++aa)
    for (int i = 0; i < 3; ++i) {
      double s = shgradgu[aa][0] * tmp2[i][0] + shgradgu[aa][1] * tmp2[i][1] +
                 shgradgu[aa][2] * tmp2[i][2];
      L->Ru[i][aa] -= (shgu[aa] * tmp1[i] + s) * w;
    }
  for (int aa = 0; aa < nshl; ++aa) {
    double s = shgradgu[aa][0] * uprime[0] + shgradgu[aa][1] * uprime[1] + shgradgu[aa][2] * uprime[2];
    L->Rp[aa] -= (shgu[aa] * divu - s) * w;
  }
}

/* ----------------------------------------------------------------------
 * Element loop of IntElmAss_NS_overset src/assembleNavSto.f90:76-336
 * (the NS-only path).  Quirks kept: uprime receives shhessgu, i.e. zeros
 * (:284-288 vs src/e3RHS.f90:4-7); kap_dc receives the constant NS_kdc_a
 * (:277-280); tauBar = 0 (:268).  Returns the largest CFL.
 * -------------------------------------------------------------------- */
double orc_elmloop_ns(const orc_mesh* m, const ovs_params* p,
                      const orc_state* A, orc_system* S, int tensor_flag,
                      int e0, int e1) {
  const int N = m->nnode, nshl = m->nshl, ngp = m->nshl;
  double gp[NGP_MAX][3], gw[NGP_MAX];
  gen_gp_gw(ngp, gp, gw);
  const int mat = (tensor_flag & OVS_TENSOR_MAT) != 0;
  const int vec = (tensor_flag & OVS_TENSOR_VEC) != 0;
  double cfl = 0.0;
  elm_arrays L;
  for (int e = e0; e < e1; ++e) {
    int eid = m->elm_id ? m->elm_id[e] : 102;
    int is_target = 0;
    if (p->subdomain_flag & 1) is_target = is_target || eid == p->elm_id_set[0];
    if (p->subdomain_flag & 2) is_target = is_target || eid == p->elm_id_set[1];
    double xl[NSHL_MAX][3], dl[NSHL_MAX][3], ul[NSHL_MAX][3], acl[NSHL_MAX][3],
        uml[NSHL_MAX][3], pl[NSHL_MAX];
    for (int a = 0; a < nshl; ++a) {
      int idx = m->ien[cm(e, m->nelem, a)] - 1;
      gather3(m->xg, N, idx, xl[a]); gather3(A->dg, N, idx, dl[a]);
      gather3(A->ug, N, idx, ul[a]); gather3(A->acg, N, idx, acl[a]);
      gather3(A->ugm, N, idx, uml[a]);
      pl[a] = A->pg[idx];
    }
    memset(&L, 0, sizeof(L));
    for (int ig = 0; ig < ngp; ++ig) {
      double shlu[NSHL_MAX], shg[NSHL_MAX][3], Gij[3][3];
      double DetJ = eval_shape_fem(nshl, gp[ig], xl, dl, shlu, shg, Gij);
      double ui[3], aci[3], umi[3], pri = 0.0, du[3][3], dp[3];
      for (int d = 0; d < 3; ++d) {
        double s1 = 0, s2 = 0, s3 = 0;
        for (int a = 0; a < nshl; ++a) {
          s1 += ul[a][d] * shlu[a]; s2 += acl[a][d] * shlu[a]; s3 += uml[a][d] * shlu[a];
        }
        ui[d] = s1; aci[d] = s2; umi[d] = s3;
      }
      for (int a = 0; a < nshl; ++a) pri += pl[a] * shlu[a];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double s = 0.0;
          for (int a = 0; a < nshl; ++a) s += ul[a][i] * shg[a][j];
          du[i][j] = s;
        }
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
        for (int a = 0; a < nshl; ++a) s += pl[a] * shg[a][j];
        dp[j] = s;
      }
      double rhoi = p->rhoa, mui = p->mua, ns_kdc = p->ns_kdc_a;
      double uadvi[3], fi[3], rm[3], rLi[3];
      for (int d = 0; d < 3; ++d) uadvi[d] = ui[d] - umi[d];
      for (int d = 0; d < 3; ++d) fi[d] = p->gravvec[d] * rhoi;
      for (int i = 0; i < 3; ++i) {
        double mv = du[i][0] * uadvi[0] + du[i][1] * uadvi[1] + du[i][2] * uadvi[2];
        rm[i] = rhoi * (aci[i] + mv) - fi[i];
        rLi[i] = rm[i] + dp[i] - mui * 0.0;  /* Hessian of a linear field is 0 */
      }
      double tauM, tauP, tauC;
      e3stab_3d(Gij, p->delt, uadvi, rhoi, mui, &tauM, &tauP, &tauC);
      double tauBar = 0.0;
      (void)e3dc_beta2(ns_kdc, Gij, rLi);  /* k_dc is computed but unused here */
      double c = e3cfl(uadvi, Gij, p->delt);
      if (c > cfl) cfl = c;
      double uprime[3] = {0.0, 0.0, 0.0};  /* = shhessgu(1:3), zeroed (:223) */
      if (mat && is_target)
        e3lhs_3d_fluid_old(p, nshl, rhoi, mui, ui, umi, rLi, tauM, tauP, tauC,
                           tauBar, ns_kdc, gw[ig], shlu, shg, DetJ, &L);
      if (vec && is_target)
        e3rhs_3d_fluid(nshl, rhoi, mui, aci, uadvi, pri, fi, du, tauC, tauBar,
                       ns_kdc, gw[ig], shlu, shg, uprime, DetJ, &L);
    }
    bclhs_3d(m, e, nshl, &L);
    if (mat) fill_sparse(m, e, nshl, &L, S, 0);
    if (vec)
      for (int b = 0; b < nshl; ++b) {
        int g = m->ien[cm(e, m->nelem, b)] - 1;
        for (int d = 0; d < 3; ++d) S->rhsu[cm(g, N, d)] += L.Ru[d][b];
        S->rhsp[g] += L.Rp[b];
      }
  }
  return cfl;
}

/* ----------------------------------------------------------------------
 * Element loop of IntElmAss_NSVOF_Quenching_STAB src/solveQuenching.f90:
 * 122-573.  The viscous RHS broadcast (:508-510: three scalars each
 * subtracted from all three momentum components) is reproduced as written.
 * -------------------------------------------------------------------- */
double orc_elmloop_nsvof(const orc_mesh* m, const ovs_params* p,
                         const orc_state* A, orc_system* S, int tensor_flag,
                         int e0, int e1) {
  const int N = m->nnode, nshl = m->nshl, ngp = m->nshl;
  double gp[NGP_MAX][3], gw[NGP_MAX];
  gen_gp_gw(ngp, gp, gw);
  const int mat = (tensor_flag & OVS_TENSOR_MAT) != 0;
  const int vec = (tensor_flag & OVS_TENSOR_VEC) != 0;
  const double fact1 = p->almi, fact2 = p->alfi * p->delt * p->gami;
  const double rhoa = p->rhoa, rhow = p->rhow;
  double cfl = 0.0;
  elm_arrays L;
  for (int e = e0; e < e1; ++e) {
    int eid = m->elm_id ? m->elm_id[e] : 102;
    int is_fluid = eid == p->fluid_elm_id;
    double xl[NSHL_MAX][3], dl[NSHL_MAX][3], ul[NSHL_MAX][3], acl[NSHL_MAX][3],
        uml[NSHL_MAX][3], pl[NSHL_MAX], phil[NSHL_MAX], rphil[NSHL_MAX],
        Tl[NSHL_MAX];
    for (int a = 0; a < nshl; ++a) {
      int idx = m->ien[cm(e, m->nelem, a)] - 1;
      gather3(m->xg, N, idx, xl[a]); gather3(A->dg, N, idx, dl[a]);
      gather3(A->ug, N, idx, ul[a]); gather3(A->acg, N, idx, acl[a]);
      gather3(A->ugm, N, idx, uml[a]);
      pl[a] = A->pg[idx]; phil[a] = A->phig[idx]; rphil[a] = A->rphig[idx];
      Tl[a] = A->tg[idx];
    }
    memset(&L, 0, sizeof(L));
    for (int ig = 0; ig < ngp; ++ig) {
      double shlu[NSHL_MAX], shg[NSHL_MAX][3], Gij[3][3];
      double DetJ = eval_shape_fem(nshl, gp[ig], xl, dl, shlu, shg, Gij);
      double DetJgw = DetJ * gw[ig];
      double ui[3], aci[3], umi[3], pri = 0, phii = 0, rphii = 0, Ti = 0;
      double du[3][3], dp[3], dphi[3];
      for (int d = 0; d < 3; ++d) {
        double s1 = 0, s2 = 0, s3 = 0;
        for (int a = 0; a < nshl; ++a) {
          s1 += ul[a][d] * shlu[a]; s2 += acl[a][d] * shlu[a]; s3 += uml[a][d] * shlu[a];
        }
        ui[d] = s1; aci[d] = s2; umi[d] = s3;
      }
      for (int a = 0; a < nshl; ++a) {
        pri += pl[a] * shlu[a]; phii += phil[a] * shlu[a];
        rphii += rphil[a] * shlu[a]; Ti += Tl[a] * shlu[a];
      }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double s = 0.0;
          for (int a = 0; a < nshl; ++a) s += ul[a][i] * shg[a][j];
          du[i][j] = s;
        }
      for (int j = 0; j < 3; ++j) {
        double s1 = 0.0, s2 = 0.0;
        for (int a = 0; a < nshl; ++a) { s1 += pl[a] * shg[a][j]; s2 += phil[a] * shg[a][j]; }
        dp[j] = s1; dphi[j] = s2;
      }
      double phic = fmax(fmin(phii, 1.0), 0.0);
      double Tic = Ti, mdot, dmdphii;
      if (Ti > p->ts) {
        mdot = p->c_evap * (1 - phic) * rhow * (Tic - p->ts) / p->ts;
        dmdphii = -p->c_evap * rhow * (Tic - p->ts) / p->ts * p->c_dmdot;
      } else {
        mdot = p->c_cond * (phic) * rhoa * (Tic - p->ts) / p->ts;
        dmdphii = p->c_cond * rhoa * (Tic - p->ts) / p->ts * p->c_dmdot;
      }
      double vdot = mdot / rhoa - mdot / rhow;
      double rhoi, mui;
      if (is_fluid) { rhoi = prop_interp(rhow, rhoa, phic); mui = prop_interp(p->muw, p->mua, phic); }
      else { rhoi = p->rhos; mui = p->mus; }
      double lambda = -2.0 / 3.0 * mui;
      if (phii < 0.0 || phii > 1.0) dmdphii = 0.0;
      double uadvi[3], fi[3], rLi[3];
      for (int d = 0; d < 3; ++d) uadvi[d] = ui[d] - umi[d];
      double divu = du[0][0] + du[1][1] + du[2][2];
      for (int d = 0; d < 3; ++d) fi[d] = p->gravvec[d] * rhoi;
      for (int i = 0; i < 3; ++i)
        rLi[i] = rhoi * aci[i] + rhoi * (du[i][0] * uadvi[0] + du[i][1] * uadvi[1] + du[i][2] * uadvi[2]) +
                 dp[i] - fi[i] - mui * 0.0 - (mui + lambda) * 0.0;
      double res_phic = rphii + (uadvi[0] * dphi[0] + uadvi[1] * dphi[1] + uadvi[2] * dphi[2]) +
                        phii * vdot - mdot / rhoa;
      double tauM, tauP, tauC, tauls;
      e3stab_3d_nsvof(Gij, p->delt, uadvi, rhoi, mui, &tauM, &tauP, &tauC, &tauls);
      double uprime[3];
      for (int d = 0; d < 3; ++d) uprime[d] = -tauM * rLi[d];
      double shconv[NSHL_MAX];
      for (int a = 0; a < nshl; ++a)
        shconv[a] = uadvi[0] * shg[a][0] + uadvi[1] * shg[a][1] + uadvi[2] * shg[a][2];
      double k_dc = 0.0;
      if (fabs(p->ns_kdc_w) + fabs(p->ns_kdc_a) > 0.0) {
        double ns_kdc = prop_interp(p->ns_kdc_w, p->ns_kdc_a, phic);
        k_dc = e3dc_beta2(ns_kdc, Gij, rLi);
      }
      double k_dc_phi = 0.0;
      if (fabs(p->lsc_kdc) > 0.0) k_dc_phi = p->lsc_kdc * fabs(res_phic) / sqrt(GG(Gij));
      double c = e3cfl(uadvi, Gij, p->delt);
      if (c > cfl) cfl = c;
      const double ira = 1.0 / rhoa - 1.0 / rhow;
      if (mat && is_fluid) {
        for (int bb = 0; bb < nshl; ++bb)
          for (int aa = 0; aa < nshl; ++aa) {
            const double* ga = shg[aa];
            const double* gb = shg[bb];
            double gab = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
            for (int i = 0; i < 3; ++i) {
              for (int j = 0; j < 3; ++j)
                L.K[3 * i + j][aa][bb] += fact2 * ga[j] * gb[i] * (mui + k_dc) * DetJgw +
                                          fact2 * ga[i] * gb[j] * (tauC + lambda) * DetJgw;
              L.K[4 * i][aa][bb] += fact1 * shlu[aa] * rhoi * shlu[bb] * DetJgw +
                                    fact2 * shlu[aa] * rhoi * shconv[bb] * DetJgw +
                                    fact2 * (mui + k_dc) * gab * DetJgw +
                                    fact1 * rhoi * shconv[aa] * tauM * rhoi * shlu[bb] * DetJgw +
                                    fact2 * rhoi * shconv[aa] * tauM * rhoi * shconv[bb] * DetJgw;
            }
            for (int d = 0; d < 3; ++d) {
              L.G[d][aa][bb] += -fact2 * ga[d] * shlu[bb] * DetJgw +
                                fact2 * rhoi * shconv[aa] * tauM * gb[d] * DetJgw;
              L.D[d][aa][bb] += fact2 * shlu[aa] * gb[d] * DetJgw +
                                ga[d] * tauM * rhoi * fact1 * shlu[bb] * DetJgw +
                                ga[d] * tauM * rhoi * fact2 * shconv[bb] * DetJgw;
            }
            L.M[aa][bb] += fact2 * tauM * gab * DetJgw;
            double wa = shlu[aa] + tauls * shconv[aa];
            L.LS[aa][bb] += wa * fact1 * shlu[bb] * DetJgw + wa * fact2 * shconv[bb] * DetJgw;
            L.LS[aa][bb] += wa * fact2 * shlu[bb] * vdot * DetJgw +
                            wa * fact2 * phii * ira * dmdphii * shlu[bb] * DetJgw -
                            wa * fact2 * dmdphii * shlu[bb] / rhoa * DetJgw;
            L.LS[aa][bb] += fact2 * k_dc_phi * gab * DetJgw;
            L.LS[aa][bb] += fact2 * dmdphii * ira * shlu[aa] * tauC * dmdphii * ira * shlu[bb] * DetJgw;
            for (int d = 0; d < 3; ++d)
              L.ULS[d][aa][bb] += fact2 * ga[d] * tauC * dmdphii * shlu[bb] * ira * DetJgw;
            L.PLS[aa][bb] += -fact2 * shlu[aa] * dmdphii * shlu[bb] * ira * DetJgw;
            for (int d = 0; d < 3; ++d) {
              L.LSU[d][aa][bb] += fact2 * wa * shlu[bb] * dphi[d] * DetJgw;
              L.LSU[d][aa][bb] += -dmdphii * ira * fact2 * shlu[aa] * tauC * gb[d] * DetJgw;
            }
          }
      }
      if (vec && is_fluid) {
        double tmp1[3];
        for (int i = 0; i < 3; ++i)
          tmp1[i] = rhoi * aci[i] + rhoi * uadvi[0] * du[i][0] + rhoi * uadvi[1] * du[i][1] +
                    rhoi * uadvi[2] * du[i][2] - fi[i];
        for (int aa = 0; aa < nshl; ++aa) {
          const double* ga = shg[aa];
          double vis[3];
          for (int k = 0; k < 3; ++k)
            vis[k] = (mui + k_dc) * (ga[0] * (du[0][k] + du[k][0]) + ga[1] * (du[1][k] + du[k][1]) +
                                     ga[2] * (du[2][k] + du[k][2]));
          for (int i = 0; i < 3; ++i)
            L.Ru[i][aa] = L.Ru[i][aa] - shlu[aa] * tmp1[i] * DetJgw -
                          ga[i] * (-pri + tauC * divu) * DetJgw + ga[i] * tauC * vdot * DetJgw -
                          ga[i] * lambda * divu * DetJgw - vis[0] * DetJgw - vis[1] * DetJgw -
                          vis[2] * DetJgw + rhoi * shconv[aa] * uprime[i] * DetJgw;
          L.Rp[aa] = L.Rp[aa] - shlu[aa] * (divu - vdot) * DetJgw +
                     (ga[0] * uprime[0] + ga[1] * uprime[1] + ga[2] * uprime[2]) * DetJgw;
          L.Rphi[aa] = L.Rphi[aa] - (shlu[aa] + tauls * shconv[aa]) * res_phic * DetJgw -
                       k_dc_phi * (ga[0] * dphi[0] + ga[1] * dphi[1] + ga[2] * dphi[2]) * DetJgw +
                       shlu[aa] * dmdphii * ira * tauC * (divu - vdot) * DetJgw;
        }
      }
    }
    if (m->quench_literal) bclhs_3d(m, e, nshl, &L); else bclhs_ns_conv(m, e, nshl, &L);
    if (mat) fill_sparse(m, e, nshl, &L, S, !m->quench_literal);
    if (vec)
      for (int b = 0; b < nshl; ++b) {  /* LocaltoGlobalNSVOF_3D src/LocaltoGlobal.f90:26-51 */
        int g = m->ien[cm(e, m->nelem, b)] - 1;
        for (int d = 0; d < 3; ++d) S->rhsu[cm(g, N, d)] += L.Ru[d][b];
        S->rhsp[g] += L.Rp[b];
        S->rhsls[g] += L.Rphi[b];
      }
  }
  return cfl;
}

/* ----------------------------------------------------------------------
 * Element loop of IntElmAss_Tem_Quenching_STAB src/solveQuenching.f90:
 * 579-882 with BCLhs_tem (src/BCLhs_3D.f90:247-274) and FillSparseMat_tem
 * (src/FillSparseMat.f90:175-201).  Returns the largest CFL of the pass.
 * -------------------------------------------------------------------- */
double orc_elmloop_tem(const orc_mesh* m, const ovs_params* p,
                       const orc_state* A, orc_system* S, int tensor_flag,
                       int e0, int e1) {
  const int N = m->nnode, nshl = m->nshl, ngp = m->nshl;
  double gp[NGP_MAX][3], gw[NGP_MAX];
  gen_gp_gw(ngp, gp, gw);
  const int mat = (tensor_flag & OVS_TENSOR_MAT) != 0;
  const int vec = (tensor_flag & OVS_TENSOR_VEC) != 0;
  const double fact1 = p->almi, fact2 = p->alfi * p->gami * p->delt;
  double cfl = 0.0;
  for (int e = e0; e < e1; ++e) {
    int eid = m->elm_id ? m->elm_id[e] : 102;
    int is_fluid = eid == p->fluid_elm_id;
    double xl[NSHL_MAX][3], dl[NSHL_MAX][3], ul[NSHL_MAX][3], uml[NSHL_MAX][3],
        phil[NSHL_MAX], Tl[NSHL_MAX], rTl[NSHL_MAX];
    for (int a = 0; a < nshl; ++a) {
      int idx = m->ien[cm(e, m->nelem, a)] - 1;
      gather3(m->xg, N, idx, xl[a]); gather3(A->dg, N, idx, dl[a]);
      gather3(A->ug, N, idx, ul[a]); gather3(A->ugm, N, idx, uml[a]);
      phil[a] = A->phig[idx]; Tl[a] = A->tg[idx]; rTl[a] = A->rtg[idx];
    }
    double xT[NSHL_MAX][NSHL_MAX], RT[NSHL_MAX];
    memset(xT, 0, sizeof(xT));
    memset(RT, 0, sizeof(RT));
    for (int ig = 0; ig < ngp; ++ig) {
      double shlu[NSHL_MAX], shg[NSHL_MAX][3], Gij[3][3];
      double DetJ = eval_shape_fem(nshl, gp[ig], xl, dl, shlu, shg, Gij);
      double DetJgw = DetJ * gw[ig];
      double phii = 0, rTi = 0, Ti = 0, ui[3], umi[3], dT[3];
      for (int a = 0; a < nshl; ++a) { phii += phil[a] * shlu[a]; rTi += rTl[a] * shlu[a]; Ti += Tl[a] * shlu[a]; }
      for (int d = 0; d < 3; ++d) {
        double s1 = 0, s2 = 0;
        for (int a = 0; a < nshl; ++a) { s1 += ul[a][d] * shlu[a]; s2 += uml[a][d] * shlu[a]; }
        ui[d] = s1; umi[d] = s2;
      }
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
        for (int a = 0; a < nshl; ++a) s += Tl[a] * shg[a][j];
        dT[j] = s;
      }
      double phic = fmax(fmin(phii, 1.0), 0.0);
      double T0c = Ti, mdot, dmdTi;
      if (Ti > p->ts) {
        mdot = p->c_evap * (1 - phic) * p->rhow * (T0c - p->ts) / p->ts;
        dmdTi = p->c_evap * (1 - phic) * p->rhow / p->ts * p->c_dmdot;
      } else {
        mdot = p->c_cond * (phic) * p->rhoa * (T0c - p->ts) / p->ts;
        dmdTi = p->c_cond * (phic) * p->rhoa / p->ts * p->c_dmdot;
      }
      double rhoi, cpi, hki, rhocpi;
      if (is_fluid) {
        rhoi = prop_interp(p->rhow, p->rhoa, phic);
        cpi = prop_interp(p->cpw, p->cpa, phic);
        hki = prop_interp(p->kappaw, p->kappaa, phic);
        rhocpi = prop_interp(p->rhow * p->cpw, p->rhoa * p->cpa, phic);
      } else {
        rhoi = p->rhos; cpi = p->cps; hki = p->kappas; rhocpi = p->rhos * p->cps;
      }
      double uadvi[3];
      for (int d = 0; d < 3; ++d) uadvi[d] = ui[d] - umi[d];
      double Se = ((p->cpw - p->cpa) * (Ti - p->ts) - p->lh) * mdot;
      double udT = uadvi[0] * dT[0] + uadvi[1] * dT[1] + uadvi[2] * dT[2];
      double res_tem1 = rhocpi * (rTi + udT) - Se - hki * 0.0;
      double tau_tem = e3stab_3d_tem(Gij, uadvi, p->delt, rhoi, cpi, hki);
      double k_dc_tem = 0.0;
      if (fabs(p->tem_kdc) > 0.0 && is_fluid)
        k_dc_tem = p->tem_kdc * fabs(res_tem1) / sqrt(GG(Gij)) / p->tref;
      double shconv[NSHL_MAX];
      for (int a = 0; a < nshl; ++a)
        shconv[a] = shg[a][0] * uadvi[0] + shg[a][1] * uadvi[1] + shg[a][2] * uadvi[2];
      double dSedTi = (p->cpw - p->cpa) * mdot + ((p->cpw - p->cpa) * (Ti - p->ts) - p->lh) * dmdTi;
      double c = e3cfl(uadvi, Gij, p->delt);
      if (c > cfl) cfl = c;
      if (mat) {
        for (int aa = 0; aa < nshl; ++aa)
          for (int bb = 0; bb < nshl; ++bb) {
            double gab = shg[aa][0] * shg[bb][0] + shg[aa][1] * shg[bb][1] + shg[aa][2] * shg[bb][2];
            if (is_fluid)
              xT[aa][bb] += shlu[aa] * rhocpi * (fact1 * shlu[bb] + fact2 * shconv[bb]) * DetJgw -
                            shlu[aa] * fact2 * dSedTi * shlu[bb] * DetJgw +
                            tau_tem * rhocpi * shconv[aa] * rhocpi * (fact1 * shlu[bb] + fact2 * shconv[bb]) * DetJgw -
                            tau_tem * rhocpi * shconv[aa] * fact2 * dSedTi * shlu[bb] * DetJgw +
                            fact2 * (hki + k_dc_tem) * gab * DetJgw;
            else
              xT[aa][bb] += shlu[aa] * rhocpi * fact1 * shlu[bb] * DetJgw + fact2 * hki * gab * DetJgw;
          }
      }
      if (vec) {
        for (int a = 0; a < nshl; ++a) {
          if (is_fluid) {
            RT[a] -= shlu[a] * rhocpi * (rTi + udT) * DetJgw;
            RT[a] += shlu[a] * Se * DetJgw;
            RT[a] -= rhocpi * tau_tem * shconv[a] * res_tem1 * DetJgw;
            RT[a] -= (hki + k_dc_tem) * shg[a][0] * dT[0] * DetJgw;
            RT[a] -= (hki + k_dc_tem) * shg[a][1] * dT[1] * DetJgw;
            RT[a] -= (hki + k_dc_tem) * shg[a][2] * dT[2] * DetJgw;
          } else {
            RT[a] -= shlu[a] * rhocpi * rTi * DetJgw;
            RT[a] -= hki * shg[a][0] * dT[0] * DetJgw;
            RT[a] -= hki * shg[a][1] * dT[1] * DetJgw;
            RT[a] -= hki * shg[a][2] * dT[2] * DetJgw;
          }
        }
      }
    }
    for (int aa = 0; aa < nshl; ++aa) {  /* BCLhs_tem */
      int cc = m->ien[cm(e, m->nelem, aa)] - 1;
      if (IBC(m, cc, 6) == 1) {
        for (int t = 0; t < nshl; ++t) { xT[aa][t] = 0.0; xT[t][aa] = 0.0; }
        xT[aa][aa] = 1.0;
        RT[aa] = 0.0;
      }
    }
    if (mat)
      for (int a = 0; a < nshl; ++a) {
        int i = m->ien[cm(e, m->nelem, a)] - 1;
        int cc = m->col[i], n = m->col[i + 1] - cc;
        for (int b = 0; b < nshl; ++b) {
          int locn = orc_sparse_mat_loc(m->row + (cc - 1), n, m->ien[cm(e, m->nelem, b)]);
          S->TEM[(size_t)(locn + cc - 1) - 1] += xT[a][b];
        }
      }
    if (vec)
      for (int a = 0; a < nshl; ++a) S->rhstem[m->ien[cm(e, m->nelem, a)] - 1] += RT[a];
  }
  return cfl;
}

/* alpha stage: src/assembleNavSto.f90:25-30, src/solveQuenching.f90:26-37 */
void orc_alpha_stage(int N, const ovs_params* p, const orc_state* s,
                     orc_state* a) {
  for (size_t i = 0; i < (size_t)N * 3; ++i) {
    a->acg[i] = s->acgold[i] + p->almi * (s->acg[i] - s->acgold[i]);
    a->acgm[i] = s->acgmold[i] + p->almi * (s->acgm[i] - s->acgmold[i]);
    a->ug[i] = s->ugold[i] + p->alfi * (s->ug[i] - s->ugold[i]);
    a->ugm[i] = s->ugmold[i] + p->alfi * (s->ugm[i] - s->ugmold[i]);
    a->dg[i] = s->dgold[i] + p->alfi * (s->dg[i] - s->dgold[i]);
  }
  for (size_t i = 0; i < (size_t)N; ++i) {
    a->pg[i] = s->pg[i];
    a->phig[i] = s->phigold[i] + p->alfi * (s->phig[i] - s->phigold[i]);
    a->rphig[i] = s->rphigold[i] + p->almi * (s->rphig[i] - s->rphigold[i]);
    a->tg[i] = s->tgold[i] + p->alfi * (s->tg[i] - s->tgold[i]);
    a->rtg[i] = s->rtgold[i] + p->almi * (s->rtg[i] - s->rtgold[i]);
  }
}

typedef struct alpha_buf { orc_state a; double* mem; } alpha_buf;
static int alpha_alloc(int N, alpha_buf* b) {
  b->mem = (double*)malloc(sizeof(double) * (size_t)N * 20);
  if (!b->mem) return -1;
  double* q = b->mem;
  b->a.acg = q; q += 3 * (size_t)N; b->a.acgm = q; q += 3 * (size_t)N;
  b->a.ug = q; q += 3 * (size_t)N; b->a.ugm = q; q += 3 * (size_t)N;
  b->a.dg = q; q += 3 * (size_t)N;
  b->a.pg = q; q += N; b->a.phig = q; q += N; b->a.rphig = q; q += N;
  b->a.tg = q; q += N; b->a.rtg = q;
  return 0;
}

/* ----------------------------------------------------------------------
 * Face assemblies (linear tets; genGPMap src/genGP_GW.f90:42-62 maps face
 * points for nshl = 4 and 6 only).
 * -------------------------------------------------------------------- */

/* genGPtritet src/genGP_GW.f90:478-572 with NGAUSSB = NSHLB = 3
 * (src/input.f90:161): volume coordinates of the three face points for
 * FACE_OR = 1..4; genGPandGWtri :453-465 gives each the weight 1/6. */
#define SIXTH 0.166666666666666666667
#define TWO3 0.666666666666666666667
static const double c_tri_mgp[4][3][3] = {
    {{SIXTH, TWO3, SIXTH}, {SIXTH, SIXTH, TWO3}, {TWO3, SIXTH, SIXTH}},
    {{0.0, SIXTH, SIXTH}, {0.0, SIXTH, TWO3}, {0.0, TWO3, SIXTH}},
    {{TWO3, 0.0, SIXTH}, {SIXTH, 0.0, TWO3}, {SIXTH, 0.0, SIXTH}},
    {{SIXTH, TWO3, 0.0}, {TWO3, SIXTH, 0.0}, {SIXTH, SIXTH, 0.0}}};
static const double c_tri_gw = SIXTH;

/* the element nodes of the face, in the order eval_faceshape_tet takes them
 * (src/eval_shape_FEM.f90:90-106), 0-based */
static const int c_face_nodes[4][3] = {{1, 2, 0}, {3, 2, 1}, {0, 2, 3}, {1, 0, 3}};

/* eval_faceshape_tet src/eval_shape_FEM.f90:66-143: tangents of the face
 * triangle (lintrishl :261-282), unit normal and DetJb (:108-126), then
 * eval_shape_fem at the face point in volume coordinates.  Returns DetJb. */
static double eval_faceshape_tet(int fo, const double* mgp, double xl[][3],
                                 double dl[][3], double* shl, double shg[][3],
                                 double dxidx[3][3], double nor[3]) {
  double bx[3][3], t1[3], t2[3], Gij[3][3];
  for (int i = 0; i < 3; ++i) {
    const int a = c_face_nodes[fo - 1][i];
    for (int d = 0; d < 3; ++d) bx[i][d] = xl[a][d] + dl[a][d];
  }
  for (int d = 0; d < 3; ++d) {
    t1[d] = bx[0][d] - bx[2][d];
    t2[d] = bx[1][d] - bx[2][d];
  }
  nor[0] = t1[1] * t2[2] - t1[2] * t2[1];
  nor[1] = t1[2] * t2[0] - t1[0] * t2[2];
  nor[2] = t1[0] * t2[1] - t1[1] * t2[0];
  const double detjb = sqrt(nor[0] * nor[0] + nor[1] * nor[1] + nor[2] * nor[2]);
  for (int d = 0; d < 3; ++d) nor[d] = nor[d] / detjb;
  eval_shape_fem_dx(4, mgp, xl, dl, shl, shg, Gij, dxidx);
  return detjb;
}

/* e3bSTAB_weak src/e3STAB.f90:256-287: tauB = 4 mu / h_n with
 * h_n = 2 / |dxi/dx n| (the non-tet branch, as written); tauNor = tauB */
static double e3bstab_weak(const double* nor, double dxidx[3][3], double mui) {
  double t[3];
  for (int i = 0; i < 3; ++i) t[i] = dxidx[i][0] * nor[0] + dxidx[i][1] * nor[1] + dxidx[i][2] * nor[2];
  const double hn = 2.0 / sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  return 4.0 * mui / hn;
}

/* e3bRHS_weak src/e3RHS.f90:105-170 */
static void e3brhs_weak(double rhoi, double mui, const double* nor, double tauB,
                        double tauNor, double gwt, double detjb, const double* shl,
                        double shg[][3], const double* ui, const double* umi, double pri,
                        double du[3][3], const double* gi, elm_arrays* L) {
  double ti[3], tmp1[3], tmp2[3][3];
  for (int i = 0; i < 3; ++i)
    ti[i] = -pri * nor[i] + mui * (du[i][0] * nor[0] + du[i][1] * nor[1] + du[i][2] * nor[2] +
                                   du[0][i] * nor[0] + du[1][i] * nor[1] + du[2][i] * nor[2]);
  double unor = (ui[0] - umi[0]) * nor[0] + (ui[1] - umi[1]) * nor[1] + (ui[2] - umi[2]) * nor[2];
  const double uneg = 0.5 * (unor - fabs(unor));
  const double gnor = gi[0] * nor[0] + gi[1] * nor[1] + gi[2] * nor[2];
  unor = ui[0] * nor[0] + ui[1] * nor[1] + ui[2] * nor[2];
  for (int i = 0; i < 3; ++i)
    tmp1[i] = -ti[i] + tauB * (ui[i] - gi[i]) - uneg * rhoi * (ui[i] - gi[i]) +
              (tauNor - tauB) * unor * nor[i];
  const double gmul = 1.0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      tmp2[a][b] = -gmul * mui * ((ui[a] - gi[a]) * nor[b] + (ui[b] - gi[b]) * nor[a]);
  for (int aa = 0; aa < 4; ++aa) {
    for (int i = 0; i < 3; ++i)
      L->Ru[i][aa] = L->Ru[i][aa] -
                     (shl[aa] * tmp1[i] + (shg[aa][0] * tmp2[i][0] + shg[aa][1] * tmp2[i][1] +
                                           shg[aa][2] * tmp2[i][2])) * detjb * gwt;
    L->Rp[aa] = L->Rp[aa] + shl[aa] * (unor - gnor) * detjb * gwt;
  }
}

/* e3bLHS_weak src/e3LHS.f90:167-294 (gmul = 1, munor = tauNor - tauB) */
static void e3blhs_weak(double rhoi, double mui, const double* ui, const double* umi,
                        double tauB, double tauNor, double gwt, double detjb,
                        const double* shl, double shg[][3], const double* nor,
                        double fact2, elm_arrays* L) {
  double tmp1[4], tmp2[4][4];
  for (int a = 0; a < 4; ++a) tmp1[a] = shg[a][0] * nor[0] + shg[a][1] * nor[1] + shg[a][2] * nor[2];
  const double unor = (ui[0] - umi[0]) * nor[0] + (ui[1] - umi[1]) * nor[1] + (ui[2] - umi[2]) * nor[2];
  const double uneg = 0.5 * (unor - fabs(unor));
  const double munor = tauNor - tauB, gmul = 1.0;
  for (int bb = 0; bb < 4; ++bb)
    for (int aa = 0; aa < 4; ++aa)
      tmp2[aa][bb] = -shl[aa] * mui * tmp1[bb] - gmul * tmp1[aa] * mui * shl[bb] +
                     shl[aa] * tauB * shl[bb] - shl[aa] * uneg * rhoi * shl[bb];
  for (int bb = 0; bb < 4; ++bb)
    for (int aa = 0; aa < 4; ++aa)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          /* xKebe((i-1)*3+j): row component i, column component j */
          double v = -shl[aa] * mui * shg[bb][i] * nor[j] - gmul * shg[aa][j] * nor[i] * mui * shl[bb] +
                     shl[aa] * nor[i] * munor * nor[j] * shl[bb];
          if (i == j) v = tmp2[aa][bb] + v;
          L->K[3 * i + j][aa][bb] += fact2 * v * detjb * gwt;
        }
  for (int bb = 0; bb < 4; ++bb)
    for (int aa = 0; aa < 4; ++aa)
      for (int d = 0; d < 3; ++d) {
        L->D[d][aa][bb] -= fact2 * shl[aa] * shl[bb] * nor[d] * detjb * gwt;
        L->G[d][aa][bb] += fact2 * shl[aa] * shl[bb] * nor[d] * detjb * gwt;
      }
}

/* FaceAssembly_NS_weak src/FaceAssembly_weak.f90:4-193 (rho_a, mu_a, wall
 * velocity g = mesh velocity, element ELM_ID selection by subdomain_flag
 * :102-109 when use_subdomain), then FaceAssembly_NS_outflow :197-409
 * (backflow term, no ELM_ID selection), each over the faces of the
 * boundaries with BCugType == 2, each face followed by BCLhs_3D and the
 * scatter (:165-176, :381-392).  tauB is evaluated at every face point; the
 * reference evaluates it only under ASSEMBLE_TENSOR_VEC (:152) although the
 * matrix terms (:160-164) read it too. */
void orc_face_ns(const orc_mesh* m, const ovs_params* p, const orc_state* A,
                 orc_system* S, int tensor_flag, int use_subdomain) {
  if (m->nface <= 0 || m->nshl != 4) return;
  const int N = m->nnode;
  const int mat = (tensor_flag & OVS_TENSOR_MAT) != 0;
  const int vec = (tensor_flag & OVS_TENSOR_VEC) != 0;
  const double fact2 = p->alfi * p->gami * p->delt;
  const double rhoi = p->rhoa, mui = p->mua;
  elm_arrays L;
  for (int pass = 0; pass < 2; ++pass) {
    for (int f = 0; f < m->nface; ++f) {
      if (!(m->fflag[f] & OVS_FACE_WEAK)) continue;
      const int e = m->f2e[f] - 1, fo = m->face_or[f];
      int is_target = 1;
      if (pass == 0 && use_subdomain) {
        const int eid = m->elm_id ? m->elm_id[e] : 102;
        is_target = 0;
        if (p->subdomain_flag & 1) is_target = is_target || eid == p->elm_id_set[0];
        if (p->subdomain_flag & 2) is_target = is_target || eid == p->elm_id_set[1];
      }
      double xl[NSHL_MAX][3], dl[NSHL_MAX][3], ul[NSHL_MAX][3], uml[NSHL_MAX][3], pl[NSHL_MAX];
      for (int a = 0; a < 4; ++a) {
        const int idx = m->ien[cm(e, m->nelem, a)] - 1;
        gather3(m->xg, N, idx, xl[a]); gather3(A->dg, N, idx, dl[a]);
        gather3(A->ug, N, idx, ul[a]); gather3(A->ugm, N, idx, uml[a]);
        pl[a] = A->pg[idx];
      }
      memset(&L, 0, sizeof(L));
      for (int ig = 0; ig < 3; ++ig) {
        double shl[NSHL_MAX], shg[NSHL_MAX][3], dxidx[3][3], nor[3];
        const double detjb = eval_faceshape_tet(fo, c_tri_mgp[fo - 1][ig], xl, dl, shl, shg, dxidx, nor);
        double ui[3], umi[3], pri = 0.0, du[3][3];
        for (int d = 0; d < 3; ++d) {
          double s1 = 0, s2 = 0;
          for (int a = 0; a < 4; ++a) { s1 += ul[a][d] * shl[a]; s2 += uml[a][d] * shl[a]; }
          ui[d] = s1; umi[d] = s2;
        }
        for (int a = 0; a < 4; ++a) pri += pl[a] * shl[a];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int a = 0; a < 4; ++a) s += ul[a][i] * shg[a][j];
            du[i][j] = s;
          }
        const double* gi = umi;
        if (pass == 0) {
          const double tauB = e3bstab_weak(nor, dxidx, mui), tauNor = tauB;
          if (vec && is_target)
            e3brhs_weak(rhoi, mui, nor, tauB, tauNor, c_tri_gw, detjb, shl, shg, ui, umi, pri, du, gi, &L);
          if (mat && is_target)
            e3blhs_weak(rhoi, mui, ui, umi, tauB, tauNor, c_tri_gw, detjb, shl, shg, nor, fact2, &L);
        } else {
          const double detjgw = detjb * c_tri_gw;
          const double unor = (ui[0] - umi[0]) * nor[0] + (ui[1] - umi[1]) * nor[1] + (ui[2] - umi[2]) * nor[2];
          const double uneg = 0.5 * (unor - fabs(unor));
          if (vec)
            for (int aa = 0; aa < 4; ++aa)
              for (int d = 0; d < 3; ++d)
                L.Ru[d][aa] = L.Ru[d][aa] + shl[aa] * rhoi * uneg * (ui[d] - gi[d]) * detjgw;
          if (mat)
            for (int bb = 0; bb < 4; ++bb)
              for (int aa = 0; aa < 4; ++aa) {
                const double t2 = -shl[aa] * uneg * rhoi * shl[bb];
                for (int ii = 0; ii < 3; ++ii) L.K[4 * ii][aa][bb] += fact2 * t2 * detjgw;
              }
        }
      }
      bclhs_3d(m, e, 4, &L);
      if (mat) fill_sparse(m, e, 4, &L, S, 0);
      if (vec)
        for (int b = 0; b < 4; ++b) {
          const int g = m->ien[cm(e, m->nelem, b)] - 1;
          for (int d = 0; d < 3; ++d) S->rhsu[cm(g, N, d)] += L.Ru[d][b];
          S->rhsp[g] += L.Rp[b];
        }
    }
  }
}

/* Convective heat flux on the temperature system, the FaceAssembly_ConvectiveH
 * the quench driver calls (src/solveQuenching.f90:92) and the reference does
 * not define: q = h (T^alpha - T_inf) on flagged faces, residual
 * -int N_a q dGamma, tangent alpha_f gamma Delt int N_a h N_b dGamma (the
 * factor of the element conductivity term), with the face points and
 * surface Jacobian of the other face routines and BCLhs_tem after each face. */
void orc_face_convh(const orc_mesh* m, const ovs_params* p, const orc_state* A,
                    orc_system* S, int tensor_flag) {
  if (m->nface <= 0 || m->nshl != 4) return;
  const int N = m->nnode;
  const int mat = (tensor_flag & OVS_TENSOR_MAT) != 0;
  const int vec = (tensor_flag & OVS_TENSOR_VEC) != 0;
  const double fact2 = p->alfi * p->gami * p->delt;
  for (int f = 0; f < m->nface; ++f) {
    if (!(m->fflag[f] & OVS_FACE_CONVH)) continue;
    const int e = m->f2e[f] - 1, fo = m->face_or[f];
    const double h = m->hconv[f], tinf = m->tinf[f];
    double xl[NSHL_MAX][3], dl[NSHL_MAX][3], Tl[NSHL_MAX];
    for (int a = 0; a < 4; ++a) {
      const int idx = m->ien[cm(e, m->nelem, a)] - 1;
      gather3(m->xg, N, idx, xl[a]); gather3(A->dg, N, idx, dl[a]);
      Tl[a] = A->tg[idx];
    }
    double xT[4][4], RT[4];
    memset(xT, 0, sizeof(xT));
    memset(RT, 0, sizeof(RT));
    for (int ig = 0; ig < 3; ++ig) {
      double shl[NSHL_MAX], shg[NSHL_MAX][3], dxidx[3][3], nor[3];
      const double detjgw = eval_faceshape_tet(fo, c_tri_mgp[fo - 1][ig], xl, dl, shl, shg, dxidx, nor) * c_tri_gw;
      double Ti = 0.0;
      for (int a = 0; a < 4; ++a) Ti += Tl[a] * shl[a];
      const double q = h * (Ti - tinf);
      if (mat)
        for (int aa = 0; aa < 4; ++aa)
          for (int bb = 0; bb < 4; ++bb) xT[aa][bb] += fact2 * shl[aa] * h * shl[bb] * detjgw;
      if (vec)
        for (int aa = 0; aa < 4; ++aa) RT[aa] -= shl[aa] * q * detjgw;
    }
    for (int aa = 0; aa < 4; ++aa) {  /* BCLhs_tem */
      const int cc = m->ien[cm(e, m->nelem, aa)] - 1;
      if (IBC(m, cc, 6) == 1) {
        for (int t = 0; t < 4; ++t) { xT[aa][t] = 0.0; xT[t][aa] = 0.0; }
        xT[aa][aa] = 1.0;
        RT[aa] = 0.0;
      }
    }
    if (mat)
      for (int a = 0; a < 4; ++a) {
        const int i = m->ien[cm(e, m->nelem, a)] - 1;
        const int cc = m->col[i], n = m->col[i + 1] - cc;
        for (int b = 0; b < 4; ++b) {
          const int locn = orc_sparse_mat_loc(m->row + (cc - 1), n, m->ien[cm(e, m->nelem, b)]);
          S->TEM[(size_t)(locn + cc - 1) - 1] += xT[a][b];
        }
      }
    if (vec)
      for (int a = 0; a < 4; ++a) S->rhstem[m->ien[cm(e, m->nelem, a)] - 1] += RT[a];
  }
}

/* setBCs_NSVOF src/setBCs.f90:172-244 and setBCs_Tem :248-278.  The *Type
 * tables are read by FACE_ID, the *Valu tables by boundary number (:212-216,
 * :230-234, :266-268), as written; Dtgl = 1/Delt (src/param.f90:488). */
void orc_set_bcs(int N, int nibc, int* ibc, const ovs_params* p, orc_state* s,
                 const ovs_bc_spec* sp, int which) {
  const double dtgl = 1.0 / p->delt, gami = p->gami;
  const int nb = sp->nbound, nt = sp->ntype;
  if (which & 1) {
    for (size_t i = 0; i < (size_t)N * nibc; ++i) ibc[i] = 0;            /* IBC = 0 */
    for (int i = 0; i < N; ++i)
      if (sp->node_id && sp->node_id[i] == 101)
        for (int c = 0; c < 5 && c < nibc; ++c) ibc[cm(i, N, c)] = 1;     /* :201-208 */
    for (int b = 0; b < nb; ++b) {
      const int fid = sp->face_id[b];
      for (int d = 0; d < 3; ++d)
        if (sp->bcug_type[cm(fid - 1, nt, d)] == 1)
          for (int j = sp->bnode_ptr[b]; j < sp->bnode_ptr[b + 1]; ++j) {
            const int k = sp->bnodes[j] - 1;
            ibc[cm(k, N, d)] = 1;
            s->ug[cm(k, N, d)] = sp->bcug_valu[cm(b, nb, d)];
            s->acg[cm(k, N, d)] = ((s->ug[cm(k, N, d)] - s->ugold[cm(k, N, d)]) * dtgl +
                                   (gami - 1.0) * s->acgold[cm(k, N, d)]) / gami;
          }
      if (sp->bcphig_type[fid - 1] == 1)
        for (int j = sp->bnode_ptr[b]; j < sp->bnode_ptr[b + 1]; ++j) {
          const int k = sp->bnodes[j] - 1;
          if (nibc > 4) ibc[cm(k, N, 4)] = 1;
          s->phig[k] = sp->bcphig_valu[b];
          s->rphig[k] = ((s->phig[k] - s->phigold[k]) * dtgl + (gami - 1.0) * s->rphigold[k]) / gami;
        }
    }
  }
  if (which & 2) {
    if (nibc > 5)
      for (int i = 0; i < N; ++i) ibc[cm(i, N, 5)] = 0;                   /* IBC(:, 6) = 0 */
    for (int b = 0; b < nb; ++b) {
      const int fid = sp->face_id[b];
      if (sp->bctg_type[fid - 1] == 1)
        for (int j = sp->bnode_ptr[b]; j < sp->bnode_ptr[b + 1]; ++j) {
          const int k = sp->bnodes[j] - 1;
          if (nibc > 5) ibc[cm(k, N, 5)] = 1;
          s->tg[k] = sp->bctg_valu[b];
          s->rtg[k] = ((s->tg[k] - s->tgold[k]) * dtgl + (gami - 1.0) * s->rtgold[k]) / gami;
        }
    }
  }
}

/* assembleNavSto src/assembleNavSto.f90:4-72 (single rank: commu is the
 * identity); the face assemblies :55-61 act on the faces flagged
 * OVS_FACE_WEAK (boundaries with BCugType == 2) */
double orc_assemble_navsto(const orc_mesh* m, const ovs_params* p,
                           const orc_state* s, orc_system* S, int tensor_flag) {
  const size_t N = (size_t)m->nnode, K = (size_t)m->icnt;
  alpha_buf b;
  if (alpha_alloc(m->nnode, &b)) return -1.0;
  orc_alpha_stage(m->nnode, p, s, &b.a);
  if (tensor_flag & OVS_TENSOR_VEC) {
    memset(S->rhsu, 0, sizeof(double) * 3 * N);
    memset(S->rhsp, 0, sizeof(double) * N);
  }
  if (tensor_flag & OVS_TENSOR_MAT) {
    memset(S->K11, 0, sizeof(double) * 9 * K); memset(S->G, 0, sizeof(double) * 3 * K);
    memset(S->D1, 0, sizeof(double) * 3 * K); memset(S->M, 0, sizeof(double) * K);
  }
  double cfl = orc_elmloop_ns(m, p, &b.a, S, tensor_flag, 0, m->nelem);
  orc_face_ns(m, p, &b.a, S, tensor_flag, 1);
  free(b.mem);
  return cfl;
}

/* assembleQuenching src/solveQuenching.f90:4-117.  Its face calls (:75-95)
 * name two routines the reference does not define (FaceAssembly_NS_weak_CF,
 * FaceAssembly_ConvectiveH) and pass 11 arguments to the 8-argument
 * FaceAssembly_NS_outflow; here the NS+VOF pass runs the defined weak and
 * outflow face routines on the velocity/pressure blocks (every element a
 * target: the quench pass has no subdomain flag) and the temperature pass
 * the convective heat term. */
double orc_assemble_quenching(const orc_mesh* m, const ovs_params* p,
                              const orc_state* s, orc_system* S,
                              int tensor_flag, int field_flag) {
  const size_t N = (size_t)m->nnode, K = (size_t)m->icnt;
  alpha_buf b;
  if (alpha_alloc(m->nnode, &b)) return -1.0;
  orc_alpha_stage(m->nnode, p, s, &b.a);
  if (tensor_flag & OVS_TENSOR_VEC) {
    if (S->rhsu) memset(S->rhsu, 0, sizeof(double) * 3 * N);
    if (S->rhsp) memset(S->rhsp, 0, sizeof(double) * N);
    if (S->rhsls) memset(S->rhsls, 0, sizeof(double) * N);
    if (S->rhstem) memset(S->rhstem, 0, sizeof(double) * N);
  }
  if (tensor_flag & OVS_TENSOR_MAT) {
    double* arr[9] = {S->K11, S->G, S->D1, S->M, S->LS, S->ULS, S->LSU, S->PLS, S->TEM};
    size_t w[9] = {9, 3, 3, 1, 1, 3, 3, 1, 1};
    for (int t = 0; t < 9; ++t) if (arr[t]) memset(arr[t], 0, sizeof(double) * w[t] * K);
  }
  double cfl = 0.0;
  if (field_flag & 3) {
    cfl = orc_elmloop_nsvof(m, p, &b.a, S, tensor_flag, 0, m->nelem);
    orc_face_ns(m, p, &b.a, S, tensor_flag, 0);
  }
  if (field_flag & 4) {
    double c2 = orc_elmloop_tem(m, p, &b.a, S, tensor_flag, 0, m->nelem);
    orc_face_convh(m, p, &b.a, S, tensor_flag);
    if (!(field_flag & 3)) cfl = c2;
  }
  free(b.mem);
  return cfl;
}

/* ----------------------------------------------------------------------
 * SpMV: SparseProdUP_3D src/SparseProd.f90:4-60, SparseProd_LS :128-161,
 * SparseProd_NS_conv :167-242.  Vectors in (N,3) + (N) layout.
 * -------------------------------------------------------------------- */
void orc_sparse_prod_up_3d(int N, const int* col, const int* row,
                           const orc_system* S, const double* xu,
                           const double* xp, double* yu, double* yp) {
  for (int a = 0; a < N; ++a) {
    double t[4] = {0, 0, 0, 0};
    for (int b = col[a] - 1; b < col[a + 1] - 1; ++b) {
      int c = row[b] - 1;
      const double* K = S->K11 + (size_t)b * 9;
      const double* G = S->G + (size_t)b * 3;
      const double* D = S->D1 + (size_t)b * 3;
      t[0] = t[0] + K[0] * xu[c] + K[1] * xu[c + N] + K[2] * xu[c + 2 * (size_t)N] + G[0] * xp[c];
      t[1] = t[1] + K[3] * xu[c] + K[4] * xu[c + N] + K[5] * xu[c + 2 * (size_t)N] + G[1] * xp[c];
      t[2] = t[2] + K[6] * xu[c] + K[7] * xu[c + N] + K[8] * xu[c + 2 * (size_t)N] + G[2] * xp[c];
      t[3] = t[3] + D[0] * xu[c] + D[1] * xu[c + N] + D[2] * xu[c + 2 * (size_t)N] + S->M[b] * xp[c];
    }
    yu[a] = t[0]; yu[a + N] = t[1]; yu[a + 2 * (size_t)N] = t[2]; yp[a] = t[3];
  }
}

void orc_sparse_prod_ns_conv(int N, const int* col, const int* row,
                             const orc_system* S, const double* xu,
                             const double* xp, const double* xls, double* yu,
                             double* yp, double* yls) {
  for (int a = 0; a < N; ++a) {
    double t[5] = {0, 0, 0, 0, 0};
    for (int b = col[a] - 1; b < col[a + 1] - 1; ++b) {
      int c = row[b] - 1;
      const double* K = S->K11 + (size_t)b * 9;
      const double* G = S->G + (size_t)b * 3;
      const double* D = S->D1 + (size_t)b * 3;
      const double* U = S->ULS + (size_t)b * 3;
      const double* V = S->LSU + (size_t)b * 3;
      double x0 = xu[c], x1 = xu[c + N], x2 = xu[c + 2 * (size_t)N];
      t[0] = t[0] + K[0] * x0 + K[1] * x1 + K[2] * x2 + U[0] * xls[c] + G[0] * xp[c];
      t[1] = t[1] + K[3] * x0 + K[4] * x1 + K[5] * x2 + U[1] * xls[c] + G[1] * xp[c];
      t[2] = t[2] + K[6] * x0 + K[7] * x1 + K[8] * x2 + U[2] * xls[c] + G[2] * xp[c];
      t[3] = t[3] + D[0] * x0 + D[1] * x1 + D[2] * x2 + S->PLS[b] * xls[c] + S->M[b] * xp[c];
      t[4] = t[4] + V[0] * x0 + V[1] * x1 + V[2] * x2 + S->LS[b] * xls[c];
    }
    yu[a] = t[0]; yu[a + N] = t[1]; yu[a + 2 * (size_t)N] = t[2]; yp[a] = t[3]; yls[a] = t[4];
  }
}

void orc_sparse_prod_ls(int N, const int* col, const int* row,
                        const double* lhs, const double* x, double* y) {
  for (int a = 0; a < N; ++a) {
    double t = 0.0;
    for (int b = col[a] - 1; b < col[a + 1] - 1; ++b) t = t + lhs[b] * x[row[b] - 1];
    y[a] = t;
  }
}

/* ----------------------------------------------------------------------
 * GMRES, one cycle, Shakib/Johan form.  The block vector of nf fields is
 * stored field-major: v[f*N + i].  The reference's dot products visit the
 * scalar fields first, then the velocity components (SparseGMRES_NS.f90:
 * 143-149, SparseGMRES_NS_conv.f:175-180).
 * -------------------------------------------------------------------- */
typedef struct gm_sys {
  int kind;  /* 1 up, 2 ns_conv, 3 tem */
  int N;
  const int *col, *row;
  const orc_system* S;
  const double* lhs_tem;
  double* Binv;    /* N*9 */
  double* pinv;    /* N   */
  double* lsinv;   /* N   */
} gm_sys;

static int gm_nf(const gm_sys* g) { return g->kind == 1 ? 4 : (g->kind == 2 ? 5 : 1); }

static double gm_dot(const gm_sys* g, const double* a, const double* b) {
  const int N = g->N;
  double rr = 0.0;
  if (g->kind == 3) {
    for (int i = 0; i < N; ++i) rr += a[i] * b[i];
    return rr;
  }
  for (int i = 0; i < N; ++i) rr += a[3 * N + i] * b[3 * N + i];      /* p   */
  if (g->kind == 2) {
    double r2 = 0.0;
    for (int i = 0; i < N; ++i) r2 += a[4 * N + i] * b[4 * N + i];    /* phi */
    rr = rr + r2;
  }
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int i = 0; i < N; ++i) s += a[d * N + i] * b[d * N + i];
    rr = rr + s;
  }
  return rr;
}

static void gm_precond(const gm_sys* g, double* v) {
  const int N = g->N;
  if (g->kind == 3) { for (int i = 0; i < N; ++i) v[i] = g->pinv[i] * v[i]; return; }
  for (int i = 0; i < N; ++i) {
    const double* B = g->Binv + (size_t)i * 9;
    double r0 = v[i], r1 = v[N + i], r2 = v[2 * N + i];
    v[i] = B[0] * r0 + B[1] * r1 + B[2] * r2;
    v[N + i] = B[3] * r0 + B[4] * r1 + B[5] * r2;
    v[2 * N + i] = B[6] * r0 + B[7] * r1 + B[8] * r2;
    v[3 * N + i] = v[3 * N + i] * g->pinv[i];
    if (g->kind == 2) v[4 * N + i] = v[4 * N + i] * g->lsinv[i];
  }
}

static void gm_matvec(const gm_sys* g, const double* x, double* y) {
  const int N = g->N;
  if (g->kind == 1) orc_sparse_prod_up_3d(N, g->col, g->row, g->S, x, x + 3 * (size_t)N, y, y + 3 * (size_t)N);
  else if (g->kind == 2)
    orc_sparse_prod_ns_conv(N, g->col, g->row, g->S, x, x + 3 * (size_t)N, x + 4 * (size_t)N, y,
                            y + 3 * (size_t)N, y + 4 * (size_t)N);
  else orc_sparse_prod_ls(N, g->col, g->row, g->lhs_tem, x, y);
}

/* diagonal block extraction + inversion: SparseGMRES_NS.f90:53-121,
 * SparseGMRES_NS_conv.f:54-139, SparseGMRES_tem.f90:38-58 */
static void gm_setup_precond(gm_sys* g) {
  const int N = g->N;
  for (int i = 0; i < N; ++i) {
    double Kd[9] = {0}, md = 0.0, lsd = 0.0;
    for (int j = g->col[i] - 1; j < g->col[i + 1] - 1; ++j)
      if (g->row[j] - 1 == i) {
        if (g->kind == 3) md = g->lhs_tem[j];
        else {
          for (int t = 0; t < 9; ++t) Kd[t] = g->S->K11[(size_t)j * 9 + t];
          md = g->S->M[j];
          if (g->kind == 2) lsd = g->S->LS[j];
        }
      }
    if (g->kind != 3) {
      double* B = g->Binv + (size_t)i * 9;
      double b11 = Kd[4] * Kd[8] - Kd[7] * Kd[5];
      double b12 = Kd[7] * Kd[2] - Kd[1] * Kd[8];
      double b13 = Kd[1] * Kd[5] - Kd[2] * Kd[4];
      double tmp2 = b11 * Kd[0] + b12 * Kd[3] + b13 * Kd[6];
      double tmp = 1.0 / tmp2;
      B[0] = b11 * tmp; B[1] = b12 * tmp; B[2] = b13 * tmp;
      B[3] = (Kd[5] * Kd[6] - Kd[3] * Kd[8]) * tmp;
      B[4] = (Kd[0] * Kd[8] - Kd[6] * Kd[2]) * tmp;
      B[5] = (Kd[3] * Kd[2] - Kd[0] * Kd[5]) * tmp;
      B[6] = (Kd[3] * Kd[7] - Kd[4] * Kd[6]) * tmp;
      B[7] = (Kd[6] * Kd[1] - Kd[0] * Kd[7]) * tmp;
      B[8] = (Kd[0] * Kd[4] - Kd[1] * Kd[3]) * tmp;
    }
    g->pinv[i] = (md == 0.0) ? 1.0 : 1.0 / md;
    if (g->kind == 2) g->lsinv[i] = (lsd == 0.0) ? 0.0 : 1.0 / lsd;
  }
}

/* The Arnoldi/MGS/Givens cycle common to SparseGMRES_up
 * (SparseGMRES_NS.f90:124-352), SparseGMRES_ns_conv (.f:142-385) and
 * SparseGMRES_tem (.f90:60-230).  rhs and sol are field-major. */
static int gm_cycle(gm_sys* g, const double* rhs, double tol, int kspace,
                    int kmin, double* sol, int* iters, double* erc_out,
                    double* res0_out) {
  const int N = g->N, nf = gm_nf(g);
  const size_t V = (size_t)N * nf;
  const int tem = g->kind == 3;
  if (tem) {
    double rr0 = 0.0;
    for (int i = 0; i < N; ++i) rr0 += rhs[i] * rhs[i];
    if (rr0 == 0.0) {  /* SparseGMRES_tem.f90:68-71 */
      for (int i = 0; i < N; ++i) sol[i] = 0.0;
      *iters = 0; *erc_out = 0.0; *res0_out = 0.0;
      return 0;
    }
  }
  double* U = (double*)calloc(V * (size_t)(kspace + 1), sizeof(double));
  double* H = (double*)calloc((size_t)(kspace + 1) * kspace, sizeof(double));
  double* e = (double*)calloc((size_t)kspace + 1, sizeof(double));
  double* y = (double*)calloc((size_t)kspace, sizeof(double));
  double* rc = (double*)calloc((size_t)kspace, sizeof(double));
  double* rs = (double*)calloc((size_t)kspace, sizeof(double));
  if (!U || !H || !e || !y || !rc || !rs) return OVS_ERR_NOMEM;
#define HH(j, k) H[(size_t)(k) * (kspace + 1) + (j)]
  memcpy(U, rhs, sizeof(double) * V);
  gm_precond(g, U);
  double unorm = sqrt(gm_dot(g, U, U));
  *res0_out = unorm;
  double epsnrm = tol * unorm;
  e[0] = unorm;
  if (tem) { double inv = 1.0 / unorm; for (size_t t = 0; t < V; ++t) U[t] *= inv; }
  else for (size_t t = 0; t < V; ++t) U[t] /= unorm;
  int iks = 0;
  double ercheck = 0.0;
  for (int ik = 1; ik <= kspace; ++ik) {
    iks = ik;
    double* w = U + V * (size_t)iks;
    gm_matvec(g, U + V * (size_t)(iks - 1), w);
    gm_precond(g, w);
    double beta = 0.0;
    for (int jk = 1; jk <= iks + 1; ++jk) {
      if (jk > 1) {
        const double* vp = U + V * (size_t)(jk - 2);
        for (size_t t = 0; t < V; ++t) w[t] = w[t] - beta * vp[t];
      }
      beta = gm_dot(g, w, U + V * (size_t)(jk - 1));
      HH(jk - 1, iks - 1) = beta;
    }
    unorm = sqrt(beta);
    HH(iks, iks - 1) = unorm;
    if (tem) { double inv = 1.0 / unorm; for (size_t t = 0; t < V; ++t) w[t] = w[t] * inv; }
    else for (size_t t = 0; t < V; ++t) w[t] = w[t] / unorm;
    for (int jk = 1; jk <= iks - 1; ++jk) {
      double tmp = rc[jk - 1] * HH(jk - 1, iks - 1) + rs[jk - 1] * HH(jk, iks - 1);
      HH(jk, iks - 1) = -rs[jk - 1] * HH(jk - 1, iks - 1) + rc[jk - 1] * HH(jk, iks - 1);
      HH(jk - 1, iks - 1) = tmp;
    }
    double a = HH(iks - 1, iks - 1), b = HH(iks, iks - 1);
    double tmp = sqrt(a * a + b * b);
    if (tem) { double t1 = 1.0 / tmp; rc[iks - 1] = a * t1; rs[iks - 1] = b * t1; }
    else { rc[iks - 1] = a / tmp; rs[iks - 1] = b / tmp; }
    HH(iks - 1, iks - 1) = tmp;
    HH(iks, iks - 1) = 0.0;
    tmp = rc[iks - 1] * e[iks - 1] + rs[iks - 1] * e[iks];
    e[iks] = -rs[iks - 1] * e[iks - 1] + rc[iks - 1] * e[iks];
    e[iks - 1] = tmp;
    ercheck = fabs(e[iks]);
    if (ercheck <= epsnrm && iks >= kmin) break;
  }
  for (int jk = iks; jk >= 1; --jk) {
    y[jk - 1] = e[jk - 1] / HH(jk - 1, jk - 1);
    for (int lk = 1; lk <= jk - 1; ++lk) e[lk - 1] = e[lk - 1] - y[jk - 1] * HH(lk - 1, jk - 1);
  }
  for (int jk = 1; jk <= iks; ++jk) {
    const double* vj = U + V * (size_t)(jk - 1);
    for (size_t t = 0; t < V; ++t) sol[t] = sol[t] + y[jk - 1] * vj[t];
  }
#undef HH
  *iters = iks;
  *erc_out = ercheck;
  free(U); free(H); free(e); free(y); free(rc); free(rs);
  return 0;
}

int orc_gmres_up(int N, const int* col, const int* row, const orc_system* S,
                 double tol, int kspace, int kspace_min, double* solu,
                 double* solp, int* iters, double* erc, double* res0) {
  gm_sys g = {1, N, col, row, S, NULL, NULL, NULL, NULL};
  g.Binv = (double*)malloc(sizeof(double) * (size_t)N * 9);
  g.pinv = (double*)malloc(sizeof(double) * (size_t)N);
  double* rhs = (double*)malloc(sizeof(double) * (size_t)N * 4);
  double* sol = (double*)malloc(sizeof(double) * (size_t)N * 4);
  memcpy(rhs, S->rhsu, sizeof(double) * 3 * (size_t)N);
  memcpy(rhs + 3 * (size_t)N, S->rhsp, sizeof(double) * (size_t)N);
  memcpy(sol, solu, sizeof(double) * 3 * (size_t)N);
  memcpy(sol + 3 * (size_t)N, solp, sizeof(double) * (size_t)N);
  gm_setup_precond(&g);
  int st = gm_cycle(&g, rhs, tol, kspace, kspace_min, sol, iters, erc, res0);
  memcpy(solu, sol, sizeof(double) * 3 * (size_t)N);
  memcpy(solp, sol + 3 * (size_t)N, sizeof(double) * (size_t)N);
  free(g.Binv); free(g.pinv); free(rhs); free(sol);
  return st;
}

int orc_gmres_ns_conv(int N, const int* col, const int* row,
                      const orc_system* S, double tol, int kspace,
                      int kspace_min, double* solu, double* solp,
                      double* solls, int* iters, double* erc, double* res0) {
  gm_sys g = {2, N, col, row, S, NULL, NULL, NULL, NULL};
  g.Binv = (double*)malloc(sizeof(double) * (size_t)N * 9);
  g.pinv = (double*)malloc(sizeof(double) * (size_t)N);
  g.lsinv = (double*)malloc(sizeof(double) * (size_t)N);
  double* rhs = (double*)malloc(sizeof(double) * (size_t)N * 5);
  double* sol = (double*)malloc(sizeof(double) * (size_t)N * 5);
  memcpy(rhs, S->rhsu, sizeof(double) * 3 * (size_t)N);
  memcpy(rhs + 3 * (size_t)N, S->rhsp, sizeof(double) * (size_t)N);
  memcpy(rhs + 4 * (size_t)N, S->rhsls, sizeof(double) * (size_t)N);
  memcpy(sol, solu, sizeof(double) * 3 * (size_t)N);
  memcpy(sol + 3 * (size_t)N, solp, sizeof(double) * (size_t)N);
  memcpy(sol + 4 * (size_t)N, solls, sizeof(double) * (size_t)N);
  gm_setup_precond(&g);
  int st = gm_cycle(&g, rhs, tol, kspace, kspace_min, sol, iters, erc, res0);
  memcpy(solu, sol, sizeof(double) * 3 * (size_t)N);
  memcpy(solp, sol + 3 * (size_t)N, sizeof(double) * (size_t)N);
  memcpy(solls, sol + 4 * (size_t)N, sizeof(double) * (size_t)N);
  free(g.Binv); free(g.pinv); free(g.lsinv); free(rhs); free(sol);
  return st;
}

int orc_gmres_tem(int N, const int* col, const int* row, const double* lhs,
                  const double* rhs, double tol, int kspace, int kspace_min,
                  double* sol, int* iters, double* erc, double* res0) {
  gm_sys g = {3, N, col, row, NULL, lhs, NULL, NULL, NULL};
  g.pinv = (double*)malloc(sizeof(double) * (size_t)N);
  gm_setup_precond(&g);
  int st = gm_cycle(&g, rhs, tol, kspace, kspace_min, sol, iters, erc, res0);
  free(g.pinv);
  return st;
}

/* Newton update: src/solveFlow.f90:99-104 (NS, VOF), :139-140 (T);
 * sol is field-major (N,nf) */
void orc_newton_update(int N, int system, const ovs_params* p, orc_state* s,
                       const double* sol) {
  const double gdt = p->gami * p->delt;
  if (system == OVS_SYS_TEM) {
    for (int i = 0; i < N; ++i) { s->rtg[i] = s->rtg[i] + sol[i]; s->tg[i] = s->tg[i] + gdt * sol[i]; }
    return;
  }
  for (size_t i = 0; i < (size_t)N * 3; ++i) {
    s->acg[i] = s->acg[i] + sol[i];
    s->ug[i] = s->ug[i] + gdt * sol[i];
  }
  for (int i = 0; i < N; ++i) s->pg[i] = s->pg[i] + p->alfi * p->gami * p->delt * sol[3 * (size_t)N + i];
  if (system == OVS_SYS_NSVOF)
    for (int i = 0; i < N; ++i) {
      s->rphig[i] = s->rphig[i] + sol[4 * (size_t)N + i];
      s->phig[i] = s->phig[i] + gdt * sol[4 * (size_t)N + i];
    }
}

/* calculate_residual src/solveFlow.f90:169-187 (sums of squares) */
void orc_calculate_residual(int N, const orc_system* S, double r[4]) {
  double a = 0, b = 0, c = 0, d = 0;
  for (size_t i = 0; i < (size_t)N * 3; ++i) a += S->rhsu[i] * S->rhsu[i];
  for (int i = 0; i < N; ++i) {
    b += S->rhsp[i] * S->rhsp[i];
    if (S->rhsls) c += S->rhsls[i] * S->rhsls[i];
    if (S->rhstem) d += S->rhstem[i] * S->rhstem[i];
  }
  r[0] = a; r[1] = b; r[2] = c; r[3] = d;
}
