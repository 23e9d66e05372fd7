/*
 * ovs_abi_driver.c - a plain C99 consumer of include/ovs.h, standing where
 * the Fortran shim would call the library (no Fortran compiler exists on
 * these machines).  It links libovs_b200.so and uses only the header.
 *
 *   ovs_abi_driver abi        stateless calls and argument checks; creates
 *                             and destroys one context when a device exists
 *                             (exit 0 either way, "device: none|present")
 *   ovs_abi_driver cavity [n] one Newton step of the NS-only lid-driven
 *                             cavity on an n^3 x 6-tet unit cube (the
 *                             reference's NS path: genSparStruc,
 *                             assembleNavSto, SparseGMRES_up, the Newton
 *                             update of src/solveFlow.f90:99-104), with
 *                             checks made here in C (exit 77: no device)
 *   ovs_abi_driver mesh n file writes the cavity's xg(N,3) doubles then
 *                             IEN(E,4) ints to `file` and prints the
 *                             closed-form pattern count (no library call)
 *
 * The mesh is built here, independently of the Python mesh module: nodes
 * lexicographic (x fastest), every cell split into the 6 Kuhn tets around
 * its (0,0,0)-(1,1,1) diagonal, each tet ordered so that
 * det[x1-x4, x2-x4, x3-x4] > 0 (the sign eval_shape_fem expects,
 * src/eval_shape_FEM.f90:54-60).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ovs.h"

static int failures = 0;

#define EXPECT(cond, ...)                                   \
  do {                                                      \
    if (!(cond)) {                                          \
      fprintf(stderr, "FAIL %s:%d: ", __FILE__, __LINE__);  \
      fprintf(stderr, __VA_ARGS__);                         \
      fprintf(stderr, "\n");                                \
      ++failures;                                           \
    }                                                       \
  } while (0)

#define CALL(expr)                                                           \
  do {                                                                       \
    int st_ = (expr);                                                        \
    if (st_ < 0) {                                                           \
      fprintf(stderr, "FAIL %s:%d: %s -> %d (%s)\n", __FILE__, __LINE__,     \
              #expr, st_, ovs_status_string(st_));                           \
      ovs_destroy(ctx);                                                      \
      return 1;                                                              \
    }                                                                        \
  } while (0)

/* ------------------------------------------------------------------ abi */

static int close_to(double a, double b) { return fabs(a - b) <= 1e-15 * fabs(b); }

static int run_abi(void) {
  int codes[] = {OVS_OK, OVS_WARN_NEG_DETJ, OVS_ERR_ARG, OVS_ERR_CUDA, OVS_ERR_NOMEM, OVS_ERR_STATE,
                 OVS_ERR_NONFINITE, OVS_ERR_PATTERN, OVS_ERR_NODEVICE, OVS_ERR_TIMEOUT};
  size_t i;
  ovs_params p;
  ovs_ctx* ctx = NULL;
  ovs_dims dims;
  int icnt = 0, st;
  double r[4];
  double rho = 0.5, almi, alfi;

  EXPECT(ovs_version() >= 10000, "version %d", ovs_version());
  for (i = 0; i < sizeof codes / sizeof codes[0]; ++i) {
    const char* s = ovs_status_string(codes[i]);
    EXPECT(s != NULL && s[0] != '\0', "no text for status %d", codes[i]);
  }

  /* generalized-alpha constants of src/param.f90:469-480 */
  memset(&p, 0, sizeof p);
  EXPECT(ovs_params_genalpha(rho, &p) == OVS_OK, "genalpha");
  almi = (3.0 - rho) / (1.0 + rho) / 2.0;
  alfi = 1.0 / (1.0 + rho);
  EXPECT(close_to(p.almi, almi) && close_to(p.alfi, alfi), "almi %.17g alfi %.17g", p.almi, p.alfi);
  EXPECT(close_to(p.gami, 0.5 + almi - alfi), "gami %.17g", p.gami);
  EXPECT(close_to(p.beti, 0.25 * (1.0 + almi - alfi) * (1.0 + almi - alfi)), "beti %.17g", p.beti);
  EXPECT(ovs_params_genalpha(2.0, &p) == OVS_OK && p.almi == 1.0 && p.alfi == 1.0 && p.gami == 1.0 &&
             p.beti == 1.0,
         "backward Euler outside [0,1]");
  EXPECT(ovs_params_genalpha(0.5, NULL) == OVS_ERR_ARG, "genalpha(NULL)");

  /* argument errors need no device */
  EXPECT(ovs_create(NULL, NULL) == OVS_ERR_ARG, "create(NULL)");
  dims.nnode = 0; dims.nelem = 10; dims.nshl = 4; dims.device = 0;
  EXPECT(ovs_create(&ctx, &dims) == OVS_ERR_ARG && ctx == NULL, "create with nnode 0");
  dims.nnode = 10; dims.nshl = 5;
  EXPECT(ovs_create(&ctx, &dims) == OVS_ERR_ARG && ctx == NULL, "create with nshl 5");
  EXPECT(ovs_destroy(NULL) == OVS_OK, "destroy(NULL)");
  EXPECT(ovs_build_pattern(NULL, &icnt) == OVS_ERR_ARG, "build_pattern(NULL)");
  EXPECT(ovs_set_params(NULL, &p) == OVS_ERR_ARG, "set_params(NULL)");
  EXPECT(ovs_assemble(NULL, OVS_ASM_NS, OVS_TENSOR_MAT | OVS_TENSOR_VEC, OVS_FP64, NULL) == OVS_ERR_ARG,
         "assemble(NULL)");
  EXPECT(ovs_residual_norms(NULL, OVS_FP64, r) == OVS_ERR_ARG, "residual_norms(NULL)");
  EXPECT(ovs_newton_update(NULL, OVS_SYS_NS) == OVS_ERR_ARG, "newton_update(NULL)");
  EXPECT(ovs_gen_spar_struc(4, 1, 4, NULL, NULL, NULL, &icnt) == OVS_ERR_ARG, "gen_spar_struc(NULL)");

  /* the stateless input checks: one tet, its four faces, two boundaries */
  {
    const int f2e[4] = {1, 1, 1, 1}, face_or[4] = {1, 2, 3, 4};
    int flags[4] = {OVS_FACE_WEAK, 0, OVS_FACE_CONVH, 0};
    const double hconv[4] = {5.0, 0.0, 5.0, 0.0}, tinf[4] = {300.0, 0.0, 300.0, 0.0};
    const int face_id[2] = {2, 1}, bnode_ptr[3] = {0, 3, 5}, bnodes[5] = {1, 2, 3, 3, 4};
    const int ut[2 * 3] = {1, 0, 1, 1, 0, 1}, pt[2] = {0, 1}, tt[2] = {1, 0};
    const double uv[2 * 3] = {0.0, 1.0, 0.0, 0.0, 0.0, 0.0}, pv[2] = {0.0, 1.0}, tv[2] = {300.0, 0.0};
    ovs_bc_spec sp;
    int bad_nodes[5] = {1, 2, 3, 3, 5};
    EXPECT(ovs_check_faces(1, 4, f2e, face_or, flags, hconv, tinf) == OVS_OK, "check_faces");
    EXPECT(ovs_check_faces(1, 4, f2e, face_or, flags, NULL, NULL) == OVS_ERR_ARG, "check_faces without tables");
    flags[1] = 8;
    EXPECT(ovs_check_faces(1, 4, f2e, face_or, flags, hconv, tinf) == OVS_ERR_ARG, "check_faces bad flag");
    memset(&sp, 0, sizeof sp);
    sp.nbound = 2; sp.ntype = 2; sp.face_id = face_id; sp.bnode_ptr = bnode_ptr; sp.bnodes = bnodes;
    sp.bcug_type = ut; sp.bcug_valu = uv; sp.bcphig_type = pt; sp.bcphig_valu = pv;
    sp.bctg_type = tt; sp.bctg_valu = tv;
    EXPECT(ovs_check_bc_spec(&sp, 4) == OVS_OK, "check_bc_spec");
    sp.bnodes = bad_nodes;
    EXPECT(ovs_check_bc_spec(&sp, 4) == OVS_ERR_ARG, "check_bc_spec node out of range");
  }

  dims.nnode = 4; dims.nelem = 1; dims.nshl = 4; dims.device = -1;
  st = ovs_create(&ctx, &dims);
  if (st == OVS_ERR_NODEVICE) {
    EXPECT(ctx == NULL, "context returned without a device");
    printf("device: none\n");
  } else {
    EXPECT(st == OVS_OK && ctx != NULL, "create -> %d (%s)", st, ovs_status_string(st));
    EXPECT(ovs_build_pattern(ctx, &icnt) == OVS_ERR_STATE, "pattern before mesh");
    EXPECT(ovs_destroy(ctx) == OVS_OK, "destroy");
    printf("device: present\n");
  }
  printf("abi checks: %d failure(s)\n", failures);
  return failures ? 1 : 0;
}

/* --------------------------------------------------------------- cavity */

typedef struct {
  int n, N, E;
  double* xg;  /* (N,3) */
  int* ien;    /* (E,4), 1-based */
} box_mesh;

static int node_id(int n, int i, int j, int k) { return i + (n + 1) * (j + (n + 1) * k); }

static double det3(const double* a, const double* b, const double* c) {
  return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]);
}

static void make_box(int n, box_mesh* m) {
  /* the 6 monotone paths from corner (0,0,0) to (1,1,1), one per axis order */
  static const int order[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  int i, j, k, t, a, d, e = 0;
  const double h = 1.0 / n;
  m->n = n;
  m->N = (n + 1) * (n + 1) * (n + 1);
  m->E = 6 * n * n * n;
  m->xg = (double*)malloc(sizeof(double) * 3 * (size_t)m->N);
  m->ien = (int*)malloc(sizeof(int) * 4 * (size_t)m->E);
  for (k = 0; k <= n; ++k)
    for (j = 0; j <= n; ++j)
      for (i = 0; i <= n; ++i) {
        int id = node_id(n, i, j, k);
        m->xg[id] = i * h;
        m->xg[m->N + id] = j * h;
        m->xg[2 * (size_t)m->N + id] = k * h;
      }
  for (k = 0; k < n; ++k)
    for (j = 0; j < n; ++j)
      for (i = 0; i < n; ++i)
        for (t = 0; t < 6; ++t) {
          int off[3] = {0, 0, 0}, v[4], tmp;
          double x[4][3], d1[3], d2[3], d3[3];
          v[0] = node_id(n, i, j, k);
          for (a = 0; a < 3; ++a) {
            off[order[t][a]] = 1;
            v[a + 1] = node_id(n, i + off[0], j + off[1], k + off[2]);
          }
          /* local order (P1, P2, P3, P0); swap P1, P2 when negatively oriented */
          tmp = v[0]; v[0] = v[1]; v[1] = v[2]; v[2] = v[3]; v[3] = tmp;
          for (a = 0; a < 4; ++a)
            for (d = 0; d < 3; ++d) x[a][d] = m->xg[(size_t)d * m->N + v[a]];
          for (d = 0; d < 3; ++d) {
            d1[d] = x[0][d] - x[3][d];
            d2[d] = x[1][d] - x[3][d];
            d3[d] = x[2][d] - x[3][d];
          }
          if (det3(d1, d2, d3) < 0.0) { tmp = v[0]; v[0] = v[1]; v[1] = tmp; }
          for (a = 0; a < 4; ++a) m->ien[(size_t)a * m->E + e] = v[a] + 1;
          ++e;
        }
}

/* entries of the node adjacency of a Kuhn-split box: every node plus both
 * directions of every edge (axis edges, one diagonal per cell face, one body
 * diagonal per cell) */
static long kuhn_nnz(int n) {
  long n1 = n + 1;
  long edges = 3L * n * n1 * n1 + 3L * n * n * n1 + (long)n * n * n;
  return n1 * n1 * n1 + 2 * edges;
}

static double dot(const double* a, const double* b, size_t len) {
  double s = 0.0;
  size_t i;
  for (i = 0; i < len; ++i) s += a[i] * b[i];
  return s;
}

static int run_cavity(int n) {
  box_mesh m;
  ovs_ctx* ctx = NULL;
  ovs_dims dims;
  ovs_params p;
  ovs_solve_info sinfo;
  ovs_gmres_info ginfo;
  int icnt = 0, icnt2 = 0, st, i, d, bad = 0;
  int *col, *row, *col2, *row2, *ibc;
  double *ug, *ugold, *acg, *sol, *sol2, *rhs, *ax;
  double r0[4], r1[4], cfl = 0.0, rel;
  unsigned long long lcg = 12345;
  size_t N, n4;

  make_box(n, &m);
  N = (size_t)m.N;
  n4 = 4 * N;
  dims.nnode = m.N; dims.nelem = m.E; dims.nshl = 4; dims.device = -1;
  st = ovs_create(&ctx, &dims);
  if (st == OVS_ERR_NODEVICE) {
    printf("cavity: no CUDA device\n");
    return 77;
  }
  CALL(st);

  /* genSparStruc, resident and stateless; both equal the closed-form count */
  CALL(ovs_upload_mesh(ctx, m.xg, m.ien, NULL));
  CALL(ovs_build_pattern(ctx, &icnt));
  EXPECT(icnt == kuhn_nnz(n), "icnt %d, expected %ld", icnt, kuhn_nnz(n));
  col = (int*)malloc(sizeof(int) * (N + 1));
  row = (int*)malloc(sizeof(int) * (size_t)icnt);
  col2 = (int*)malloc(sizeof(int) * (N + 1));
  row2 = (int*)malloc(sizeof(int) * (size_t)icnt);
  CALL(ovs_get_pattern(ctx, col, row));
  EXPECT(col[0] == 1 && col[N] == icnt + 1, "row pointer ends %d %d", col[0], col[N]);
  for (i = 0; i < m.N && !bad; ++i) {
    int k, self = 0;
    for (k = col[i] - 1; k < col[i + 1] - 1; ++k) {
      if (row[k] < 1 || row[k] > m.N || (k > col[i] - 1 && row[k] <= row[k - 1])) bad = 1;
      if (row[k] == i + 1) self = 1;
    }
    if (!self) bad = 1;
  }
  EXPECT(!bad, "pattern rows not sorted, unique, 1-based and holding the diagonal");
  icnt2 = icnt;
  CALL(ovs_gen_spar_struc(m.N, m.E, 4, m.ien, col2, row2, &icnt2));
  EXPECT(icnt2 == icnt && !memcmp(col, col2, sizeof(int) * (N + 1)) &&
             !memcmp(row, row2, sizeof(int) * (size_t)icnt),
         "ovs_gen_spar_struc differs from the resident pattern");

  /* config-1 physics: rho = 1, mu = 0.01, Delt = 0.01, rho_inf = 0.5 */
  memset(&p, 0, sizeof p);
  CALL(ovs_params_genalpha(0.5, &p));
  p.delt = 0.01;
  p.rhow = p.rhoa = 1.0;
  p.muw = p.mua = 0.01;
  p.rhos = 2700.0; p.mus = 1.0;
  p.cpw = 4180.0; p.cpa = 1000.0; p.cps = 900.0;
  p.kappaw = 0.6; p.kappaa = 0.03; p.kappas = 200.0;
  p.ts = 373.0; p.lh = 2.26e6; p.c_dmdot = 1.0; p.tref = 1.0;
  p.gravvec[2] = -9.81;
  p.fluid_elm_id = 102; p.subdomain_flag = 1; p.elm_id_set[0] = 102;
  CALL(ovs_set_params(ctx, &p));

  /* predictor ug = ugold (acgold = 0, so acg = 0); walls u = 0, lid z = 1
   * u = (1,0,0), with acg from setBCs_NSVOF (src/setBCs.f90:210-220); the
   * pressure is held on the lid (IBC column 4), which removes the constant
   * pressure mode of the closed cavity */
  ug = (double*)calloc(3 * N, sizeof(double));
  ugold = (double*)calloc(3 * N, sizeof(double));
  acg = (double*)calloc(3 * N, sizeof(double));
  ibc = (int*)calloc(8 * N, sizeof(int));
  for (i = 0; i < 3 * m.N; ++i) {
    lcg = lcg * 6364136223846793005ULL + 1442695040888963407ULL;
    ugold[i] = ug[i] = ((double)(lcg >> 11) / 9007199254740992.0 - 0.5) * 0.02;
  }
  for (i = 0; i < m.N; ++i) {
    int ii = i % (n + 1), jj = (i / (n + 1)) % (n + 1), kk = i / ((n + 1) * (n + 1));
    if (ii == 0 || ii == n || jj == 0 || jj == n || kk == 0 || kk == n) {
      for (d = 0; d < 3; ++d) {
        size_t q = (size_t)d * N + i;
        ibc[q] = 1;
        ug[q] = (kk == n && d == 0) ? 1.0 : 0.0;
        acg[q] = ((ug[q] - ugold[q]) / p.delt) / p.gami;
      }
      if (kk == n) ibc[3 * N + i] = 1;
    }
  }
  CALL(ovs_set_ibc(ctx, ibc, 8));
  CALL(ovs_set_field(ctx, OVS_F_UGOLD, ugold));
  CALL(ovs_set_field(ctx, OVS_F_UG, ug));
  CALL(ovs_set_field(ctx, OVS_F_ACG, acg));

  /* assembleNavSto(MAT+VEC); the reference GMRES cycle; a refined solve */
  st = ovs_assemble(ctx, OVS_ASM_NS, OVS_TENSOR_MAT | OVS_TENSOR_VEC, OVS_FP64, &cfl);
  CALL(st);
  EXPECT(st == OVS_OK, "assembly warning %d", st);
  EXPECT(cfl > 0.0 && cfl < 1e3, "cfl %g", cfl);
  CALL(ovs_residual_norms(ctx, OVS_FP64, r0));
  EXPECT(r0[0] > 0.0 && isfinite(r0[0]) && isfinite(r0[1]), "residual %g %g", r0[0], r0[1]);

  sol = (double*)calloc(n4, sizeof(double));
  sol2 = (double*)calloc(n4, sizeof(double));
  rhs = (double*)malloc(sizeof(double) * n4);
  ax = (double*)malloc(sizeof(double) * n4);
  CALL(ovs_gmres(ctx, OVS_SYS_NS, 1e-6, 50, 1, sol2, &ginfo));
  EXPECT(ginfo.iterations >= 1 && ginfo.iterations <= 50 && ginfo.res0 > 0.0, "gmres its %d res0 %g",
         ginfo.iterations, ginfo.res0);
  EXPECT(!ginfo.converged || ginfo.ercheck <= 1e-6 * ginfo.res0, "gmres ercheck %g", ginfo.ercheck);

  CALL(ovs_solve(ctx, OVS_SYS_NS, OVS_FP64, 1e-8, 50, 40, sol, &sinfo));
  EXPECT(sinfo.converged && sinfo.rel_residual <= 1e-8, "solve rel %g", sinfo.rel_residual);
  /* the true residual, recomputed here from the assembled system */
  CALL(ovs_get_rhs(ctx, OVS_SYS_NS, OVS_FP64, rhs));
  CALL(ovs_spmv(ctx, OVS_SYS_NS, OVS_FP64, sol, ax));
  for (i = 0; i < (int)n4; ++i) ax[i] = rhs[i] - ax[i];
  rel = sqrt(dot(ax, ax, n4) / dot(rhs, rhs, n4));
  EXPECT(rel <= 1e-7, "||b - A x|| / ||b|| = %g", rel);
  for (i = 0, bad = 0; i < m.N; ++i)
    for (d = 0; d < 3; ++d)
      if (ibc[(size_t)d * N + i] && sol[(size_t)d * N + i] != 0.0) bad = 1;
  EXPECT(!bad, "non-zero update at a Dirichlet velocity dof");

  /* Newton update, then the residual of the updated state */
  CALL(ovs_newton_update(ctx, OVS_SYS_NS));
  CALL(ovs_assemble(ctx, OVS_ASM_NS, OVS_TENSOR_VEC, OVS_FP64, NULL));
  CALL(ovs_residual_norms(ctx, OVS_FP64, r1));
  EXPECT(r1[0] < 1e-2 * r0[0], "momentum residual %g -> %g", r0[0], r1[0]);

  printf("cavity n=%d N=%d E=%d icnt=%d gmres_its=%d solve_its=%d rel=%.3e res %.3e -> %.3e\n", n, m.N, m.E,
         icnt, ginfo.iterations, sinfo.iterations, rel, r0[0], r1[0]);
  printf("cavity checks: %d failure(s)\n", failures);
  ovs_destroy(ctx);
  free(m.xg); free(m.ien); free(col); free(row); free(col2); free(row2); free(ibc);
  free(ug); free(ugold); free(acg); free(sol); free(sol2); free(rhs); free(ax);
  return failures ? 1 : 0;
}

static int run_mesh(int n, const char* path) {
  box_mesh m;
  FILE* f = fopen(path, "wb");
  size_t ok;
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    return 2;
  }
  make_box(n, &m);
  ok = fwrite(m.xg, sizeof(double), 3 * (size_t)m.N, f) == 3 * (size_t)m.N &&
       fwrite(m.ien, sizeof(int), 4 * (size_t)m.E, f) == 4 * (size_t)m.E;
  fclose(f);
  printf("mesh n=%d N=%d E=%d nnz=%ld\n", n, m.N, m.E, kuhn_nnz(n));
  free(m.xg);
  free(m.ien);
  return ok ? 0 : 1;
}

int main(int argc, char** argv) {
  if (argc >= 2 && !strcmp(argv[1], "abi")) return run_abi();
  if (argc >= 4 && !strcmp(argv[1], "mesh")) {
    int n = atoi(argv[2]);
    if (n < 1 || n > 256) {
      fprintf(stderr, "mesh size out of range\n");
      return 2;
    }
    return run_mesh(n, argv[3]);
  }
  if (argc >= 2 && !strcmp(argv[1], "cavity")) {
    int n = argc >= 3 ? atoi(argv[2]) : 8;
    if (n < 1 || n > 256) {
      fprintf(stderr, "cavity size out of range\n");
      return 2;
    }
    return run_cavity(n);
  }
  fprintf(stderr, "usage: %s abi | cavity [n] | mesh n file\n", argv[0]);
  return 2;
}
