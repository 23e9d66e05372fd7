// Face assemblies on boundary faces of linear tets:
//   FaceAssembly_NS_weak (Nitsche weak Dirichlet) and FaceAssembly_NS_outflow
//   (backflow), src/FaceAssembly_weak.f90:4-409, with e3bSTAB_weak
//   src/e3STAB.f90:256-287, e3bLHS_weak src/e3LHS.f90:167-294, e3bRHS_weak
//   src/e3RHS.f90:105-170, eval_faceshape_tet src/eval_shape_FEM.f90:66-143,
//   the face rules genGPandGWtri / genGPtritet src/genGP_GW.f90:436-572;
//   and the convective heat flux h (T - T_inf) on the temperature system that
//   the quench driver calls as FaceAssembly_ConvectiveH
//   (src/solveQuenching.f90:92) and the reference never defines.
//
// Boundary faces number O(N^(2/3)), so this pass is laid out for
// determinism rather than bandwidth:
//   face_ns_kernel / face_tem_kernel: one thread per face builds the face's
//     element arrays in FP64 (both NS face routines, one after the other),
//     applies BCLhs_3D / BCLhs_tem (which, as in the reference, also puts 1 on
//     the diagonal of every constrained node the face element touches) and
//     stores them at the precision of the system;
//   face_scatter_kernel: one thread per node touched by a face element adds
//     its rows in the reference's order (all weak-face terms in face order,
//     then all outflow terms), after the element pass has written the rows,
//     so the sums are reproducible bit for bit without atomics.
#include "ovs_internal.cuh"

#include <math.h>

#include <algorithm>
#include <utility>
#include <vector>

namespace {

constexpr int FW = 272;   // one NS face routine: 16 (a, b) blocks x 16 slot values + 4 nodes x (u1 u2 u3 p)
constexpr int FT = 20;    // temperature: 4 x 4 matrix + 4 RHS values
constexpr uint8_t PB = 8, TB = 32;   // IBC bits: pressure (column 4), temperature (column 6)

// element-local nodes of the face FACE_OR = 1..4 in eval_faceshape_tet order
__constant__ int c_fnodes[4][3] = {{1, 2, 0}, {3, 2, 1}, {0, 2, 3}, {1, 0, 3}};
// genGPtritet, ngp = 3: volume coordinates of the face points per FACE_OR
#define F6 0.166666666666666666667
#define F23 0.666666666666666666667
__constant__ double c_fmgp[4][3][3] = {
    {{F6, F23, F6}, {F6, F6, F23}, {F23, F6, F6}},
    {{0.0, F6, F6}, {0.0, F6, F23}, {0.0, F23, F6}},
    {{F23, 0.0, F6}, {F6, 0.0, F23}, {F6, 0.0, F6}},
    {{F6, F23, 0.0}, {F23, F6, 0.0}, {F6, F6, 0.0}}};
constexpr double c_fgw = F6;   // genGPandGWtri weights

struct FaceArgs {
  const double* f[OVS_F_COUNT];
  const int* ien;
  const int* elm_id;
  const uint8_t* ibc;
  const int* face_e;
  const int* face_info;     // (FACE_OR - 1) | flags << 2
  const double* face_h;     // (h, T_inf) per face
  void* out;
  int nface, N;
  int mat, vec, use_subdomain;
  double alfi, fact2, rhoa, mua;
  int subdomain_flag, elm_id_set0, elm_id_set1;
};

// Face geometry shared by the face points of a linear tet: alpha-stage
// coordinates x + d, global shape gradients and dxi/dx from eval_shape_fem
// (src/eval_shape_FEM.f90:4-61, get_inverse_3x3 src/eval_shape.f90:85-112;
// constant on the element), the unit normal and DetJb of the face triangle.
struct FaceGeo {
  double shg[4][3];
  double dxidx[3][3];
  double nor[3];
  double detjb;
};

__device__ void face_geometry(const FaceArgs& a, const int node[4], int fo, FaceGeo& g) {
  const size_t N = a.N;
  double xl[4][3];
  for (int k = 0; k < 4; ++k)
    for (int d = 0; d < 3; ++d) {
      const size_t i = node[k] + N * d;
      const double dga = a.f[OVS_F_DGOLD][i] + a.alfi * (a.f[OVS_F_DG][i] - a.f[OVS_F_DGOLD][i]);
      xl[k][d] = a.f[OVS_F_XG][i] + dga;
    }
  // lintetshl gradients: node 1..3 unit vectors, node 4 = -(1,1,1)
  double J[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) J[i][j] = xl[j][i] - xl[3][i];
  double Ai[3][3];
  Ai[0][0] = J[1][1] * J[2][2] - J[2][1] * J[1][2];
  Ai[0][1] = J[2][1] * J[0][2] - J[0][1] * J[2][2];
  Ai[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  const double tmp = 1.0 / (Ai[0][0] * J[0][0] + Ai[0][1] * J[1][0] + Ai[0][2] * J[2][0]);
  Ai[0][0] *= tmp; Ai[0][1] *= tmp; Ai[0][2] *= tmp;
  Ai[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * tmp;
  Ai[1][1] = (J[0][0] * J[2][2] - J[2][0] * J[0][2]) * tmp;
  Ai[1][2] = (J[1][0] * J[0][2] - J[0][0] * J[1][2]) * tmp;
  Ai[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * tmp;
  Ai[2][1] = (J[2][0] * J[0][1] - J[0][0] * J[2][1]) * tmp;
  Ai[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * tmp;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) g.dxidx[i][j] = Ai[i][j];
  for (int j = 0; j < 3; ++j) {
    g.shg[0][j] = Ai[0][j];
    g.shg[1][j] = Ai[1][j];
    g.shg[2][j] = Ai[2][j];
    g.shg[3][j] = -Ai[0][j] - Ai[1][j] - Ai[2][j];
  }
  double t1[3], t2[3];
  const int* fn = c_fnodes[fo];
  for (int d = 0; d < 3; ++d) {
    t1[d] = xl[fn[0]][d] - xl[fn[2]][d];
    t2[d] = xl[fn[1]][d] - xl[fn[2]][d];
  }
  double n[3];
  n[0] = t1[1] * t2[2] - t1[2] * t2[1];
  n[1] = t1[2] * t2[0] - t1[0] * t2[2];
  n[2] = t1[0] * t2[1] - t1[1] * t2[0];
  g.detjb = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (int d = 0; d < 3; ++d) g.nor[d] = n[d] / g.detjb;
}

__device__ inline void face_shl(int fo, int ig, double shl[4]) {
  const double* m = c_fmgp[fo][ig];
  shl[0] = m[0];
  shl[1] = m[1];
  shl[2] = m[2];
  shl[3] = 1.0 - m[0] - m[1] - m[2];
}

// BCLhs_3D (src/BCLhs_3D.f90:4-122) on one (a, b) block in slot positions
// 0..15 (K(i,j) at 4i+j, G(i) at 4i+3, D(j) at 12+j, M at 15): zero the
// constrained rows of node a and columns of node b, then 1 on the diagonal.
__device__ inline void bclhs_block(double v[16], uint8_t ra, uint8_t rb, bool same) {
  for (int i = 0; i < 3; ++i)
    if (ra & (1u << i)) { v[4 * i] = v[4 * i + 1] = v[4 * i + 2] = v[4 * i + 3] = 0.0; }
  for (int j = 0; j < 3; ++j)
    if (rb & (1u << j)) { v[j] = v[4 + j] = v[8 + j] = v[12 + j] = 0.0; }
  if (ra & PB) { v[12] = v[13] = v[14] = v[15] = 0.0; }
  if (rb & PB) { v[3] = v[7] = v[11] = 0.0; }
  if (same) {
    for (int i = 0; i < 3; ++i)
      if (ra & (1u << i)) v[5 * i] = 1.0;
    if (ra & PB) v[15] = 1.0;
  }
}

template <typename T>
__global__ void __launch_bounds__(128) face_ns_kernel(const FaceArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.nface) return;
  const int info = a.face_info[f];
  if (!((info >> 2) & OVS_FACE_WEAK)) return;
  const int e = a.face_e[f], fo = info & 3;
  const int4 nd = reinterpret_cast<const int4*>(a.ien)[e];
  const int node[4] = {nd.x, nd.y, nd.z, nd.w};
  const size_t N = a.N;
  FaceGeo g;
  face_geometry(a, node, fo, g);
  double ul[4][3], uml[4][3], pl[4];
  uint8_t bits[4];
  for (int k = 0; k < 4; ++k) {
    for (int d = 0; d < 3; ++d) {
      const size_t i = node[k] + N * d;
      ul[k][d] = a.f[OVS_F_UGOLD][i] + a.alfi * (a.f[OVS_F_UG][i] - a.f[OVS_F_UGOLD][i]);
      uml[k][d] = a.f[OVS_F_UGMOLD][i] + a.alfi * (a.f[OVS_F_UGM][i] - a.f[OVS_F_UGMOLD][i]);
    }
    pl[k] = a.f[OVS_F_PG][node[k]];
    bits[k] = a.ibc[node[k]];
  }
  // per face point: shape values, u, u_mesh (= wall velocity g), p, u_n^-
  double shl[3][4], ui[3][3], gi[3][3], pri[3], uneg[3];
  for (int ig = 0; ig < 3; ++ig) {
    face_shl(fo, ig, shl[ig]);
    pri[ig] = 0.0;
    for (int d = 0; d < 3; ++d) {
      double s1 = 0.0, s2 = 0.0;
      for (int k = 0; k < 4; ++k) { s1 += ul[k][d] * shl[ig][k]; s2 += uml[k][d] * shl[ig][k]; }
      ui[ig][d] = s1;
      gi[ig][d] = s2;
    }
    for (int k = 0; k < 4; ++k) pri[ig] += pl[k] * shl[ig][k];
    const double unor = (ui[ig][0] - gi[ig][0]) * g.nor[0] + (ui[ig][1] - gi[ig][1]) * g.nor[1] +
                        (ui[ig][2] - gi[ig][2]) * g.nor[2];
    uneg[ig] = 0.5 * (unor - fabs(unor));
  }
  double du[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += ul[k][i] * g.shg[k][j];
      du[i][j] = s;
    }
  bool is_target = true;
  if (a.use_subdomain) {
    const int eid = a.elm_id ? a.elm_id[e] : 102;
    is_target = false;
    if (a.subdomain_flag & 1) is_target = is_target || eid == a.elm_id_set0;
    if (a.subdomain_flag & 2) is_target = is_target || eid == a.elm_id_set1;
  }
  // e3bSTAB_weak: h_n = 2 / |dxi/dx n|, tauB = 4 mu / h_n, tauNor = tauB
  double tt[3];
  for (int i = 0; i < 3; ++i)
    tt[i] = g.dxidx[i][0] * g.nor[0] + g.dxidx[i][1] * g.nor[1] + g.dxidx[i][2] * g.nor[2];
  const double hn = 2.0 / sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
  const double mui = a.mua, rhoi = a.rhoa, fact2 = a.fact2;
  const double tauB = 4.0 * mui / hn, tauNor = tauB, munor = tauNor - tauB, gmul = 1.0;
  double tmpn[4];   // grad N_a . n
  for (int k = 0; k < 4; ++k) tmpn[k] = g.shg[k][0] * g.nor[0] + g.shg[k][1] * g.nor[1] + g.shg[k][2] * g.nor[2];
  const double* nor = g.nor;
  T* out = reinterpret_cast<T*>(a.out) + (size_t)f * 2 * FW;
  for (int pass = 0; pass < 2; ++pass) {
    T* o = out + pass * FW;
    const bool on = pass == 1 || is_target;
    if (a.mat) {
      for (int aa = 0; aa < 4; ++aa)
        for (int bb = 0; bb < 4; ++bb) {
          double v[16];
          for (int t = 0; t < 16; ++t) v[t] = 0.0;
          if (on)
            for (int ig = 0; ig < 3; ++ig) {
              const double* s = shl[ig];
              if (pass == 0) {   // e3bLHS_weak
                const double wt = g.detjb * c_fgw;
                const double t2 = -s[aa] * mui * tmpn[bb] - gmul * tmpn[aa] * mui * s[bb] +
                                  s[aa] * tauB * s[bb] - s[aa] * uneg[ig] * rhoi * s[bb];
                for (int i = 0; i < 3; ++i)
                  for (int j = 0; j < 3; ++j) {
                    double w = -s[aa] * mui * g.shg[bb][i] * nor[j] - gmul * g.shg[aa][j] * nor[i] * mui * s[bb] +
                               s[aa] * nor[i] * munor * nor[j] * s[bb];
                    if (i == j) w = t2 + w;
                    v[4 * i + j] += fact2 * w * wt;
                  }
                for (int d = 0; d < 3; ++d) {
                  v[12 + d] -= fact2 * s[aa] * s[bb] * nor[d] * wt;
                  v[4 * d + 3] += fact2 * s[aa] * s[bb] * nor[d] * wt;
                }
              } else {           // FaceAssembly_NS_outflow :361-373
                const double detjgw = g.detjb * c_fgw;
                const double t2 = -s[aa] * uneg[ig] * rhoi * s[bb];
                for (int i = 0; i < 3; ++i) v[5 * i] += fact2 * t2 * detjgw;
              }
            }
          bclhs_block(v, bits[aa], bits[bb], aa == bb);
          T* ob = o + (aa * 4 + bb) * 16;
          for (int t = 0; t < 16; ++t) ob[t] = (T)v[t];
        }
    }
    if (a.vec) {
      for (int aa = 0; aa < 4; ++aa) {
        double r[4] = {0.0, 0.0, 0.0, 0.0};
        if (on)
          for (int ig = 0; ig < 3; ++ig) {
            const double* s = shl[ig];
            const double* u = ui[ig];
            const double* gv = gi[ig];
            if (pass == 0) {   // e3bRHS_weak
              const double wt = g.detjb * c_fgw;
              double ti[3], t1[3], t2[3][3];
              for (int i = 0; i < 3; ++i)
                ti[i] = -pri[ig] * nor[i] + mui * (du[i][0] * nor[0] + du[i][1] * nor[1] + du[i][2] * nor[2] +
                                                   du[0][i] * nor[0] + du[1][i] * nor[1] + du[2][i] * nor[2]);
              const double gnor = gv[0] * nor[0] + gv[1] * nor[1] + gv[2] * nor[2];
              const double unor = u[0] * nor[0] + u[1] * nor[1] + u[2] * nor[2];
              for (int i = 0; i < 3; ++i)
                t1[i] = -ti[i] + tauB * (u[i] - gv[i]) - uneg[ig] * rhoi * (u[i] - gv[i]) +
                        (tauNor - tauB) * unor * nor[i];
              for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q)
                  t2[p][q] = -gmul * mui * ((u[p] - gv[p]) * nor[q] + (u[q] - gv[q]) * nor[p]);
              for (int i = 0; i < 3; ++i)
                r[i] = r[i] - (s[aa] * t1[i] + (g.shg[aa][0] * t2[i][0] + g.shg[aa][1] * t2[i][1] +
                                                g.shg[aa][2] * t2[i][2])) * g.detjb * c_fgw;
              r[3] = r[3] + s[aa] * (unor - gnor) * wt;
            } else {           // FaceAssembly_NS_outflow :353-358
              const double detjgw = g.detjb * c_fgw;
              for (int d = 0; d < 3; ++d) r[d] = r[d] + s[aa] * rhoi * uneg[ig] * (u[d] - gv[d]) * detjgw;
            }
          }
        for (int d = 0; d < 3; ++d)
          if (bits[aa] & (1u << d)) r[d] = 0.0;
        if (bits[aa] & PB) r[3] = 0.0;
        for (int k = 0; k < 4; ++k) o[256 + aa * 4 + k] = (T)r[k];
      }
    }
  }
}

// Convective heat flux q = h (T^alpha - T_inf): residual -int N_a q, tangent
// alpha_f gamma Delt int N_a h N_b (the factor of the element conductivity
// term), face points and DetJb as above, then BCLhs_tem.
template <typename T>
__global__ void __launch_bounds__(128) face_tem_kernel(const FaceArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.nface) return;
  const int info = a.face_info[f];
  if (!((info >> 2) & OVS_FACE_CONVH)) return;
  const int e = a.face_e[f], fo = info & 3;
  const int4 nd = reinterpret_cast<const int4*>(a.ien)[e];
  const int node[4] = {nd.x, nd.y, nd.z, nd.w};
  FaceGeo g;
  face_geometry(a, node, fo, g);
  const double h = a.face_h[2 * (size_t)f], tinf = a.face_h[2 * (size_t)f + 1];
  double Tl[4];
  uint8_t bits[4];
  for (int k = 0; k < 4; ++k) {
    const int i = node[k];
    Tl[k] = a.f[OVS_F_TGOLD][i] + a.alfi * (a.f[OVS_F_TG][i] - a.f[OVS_F_TGOLD][i]);
    bits[k] = a.ibc[i];
  }
  double xT[4][4] = {}, RT[4] = {};
  for (int ig = 0; ig < 3; ++ig) {
    double s[4];
    face_shl(fo, ig, s);
    const double detjgw = g.detjb * c_fgw;
    double Ti = 0.0;
    for (int k = 0; k < 4; ++k) Ti += Tl[k] * s[k];
    const double q = h * (Ti - tinf);
    if (a.mat)
      for (int aa = 0; aa < 4; ++aa)
        for (int bb = 0; bb < 4; ++bb) xT[aa][bb] += a.fact2 * s[aa] * h * s[bb] * detjgw;
    if (a.vec)
      for (int aa = 0; aa < 4; ++aa) RT[aa] -= s[aa] * q * detjgw;
  }
  for (int aa = 0; aa < 4; ++aa)
    if (bits[aa] & TB) {
      for (int t = 0; t < 4; ++t) { xT[aa][t] = 0.0; xT[t][aa] = 0.0; }
      xT[aa][aa] = 1.0;
      RT[aa] = 0.0;
    }
  T* o = reinterpret_cast<T*>(a.out) + (size_t)f * FT;
  for (int aa = 0; aa < 4; ++aa) {
    for (int bb = 0; bb < 4; ++bb) o[aa * 4 + bb] = (T)xT[aa][bb];
    o[16 + aa] = (T)RT[aa];
  }
}

struct ScatterArgs {
  const int* fnode;     // nodes touched by a face element, ascending
  const int* fptr;      // entries of fnode[i]: [fptr[i], fptr[i+1])
  const int* fent;      // (face << 2) | local node, ascending face
  const int* face_e;
  const int* face_info;
  const int* ien;
  const int* rowptr;
  const int* colidx;
  const void* buf;
  void* vals;
  void* rhs;
  int* bad;             // set when a face column is missing from the row
  int nfnode, N, nv;
  int nvb, nrhs, npass, fstride, pstride, flag;
  int mat, vec;
};

template <typename T>
__global__ void __launch_bounds__(128) face_scatter_kernel(const ScatterArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nfnode) return;
  const int A = a.fnode[i];
  const int r0 = a.rowptr[A], r1 = a.rowptr[A + 1];
  const int k0 = a.fptr[i], k1 = a.fptr[i + 1];
  T* vals = reinterpret_cast<T*>(a.vals);
  T* rhs = reinterpret_cast<T*>(a.rhs);
  const T* buf = reinterpret_cast<const T*>(a.buf);
  for (int pass = 0; pass < a.npass; ++pass)
    for (int k = k0; k < k1; ++k) {
      const int ent = a.fent[k], f = ent >> 2, la = ent & 3;
      if (!((a.face_info[f] >> 2) & a.flag)) continue;
      const int e = a.face_e[f];
      const T* src = buf + (size_t)f * a.fstride + (size_t)pass * a.pstride;
      if (a.mat)
        for (int b = 0; b < 4; ++b) {
          const int B = a.ien[4 * (size_t)e + b];
          int slot = r0;
          while (slot < r1 && a.colidx[slot] != B) ++slot;
          if (slot == r1) { *a.bad = 1; continue; }
          T* dst = vals + (size_t)slot * a.nv;
          const T* s = src + (la * 4 + b) * a.nvb;
          for (int t = 0; t < a.nvb; ++t) dst[t] += s[t];
        }
      if (a.vec) {
        const T* s = src + 16 * a.nvb + la * a.nrhs;
        for (int q = 0; q < a.nrhs; ++q) rhs[A + (size_t)a.N * q] += s[q];
      }
    }
}

__global__ void face_nodes_kernel(const int* __restrict__ ien, const int* __restrict__ face_e, int nface,
                                  int* __restrict__ out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nface) return;
  const int4 nd = reinterpret_cast<const int4*>(ien)[face_e[f]];
  out[4 * (size_t)f + 0] = nd.x;
  out[4 * (size_t)f + 1] = nd.y;
  out[4 * (size_t)f + 2] = nd.z;
  out[4 * (size_t)f + 3] = nd.w;
}

void free_faces(ovs_ctx* c) {
  void* ptrs[] = {c->face_e, c->face_info, c->face_h, c->fnode, c->fnode_ptr, c->fnode_ent,
                  c->fbuf[0], c->fbuf[1]};
  for (void* p : ptrs) if (p) cudaFree(p);
  c->face_e = c->face_info = c->fnode = c->fnode_ptr = c->fnode_ent = nullptr;
  c->face_h = nullptr;
  c->fbuf[0] = c->fbuf[1] = nullptr;
  c->nface = c->nfnode = 0;
  c->face_flags_all = 0;
}

}  // namespace

void ovs_faces_free(ovs_ctx* c) { free_faces(c); }

namespace {
// The per-face checks of a face set on a tet mesh of nelem elements: owning
// elements in 1..nelem, FACE_OR in 1..4, known flag bits, and the convective
// tables present when a face carries the convective term.
int validate_faces(int nelem, int nface, const int* f2e, const int* face_or, const int* flags, const double* hconv,
                   const double* tinf) {
  if (nface > (1 << 28)) return OVS_ERR_ARG;
  int all = 0;
  for (int f = 0; f < nface; ++f) {
    if (f2e[f] < 1 || f2e[f] > nelem || face_or[f] < 1 || face_or[f] > 4) return OVS_ERR_ARG;
    if (flags[f] & ~(OVS_FACE_WEAK | OVS_FACE_CONVH)) return OVS_ERR_ARG;
    all |= flags[f];
  }
  if ((all & OVS_FACE_CONVH) && (!hconv || !tinf)) return OVS_ERR_ARG;
  return OVS_OK;
}
}  // namespace

int ovs_check_faces(int nelem, int nface, const int* f2e, const int* face_or, const int* flags, const double* hconv,
                    const double* tinf) {
  if (nelem <= 0 || nface < 0) return OVS_ERR_ARG;
  if (nface > 0 && (!f2e || !face_or || !flags)) return OVS_ERR_ARG;
  return validate_faces(nelem, nface, f2e, face_or, flags, hconv, tinf);
}

int ovs_faces_set_impl(ovs_ctx* c, int nface, const int* f2e, const int* face_or, const int* flags,
                       const double* hconv, const double* tinf) {
  if (nface < 0) return OVS_ERR_ARG;
  if (nface > 0 && (!f2e || !face_or || !flags)) return OVS_ERR_ARG;
  if (nface > 0 && c->nshl != 4) return OVS_ERR_ARG;   // face rules exist for tets (and prisms) only
  if (nface > 0 && !c->have_mesh) return OVS_ERR_STATE;
  int st;
  if ((st = validate_faces(c->E, nface, f2e, face_or, flags, hconv, tinf))) return st;
  int all = 0;   // the face kinds present, for the assembly dispatch
  for (int f = 0; f < nface; ++f) all |= flags[f];
  if ((st = ovs_activate(c))) return st;
  cudaStream_t s = c->stream;
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  free_faces(c);
  if (nface == 0) return OVS_OK;
  std::vector<int> he(nface), hi(nface);
  std::vector<double> hh(2 * (size_t)nface, 0.0);
  for (int f = 0; f < nface; ++f) {
    he[f] = f2e[f] - 1;
    hi[f] = (face_or[f] - 1) | (flags[f] << 2);
    if (flags[f] & OVS_FACE_CONVH) { hh[2 * (size_t)f] = hconv[f]; hh[2 * (size_t)f + 1] = tinf[f]; }
  }
  if ((st = ovs_ensure((void**)&c->face_e, sizeof(int) * nface))) return st;
  if ((st = ovs_ensure((void**)&c->face_info, sizeof(int) * nface))) return st;
  if ((st = ovs_ensure((void**)&c->face_h, sizeof(double) * 2 * nface))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->face_e, he.data(), sizeof(int) * nface, cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->face_info, hi.data(), sizeof(int) * nface, cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->face_h, hh.data(), sizeof(double) * 2 * nface, cudaMemcpyHostToDevice, s));
  // nodes of every face element, then the node -> face entries in face order
  int* dn = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&dn, sizeof(int) * 4 * (size_t)nface, s));
  face_nodes_kernel<<<ovs_grid(nface, 128, 1 << 30), 128, 0, s>>>(c->ien, c->face_e, nface, dn);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  std::vector<int> nodes(4 * (size_t)nface);
  OVS_CUDA_TRY(cudaMemcpyAsync(nodes.data(), dn, sizeof(int) * 4 * (size_t)nface, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaFreeAsync(dn, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<std::pair<int, int>> ent(4 * (size_t)nface);
  for (size_t k = 0; k < ent.size(); ++k) ent[k] = {nodes[k], (int)k};   // k = 4 f + a
  std::sort(ent.begin(), ent.end());
  std::vector<int> fn, fp, fe(ent.size());
  for (size_t k = 0; k < ent.size(); ++k) {
    if (k == 0 || ent[k].first != ent[k - 1].first) { fn.push_back(ent[k].first); fp.push_back((int)k); }
    fe[k] = ent[k].second;
  }
  fp.push_back((int)ent.size());
  c->nfnode = (int)fn.size();
  if ((st = ovs_ensure((void**)&c->fnode, sizeof(int) * fn.size()))) return st;
  if ((st = ovs_ensure((void**)&c->fnode_ptr, sizeof(int) * fp.size()))) return st;
  if ((st = ovs_ensure((void**)&c->fnode_ent, sizeof(int) * fe.size()))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->fnode, fn.data(), sizeof(int) * fn.size(), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->fnode_ptr, fp.data(), sizeof(int) * fp.size(), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->fnode_ent, fe.data(), sizeof(int) * fe.size(), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  c->nface = nface;
  c->face_flags_all = all;
  return OVS_OK;
}

// Adds the face terms of `kernel` to the system just assembled (rows
// written by the element pass).
int ovs_faces_assemble(ovs_ctx* c, int kernel, int prec, int mat, int vec) {
  const bool tem = kernel == OVS_ASM_TEM;
  const int flag = tem ? OVS_FACE_CONVH : OVS_FACE_WEAK;
  if (!c->nface || !(c->face_flags_all & flag) || !(mat || vec)) return OVS_OK;
  const int sys = kernel == OVS_ASM_NS ? OVS_SYS_NS : (kernel == OVS_ASM_NSVOF ? OVS_SYS_NSVOF : OVS_SYS_TEM);
  const size_t ts = prec == OVS_FP64 ? 8 : 4;
  int st;
  if ((st = ovs_ensure(&c->fbuf[prec], ts * (size_t)c->nface * 2 * FW))) return st;
  cudaStream_t s = c->stream;
  const ovs_params& p = c->params;
  FaceArgs fa;
  for (int k = 0; k < OVS_F_COUNT; ++k) fa.f[k] = c->field[k];
  fa.ien = c->ien;
  fa.elm_id = c->elm_id;
  fa.ibc = c->ibc;
  fa.face_e = c->face_e;
  fa.face_info = c->face_info;
  fa.face_h = c->face_h;
  fa.out = c->fbuf[prec];
  fa.nface = c->nface;
  fa.N = c->N;
  fa.mat = mat;
  fa.vec = vec;
  fa.use_subdomain = kernel == OVS_ASM_NS;
  fa.alfi = p.alfi;
  fa.fact2 = p.alfi * p.gami * p.delt;
  fa.rhoa = p.rhoa;
  fa.mua = p.mua;
  fa.subdomain_flag = p.subdomain_flag;
  fa.elm_id_set0 = p.elm_id_set[0];
  fa.elm_id_set1 = p.elm_id_set[1];
  const int g1 = ovs_grid(c->nface, 128, 1 << 30);
  if (tem) {
    if (prec == OVS_FP64) face_tem_kernel<double><<<g1, 128, 0, s>>>(fa);
    else face_tem_kernel<float><<<g1, 128, 0, s>>>(fa);
  } else {
    if (prec == OVS_FP64) face_ns_kernel<double><<<g1, 128, 0, s>>>(fa);
    else face_ns_kernel<float><<<g1, 128, 0, s>>>(fa);
  }
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  SysStore& S = c->sys[sys][prec];
  ScatterArgs sa;
  sa.fnode = c->fnode;
  sa.fptr = c->fnode_ptr;
  sa.fent = c->fnode_ent;
  sa.face_e = c->face_e;
  sa.face_info = c->face_info;
  sa.ien = c->ien;
  sa.rowptr = c->rowptr;
  sa.colidx = c->colidx;
  sa.buf = c->fbuf[prec];
  sa.vals = S.vals;
  sa.rhs = S.rhs;
  sa.bad = c->flags + 3;
  sa.nfnode = c->nfnode;
  sa.N = c->N;
  sa.nv = ovs_sys_nv(sys);
  sa.nvb = tem ? 1 : 16;
  sa.nrhs = tem ? 1 : 4;
  sa.npass = tem ? 1 : 2;
  sa.fstride = tem ? FT : 2 * FW;
  sa.pstride = tem ? 0 : FW;
  sa.flag = flag;
  sa.mat = mat;
  sa.vec = vec;
  const int g2 = ovs_grid(c->nfnode, 128, 1 << 30);
  if (prec == OVS_FP64) face_scatter_kernel<double><<<g2, 128, 0, s>>>(sa);
  else face_scatter_kernel<float><<<g2, 128, 0, s>>>(sa);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}
