// Element assembly into the node-block CSR system (sm_100a).
//
// Replaces the element loops of
//   IntElmAss_NS_overset            src/assembleNavSto.f90:76-336 (+e3LHS/e3RHS)
//   IntElmAss_NSVOF_Quenching_STAB  src/solveQuenching.f90:122-573
//   IntElmAss_Tem_Quenching_STAB    src/solveQuenching.f90:579-882
// together with the element Dirichlet treatment (BCLhs_3D / BCLhs_NS_conv /
// BCLhs_tem, src/BCLhs_3D.f90) and the scatter (FillSparseMat_*,
// LocaltoGlobalNSVOF_3D).
//
// Scheme (row owner, deterministic, atomic-free):
//   * one warp owns one CSR row, i.e. one node A;
//   * phase 1: lane l takes the l-th element of A's element list (sorted by
//     element id) and evaluates A's row of that element's matrix, i.e. the
//     nshl node-pair blocks (A, b), plus A's residual entries, from the
//     gathered node records; results go to shared memory;
//   * phase 2: the warp adds the element rows into a shared accumulator of
//     A's CSR slots, element by element in ascending element id, so every
//     slot is summed in the same order on every run;
//   * the Dirichlet treatment of the reference zeroes element rows/columns
//     and puts 1 on the element diagonal; both commute with the sum, so they
//     are applied once at the row write: masked entries are 0, a constrained
//     diagonal entry equals the number of elements around A;
//   * the row (contiguous in the CSR value array) is written with vector
//     stores.
// Gauss-point physics is recomputed by each of the element's nshl rows
// instead of being staged through HBM.
#include "dual.cuh"
#include "ovs_internal.cuh"

#include <math.h>
#include <string.h>

#include <type_traits>
#include <vector>

namespace {

// ------------------------------------------------------------------ params
struct AsmArgs {
  const void* rec;        // alpha-stage node records, REC values per node
  const int* ien;         // E*nshl element-major, 0-based
  const int* elm_id;      // E
  const uint8_t* ibc;     // N
  const int* rowptr;
  const int* colidx;
  const int* n2e_ptr;
  const int* n2e;
  const unsigned* n2s;    // slots of each entry's element nodes in the row
  const int4* row_rec;    // per row in processing order: {A, rowptr[A], n2e_ptr[A], deg | sd << 8 | ne << 16}
  const int* cptr;        // off-diagonal contribution lists (tets): offsets per CSR entry
  const int* clist;       //   entries (e << 4) | (la << 2) | b
  void* vals;             // nnz*NV
  void* rhs;              // NF*N field-major
  const void* kbuf;       // hex tensor-core block values (E x 64 x 24), or null
  int* flags;             // [0] non-positive DetJ count, [1] non-finite residual
  unsigned long long* cfl_bits;
  int N;
  int nrows;              // row records the row pass visits (N, or the rows a tile cannot hold)
  int mat, vec;
  int max_deg;
  ovs_params p;
};

// value position tables of the internal slot layout (24 values per slot):
//   0..3  K(1,1) K(1,2) K(1,3) G(1)     row u1
//   4..7  K(2,1) K(2,2) K(2,3) G(2)     row u2
//   8..11 K(3,1) K(3,2) K(3,3) G(3)     row u3
//  12..15 D(1)   D(2)   D(3)   M        row p
//  16..19 LSU(1) LSU(2) LSU(3) LS       row phi
//  20..23 ULS(1) ULS(2) ULS(3) PLS      column phi
// The NS system keeps the first 16, the temperature system one value.
// IBC bit d <=> IBC(:, d+1) == 1: bits 0-2 velocity, 3 pressure, 4 VOF, 5 T.
// rowbits: A-side constraints that zero the entry (element row zeroing),
// colbits: B-side constraints (element column zeroing), diagbit: the entry
// set to 1 on the element diagonal.  Row/column rules follow BCLhs_3D
// (src/BCLhs_3D.f90:18-120) and BCLhs_NS_conv (:295-424) with the pressure at
// IBC column 4 and VOF at column 5; note M is only row-zeroed, ULS only
// column-zeroed, and LSU(i) is also zeroed by the u_i constraint of the ROW
// node (BCLhs_NS_conv :313,:345,:377).
constexpr uint8_t U0 = 1, U1 = 2, U2 = 4, PB = 8, FB = 16, TB = 32;
__constant__ uint8_t c_rowbits[24] = {U0, U0, U0, U0, U1, U1, U1, U1, U2, U2, U2, U2,
                                      PB, PB, PB, PB, FB | U0, FB | U1, FB | U2, FB, 0, 0, 0, PB};
__constant__ uint8_t c_colbits[24] = {U0, U1, U2, PB, U0, U1, U2, PB, U0, U1, U2, PB,
                                      U0, U1, U2, 0, U0, U1, U2, FB, FB, FB, FB, FB};
__constant__ uint8_t c_diagbit[24] = {U0, 0, 0, 0, 0, U1, 0, 0, 0, 0, U2, 0,
                                      0, 0, 0, PB, 0, 0, 0, FB, 0, 0, 0, 0};

// tet 4-point rule (src/genGP_GW.f90:332-353); N = (xi, eta, zeta, 1-xi-eta-zeta)
template <typename T>
__device__ __forceinline__ void tet_shape(int g, T N[4]) {
  const T a = (T)0.5854101966249685, b = (T)0.1381966011250105;
  T xi = (g == 0) ? a : b, eta = (g == 1) ? a : b, ze = (g == 2) ? a : b;
  N[0] = xi; N[1] = eta; N[2] = ze;
  N[3] = (T)1.0 - xi - eta - ze;
}

// FP64 node records held in shared memory instead of registers (64 values
// per element, transposed so a warp's accesses hit 32 consecutive banks),
// and zero rounding remainders: the FP64 element routines otherwise need
// more registers than a thread has.
template <typename T> struct SmemRecRow {
  const volatile T* p;   // volatile: read where used, not hoisted into registers
  __device__ __forceinline__ T operator[](int k) const { return p[(size_t)k * 128]; }
};
template <typename T> struct SmemRecs {
  const T* p;   // this thread's column of a [64][128] block array
  __device__ __forceinline__ SmemRecRow<T> operator[](int n) const { return SmemRecRow<T>{p + (size_t)n * 16 * 128}; }
};
template <typename T> struct ZeroRow {
  __device__ __forceinline__ T operator[](int) const { return (T)0; }
};
template <typename T> struct ZeroRecs {
  __device__ __forceinline__ ZeroRow<T> operator[](int) const { return ZeroRow<T>{}; }
};

// SMEMREC (FP64 only): the node records through shared memory (a 3-block
// register bound) instead of registers (255 registers, 2 blocks)
// Type of the VOF value and of the property blend: FP64 for the FP32 and
// FP64 routines, the dual number itself for the adjoint.
template <typename T> struct Wide { using type = double; };
template <> struct Wide<Dual> { using type = Dual; };

// VOF field at tet Gauss point g in FP64 from the record value (slot k)
// plus its rounding remainder (lo[.][3]): sum_a N_a phi_a, in node order
template <typename T, typename RA, typename LA>
__device__ __forceinline__ typename Wide<T>::type gp_phi(const RA& r, const LA& lo, int k, int g) {
  using W = typename Wide<T>::type;
  const double a = 0.5854101966249685, b = 0.1381966011250105;
  const double xi = (g == 0) ? a : b, eta = (g == 1) ? a : b, ze = (g == 2) ? a : b;
  const double N[4] = {xi, eta, ze, 1.0 - xi - eta - ze};
  W s = 0.0;
#pragma unroll
  for (int n = 0; n < 4; ++n) s += ((W)r[n][k] + (W)lo[n][3]) * N[n];
  return s;
}

// the clamp of prop_interp (src/e3int.f90:4-13): phic = min(max(phi, 0), 1)
__device__ __forceinline__ double clamp01(double x) { return fmax(fmin(x, 1.0), 0.0); }
__device__ __forceinline__ Dual clamp01(const Dual& x) {
  return x.v < 0.0 ? Dual(0.0) : (x.v > 1.0 ? Dual(1.0) : x);
}

// store NV (multiple of 4) register values to 16-byte aligned shared memory
template <int NV>
__device__ __forceinline__ void store_row(float* dst, const float* v) {
#pragma unroll
  for (int k = 0; k < NV; k += 4)
    *reinterpret_cast<float4*>(dst + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
}
template <int NV>
__device__ __forceinline__ void store_row(double* dst, const double* v) {
#pragma unroll
  for (int k = 0; k < NV; k += 2)
    *reinterpret_cast<double2*>(dst + k) = make_double2(v[k], v[k + 1]);
}

// 4 values to global memory with the streaming cache hint (st.global.cs):
// the CSR values are written once and not read again by the pass, so they
// should not evict the element summaries the pass still reads from L2
__device__ __forceinline__ void store4_cs(float* dst, const float* v) {
  __stcs(reinterpret_cast<float4*>(dst), make_float4(v[0], v[1], v[2], v[3]));
}
__device__ __forceinline__ void store4_cs(double* dst, const double* v) {
  __stcs(reinterpret_cast<double2*>(dst), make_double2(v[0], v[1]));
  __stcs(reinterpret_cast<double2*>(dst) + 1, make_double2(v[2], v[3]));
}

template <typename T>
__device__ __forceinline__ T pick4(const T v[4], int i) {
  return i == 0 ? v[0] : (i == 1 ? v[1] : (i == 2 ? v[2] : v[3]));
}

// Node records: REC = 20 values per node.  0-2: x+d (rounded to T),
// 3-15: the fields of the pass, 16-18: the rounding remainder of x+d, 19:
// the rounding remainder of the VOF field.  With the remainders, edge
// vectors x_j - x_k keep full T accuracy on fine meshes far from the origin,
// and the VOF value that blends properties 1000:1 is exact to FP64 (in FP64
// the remainders are 0).
constexpr int REC = 20;
__device__ __forceinline__ void load_rec(const float* rec, int node, float r[16], float lo[4]) {
  const float4* p = reinterpret_cast<const float4*>(rec) + (size_t)node * 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float4 v = __ldg(p + k);
    r[4 * k] = v.x; r[4 * k + 1] = v.y; r[4 * k + 2] = v.z; r[4 * k + 3] = v.w;
  }
  float4 v = __ldg(p + 4);
  lo[0] = v.x; lo[1] = v.y; lo[2] = v.z; lo[3] = v.w;
}
__device__ __forceinline__ void load_rec(const double* rec, int node, double r[16], double lo[4]) {
  const double2* p = reinterpret_cast<const double2*>(rec) + (size_t)node * 10;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double2 v = __ldg(p + k);
    r[2 * k] = v.x; r[2 * k + 1] = v.y;
  }
  // FP64 records round nothing: their remainders (slots 16-19) are exactly 0
  lo[0] = lo[1] = lo[2] = lo[3] = 0.0;
}

// Geometry of a linear tet on the current configuration x+d
// (eval_shape_fem, src/eval_shape_FEM.f90:4-61, with get_inverse_3x3,
// src/eval_shape.f90:85-112).  xd[a][i] = x+d of node a.  The Jacobian of a
// linear tet is the same at every Gauss point, so it is evaluated once.
template <typename T, typename LA>
__device__ __forceinline__ T tet_geometry(const T xd[4][3], const LA& lo, T g[4][3], T G[3][3]) {
  T A[3][3], Ai[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) A[i][j] = (xd[j][i] - xd[3][i]) + (lo[j][i] - lo[3][i]);
  Ai[0][0] = A[1][1] * A[2][2] - A[2][1] * A[1][2];
  Ai[0][1] = A[2][1] * A[0][2] - A[0][1] * A[2][2];
  Ai[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  T tmp = (T)1.0 / (Ai[0][0] * A[0][0] + Ai[0][1] * A[1][0] + Ai[0][2] * A[2][0]);
  Ai[0][0] *= tmp; Ai[0][1] *= tmp; Ai[0][2] *= tmp;
  Ai[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * tmp;
  Ai[1][1] = (A[0][0] * A[2][2] - A[2][0] * A[0][2]) * tmp;
  Ai[1][2] = (A[1][0] * A[0][2] - A[0][0] * A[1][2]) * tmp;
  Ai[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * tmp;
  Ai[2][1] = (A[2][0] * A[0][1] - A[0][0] * A[2][1]) * tmp;
  Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * tmp;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    g[0][j] = Ai[0][j]; g[1][j] = Ai[1][j]; g[2][j] = Ai[2][j];
    g[3][j] = (-Ai[0][j] - Ai[1][j]) - Ai[2][j];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      G[i][j] = Ai[0][i] * Ai[0][j] + Ai[1][i] * Ai[1][j] + Ai[2][i] * Ai[2][j];
  return (T)1.0 / tmp;
}

template <typename T>
__device__ __forceinline__ T quad_uGu(const T u[3], const T G[3][3]) {
  T t = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) t += u[i] * G[i][j] * u[j];
  return t;
}

// e3DC_beta2's INTEGER dummy receiving a real(8) (src/e3STAB.f90:175-189):
// the callee reads the low 4 bytes of the double.
__device__ __forceinline__ int low_word(double v) {
  return (int)(unsigned)(__double_as_longlong(v) & 0xffffffffULL);
}

__device__ __forceinline__ void cfl_max(unsigned long long* bits, double v) {
  if (v >= 0.0) atomicMax(bits, (unsigned long long)__double_as_longlong(v));
}

// ----------------------------------------------------- element summaries
// Pass 1 (one thread per element) evaluates everything the element matrix
// needs from its Gauss points, once, plus the element's residual rows, and
// stores it as a compact summary of SW values.  Pass 2 (one warp per CSR
// row) expands A's row of each element matrix from the summaries.  Inactive
// elements (solid on the NS+VOF pass, non-target on the NS pass) store zero
// sums and zero residuals, which makes every expanded block exactly zero.
// NS / NS+VOF: the Gauss-point sums of the block formulas (see
// expand_block), which pass 1 forms once per element:
//   [0, ND0)     per (row node a, column node b), PW values at PW (4a + b):
//                NS+VOF {S_ab, L1_ab + E_ab, PL_ab, V_ab}, NS {S_ab}
//   [ND0, C0)    per node n, 8 values: grad N_n (3), PR_n, T_n, U_n, Q_n, 0
//   [C0, RHS0)   KA KB MM, then NS+VOF: KDP dphi (3) 0; NS: 0
//   [RHS0, SW)   the residual, NF values per node
// (PR_n is both P_b and R_a of the block formulas, U_n both U_b and W_a)
//   TEM  : the 4x4 element matrix itself, row-major (a, b) | residual 4 = 20
//          (a scalar system: its element matrix is smaller than the
//          Gauss-point records it would be expanded from)
// GQ: the values pass 1 keeps per Gauss point for the sums: uadv (3) and
// rt = rho tauM; NS+VOF: uadv (3) rho rt tauLS src eps ufac plfac (the
// factors of the phase-change terms).
template <int KIND> struct Lay;
template <> struct Lay<OVS_ASM_NS> {
  static constexpr int PW = 1, ND0 = 16, C0 = 48, RHS0 = 52, SW = 68, NF = 4, NV = 16, GQ = 4;
};
template <> struct Lay<OVS_ASM_NSVOF> {
  static constexpr int PW = 4, ND0 = 64, C0 = 96, RHS0 = 104, SW = 124, NF = 5, NV = 24, GQ = 10;
};
template <> struct Lay<OVS_ASM_TEM> {
  static constexpr int SW = 20, RHS0 = 16, NF = 1, NV = 1;
};

// 4 values of an element summary (global memory; 16-byte aligned in FP32,
// 32-byte aligned in FP64, where every 4-value group of a summary sits on
// a 32-byte boundary) with one vector store.  FP64 uses the 256-bit global
// store of sm_100: one instruction instead of two 128-bit stores, measured
// 5.9 against 7.1 ms for the FP64 NS+VOF element pass at 128^3 (the pass
// writes 31 such groups per tet).  The asm carries no memory clobber: the
// element pass never reads a summary it writes, and the row pass that
// reads it is a later launch
template <typename T>
__device__ __forceinline__ void put4(T* d, T a, T b, T c, T e) {
  d[0] = a; d[1] = b; d[2] = c; d[3] = e;
}
__device__ __forceinline__ void put4(float* d, float a, float b, float c, float e) {
  *reinterpret_cast<float4*>(d) = make_float4(a, b, c, e);
}
__device__ __forceinline__ void put4(double* d, double a, double b, double c, double e) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(d), "d"(a), "d"(b), "d"(c), "d"(e));
}

// The Gauss-point sums of the NS / NS+VOF block formulas (expand_block)
// from the per-point values q (layout GQ above), the shape gradients g and
// the weight w, written to the summary o: with c_n = uadv . grad N_n,
//   S_ab  = sum w rho (Na + rt ca)(fact1 Nb + fact2 cb)
//   L1_ab = sum w (Na + tauLS ca)(fact1 Nb + fact2 cb + fact2 Nb src)
//   E_ab  = sum eps Na Nb      PL_ab = -sum plfac Na Nb
//   V_ab  = sum fact2 w (Na + tauLS ca) Nb
//   PR_n  = sum fact2 w Nn     T_n = sum w rt (fact1 Nn + fact2 cn)
//   U_n   = sum ufac Nn        Q_n = sum fact2 w rt cn
// (rho = rho_ns on the NS pass).  Each sum is formed once per element here
// instead of once per block in the row pass.  block_sums_row writes the
// pairs of row node a and node a's record (a may vary per lane: the
// per-node values are picked by selects, which fold for a constant a).
template <typename T, int KIND>
__device__ __forceinline__ void block_sums_row(const T (&q)[4][Lay<KIND>::GQ], const T (&g)[4][3], T w, T fact1,
                                               T fact2, T rho_ns, int a, T* o) {
  using L = Lay<KIND>;
  constexpr bool vof = KIND == OVS_ASM_NSVOF;
  T c[4][4];
#pragma unroll
  for (int gp = 0; gp < 4; ++gp)
#pragma unroll
    for (int n = 0; n < 4; ++n) c[gp][n] = q[gp][0] * g[n][0] + q[gp][1] * g[n][1] + q[gp][2] * g[n][2];
  T S[4], L1[4], PL[4], V[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) S[b] = L1[b] = PL[b] = V[b] = 0;
#pragma unroll
  for (int gp = 0; gp < 4; ++gp) {
    T N[4];
    tet_shape<T>(gp, N);
    const T Na = pick4<T>(N, a), ca = pick4<T>(c[gp], a);
    const T rho = vof ? q[gp][3] : rho_ns;
    const T rt = vof ? q[gp][4] : q[gp][3];
    const T alpha = w * rho * (Na + rt * ca);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const T beta = fact1 * N[b] + fact2 * c[gp][b];
      S[b] += alpha * beta;
      if constexpr (vof) {
        const T gam = w * (Na + q[gp][5] * ca);
        L1[b] += gam * (beta + fact2 * N[b] * q[gp][6]) + q[gp][7] * Na * N[b];
        PL[b] -= q[gp][9] * Na * N[b];
        V[b] += fact2 * gam * N[b];
      }
    }
  }
  if constexpr (vof) {
#pragma unroll
    for (int b = 0; b < 4; ++b) put4(o + L::PW * (4 * a + b), S[b], L1[b], PL[b], V[b]);
  } else {
    put4(o + L::PW * 4 * a, S[0], S[1], S[2], S[3]);
  }
  T PR = 0, Tn = 0, U = 0, Q = 0;
#pragma unroll
  for (int gp = 0; gp < 4; ++gp) {
    T N[4];
    tet_shape<T>(gp, N);
    const T Nn = pick4<T>(N, a), cn = pick4<T>(c[gp], a);
    const T rt = vof ? q[gp][4] : q[gp][3];
    PR += fact2 * w * Nn;
    Tn += w * rt * (fact1 * Nn + fact2 * cn);
    Q += fact2 * w * rt * cn;
    if constexpr (vof) U += q[gp][8] * Nn;
  }
  T ga[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const T col[4] = {g[0][d], g[1][d], g[2][d], g[3][d]};
    ga[d] = pick4<T>(col, a);
  }
  put4(o + L::ND0 + 8 * a, ga[0], ga[1], ga[2], PR);
  put4(o + L::ND0 + 8 * a + 4, Tn, U, Q, (T)0);
}

// all four rows of the element (one thread per element)
template <typename T, int KIND>
__device__ __forceinline__ void block_sums(const T (&q)[4][Lay<KIND>::GQ], const T (&g)[4][3], T w, T fact1,
                                           T fact2, T rho_ns, T* o) {
#pragma unroll
  for (int a = 0; a < 4; ++a) block_sums_row<T, KIND>(q, g, w, fact1, fact2, rho_ns, a, o);
}

// The CFL number delt sqrt(taua), largest over an element's points: the
// point routines keep the largest taua and the element kernel takes one
// square root of it (sqrt and the product are monotone and correctly
// rounded, so this is the largest point value exactly; measured FP64
// NS+VOF 4.24 -> 4.12 ms, T 1.62 -> 1.49 ms, FP32 T 0.91 -> 0.79 ms).
// The FP32 NS+VOF pass keeps the value per point: the same change made
// that kernel slower (2.79 -> 3.05 ms at its 3-block bound, 3.26 at 4,
// 3.30 at 2).
template <typename T, int KIND> struct CflPerPoint { static constexpr bool v = false; };
template <> struct CflPerPoint<float, OVS_ASM_NSVOF> { static constexpr bool v = true; };

// 1 / sqrt(x): the reciprocal square root (FP64, FP32), and for the dual
// numbers of the adjoint the quotient
__device__ __forceinline__ double inv_sqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float inv_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ Dual inv_sqrt(const Dual& x) { return 1.0 / sqrt(x); }

struct SumArgs {
  const void* rec;
  const int* ien;
  const int* elm_id;
  void* sum;
  int* flags;
  unsigned long long* cfl_bits;
  int E;
  ovs_params p;
};

template <typename T, typename RA, typename LA>
__device__ __forceinline__ void element_geometry(const RA& r, const LA& lo, T g[4][3], T G[3][3],
                                                 T& detj, T& GG, T& trG) {
  T xd[4][3];
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int i = 0; i < 3; ++i) xd[n][i] = r[n][i];
  detj = tet_geometry<T>(xd, lo, g, G);
  GG = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) GG += G[i][j] * G[i][j];
  trG = G[0][0] + G[1][1] + G[2][2];
}

// pass 1, NS-only: IntElmAss_NS_overset's Gauss loop with e3LHS_3D_fluid_Old /
// e3Rhs_3D_fluid (quirks: uprime = 0, kap_dc = NS_kdc_a, tauBar = 0)
template <typename T, typename RA, typename LA>
__device__ void summarize_ns(const SumArgs& a, const RA& r, const LA& lo, bool target, T* o,
                             double& tamax, T& detj_out) {
  const ovs_params& p = a.p;
  T g[4][3], G[3][3], detj, GG, trG;
  element_geometry<T>(r, lo, g, G, detj, GG, trG);
  detj_out = detj;
  const T w = detj * (T)(0.25 / 6.0);
  T du[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      du[i][j] = r[0][3 + i] * g[0][j] + r[1][3 + i] * g[1][j] + r[2][3 + i] * g[2][j] + r[3][3 + i] * g[3][j];
  const T divu = du[0][0] + du[1][1] + du[2][2];
  const T rho = (T)p.rhoa, mu = (T)p.mua, mupkdc = mu + (T)p.ns_kdc_a;
  const T fact2 = (T)(p.alfi * p.gami * p.delt);
  const T taut = (T)(4.0 / (p.delt * p.delt));
  // the element's constants as reciprocals (rho, mu and trG are fixed over
  // its points): products instead of per-point divisions
  const T irho = (T)1.0 / rho, itrG = (T)1.0 / trG;
  const T nu = mu * irho;
  T KA = 0, KB = 0, MM = 0;
  T ru[4][3], rp[4], q[4][Lay<OVS_ASM_NS>::GQ];
#pragma unroll
  for (int n = 0; n < 4; ++n) { ru[n][0] = ru[n][1] = ru[n][2] = 0; rp[n] = 0; }
#pragma unroll
  for (int gp = 0; gp < 4; ++gp) {
    T N[4];
    tet_shape<T>(gp, N);
    T ui[3], umi[3], aci[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      ui[d] = r[0][3 + d] * N[0] + r[1][3 + d] * N[1] + r[2][3 + d] * N[2] + r[3][3 + d] * N[3];
      umi[d] = r[0][6 + d] * N[0] + r[1][6 + d] * N[1] + r[2][6 + d] * N[2] + r[3][6 + d] * N[3];
      aci[d] = r[0][9 + d] * N[0] + r[1][9 + d] * N[1] + r[2][9 + d] * N[2] + r[3][9 + d] * N[3];
    }
    const T pri = r[0][12] * N[0] + r[1][12] * N[1] + r[2][12] * N[2] + r[3][12] * N[3];
    const T uadv[3] = {ui[0] - umi[0], ui[1] - umi[1], ui[2] - umi[2]};
    const T taua = quad_uGu<T>(uadv, G);
    const T taud = nu * nu * (T)12.0 * GG;
    const T tauM = irho * inv_sqrt(taut + taua + taud);
    const T tauC = rho * sqrt(taua + taud) * itrG;
    if ((double)taua > tamax) tamax = (double)taua;   // CFL number: delt sqrt(max taua), in the kernel
    q[gp][0] = uadv[0]; q[gp][1] = uadv[1]; q[gp][2] = uadv[2]; q[gp][3] = rho * tauM;
    if (target) {
      KA += fact2 * mupkdc * w;
      KB += fact2 * tauC * w;
      MM += fact2 * w * tauM;
      const T ptot = pri - tauC * divu;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const T tmp1 = rho * (aci[i] + uadv[0] * du[i][0] + uadv[1] * du[i][1] + uadv[2] * du[i][2]) - (T)p.gravvec[i] * rho;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
          const T sym = mupkdc * (g[n][0] * (du[i][0] + du[0][i]) + g[n][1] * (du[i][1] + du[1][i]) +
                                  g[n][2] * (du[i][2] + du[2][i]));
          ru[n][i] -= (N[n] * tmp1 + (sym - g[n][i] * ptot)) * w;
        }
      }
#pragma unroll
      for (int n = 0; n < 4; ++n) rp[n] -= (N[n] * divu) * w;
    }
  }
  using L = Lay<OVS_ASM_NS>;
#pragma unroll
  for (int n = 0; n < 4; ++n) put4(o + L::RHS0 + 4 * n, ru[n][0], ru[n][1], ru[n][2], rp[n]);
  put4(o + L::C0, KA, KB, MM, (T)0);
  if constexpr (!std::is_same<T, Dual>::value)
    block_sums<T, OVS_ASM_NS>(q, g, target ? w : (T)0, (T)p.almi, fact2, rho, o);
}

// One Gauss point of the NS+VOF quench routine (src/solveQuenching.f90:
// 295-523): the point values q (layout GQ of Lay<NSVOF>) and, on fluid
// elements, the point's terms of KA, KB, MM, KDP and of the residual rows,
// added to the accumulators.  The viscous RHS broadcast (:508-510) is kept:
// the three scalars sum_j gN_a,j (du(j,k) + du(k,j)), k = 1..3, are
// subtracted from every momentum component.  ui, umi, aci, pri, phid (FP64),
// rphii, Ti: the fields at the point; N: its shape values.
// Reciprocals taken once per element for the Gauss-point routines: of the
// launch constants ts, rhoa, rhow, tref and of the element's trG, GG and
// sqrt(GG).  The point formulas multiply by them where the reference
// divides (a quotient and the product with the reciprocal differ by
// rounding only); each FP64 division is a reciprocal sequence of its own.
// At a point, one reciprocal of rho (rho cp for the temperature) serves
// nu, tauM (kk, tauT), and 1/sqrt is the reciprocal square root
// (inv_sqrt).  Measured for the FP64 element passes at 128^3: NS+VOF 5.9
// -> 4.35 ms with the per-element reciprocals -> 4.24 ms with the point
// ones, T 2.45 -> 1.74 -> 1.62 ms (FP32: 3.83 -> 2.78 and 1.25 -> 0.91).
template <typename T> struct PointInv {
  T ts, rhoa, rhow, tref, trG, GG, sGG, taut;   // taut = 4 / delt^2 itself
};
template <typename T>
__device__ __forceinline__ PointInv<T> point_inv(const ovs_params& p, T trG, T GG) {
  PointInv<T> iv;
  iv.taut = (T)(4.0 / (p.delt * p.delt));
  iv.ts = (T)(1.0 / p.ts);
  iv.rhoa = (T)(1.0 / p.rhoa);
  iv.rhow = (T)(1.0 / p.rhow);
  iv.tref = (T)(1.0 / p.tref);
  iv.trG = (T)1.0 / trG;
  iv.GG = (T)1.0 / GG;
  iv.sGG = (T)1.0 / sqrt(GG);
  return iv;
}

template <typename T>
__device__ __forceinline__ void nsvof_point(const ovs_params& p, bool fluid, const T (&N)[4], const T (&g)[4][3],
                                            const T (&G)[3][3], T GG, T trG, T w, const T (&du)[3][3],
                                            const T (&dp)[3], const T (&dphi)[3], T divu, const T (&svis)[4],
                                            const T (&gdphi)[4], const T (&ui)[3], const T (&umi)[3],
                                            const T (&aci)[3], T pri, typename Wide<T>::type phid, T rphii, T Ti,
                                            T* q, T& KA, T& KB, T& MM, T& KDP, T (&ru)[4][3], T (&rp)[4],
                                            T (&rf)[4], double& tamax, const PointInv<T>& iv) {
  using W = typename Wide<T>::type;
  const T fact2 = (T)(p.alfi * p.delt * p.gami);
  const T taut = iv.taut;
  const T rhoa = (T)p.rhoa, rhow = (T)p.rhow, ts = (T)p.ts;
  const T ira = iv.rhoa - iv.rhow;
  const bool kdc_on = fabs(p.ns_kdc_w) + fabs(p.ns_kdc_a) > 0.0;
  const bool kdcphi_on = fabs(p.lsc_kdc) > 0.0;
  const T phii = (T)phid;
  const W phicd = clamp01(phid);
  const T phic = (T)phicd;
  T mdot, dmd;
  if (Ti > ts) {
    mdot = (T)p.c_evap * (T)(1.0 - phicd) * rhow * (Ti - ts) * iv.ts;
    dmd = -(T)p.c_evap * rhow * (Ti - ts) * iv.ts * (T)p.c_dmdot;
  } else {
    mdot = (T)p.c_cond * phic * rhoa * (Ti - ts) * iv.ts;
    dmd = (T)p.c_cond * rhoa * (Ti - ts) * iv.ts * (T)p.c_dmdot;
  }
  const T vdot = mdot * iv.rhoa - mdot * iv.rhow;
  T rho, mu;
  if (fluid) {
    rho = (T)(p.rhow * (1.0 - phicd) + p.rhoa * phicd);
    mu = (T)(p.muw * (1.0 - phicd) + p.mua * phicd);
  } else {
    rho = (T)p.rhos; mu = (T)p.mus;
  }
  const T lambda = (T)(-2.0 / 3.0) * mu;
  if (phid < 0.0 || phid > 1.0) dmd = 0;
  const T uadv[3] = {ui[0] - umi[0], ui[1] - umi[1], ui[2] - umi[2]};
  T tmp1[3], rL[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T conv = du[i][0] * uadv[0] + du[i][1] * uadv[1] + du[i][2] * uadv[2];
    tmp1[i] = rho * aci[i] + rho * conv - (T)p.gravvec[i] * rho;
    rL[i] = tmp1[i] + dp[i];
  }
  const T res_phi = rphii + (uadv[0] * dphi[0] + uadv[1] * dphi[1] + uadv[2] * dphi[2]) + phii * vdot - mdot * iv.rhoa;
  const T taua = quad_uGu<T>(uadv, G);
  const T irho = (T)1.0 / rho;
  const T nu = mu * irho;
  const T taud = nu * nu * (T)12.0 * GG;
  const T tauM = irho * inv_sqrt(taut + taua + taud);
  const T tauLS = inv_sqrt(taut + taua);
  const T tauC = rho * sqrt(taua + taud) * iv.trG;
  if constexpr (CflPerPoint<T, OVS_ASM_NSVOF>::v) {
    const double cf = (double)p.delt * sqrt((double)taua);
    if (cf > tamax) tamax = cf;
  } else if ((double)taua > tamax) {
    tamax = (double)taua;   // CFL number: delt sqrt(max taua), in the kernel
  }
  T kdc = 0;
  if (kdc_on) {
    const double nk = (double)(p.ns_kdc_w * (1.0 - phicd) + p.ns_kdc_a * phicd);
    const T rr = rL[0] * rL[0] + rL[1] * rL[1] + rL[2] * rL[2];
    kdc = (T)low_word(nk) * sqrt(rr * iv.GG);
  }
  T kdphi = 0;
  if (kdcphi_on) kdphi = (T)p.lsc_kdc * fabs(res_phi) * iv.sGG;
  const T mupk = mu + kdc;
  const T dmdi = dmd * ira;
  q[0] = uadv[0]; q[1] = uadv[1]; q[2] = uadv[2];
  q[3] = rho; q[4] = rho * tauM; q[5] = tauLS;
  q[6] = vdot + phii * ira * dmd - dmd * iv.rhoa;
  const T wf = fluid ? w : (T)0;   // solid elements contribute nothing
  q[7] = fact2 * wf * tauC * dmdi * dmdi;
  q[8] = fact2 * tauC * dmdi * wf;
  q[9] = fact2 * dmdi * wf;
  if (!fluid) return;
  KA += fact2 * mupk * w;
  KB += fact2 * (tauC + lambda) * w;
  MM += fact2 * w * tauM;
  KDP += fact2 * w * kdphi;
  T c[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) c[n] = uadv[0] * g[n][0] + uadv[1] * g[n][1] + uadv[2] * g[n][2];
  const T tdiv = -pri + tauC * divu;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
      ru[n][i] += w * (-N[n] * tmp1[i] - g[n][i] * tdiv + g[n][i] * tauC * vdot - g[n][i] * lambda * divu -
                       mupk * svis[n] + rho * c[n] * (-tauM * rL[i]));
    rp[n] += w * (-N[n] * (divu - vdot) + (g[n][0] * rL[0] + g[n][1] * rL[1] + g[n][2] * rL[2]) * (-tauM));
    rf[n] += w * (-(N[n] + tauLS * c[n]) * res_phi - kdphi * gdphi[n] + N[n] * dmdi * tauC * (divu - vdot));
  }
}

// svis (the viscous broadcast) and g . grad phi per node, from the
// gradients
template <typename T>
__device__ __forceinline__ void nsvof_node_terms(const T (&g)[4][3], const T (&du)[3][3], const T (&dphi)[3],
                                                 T (&svis)[4], T (&gdphi)[4]) {
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    T sv = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      sv += g[n][0] * (du[0][k] + du[k][0]) + g[n][1] * (du[1][k] + du[k][1]) + g[n][2] * (du[2][k] + du[k][2]);
    svis[n] = sv;
    gdphi[n] = g[n][0] * dphi[0] + g[n][1] * dphi[1] + g[n][2] * dphi[2];
  }
}

// pass 1, NS+VOF quench (src/solveQuenching.f90:295-523), one thread per
// element: geometry and gradients, the four Gauss points (nsvof_point),
// then the residual rows, the element constants and the block sums
template <typename T, typename RA, typename LA>
__device__ void summarize_nsvof(const SumArgs& a, const RA& r, const LA& lo, bool fluid, T* o,
                                double& tamax, T& detj_out) {
  using W = typename Wide<T>::type;
  const ovs_params& p = a.p;
  T g[4][3], G[3][3], detj, GG, trG;
  element_geometry<T>(r, lo, g, G, detj, GG, trG);
  detj_out = detj;
  const T w = detj * (T)(0.25 / 6.0);
  T du[3][3], dp[3], dphi[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      du[i][j] = r[0][3 + i] * g[0][j] + r[1][3 + i] * g[1][j] + r[2][3 + i] * g[2][j] + r[3][3 + i] * g[3][j];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    dp[j] = r[0][12] * g[0][j] + r[1][12] * g[1][j] + r[2][12] * g[2][j] + r[3][12] * g[3][j];
    dphi[j] = r[0][13] * g[0][j] + r[1][13] * g[1][j] + r[2][13] * g[2][j] + r[3][13] * g[3][j];
  }
  const T divu = du[0][0] + du[1][1] + du[2][2];
  T svis[4], gdphi[4];
  nsvof_node_terms<T>(g, du, dphi, svis, gdphi);
  const PointInv<T> iv = point_inv<T>(p, trG, GG);
  T KA = 0, KB = 0, MM = 0, KDP = 0;
  T ru[4][3], rp[4], rf[4], q[4][Lay<OVS_ASM_NSVOF>::GQ];
#pragma unroll
  for (int n = 0; n < 4; ++n) { ru[n][0] = ru[n][1] = ru[n][2] = 0; rp[n] = 0; rf[n] = 0; }
#pragma unroll (std::is_same<RA, SmemRecs<T>>::value ? 1 : 4)
  for (int gp = 0; gp < 4; ++gp) {
    T N[4];
    tet_shape<T>(gp, N);
    T ui[3], umi[3], aci[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      ui[d] = r[0][3 + d] * N[0] + r[1][3 + d] * N[1] + r[2][3 + d] * N[2] + r[3][3 + d] * N[3];
      umi[d] = r[0][6 + d] * N[0] + r[1][6 + d] * N[1] + r[2][6 + d] * N[2] + r[3][6 + d] * N[3];
      aci[d] = r[0][9 + d] * N[0] + r[1][9 + d] * N[1] + r[2][9 + d] * N[2] + r[3][9 + d] * N[3];
    }
    const T pri = r[0][12] * N[0] + r[1][12] * N[1] + r[2][12] * N[2] + r[3][12] * N[3];
    const W phid = gp_phi<T>(r, lo, 13, gp);   // VOF in FP64 for the 1000:1 property blend
    const T rphii = r[0][14] * N[0] + r[1][14] * N[1] + r[2][14] * N[2] + r[3][14] * N[3];
    const T Ti = r[0][15] * N[0] + r[1][15] * N[1] + r[2][15] * N[2] + r[3][15] * N[3];
    nsvof_point<T>(p, fluid, N, g, G, GG, trG, w, du, dp, dphi, divu, svis, gdphi, ui, umi, aci, pri, phid, rphii, Ti,
                   q[gp], KA, KB, MM, KDP, ru, rp, rf, tamax, iv);
  }
  using L = Lay<OVS_ASM_NSVOF>;
  {
    T rh[20];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      rh[5 * n] = ru[n][0]; rh[5 * n + 1] = ru[n][1]; rh[5 * n + 2] = ru[n][2];
      rh[5 * n + 3] = rp[n]; rh[5 * n + 4] = rf[n];
    }
#pragma unroll
    for (int k = 0; k < 20; k += 4) put4(o + L::RHS0 + k, rh[k], rh[k + 1], rh[k + 2], rh[k + 3]);
  }
  put4(o + L::C0, KA, KB, MM, KDP);
  put4(o + L::C0 + 4, dphi[0], dphi[1], dphi[2], (T)0);
  if constexpr (!std::is_same<T, Dual>::value)
    block_sums<T, OVS_ASM_NSVOF>(q, g, fluid ? w : (T)0, (T)p.almi, (T)(p.alfi * p.delt * p.gami), (T)0, o);
}

// pass 1, temperature (src/solveQuenching.f90:712-856).  Record layout of
// this pass: xd(0:2) u(3:5) um(6:8) phi(9) T(10) rT(11).  The element matrix
// (:814-839) is formed here, per Gauss point
//   K(a,b) += w (Na + trc ca) (rcp (fact1 Nb + fact2 cb) - fact2 dSe Nb)
// with trc = tauT rho cp, c_n = uadv . grad N_n, then K(a,b) += HK gab; solid
// elements take uadv = dSe = trc = 0, which turns the fluid block formula
// into the solid one.  The adjoint instantiation (dual numbers) needs the
// residual only and skips the matrix.
template <typename T, typename RA, typename LA>
__device__ void summarize_tem(const SumArgs& a, const RA& r, const LA& lo, bool fluid, T* o,
                              double& tamax, T& detj_out) {
  using W = typename Wide<T>::type;
  const ovs_params& p = a.p;
  T g[4][3], G[3][3], detj, GG, trG;
  element_geometry<T>(r, lo, g, G, detj, GG, trG);
  detj_out = detj;
  const T w = detj * (T)(0.25 / 6.0);
  const PointInv<T> iv = point_inv<T>(p, trG, GG);
  T dT[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) dT[j] = r[0][10] * g[0][j] + r[1][10] * g[1][j] + r[2][10] * g[2][j] + r[3][10] * g[3][j];
  const T fact2 = (T)(p.alfi * p.gami * p.delt);
  const T ts = (T)p.ts, cpw = (T)p.cpw, cpa = (T)p.cpa, lh = (T)p.lh;
  T gdT[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) gdT[n] = g[n][0] * dT[0] + g[n][1] * dT[1] + g[n][2] * dT[2];
  T HK = 0, rt[4] = {0, 0, 0, 0};
  const T fact1 = (T)p.almi;
  T K[4][4];
#pragma unroll
  for (int ia = 0; ia < 4; ++ia)
#pragma unroll
    for (int ib = 0; ib < 4; ++ib) K[ia][ib] = (T)0;
  const bool kdc_on = fabs(p.tem_kdc) > 0.0;
#pragma unroll
  for (int gp = 0; gp < 4; ++gp) {
    T N[4];
    tet_shape<T>(gp, N);
    const W phid = gp_phi<T>(r, lo, 9, gp);
    const T Ti = r[0][10] * N[0] + r[1][10] * N[1] + r[2][10] * N[2] + r[3][10] * N[3];
    const T rTi = r[0][11] * N[0] + r[1][11] * N[1] + r[2][11] * N[2] + r[3][11] * N[3];
    T ui[3], umi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      ui[d] = r[0][3 + d] * N[0] + r[1][3 + d] * N[1] + r[2][3 + d] * N[2] + r[3][3 + d] * N[3];
      umi[d] = r[0][6 + d] * N[0] + r[1][6 + d] * N[1] + r[2][6 + d] * N[2] + r[3][6 + d] * N[3];
    }
    const W phicd = clamp01(phid);
    const T phic = (T)phicd;
    T mdot, dmdT;
    if (Ti > ts) {
      mdot = (T)p.c_evap * (T)(1.0 - phicd) * (T)p.rhow * (Ti - ts) * iv.ts;
      dmdT = (T)p.c_evap * (T)(1.0 - phicd) * (T)p.rhow * iv.ts * (T)p.c_dmdot;
    } else {
      mdot = (T)p.c_cond * phic * (T)p.rhoa * (Ti - ts) * iv.ts;
      dmdT = (T)p.c_cond * phic * (T)p.rhoa * iv.ts * (T)p.c_dmdot;
    }
    T rho, cp, hk, rcp;
    if (fluid) {
      rho = (T)(p.rhow * (1.0 - phicd) + p.rhoa * phicd);
      cp = (T)(p.cpw * (1.0 - phicd) + p.cpa * phicd);
      hk = (T)(p.kappaw * (1.0 - phicd) + p.kappaa * phicd);
      rcp = (T)((p.rhow * p.cpw) * (1.0 - phicd) + (p.rhoa * p.cpa) * phicd);
    } else {
      rho = (T)p.rhos; cp = (T)p.cps; hk = (T)p.kappas; rcp = (T)(p.rhos * p.cps);
    }
    const T uadv[3] = {ui[0] - umi[0], ui[1] - umi[1], ui[2] - umi[2]};
    const T Se = ((cpw - cpa) * (Ti - ts) - lh) * mdot;
    const T udT = uadv[0] * dT[0] + uadv[1] * dT[1] + uadv[2] * dT[2];
    const T res = rcp * (rTi + udT) - Se;
    const T taua = quad_uGu<T>(uadv, G);
    T tt = taua + iv.taut;
    const T ircp = (T)1.0 / (rho * cp);
    const T kk = hk * ircp;
    tt = tt + kk * kk * (T)12.0 * GG;
    const T tauT = ircp * inv_sqrt(tt);
    if ((double)taua > tamax) tamax = (double)taua;   // CFL number: delt sqrt(max taua), in the kernel
    T kdcT = 0;
    if (kdc_on && fluid) kdcT = (T)p.tem_kdc * fabs(res) * iv.sGG * iv.tref;
    const T dSe = (cpw - cpa) * mdot + ((cpw - cpa) * (Ti - ts) - lh) * dmdT;
    if constexpr (!std::is_same<T, Dual>::value) {
      const T uq[3] = {fluid ? uadv[0] : (T)0, fluid ? uadv[1] : (T)0, fluid ? uadv[2] : (T)0};
      const T dSq = fluid ? dSe : (T)0, trq = fluid ? tauT * rcp : (T)0;
      T cq[4];
#pragma unroll
      for (int n = 0; n < 4; ++n) cq[n] = g[n][0] * uq[0] + g[n][1] * uq[1] + g[n][2] * uq[2];
#pragma unroll
      for (int ia = 0; ia < 4; ++ia) {
        const T aw = w * (N[ia] + trq * cq[ia]);
#pragma unroll
        for (int ib = 0; ib < 4; ++ib) K[ia][ib] += aw * (rcp * (fact1 * N[ib] + fact2 * cq[ib]) - fact2 * dSq * N[ib]);
      }
    }
    if (fluid) {
      HK += fact2 * (hk + kdcT) * w;
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const T cn = uadv[0] * g[n][0] + uadv[1] * g[n][1] + uadv[2] * g[n][2];
        rt[n] += w * (-N[n] * rcp * (rTi + udT) + N[n] * Se - rcp * tauT * cn * res - (hk + kdcT) * gdT[n]);
      }
    } else {
      HK += fact2 * hk * w;
#pragma unroll
      for (int n = 0; n < 4; ++n) rt[n] += w * (-N[n] * rcp * rTi - hk * gdT[n]);
    }
  }
  if constexpr (!std::is_same<T, Dual>::value) {
#pragma unroll
    for (int ia = 0; ia < 4; ++ia)
#pragma unroll
      for (int ib = 0; ib < 4; ++ib)
        o[4 * ia + ib] = K[ia][ib] + HK * (g[ia][0] * g[ib][0] + g[ia][1] * g[ib][1] + g[ia][2] * g[ib][2]);
  }
#pragma unroll
  for (int n = 0; n < 4; ++n) o[Lay<OVS_ASM_TEM>::RHS0 + n] = rt[n];
}

// -------------------------------------------------- pass 2: block expansion
// Blocks of row A (local node la) of one element from its summary, for a
// column node b (formulas factored from the reference's per Gauss point
// sums, with the sums of block_sums):
//   K(i,j) = KA ga_j gb_i + KB ga_i gb_j + delta_ij (KA gab + S_ab)
//   G(i) = -ga_i PR_b + gb_i Q_a      D(i) = gb_i PR_a + ga_i T_b
//   M = MM gab    LS = L1_ab + E_ab + KDP gab    ULS(i) = ga_i U_b
//   PLS = PL_ab   LSU(i) = dphi_i V_ab - gb_i U_a
// 4 consecutive values: read-only global loads (SMEM = false) or loads from
// the warp's shared-memory stage (SMEM = true)
template <typename T, bool SMEM = false>
__device__ __forceinline__ void ldv4(const T* p, T* d) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = SMEM ? *reinterpret_cast<const float4*>(p) : __ldg(reinterpret_cast<const float4*>(p));
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
  } else {
    const double2 a = SMEM ? reinterpret_cast<const double2*>(p)[0] : __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = SMEM ? reinterpret_cast<const double2*>(p)[1] : __ldg(reinterpret_cast<const double2*>(p) + 1);
    d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y;
  }
}
template <typename T, bool SMEM = false>
__device__ __forceinline__ T ld1(const T* p) {
  if constexpr (SMEM) return *p;
  else return __ldg(p);
}

// the summary values an NS/NS+VOF block (la, b) is formed from: node la's
// record, the element constants, node b's record and the pair sums
template <typename T> struct BlockIn {
  T na[8], cs[8], nb[8], pr[4];
};

template <typename T, int KIND, bool SMEM>
__device__ __forceinline__ void load_block(const T* sm, int la, int b, BlockIn<T>& in) {
  using L = Lay<KIND>;
  constexpr bool vof = KIND == OVS_ASM_NSVOF;
  ldv4<T, SMEM>(sm + L::ND0 + 8 * la, in.na);
  ldv4<T, SMEM>(sm + L::ND0 + 8 * la + 4, in.na + 4);
  ldv4<T, SMEM>(sm + L::C0, in.cs);
  ldv4<T, SMEM>(sm + L::ND0 + 8 * b, in.nb);
  ldv4<T, SMEM>(sm + L::ND0 + 8 * b + 4, in.nb + 4);
  if constexpr (vof) {
    ldv4<T, SMEM>(sm + L::C0 + 4, in.cs + 4);
    ldv4<T, SMEM>(sm + L::PW * (4 * la + b), in.pr);
  } else {
    in.pr[0] = ld1<T, SMEM>(sm + L::PW * (4 * la + b));
  }
}

template <typename T, int KIND>
__device__ __forceinline__ void form_block(const BlockIn<T>& in, T (&o)[Lay<KIND>::NV]) {
  constexpr bool vof = KIND == OVS_ASM_NSVOF;
  const T ga[3] = {in.na[0], in.na[1], in.na[2]};
  const T Ra = in.na[3], Wa = in.na[5], Qa = in.na[6];
  const T KA = in.cs[0], KB = in.cs[1], MM = in.cs[2];
  const T gk[3] = {in.nb[0], in.nb[1], in.nb[2]};
  const T Pb = in.nb[3], Tb = in.nb[4], Ub = in.nb[5];
  const T gab = ga[0] * gk[0] + ga[1] * gk[1] + ga[2] * gk[2];
  const T dg = KA * gab + in.pr[0];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) o[4 * i + j] = KA * ga[j] * gk[i] + KB * ga[i] * gk[j] + (i == j ? dg : (T)0);
    o[4 * i + 3] = -ga[i] * Pb + gk[i] * Qa;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) o[12 + d] = gk[d] * Ra + ga[d] * Tb;
  o[15] = MM * gab;
  if constexpr (vof) {
    const T KDP = in.cs[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) o[16 + d] = in.cs[4 + d] * in.pr[3] - gk[d] * Wa;
    o[19] = in.pr[1] + KDP * gab;
#pragma unroll
    for (int d = 0; d < 3; ++d) o[20 + d] = ga[d] * Ub;
    o[23] = in.pr[2];
  }
}

// Blocks (row node la, column nodes b0 + k*BS, k < NC) of an element from
// its summary.  The 4 lanes of an NS/NS+VOF element take one column each
// (NC = 1); a T lane takes all four.  sm: the element's summary (global
// memory, or its matrix part staged in shared memory with SMEM); the
// residual rows behind it are read by the caller
template <typename T, int KIND, int NC, bool SMEM = false>
__device__ __forceinline__ void expand_block(const T* sm, int la, int b0, int BS,
                                             T (&o)[NC][Lay<KIND>::NV < 4 ? 1 : Lay<KIND>::NV]) {
  if constexpr (KIND == OVS_ASM_TEM) {
    // the element pass stored the element matrix: row la, columns b
#pragma unroll
    for (int k = 0; k < NC; ++k) o[k][0] = sm[4 * la + b0 + k * BS];
  } else {
#pragma unroll
    for (int k = 0; k < NC; ++k) {
      BlockIn<T> in;
      load_block<T, KIND, SMEM>(sm, la, b0 + k * BS, in);
      form_block<T, KIND>(in, o[k]);
    }
  }
}

template <typename T> struct Vec4 {};
template <> struct Vec4<float> {
  __device__ static void add(float* dst, const float* src) {
    float4 a = *reinterpret_cast<float4*>(dst);
    float4 b = *reinterpret_cast<const float4*>(src);
    a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w;
    *reinterpret_cast<float4*>(dst) = a;
  }
};
template <> struct Vec4<double> {
  __device__ static void add(double* dst, const double* src) {
    double2 a0 = reinterpret_cast<double2*>(dst)[0], a1 = reinterpret_cast<double2*>(dst)[1];
    double2 b0 = reinterpret_cast<const double2*>(src)[0], b1 = reinterpret_cast<const double2*>(src)[1];
    a0.x += b0.x; a0.y += b0.y; a1.x += b1.x; a1.y += b1.y;
    reinterpret_cast<double2*>(dst)[0] = a0;
    reinterpret_cast<double2*>(dst)[1] = a1;
  }
};

// shared-memory layout per warp: the blocks of the chunk's elements
// [CH elements][4 columns][BSTR] (stride padded so the 16-byte stores of a
// quarter warp hit distinct banks), their RHS rows [CH][RSTR], the row
// accumulator [max_deg][NVP], then the slot words of the chunk's elements
// [CH], the columns [max_deg] and their Dirichlet masks [max_deg]
template <typename T, int KIND> struct Smem {
  static constexpr int NV = Lay<KIND>::NV, NF = Lay<KIND>::NF;
  static constexpr int LPE = (NV < 4) ? 1 : 4;       // lanes per element
  static constexpr int CH = 32 / LPE;                // elements per chunk
  static constexpr int NVP = (NV < 4) ? 1 : NV;
  static constexpr int BSTR = (NV < 4) ? 1 : NV + 16 / (int)sizeof(T);
  static constexpr int RSTR = NF + 1;
  // the stage buffer of the staged row pass: the chunk's CH element
  // summaries, copied in with one round of asynchronous 16-byte copies
  static constexpr int SW = Lay<KIND>::SW;
  // values staged per element: the matrix part of the summary (the residual
  // rows behind it are read from global memory by the lanes that need them)
  static constexpr int SWS = (KIND == OVS_ASM_TEM) ? SW : Lay<KIND>::RHS0;
  __host__ __device__ static size_t ints_offset(int max_deg) {
    const size_t b = sizeof(T) * ((size_t)4 * CH * BSTR + (size_t)CH * RSTR + (size_t)max_deg * NVP);
    return (b + 15) & ~(size_t)15;
  }
  __host__ __device__ static size_t bytes(int max_deg, bool staged = false) {
    size_t b = ints_offset(max_deg) + sizeof(int) * ((size_t)CH + 2 * (size_t)max_deg);
    b = (b + 15) & ~(size_t)15;
    if (staged) b += sizeof(T) * (size_t)CH * SWS;
    return b;
  }
  __host__ __device__ static size_t stage_offset(int max_deg) { return bytes(max_deg, false); }
};

// 16-byte asynchronous global -> shared copy (cp.async, no register
// staging) and 4-byte variant; completion by cp_async_wait_all
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// ---------------------------------------------------------- pass 1 kernel
// blocks per SM the element pass is compiled for: the FP32 NS+VOF pass at 3
// (168 registers, measured faster than the unbounded 178 and than 2 or 4),
// the FP32 temperature pass at 4 (1.25 against 1.45 ms at 160 registers),
// the others as the compiler chooses (the FP64 temperature pass measured
// slower at 3)
template <typename T, int KIND> struct SumMinBlocks { static constexpr int v = 1; };
template <> struct SumMinBlocks<float, OVS_ASM_NSVOF> { static constexpr int v = 3; };
template <> struct SumMinBlocks<float, OVS_ASM_TEM> { static constexpr int v = 4; };

template <typename T, int KIND, bool SMEMREC> struct SumBlocks { static constexpr int v = SumMinBlocks<T, KIND>::v; };
// FP64 with the node records in shared memory: 2 blocks (up to 255
// registers, measured 7.1 ms for NS+VOF at 128^3 against 7.6 ms at 3
// blocks and 10.2 ms at 4)
template <int KIND> struct SumBlocks<double, KIND, true> { static constexpr int v = 2; };

template <typename T, int KIND, bool SMEMREC>
__global__ void __launch_bounds__(128, (SumBlocks<T, KIND, SMEMREC>::v))
element_summary_kernel(const SumArgs a) {
  using L = Lay<KIND>;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double tamax = 0.0;   // the element's largest taua over its points (CflPerPoint: largest CFL number)
  int nbad = 0;
  if (e < a.E) {
    const int4 nd = __ldg(reinterpret_cast<const int4*>(a.ien) + e);
    const int nodes[4] = {nd.x, nd.y, nd.z, nd.w};
    const T* rec = reinterpret_cast<const T*>(a.rec);
    const int eid = __ldg(a.elm_id + e);
    T detj;
    auto run = [&](const auto& r, const auto& lo, T* o) {
      if constexpr (KIND == OVS_ASM_NS) {
        const bool target = ((a.p.subdomain_flag & 1) && eid == a.p.elm_id_set[0]) ||
                            ((a.p.subdomain_flag & 2) && eid == a.p.elm_id_set[1]);
        summarize_ns<T>(a, r, lo, target, o, tamax, detj);
      } else if constexpr (KIND == OVS_ASM_NSVOF) {
        summarize_nsvof<T>(a, r, lo, eid == a.p.fluid_elm_id, o, tamax, detj);
      } else {
        summarize_tem<T>(a, r, lo, eid == a.p.fluid_elm_id, o, tamax, detj);
      }
    };
    if constexpr (SMEMREC && sizeof(T) == 8) {
      // records through shared memory; the summary written straight to
      // global memory as its values are produced
      extern __shared__ __align__(16) unsigned char sm_elem[];
      T* col = reinterpret_cast<T*>(sm_elem) + threadIdx.x;
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const double2* q = reinterpret_cast<const double2*>(rec) + (size_t)nodes[n] * (REC / 2);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double2 v = __ldg(q + k);
          col[(size_t)(n * 16 + 2 * k) * 128] = v.x;
          col[(size_t)(n * 16 + 2 * k + 1) * 128] = v.y;
        }
      }
      run(SmemRecs<T>{col}, ZeroRecs<T>{}, reinterpret_cast<T*>(a.sum) + (size_t)e * L::SW);
    } else {
      T r[4][16], lo[4][4];
#pragma unroll
      for (int n = 0; n < 4; ++n) load_rec(rec, nodes[n], r[n], lo[n]);
      if constexpr (KIND == OVS_ASM_TEM) {
        T o[L::SW];
        run(r, lo, o);
        // 20 values per tet: 5 groups of 4 (256-bit stores in FP64, the
        // summary 32-byte aligned; 2.45 against 2.52 ms at 128^3)
        T* dst = reinterpret_cast<T*>(a.sum) + (size_t)e * L::SW;
        if constexpr (sizeof(T) == 8) {
#pragma unroll
          for (int k = 0; k < L::SW; k += 4) put4(dst + k, o[k], o[k + 1], o[k + 2], o[k + 3]);
        } else {
          store_row<L::SW>(dst, o);
        }
      } else {
        // NS / NS+VOF write their summary with vector stores as its parts
        // are formed
        run(r, lo, reinterpret_cast<T*>(a.sum) + (size_t)e * L::SW);
      }
    }
    if (!(detj > (T)0)) nbad = 1;
  }
  // the CFL number of the element (CflPerPoint: already the number itself)
  double cfl = CflPerPoint<T, KIND>::v ? tamax : (double)a.p.delt * sqrt(tamax);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    cfl = fmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
    nbad += __shfl_xor_sync(0xffffffffu, nbad, off);
  }
  if ((threadIdx.x & 31) == 0) {
    cfl_max(a.cfl_bits, cfl);
    if (nbad) atomicAdd(a.flags, nbad);
  }
}

// ---------------------------------------------------------- pass 2 kernel
// The masks of the Dirichlet treatment, per value position v:
// bits 0-7 row (A) constraints, 8-15 column (B) constraints, 16-23 the
// diagonal entry set to 1 per element.
__device__ __forceinline__ unsigned mask_of(int v) {
  return (unsigned)c_rowbits[v] | ((unsigned)c_colbits[v] << 8) | ((unsigned)c_diagbit[v] << 16);
}

// One warp per CSR row, the rows in the order of the row records (Morton
// order of the nodes, so that the rows sharing an element run close
// together in time and its summary comes from L2).  Per chunk of CH of the
// row's elements: phase 1 expands block (A's row, column b) of each element
// into shared memory (lane = element, column), phase 2 adds them into the
// row accumulator, each lane owning value groups of whole slots and adding
// the chunk's blocks that fall in its slot in ascending element order (so
// every entry is summed in the same order on every run).  The next row's
// record and its first element ids are loaded while the current row runs,
// and the Dirichlet masks of the row's columns while its first chunk runs.
// STAGED: the warp first copies the chunk's element summaries into its
// shared-memory stage with one round of asynchronous 16-byte copies (all in
// flight together, no registers held); the block expansion then reads
// shared memory.  Otherwise every lane reads its element's summary from
// global memory.
template <typename T, int KIND, int WARPS, bool STAGED>
__global__ void __launch_bounds__(WARPS * 32)
assemble_rows_kernel(const AsmArgs a) {
  using S = Smem<T, KIND>;
  using L = Lay<KIND>;
  constexpr int NV = S::NV, NF = S::NF, NVP = S::NVP, BSTR = S::BSTR, RSTR = S::RSTR, CH = S::CH;
  constexpr int NG = (NV >= 4) ? NV / 4 : 1;   // value groups per slot: 4 values (T: the value)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned masks[24];
  if (threadIdx.x < 24) masks[threadIdx.x] = (KIND == OVS_ASM_TEM) ? (TB | (TB << 8) | (TB << 16)) : mask_of(threadIdx.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* base = smem_raw + (size_t)wid * S::bytes(a.max_deg, STAGED);
  T* stage = reinterpret_cast<T*>(base + S::stage_offset(a.max_deg));   // [CH][SWS] (STAGED)
  T* blk = reinterpret_cast<T*>(base);                 // [CH][4][BSTR]
  T* rvs = blk + 4 * CH * BSTR;                        // [CH][RSTR]
  T* acc = rvs + CH * RSTR;                            // [max_deg][NVP]
  unsigned* sl4 = reinterpret_cast<unsigned*>(base + S::ints_offset(a.max_deg));   // [CH]
  int* cols = reinterpret_cast<int*>(sl4 + CH);        // [max_deg]
  unsigned* cib = reinterpret_cast<unsigned*>(cols + a.max_deg);                 // [max_deg]

  const T* sum = reinterpret_cast<const T*>(a.rec);
  const int W = gridDim.x * WARPS;
  // lane = (element jl of the chunk, first column node bl0 of that element);
  // with one lane per element (T) a lane takes all 4 columns
  constexpr int LPE = S::LPE, CPL = 4 / LPE;
  const int jl = lane / LPE, bl0 = lane % LPE;
  constexpr int SWS = S::SWS;
  constexpr int U16 = SWS * (int)sizeof(T) / 16;            // 16-byte units staged per summary
  static_assert(SWS * sizeof(T) % 16 == 0, "staged summaries must be whole 16-byte units");
  static_assert(L::SW * sizeof(T) % 16 == 0, "summaries must be whole 16-byte units");
  int t = blockIdx.x * WARPS + wid;
  // row record {A, rowptr[A], n2e_ptr[A], deg | sd << 8 | ne << 16} and the element
  // ids of the first chunk (lanes j < nc hold entry j)
  int4 rr = make_int4(0, 0, 0, 0);
  if (t < a.nrows) rr = __ldg(a.row_rec + t);
  int pk_n = 0;
  unsigned s4_n = 0;
  if (t < a.nrows && lane < min(CH, rr.w >> 16)) {
    pk_n = __ldg(a.n2e + rr.z + lane);
    s4_n = __ldg(a.n2s + rr.z + lane);
  }
  for (; t < a.nrows; t += W) {
    const int A = rr.x, rp = rr.y, ep = rr.z, deg = rr.w & 0xff, ne = rr.w >> 16;
    int4 rn = make_int4(0, 0, 0, 0);
    if (t + W < a.nrows) rn = __ldg(a.row_rec + t + W);
    const unsigned ibA = __ldg(a.ibc + A);
    for (int s = lane; s < deg; s += 32) cp_async4(cols + s, a.colidx + rp + s);
    for (int q = lane; q < deg * NVP; q += 32) acc[q] = (T)0;
    T racc = (T)0;
    unsigned ib0 = 0, ib1 = 0;   // masks of columns lane and lane + 32
    __syncwarp();
    for (int c0 = 0; c0 < ne; c0 += CH) {
      const int nc = min(CH, ne - c0);
      const int pk_c = pk_n;
      const unsigned s4_c = s4_n;
      // the next chunk's ids travel while this one is expanded
      if (c0 + CH < ne && lane < min(CH, ne - c0 - CH)) {
        pk_n = __ldg(a.n2e + ep + c0 + CH + lane);
        s4_n = __ldg(a.n2s + ep + c0 + CH + lane);
      }
      if constexpr (STAGED) {
        // every lane runs the same trip count: the shuffle needs the full warp
        for (int it = 0; it < (CH * U16 + 31) / 32; ++it) {
          const int u = lane + 32 * it;
          const int j = min(u / U16, CH - 1);
          const int e = __shfl_sync(0xffffffffu, pk_c, j) >> 3;
          if (u < nc * U16) {
            const int k = u - j * U16;
            cp_async16(reinterpret_cast<unsigned char*>(stage + (size_t)j * SWS) + 16 * k,
                       reinterpret_cast<const unsigned char*>(sum + (size_t)e * L::SW) + 16 * k);
          }
        }
        cp_async_wait_all();
        __syncwarp();
      }
      // ---------------- phase 1: block (A's row, column bl) of element jl
      const int packed = __shfl_sync(0xffffffffu, pk_c, min(jl, CH - 1));
      const unsigned slots4 = __shfl_sync(0xffffffffu, s4_c, min(jl, CH - 1));
      if (jl < nc) {
        const int e = packed >> 3, la = packed & 7;
        T o[CPL][NVP];
        if constexpr (STAGED)
          expand_block<T, KIND, CPL, true>(stage + (size_t)jl * SWS, la, bl0, LPE, o);
        else
          expand_block<T, KIND, CPL>(sum + (size_t)e * L::SW, la, bl0, LPE, o);
#pragma unroll
        for (int k = 0; k < CPL; ++k) {
          T* dst = blk + (jl * 4 + bl0 + k * LPE) * BSTR;
          if constexpr (NV >= 4) {
#pragma unroll
            for (int v = 0; v < NV; v += 4) store_row<4>(dst + v, o[k] + v);
          } else {
            dst[0] = o[k][0];
          }
        }
        if (bl0 == 0) {   // the element's slot word and residual rows of node la
          sl4[jl] = slots4;
          const T* r = sum + (size_t)e * L::SW + L::RHS0 + NF * la;
#pragma unroll
          for (int f = 0; f < NF; ++f) rvs[jl * RSTR + f] = r[f];
        }
      }
      if (c0 == 0) {
        // the columns have arrived (their copies were issued at the row's
        // start); their masks travel while the row is assembled
        if constexpr (!STAGED) cp_async_wait_all();
        __syncwarp();
        if (lane < deg) ib0 = __ldg(a.ibc + cols[lane]);
        if (lane + 32 < deg) ib1 = __ldg(a.ibc + cols[lane + 32]);
      }
      __syncwarp();
      // ---------------- phase 2: ordered reduction into acc
      // task q = (slot s, value group g); the 4 blocks of one element go to
      // distinct slots (elements with a repeated node are rejected at upload)
      for (int q = lane; q < deg * NG; q += 32) {
        const int s = q / NG, g = q - s * NG;
        const unsigned key = (unsigned)s * 0x01010101u;
        if constexpr (NV >= 4) {
          T v[4];
          ldv4<T, true>(acc + s * NVP + 4 * g, v);
          for (int j = 0; j < nc; ++j) {
            const unsigned m = __vcmpeq4(sl4[j], key);
            if (m) {
              const int b = (__ffs(m) - 1) >> 3;
              T x[4];
              ldv4<T, true>(blk + (j * 4 + b) * BSTR + 4 * g, x);
              v[0] += x[0]; v[1] += x[1]; v[2] += x[2]; v[3] += x[3];
            }
          }
          store_row<4>(acc + s * NVP + 4 * g, v);
        } else {
          T v = acc[s];
          for (int j = 0; j < nc; ++j) {
            const unsigned m = __vcmpeq4(sl4[j], key);
            if (m) v += blk[j * 4 + ((__ffs(m) - 1) >> 3)];
          }
          acc[s] = v;
        }
      }
      if (lane < NF)
        for (int j = 0; j < nc; ++j) racc += rvs[j * RSTR + lane];
      __syncwarp();
    }
    if (ne == 0) {   // a node without elements: only the Dirichlet rows
      cp_async_wait_all();
      __syncwarp();
      if (lane < deg) ib0 = __ldg(a.ibc + cols[lane]);
      if (lane + 32 < deg) ib1 = __ldg(a.ibc + cols[lane + 32]);
    }
    // the next row's first element ids travel while this row is written
    pk_n = 0;
    s4_n = 0;
    if (t + W < a.nrows && lane < min(CH, rn.w >> 16)) {
      pk_n = __ldg(a.n2e + rn.z + lane);
      s4_n = __ldg(a.n2s + rn.z + lane);
    }
    // ---------------- row write with the Dirichlet treatment
    if (a.mat) {
      if (lane < deg) cib[lane] = ib0;
      if (lane + 32 < deg) cib[lane + 32] = ib1;
      for (int s = lane + 64; s < deg; s += 32) cib[s] = __ldg(a.ibc + cols[s]);
      __syncwarp();
      T* out = reinterpret_cast<T*>(a.vals) + (size_t)rp * NV;
      const T cnt = (T)ne;
      if constexpr (NV >= 4) {
        // one 4-value group per lane and step, 16-byte aligned (NV % 4 == 0)
        for (int q = lane; q < deg * NG; q += 32) {
          const int s = q / NG, gidx = q - s * NG;
          const unsigned ibB = cib[s];
          const bool dg = cols[s] == A;
          T v4[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const unsigned m = masks[4 * gidx + u];
            T val = acc[s * NVP + 4 * gidx + u];
            if ((ibA & m & 0xffu) || ((ibB << 8) & m & 0xff00u)) val = (T)0;
            if (dg && ((ibA << 16) & m & 0xff0000u)) val = cnt;
            v4[u] = val;
          }
          store4_cs(out + (size_t)s * NV + 4 * gidx, v4);
        }
      } else {
        for (int q = lane; q < deg; q += 32) {
          const int B = cols[q];
          const unsigned ibB = cib[q];
          T val = acc[q];
          if ((ibA & TB) || (ibB & TB)) val = (T)0;
          if (B == A && (ibA & TB)) val = cnt;
          __stcs(out + q, val);
        }
      }
    }
    if (a.vec && lane < NF) {
      unsigned bit;
      if (KIND == OVS_ASM_TEM) bit = TB;
      else bit = (lane < 3) ? (1u << lane) : (lane == 3 ? PB : FB);
      T v = (ibA & bit) ? (T)0 : racc;
      if (!isfinite((double)v)) atomicOr(a.flags + 1, 1);
      __stcs(reinterpret_cast<T*>(a.rhs) + (size_t)lane * a.N + A, v);
    }
    rr = rn;
    __syncwarp();
  }
}

// A block of NV values to its CSR slot with the Dirichlet treatment of the
// row (ibA) and column (ibB) masks; dg: the diagonal entry (cnt, the row's
// element count, on constrained diagonal positions)
template <typename T, int NV>
__device__ __forceinline__ void write_block(T* dst, const T* v, const unsigned* masks, unsigned ibA, unsigned ibB,
                                            bool dg, T cnt) {
  const bool plain = (ibA | ibB) == 0u;
  if constexpr (NV >= 4) {
#pragma unroll
    for (int g = 0; g < NV; g += 4) {
      T v4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        T val = v[g + u];
        if (!plain) {
          const unsigned m = masks[g + u];
          if ((ibA & m & 0xffu) || ((ibB << 8) & m & 0xff00u)) val = (T)0;
          if (dg && ((ibA << 16) & m & 0xff0000u)) val = cnt;
        }
        v4[u] = val;
      }
      store4_cs(dst + g, v4);
    }
  } else {
    T val = v[0];
    if ((ibA & TB) || (ibB & TB)) val = (T)0;
    if (dg && (ibA & TB)) val = cnt;
    __stcs(dst, val);
  }
}

// Gather row pass (tets): one warp per CSR row, every lane summing whole
// blocks of the row in registers, so that no element block passes through
// shared memory.  The work of a row is its off-diagonal entries'
// contribution lists (the elements holding both nodes, ascending) and the
// diagonal entry's list (all the row's elements, ascending, with the
// residual rows).  Each list is cut into pieces of at most R consecutive
// entries, R the fewest rounds for which the pieces fit the 32 lanes (an
// interior Kuhn-mesh row: 96 entries, lists of 4, 6 and 24, R = 4); a lane
// adds its piece one entry per round, loading the next entry while the
// current block is expanded.  The pieces' sums then meet in the warp's
// shared memory, and each output task (entry, 4-value group) adds its
// entry's pieces in order and writes the group, consecutive lanes writing
// consecutive groups.  Every entry is summed in an order fixed by the mesh,
// the same on every run.  A row with more than 31 off-diagonal entries
// takes further passes.  TILED: the element summaries come from the CTA's
// shared-memory stage (tile-local element numbers in n2e_loc / clist_loc),
// otherwise from global memory (element ids in n2e / clist).
template <typename T, int KIND> struct GatherGeom {
  static constexpr int NV = Lay<KIND>::NV, NF = Lay<KIND>::NF;
  static constexpr int NVP = NV < 4 ? 1 : NV;
  static constexpr int PSTR = ((NVP + NF) * (int)sizeof(T) + 15) / 16 * 16 / (int)sizeof(T);
};
// per warp: the lanes' piece sums and the pass's entry table (slot, first
// lane, lanes, column mask; the diagonal last)
template <typename T, int KIND> struct GatherSmem {
  T part[32][GatherGeom<T, KIND>::PSTR];
  int slot[33], first[33], nl[33];
  unsigned ib[33];
};

__device__ __forceinline__ int warp_excl_scan(int v, int lane) {
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  return x - v;
}


template <typename T, int KIND, bool TILED>
__device__ __forceinline__ void gather_row(const AsmArgs& a, const int4 rr, const T* base, int str,
                                           const uint16_t* n2e_loc, const uint16_t* clist_loc,
                                           GatherSmem<T, KIND>& w, const unsigned* masks, int lane) {
  using L = Lay<KIND>;
  using Q = GatherGeom<T, KIND>;
  constexpr int NV = Q::NV, NF = Q::NF, NVP = Q::NVP;
  constexpr int NG = NV >= 4 ? NV / 4 : 1, GW = NV >= 4 ? 4 : 1;
  constexpr unsigned FULL = 0xffffffffu;
  const int A = rr.x, rp = rr.y, ep = rr.z, deg = rr.w & 0xff, sd = (rr.w >> 8) & 0xff, ne = rr.w >> 16;
  const unsigned ibA = __ldg(a.ibc + A);
  const int nod = deg > 0 ? deg - 1 : 0;
  T* out = reinterpret_cast<T*>(a.vals) + (size_t)rp * NV;
  const T cnt = (T)ne;
  for (int o0 = 0; o0 == 0 || o0 < nod;) {
    const bool wd = o0 == 0;                        // this pass also takes the diagonal and the residual
    const int nsl = min(nod - o0, wd ? 31 : 32);    // the pass's off-diagonal entries
    int s = 0, c0 = 0, len = 0;                     // lane j < nsl: entry j
    unsigned ibB = 0;
    if (lane < nsl) {
      const int o = o0 + lane;
      s = o < sd ? o : o + 1;
      c0 = __ldg(a.cptr + rp + s);
      len = __ldg(a.cptr + rp + s + 1) - c0;
      ibB = __ldg(a.ibc + __ldg(a.colidx + rp + s));
    }
    const int nd = wd ? ne : 0;
    int R = max(1, (__reduce_add_sync(FULL, len) + nd + 31) / 32);
    while (__reduce_add_sync(FULL, (len + R - 1) / R) + (nd + R - 1) / R > 32) ++R;
    const int P = (len + R - 1) / R;                // lanes of entry j
    const int F = warp_excl_scan(P, lane);          // its first lane
    const int Fd = __reduce_add_sync(FULL, P);      // the diagonal's first lane
    const int PD = (nd + R - 1) / R;
    if (lane < nsl) {
      w.slot[lane] = s; w.first[lane] = F; w.nl[lane] = P; w.ib[lane] = ibB;
    }
    if (wd && lane == 0) {
      w.slot[nsl] = sd; w.first[nsl] = Fd; w.nl[nsl] = PD; w.ib[nsl] = ibA;
    }
    // this lane's piece: of entry k (the last with first lane <= lane), or
    // of the diagonal list
    int k = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int j = k + step;
      const int Fj = __shfl_sync(FULL, F, j & 31);
      if (j < nsl && Fj <= lane) k = j;
    }
    const int Fk = __shfl_sync(FULL, F, k), c0k = __shfl_sync(FULL, c0, k), lenk = __shfl_sync(FULL, len, k);
    const bool dl = lane >= Fd && lane < Fd + PD;  // a diagonal piece
    int pc0 = 0, plen = 0;
    if (lane < Fd) {
      pc0 = c0k + (lane - Fk) * R;
      plen = min(R, lenk - (lane - Fk) * R);
    } else if (dl) {
      pc0 = ep + (lane - Fd) * R;
      plen = min(R, ne - (lane - Fd) * R);
    }
    T acc[NVP], racc[NF];
#pragma unroll
    for (int v = 0; v < NVP; ++v) acc[v] = (T)0;
#pragma unroll
    for (int f = 0; f < NF; ++f) racc[f] = (T)0;
    // entry i of the piece: off-diagonal (e << 4) | (la << 2) | b, diagonal
    // (e << 3) | la (tiled: (tile-local element << 2) | la)
    auto entry = [&](int i) -> int {
      if constexpr (TILED) return dl ? (int)__ldg(n2e_loc + pc0 + i) : (int)__ldg(clist_loc + pc0 + i);
      else return dl ? __ldg(a.n2e + pc0 + i) : __ldg(a.clist + pc0 + i);
    };
    // one entry per round, the next round's entry loaded ahead (a second
    // buffer of summary loads in flight measured slower in FP64, 13.3 vs
    // 12.7 ms at 128^3: 235 registers and 8 warps per SM against 128 and 16)
    int ent = plen > 0 ? entry(0) : 0;
    for (int r = 0; r < R; ++r) {
      const int cur = ent;
      if (r + 1 < plen) ent = entry(r + 1);
      if (r < plen) {
        int e, la, b;
        if (!dl) {
          e = cur >> 4; la = (cur >> 2) & 3; b = cur & 3;
        } else if constexpr (TILED) {
          e = cur >> 2; la = cur & 3; b = la;
        } else {
          e = cur >> 3; la = cur & 7; b = la;
        }
        const T* se = base + (size_t)e * str;
        T ob[1][NVP];
        expand_block<T, KIND, 1, TILED>(se, la, b, 0, ob);
#pragma unroll
        for (int v = 0; v < NVP; ++v) acc[v] += ob[0][v];
        if (dl) {
#pragma unroll
          for (int f = 0; f < NF; ++f) racc[f] += ld1<T, TILED>(se + L::RHS0 + NF * la + f);
        }
      }
    }
    if (plen > 0) {
#pragma unroll
      for (int v = 0; v < NVP; ++v) w.part[lane][v] = acc[v];
      if (dl) {
#pragma unroll
        for (int f = 0; f < NF; ++f) w.part[lane][NVP + f] = racc[f];
      }
    }
    __syncwarp();
    // output tasks (entry j, group g): the entry's pieces added in order
    if (a.mat && deg > 0) {
      const int nt = (nsl + (wd ? 1 : 0)) * NG;
      for (int q = lane; q < nt; q += 32) {
        const int j = q / NG, g = q - j * NG;
        const int f0 = w.first[j], n = w.nl[j];
        const unsigned ib = w.ib[j];
        const bool dg = wd && j == nsl;
        T v[GW];
#pragma unroll
        for (int u = 0; u < GW; ++u) v[u] = (T)0;
        for (int pp = 0; pp < n; ++pp)
#pragma unroll
          for (int u = 0; u < GW; ++u) v[u] += w.part[f0 + pp][GW * g + u];
        T* dst = out + (size_t)w.slot[j] * NV + GW * g;
        if constexpr (NV >= 4) {
          if ((ibA | ib) != 0u) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const unsigned m = masks[4 * g + u];
              if ((ibA & m & 0xffu) || ((ib << 8) & m & 0xff00u)) v[u] = (T)0;
              if (dg && ((ibA << 16) & m & 0xff0000u)) v[u] = cnt;
            }
          }
          store4_cs(dst, v);
        } else {
          if ((ibA & TB) || (ib & TB)) v[0] = (T)0;
          if (dg && (ibA & TB)) v[0] = cnt;
          __stcs(dst, v[0]);
        }
      }
    }
    if (wd && a.vec && lane < NF) {
      T v = (T)0;
      for (int pp = 0; pp < PD; ++pp) v += w.part[Fd + pp][NVP + lane];
      unsigned bit;
      if (KIND == OVS_ASM_TEM) bit = TB;
      else bit = (lane < 3) ? (1u << lane) : (lane == 3 ? PB : FB);
      if (ibA & bit) v = (T)0;
      if (!isfinite((double)v)) atomicOr(a.flags + 1, 1);
      __stcs(reinterpret_cast<T*>(a.rhs) + (size_t)lane * a.N + A, v);
    }
    __syncwarp();
    o0 += nsl;
  }
}

// Interleaved form of the gather scheme (the temperature rows, whose
// blocks are single values: the piece bookkeeping above costs more than it
// saves there).  Lanes 0..GD-1 take the off-diagonal entries (lane l the
// l-th, counting past the diagonal slot; a row with more than GD of them
// takes further passes) and add each entry's whole list, one block per
// round; lanes GD..31 share the diagonal block and the residual rows, lane
// GD + i taking the row's elements i, i + ND, ... in ascending order, the ND
// partial sums then added in lane order.
template <typename T, int KIND, bool TILED>
__device__ __forceinline__ void gather_row_il(const AsmArgs& a, const int4 rr, const T* base, int str,
                                              const uint16_t* n2e_loc, const uint16_t* clist_loc,
                                              GatherSmem<T, KIND>& w, const unsigned* masks, int lane) {
  using L = Lay<KIND>;
  using Q = GatherGeom<T, KIND>;
  constexpr int NV = Q::NV, NF = Q::NF, NVP = Q::NVP, ND = 8, GD = 32 - ND;
  T(*pw)[Q::PSTR] = w.part;
  const bool diagl = lane >= GD;
  const int di = lane - GD;   // the diagonal lane's index
  const int A = rr.x, rp = rr.y, ep = rr.z, deg = rr.w & 0xff, sd = (rr.w >> 8) & 0xff, ne = rr.w >> 16;
  const unsigned ibA = __ldg(a.ibc + A);
  const int nod = deg > 0 ? deg - 1 : 0;
  T* out = reinterpret_cast<T*>(a.vals) + (size_t)rp * NV;
  const T cnt = (T)ne;
  for (int o0 = 0; o0 == 0 || o0 < nod; o0 += GD) {
    const int o = o0 + lane;   // off-diagonal ordinal of the lane
    const bool offl = !diagl && o < nod;
    const int s = o < sd ? o : o + 1;
    int c0 = 0, len = 0;
    unsigned ibB = 0;
    if (offl) {
      c0 = __ldg(a.cptr + rp + s);
      len = __ldg(a.cptr + rp + s + 1) - c0;
      ibB = __ldg(a.ibc + __ldg(a.colidx + rp + s));
    } else if (diagl && o0 == 0) {
      len = ne > di ? (ne - di + ND - 1) / ND : 0;
    }
    const int rounds = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
    T acc[NVP], racc[NF];
#pragma unroll
    for (int v = 0; v < NVP; ++v) acc[v] = (T)0;
#pragma unroll
    for (int f = 0; f < NF; ++f) racc[f] = (T)0;
    // entry k of the lane's list: off-diagonal (e << 4) | (la << 2) | b,
    // diagonal (e << 3) | la (tiled: the tile-local element number)
    auto entry = [&](int k) -> int {
      if constexpr (TILED) return offl ? (int)__ldg(clist_loc + c0 + k) : (int)__ldg(n2e_loc + ep + di + k * ND);
      else return offl ? __ldg(a.clist + c0 + k) : __ldg(a.n2e + ep + di + k * ND);
    };
    int ent = len > 0 ? entry(0) : 0;
    for (int k = 0; k < rounds; ++k) {
      const int cur = ent;
      if (k + 1 < len) ent = entry(k + 1);
      if (k < len) {
        int e, la, b;
        if (offl) {
          e = cur >> 4; la = (cur >> 2) & 3; b = cur & 3;
        } else if constexpr (TILED) {
          e = cur >> 2; la = cur & 3; b = la;
        } else {
          e = cur >> 3; la = cur & 7; b = la;
        }
        const T* se = base + (size_t)e * str;
        T ob[1][NVP];
        expand_block<T, KIND, 1, TILED>(se, la, b, 0, ob);
#pragma unroll
        for (int v = 0; v < NVP; ++v) acc[v] += ob[0][v];
        if (diagl) {
#pragma unroll
          for (int f = 0; f < NF; ++f) racc[f] += ld1<T, TILED>(se + L::RHS0 + NF * la + f);
        }
      }
    }
    if (offl && a.mat) write_block<T, NV>(out + (size_t)s * NV, acc, masks, ibA, ibB, false, cnt);
    if (o0 == 0) {
      if (diagl) {
#pragma unroll
        for (int v = 0; v < NVP; ++v) pw[di][v] = acc[v];
#pragma unroll
        for (int f = 0; f < NF; ++f) pw[di][NVP + f] = racc[f];
      }
      __syncwarp();
      constexpr int NG = NV >= 4 ? NV / 4 : 1;
      if (a.mat && deg > 0 && lane < NG) {
        constexpr int GW = NV >= 4 ? 4 : 1;
        T v4[GW];
#pragma unroll
        for (int u = 0; u < GW; ++u) v4[u] = pw[0][GW * lane + u];
        for (int i = 1; i < ND; ++i)
#pragma unroll
          for (int u = 0; u < GW; ++u) v4[u] += pw[i][GW * lane + u];
        if constexpr (NV >= 4) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const unsigned m = masks[4 * lane + u];
            if (ibA & m & 0xffu) v4[u] = (T)0;
            if ((ibA << 8) & m & 0xff00u) v4[u] = (T)0;
            if ((ibA << 16) & m & 0xff0000u) v4[u] = cnt;
          }
          store4_cs(out + (size_t)sd * NV + 4 * lane, v4);
        } else {
          T val = v4[0];
          if (ibA & TB) val = cnt;
          __stcs(out + sd, val);
        }
      }
      if (a.vec && lane >= 32 - NF) {
        const int f = lane - (32 - NF);
        T v = pw[0][NVP + f];
        for (int i = 1; i < ND; ++i) v += pw[i][NVP + f];
        unsigned bit;
        if (KIND == OVS_ASM_TEM) bit = TB;
        else bit = (f < 3) ? (1u << f) : (f == 3 ? PB : FB);
        if (ibA & bit) v = (T)0;
        if (!isfinite((double)v)) atomicOr(a.flags + 1, 1);
        __stcs(reinterpret_cast<T*>(a.rhs) + (size_t)f * a.N + A, v);
      }
      __syncwarp();
    }
  }
}

template <typename T, int KIND>
__global__ void __launch_bounds__(128) gather_rows_kernel(const AsmArgs a) {
  __shared__ unsigned masks[24];
  __shared__ __align__(16) GatherSmem<T, KIND> gw[4];
  if (threadIdx.x < 24) masks[threadIdx.x] = (KIND == OVS_ASM_TEM) ? (TB | (TB << 8) | (TB << 16)) : mask_of(threadIdx.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const T* sum = reinterpret_cast<const T*>(a.rec);
  const int W = gridDim.x * 4;
  for (int t = blockIdx.x * 4 + wid; t < a.nrows; t += W)
    if constexpr (KIND == OVS_ASM_TEM)
      gather_row_il<T, KIND, false>(a, __ldg(a.row_rec + t), sum, Lay<KIND>::SW, nullptr, nullptr, gw[wid], masks,
                                    lane);
    else
      gather_row<T, KIND, false>(a, __ldg(a.row_rec + t), sum, Lay<KIND>::SW, nullptr, nullptr, gw[wid], masks, lane);
}

// ---------------------------------------------------------- tiled row pass
// One CTA per row tile (ovs_tiles_build): the summaries of the tile's
// elements are copied into shared memory by bulk asynchronous copies
// (cp.async.bulk, completing on one mbarrier; from this GPU's own memory, no
// multicast), then the four warps take the tile's rows by the gather scheme
// above, reading the summaries from shared memory.  Each summary is fetched
// in whole 16-byte units, once per tile that uses it, instead of lane by
// lane in scattered 16-byte loads.
struct TileArgs {
  const int* rptr;
  const int* rows;
  const int* eptr;
  const int* elems;
  const uint16_t* n2e_loc;
  const uint16_t* clist_loc;
};

// a staged summary's stride in shared memory: an odd number of 16-byte
// units, so the lanes reading different elements spread over the banks
template <typename T, int KIND> struct TileStage {
  static constexpr int SWB = Lay<KIND>::SW * (int)sizeof(T);
  static constexpr int STRB = 16 * ((SWB / 16) | 1);
  static constexpr int STR = STRB / (int)sizeof(T);
  static_assert(SWB % 16 == 0, "summaries must be whole 16-byte units");
};

constexpr long TILE_WAIT_LIMIT = 1L << 26;   // bounded mbarrier wait (polls)

template <typename T, int KIND>
__global__ void __launch_bounds__(128) tiled_rows_kernel(const AsmArgs a, const TileArgs ta) {
  using G = TileStage<T, KIND>;
  extern __shared__ __align__(128) unsigned char tile_smem[];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ unsigned masks[24];
  __shared__ __align__(16) GatherSmem<T, KIND> gw[4];
  T* stage = reinterpret_cast<T*>(tile_smem);
  const int tile = blockIdx.x;
  const int k0 = __ldg(ta.eptr + tile), nel = __ldg(ta.eptr + tile + 1) - k0;
  const unsigned barp = (unsigned)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barp));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 24) masks[threadIdx.x] = (KIND == OVS_ASM_TEM) ? (TB | (TB << 8) | (TB << 16)) : mask_of(threadIdx.x);
  __syncthreads();
  if (threadIdx.x == 0)
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(barp), "r"((unsigned)(nel * G::SWB))
                 : "memory");
  __syncthreads();   // the expected bytes are registered before any copy completes
  const T* sum = reinterpret_cast<const T*>(a.rec);
  for (int k = threadIdx.x; k < nel; k += blockDim.x) {
    const int e = __ldg(ta.elems + k0 + k);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"((unsigned)__cvta_generic_to_shared(stage + (size_t)k * G::STR)), "l"(sum + (size_t)e * Lay<KIND>::SW),
                 "r"((unsigned)G::SWB), "r"(barp)
                 : "memory");
  }
  unsigned done = 0;
  for (long it = 0; it < TILE_WAIT_LIMIT && !done; ++it)
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(barp) : "memory");
  if (!done) {   // the copies did not land: report, assemble nothing
    if (threadIdx.x == 0) atomicOr(a.flags + 2, 1);
    return;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int r1 = __ldg(ta.rptr + tile + 1);
  for (int r = __ldg(ta.rptr + tile) + wid; r < r1; r += 4) {
    const int4 rr = __ldg(a.row_rec + __ldg(ta.rows + r));
    if constexpr (KIND == OVS_ASM_TEM)
      gather_row_il<T, KIND, true>(a, rr, stage, G::STR, ta.n2e_loc, ta.clist_loc, gw[wid], masks, lane);
    else
      gather_row<T, KIND, true>(a, rr, stage, G::STR, ta.n2e_loc, ta.clist_loc, gw[wid], masks, lane);
  }
}

// ---------------------------------------------------- alpha-stage records
// assembleQuenching / assembleNavSto alpha stage (src/solveQuenching.f90:26-37,
// src/assembleNavSto.f90:25-30) fused with the packing of the values the
// element kernels gather, 16 per node.
struct AlphaArgs {
  const double* f[OVS_F_COUNT];
  const double* xg;
  void* rec;
  int N;
  int tem;   // record layout of the temperature pass
  double almi, alfi;
};

template <typename T>
__global__ void alpha_records_kernel(const AlphaArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const size_t N = a.N;
  const double am = a.almi, af = a.alfi;
  T r[REC];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const size_t k = i + N * d;
    const double dga = a.f[OVS_F_DGOLD][k] + af * (a.f[OVS_F_DG][k] - a.f[OVS_F_DGOLD][k]);
    const double xd = a.xg[k] + dga;   // xl + dl of eval_shape_fem (:34)
    r[d] = (T)xd;
    r[16 + d] = (T)(xd - (double)r[d]);
    r[3 + d] = (T)(a.f[OVS_F_UGOLD][k] + af * (a.f[OVS_F_UG][k] - a.f[OVS_F_UGOLD][k]));
    r[6 + d] = (T)(a.f[OVS_F_UGMOLD][k] + af * (a.f[OVS_F_UGM][k] - a.f[OVS_F_UGMOLD][k]));
    if (!a.tem) r[9 + d] = (T)(a.f[OVS_F_ACGOLD][k] + am * (a.f[OVS_F_ACG][k] - a.f[OVS_F_ACGOLD][k]));
  }
  const double phia = a.f[OVS_F_PHIGOLD][i] + af * (a.f[OVS_F_PHIG][i] - a.f[OVS_F_PHIGOLD][i]);
  const double ta = a.f[OVS_F_TGOLD][i] + af * (a.f[OVS_F_TG][i] - a.f[OVS_F_TGOLD][i]);
  r[19] = (T)(phia - (double)(T)phia);
  if (!a.tem) {
    r[12] = (T)a.f[OVS_F_PG][i];
    r[13] = (T)phia;
    r[14] = (T)(a.f[OVS_F_RPHIGOLD][i] + am * (a.f[OVS_F_RPHIG][i] - a.f[OVS_F_RPHIGOLD][i]));
    r[15] = (T)ta;
  } else {
    r[9] = (T)phia;
    r[10] = (T)ta;
    r[11] = (T)(a.f[OVS_F_RTGOLD][i] + am * (a.f[OVS_F_RTG][i] - a.f[OVS_F_RTGOLD][i]));
    r[12] = r[13] = r[14] = r[15] = (T)0;
  }
  T* o = reinterpret_cast<T*>(a.rec) + (size_t)i * REC;
#pragma unroll
  for (int k = 0; k < REC; ++k) o[k] = r[k];
}

template <typename T, int KIND, int WARPS, bool STAGED>
int launch_rows(ovs_ctx* c, const AsmArgs& a) {
  using S = Smem<T, KIND>;
  const size_t smem = S::bytes(a.max_deg, STAGED) * WARPS;
  auto kern = assemble_rows_kernel<T, KIND, WARPS, STAGED>;
  OVS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem));
  if (per_sm < 1) return OVS_ERR_ARG;
  long need = ((long)c->N + WARPS - 1) / WARPS;
  long grid = (long)per_sm * c->num_sms * 4;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(int)grid, WARPS * 32, smem, c->stream>>>(a);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

template <typename T, int KIND>
int launch_gather(ovs_ctx* c, const AsmArgs& a) {
  auto kern = gather_rows_kernel<T, KIND>;
  int per_sm = 0;
  OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0));
  if (per_sm < 1) return OVS_ERR_ARG;
  long need = ((long)a.nrows + 3) / 4;
  long grid = (long)per_sm * c->num_sms * 4;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(int)grid, 128, 0, c->stream>>>(a);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

template <typename T, int KIND>
int launch_tiled(ovs_ctx* c, const AsmArgs& a) {
  int st;
  if ((st = ovs_tiles_build(c, c->tile_elems_opt))) return st;
  using G = TileStage<T, KIND>;
  const size_t smem = (size_t)c->tile_maxe * G::STRB;
  auto kern = tiled_rows_kernel<T, KIND>;
  OVS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const TileArgs ta{c->tile_rptr, c->tile_rows, c->tile_eptr, c->tile_elems, c->n2e_loc, c->clist_loc};
  if (c->ntiles > 0) {
    kern<<<c->ntiles, 128, smem, c->stream>>>(a, ta);
    ++c->launches;
    OVS_CUDA_TRY(cudaGetLastError());
  }
  if (c->nbig > 0) {   // rows with more elements than a tile holds
    AsmArgs b = a;
    b.row_rec = c->big_rec;
    b.nrows = c->nbig;
    return launch_gather<T, KIND>(c, b);
  }
  return OVS_OK;
}

// parts: bit 0 the element pass, bit 1 the row pass
template <typename T, int KIND>
int launch_assemble(ovs_ctx* c, const AsmArgs& a, const SumArgs& sa, int parts = 3) {
  // pass 1: element summaries
  if (parts & 1) {
    if (sizeof(T) == 8 && (c->elem_smem > 0 || (c->elem_smem < 0 && KIND == OVS_ASM_NSVOF))) {
      // the node records of the block's 128 elements in shared memory
      const size_t esm = sizeof(T) * 64 * 128;
      OVS_CUDA_TRY(cudaFuncSetAttribute(element_summary_kernel<T, KIND, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esm));
      element_summary_kernel<T, KIND, true><<<(sa.E + 127) / 128, 128, esm, c->stream>>>(sa);
    } else {
      element_summary_kernel<T, KIND, false><<<(sa.E + 127) / 128, 128, 0, c->stream>>>(sa);
    }
    ++c->launches;
    OVS_CUDA_TRY(cudaGetLastError());
  }
  if (!(parts & 2)) return OVS_OK;
  // pass 2: rows
  // the temperature summaries (20 values, one lane per element) gain
  // nothing from staging: measured slower, so it reads them directly
  if (c->rows_tiled && c->cptr) return launch_tiled<T, KIND>(c, a);
  if (c->rows_gather && c->cptr) return launch_gather<T, KIND>(c, a);
  if (c->rows_staged && KIND != OVS_ASM_TEM) return launch_rows<T, KIND, 4, true>(c, a);
  return launch_rows<T, KIND, 4, false>(c, a);
}


// ------------------------------------------------ adjoint of the residual
// VJP of the assembled residual (the RHS the row pass writes, FP64) with
// respect to the nodal state.  One thread per element recomputes the
// element's residual rows on dual numbers once per nodal input of the
// element (Gauss-point quantities are recomputed, not stored) and contracts
// the tangent rows with the cotangent, which is zero on Dirichlet rows (the
// row pass writes 0 there).  A node pass then sums the element terms in
// ascending element id (deterministic) and applies the alpha-stage chain
// factors: x+d_a = xg + ..., u_a = .. + alfi ug, p, phi_a = .. + alfi phig,
// T_a = .. + alfi Tg, a_a = .. + almi acg, phidot_a = .. + almi rphig,
// Tdot_a = .. + almi rTg (src/solveQuenching.f90:26-37).
struct VjpArgs {
  const double* rec;      // FP64 alpha-stage records of the kernel's layout
  const int* ien;
  const int* elm_id;
  const uint8_t* ibc;
  const double* cot;      // NF*N field-major
  double* ge;             // E*4*NC element terms
  int E, N;
  ovs_params p;
};

template <int KIND> struct VjpMap;
// record slot, output field (OVS_VJP_* order), chain factor kind (0: 1, 1: alfi, 2: almi)
template <> struct VjpMap<OVS_ASM_NSVOF> {
  static constexpr int NC = 13;
  __device__ static int slot(int q) { const int s[13] = {0, 1, 2, 3, 4, 5, 12, 13, 15, 9, 10, 11, 14}; return s[q]; }
};
template <> struct VjpMap<OVS_ASM_TEM> {
  static constexpr int NC = 9;
  __device__ static int slot(int q) { const int s[9] = {0, 1, 2, 3, 4, 5, 9, 10, 11}; return s[q]; }
};
static const int h_vjp_out_nsvof[13] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12};
static const int h_vjp_fac_nsvof[13] = {0, 0, 0, 1, 1, 1, 0, 1, 1, 2, 2, 2, 2};
static const int h_vjp_out_tem[9] = {0, 1, 2, 3, 4, 5, 7, 8, 13};
static const int h_vjp_fac_tem[9] = {0, 0, 0, 1, 1, 1, 1, 1, 2};

template <int KIND>
__global__ void __launch_bounds__(128) residual_vjp_kernel(const VjpArgs a) {
  using L = Lay<KIND>;
  using M = VjpMap<KIND>;
  constexpr int NF = L::NF;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.E) return;
  const int4 nd = __ldg(reinterpret_cast<const int4*>(a.ien) + e);
  const int nodes[4] = {nd.x, nd.y, nd.z, nd.w};
  double r[4][16], lo[4][4];
#pragma unroll
  for (int n = 0; n < 4; ++n) load_rec(a.rec, nodes[n], r[n], lo[n]);
  const bool fluid = __ldg(a.elm_id + e) == a.p.fluid_elm_id;
  double vv[4][NF];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const unsigned ib = __ldg(a.ibc + nodes[m]);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const unsigned bit = KIND == OVS_ASM_TEM ? TB : (f < 3 ? (1u << f) : (f == 3 ? PB : FB));
      vv[m][f] = (ib & bit) ? 0.0 : a.cot[(size_t)f * a.N + nodes[m]];
    }
  }
  SumArgs sa;
  sa.p = a.p;
  for (int n = 0; n < 4; ++n) {
    for (int q = 0; q < M::NC; ++q) {
      Dual rd[4][16], ld[4][4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
#pragma unroll
        for (int k = 0; k < 16; ++k) rd[m][k] = Dual(r[m][k]);
#pragma unroll
        for (int k = 0; k < 4; ++k) ld[m][k] = Dual(lo[m][k]);
      }
      rd[n][M::slot(q)].d = 1.0;
      Dual o[L::SW];
      double cfl = 0.0;
      Dual detj;
      if constexpr (KIND == OVS_ASM_NSVOF) summarize_nsvof<Dual>(sa, rd, ld, fluid, o, cfl, detj);
      else summarize_tem<Dual>(sa, rd, ld, fluid, o, cfl, detj);
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int f = 0; f < NF; ++f) acc += vv[m][f] * o[L::RHS0 + NF * m + f].d;
      a.ge[((size_t)e * 4 + n) * M::NC + q] = acc;
    }
  }
}

struct VjpGatherArgs {
  const int* n2e_ptr;
  const int* n2e;
  const double* ge;
  double* grad;           // OVS_VJP_COUNT*N field-major
  int N, NC;
  int out[16];
  double fac[16];
};

__global__ void vjp_gather_kernel(const VjpGatherArgs a) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= a.N) return;
  double s[16];
  for (int q = 0; q < a.NC; ++q) s[q] = 0.0;
  for (int k = a.n2e_ptr[A]; k < a.n2e_ptr[A + 1]; ++k) {
    const int packed = a.n2e[k];
    const double* g = a.ge + ((size_t)(packed >> 3) * 4 + (packed & 7)) * a.NC;
    for (int q = 0; q < a.NC; ++q) s[q] += g[q];
  }
  for (int f = 0; f < OVS_VJP_COUNT; ++f) a.grad[(size_t)f * a.N + A] = 0.0;
  for (int q = 0; q < a.NC; ++q) a.grad[(size_t)a.out[q] * a.N + A] = a.fac[q] * s[q];
}

#include "assemble_hex.cuh"

}  // namespace

// W = f_g (x) f_g of the hex tensor-core pass, split into TF32 hi + lo, in
// the canonical K-major no-swizzle layout: row n = 8 a + b, k = 16 g + 4 r + s,
// byte offset (k / 4) * 1024 + (n / 8) * 128 + (n % 8) * 16 + (k % 4) * 4.
static float host_tf32(double x) {   // round to the nearest TF32, ties away (cvt.rna)
  float f = (float)x;
  uint32_t b;
  memcpy(&b, &f, 4);
  b = (b + 0x1000u) & 0xFFFFE000u;
  memcpy(&f, &b, 4);
  return f;
}

int hex_tc_prepare(ovs_ctx* c) {
  int st;
  if ((st = ovs_ensure(&c->hex_kbuf, sizeof(float) * (size_t)c->E * 64 * 24))) return st;
  if (c->hex_w) return OVS_OK;
  static const int sgn[8][3] = {{-1, 1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1},
                                {-1, -1, -1}, {1, -1, -1}, {1, -1, 1}, {-1, -1, 1}};
  const double q = 0.57735026918963;   // the 2x2x2 points of hex_gp
  double f[8][4][8];
  for (int g = 0; g < 8; ++g) {
    const double xi = (g & 1) ? q : -q, eta = (g & 2) ? q : -q, ze = (g & 4) ? q : -q;
    for (int a = 0; a < 8; ++a) {
      const double sx = sgn[a][0], sy = sgn[a][1], sz = sgn[a][2];
      f[g][0][a] = (1.0 + sx * xi) * (1.0 + sy * eta) * (1.0 + sz * ze) * 0.125;
      f[g][1][a] = sx * (1.0 + sy * eta) * (1.0 + sz * ze) * 0.125;
      f[g][2][a] = sy * (1.0 + sx * xi) * (1.0 + sz * ze) * 0.125;
      f[g][3][a] = sz * (1.0 + sx * xi) * (1.0 + sy * eta) * 0.125;
    }
  }
  std::vector<float> hw(2 * 8192, 0.f);
  for (int n = 0; n < 64; ++n)
    for (int k = 0; k < 128; ++k) {
      const int a = n >> 3, b = n & 7, g = k >> 4, r = (k >> 2) & 3, s = k & 3;
      const double v = f[g][r][a] * f[g][s][b];
      const float hi = host_tf32(v), lo = host_tf32(v - (double)hi);
      const size_t off = ((size_t)(k >> 2) * 1024 + (n >> 3) * 128 + (n & 7) * 16 + (k & 3) * 4) / 4;
      hw[off] = hi;
      hw[8192 + off] = lo;
    }
  if ((st = ovs_ensure((void**)&c->hex_w, sizeof(float) * 2 * 8192))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->hex_w, hw.data(), sizeof(float) * 2 * 8192, cudaMemcpyHostToDevice, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

static int dispatch_assemble(ovs_ctx* c, int kernel, int prec, const AsmArgs& a, const SumArgs& sa,
                             int parts = 3) {
  if (c->nshl == 8) {   // trilinear hexahedra: NS+VOF and temperature passes
    if (kernel == OVS_ASM_NS) return OVS_ERR_ARG;
    if (prec == OVS_FP64)
      return kernel == OVS_ASM_NSVOF ? launch_assemble_hex<double, OVS_ASM_NSVOF>(c, a, sa, parts)
                                     : launch_assemble_hex<double, OVS_ASM_TEM>(c, a, sa, parts);
    return kernel == OVS_ASM_NSVOF ? launch_assemble_hex<float, OVS_ASM_NSVOF>(c, a, sa, parts)
                                   : launch_assemble_hex<float, OVS_ASM_TEM>(c, a, sa, parts);
  }
  if (prec == OVS_FP64) {
    if (kernel == OVS_ASM_NS) return launch_assemble<double, OVS_ASM_NS>(c, a, sa, parts);
    if (kernel == OVS_ASM_NSVOF) return launch_assemble<double, OVS_ASM_NSVOF>(c, a, sa, parts);
    return launch_assemble<double, OVS_ASM_TEM>(c, a, sa, parts);
  }
  if (kernel == OVS_ASM_NS) return launch_assemble<float, OVS_ASM_NS>(c, a, sa, parts);
  if (kernel == OVS_ASM_NSVOF) return launch_assemble<float, OVS_ASM_NSVOF>(c, a, sa, parts);
  return launch_assemble<float, OVS_ASM_TEM>(c, a, sa, parts);
}

static void fill_args(ovs_ctx* c, int prec, SysStore& S, int tensor_flag, AsmArgs& a, SumArgs& sa) {
  sa.rec = c->rec[prec];
  sa.ien = c->ien;
  sa.elm_id = c->elm_id;
  sa.sum = c->esum[prec];
  sa.flags = c->flags;
  sa.cfl_bits = c->cfl_bits;
  sa.E = c->E;
  sa.p = c->params;
  a.rec = c->esum[prec];     // pass 2 reads the summaries
  a.ien = c->ien;
  a.elm_id = c->elm_id;
  a.ibc = c->ibc;
  a.rowptr = c->rowptr;
  a.colidx = c->colidx;
  a.n2e_ptr = c->n2e_ptr;
  a.n2e = c->n2e;
  a.vals = S.vals;
  a.rhs = S.rhs;
  a.flags = c->flags;
  a.cfl_bits = c->cfl_bits;
  a.N = c->N;
  a.nrows = c->N;
  a.mat = (tensor_flag & OVS_TENSOR_MAT) != 0;
  a.vec = (tensor_flag & OVS_TENSOR_VEC) != 0;
  a.n2s = c->n2s;
  a.row_rec = c->row_rec;
  a.cptr = c->cptr;
  a.clist = c->clist;
  a.max_deg = c->max_deg;
  a.p = c->params;
  a.kbuf = nullptr;
}

// parts: 3 both passes, 1 the element pass, 2 the row pass (on the summaries
// of the warm-up run)
int ovs_profile_assemble(ovs_ctx* c, int kernel, int prec, int reps, double* ms, int parts) {
  if (kernel != OVS_ASM_NS && kernel != OVS_ASM_NSVOF && kernel != OVS_ASM_TEM) return OVS_ERR_ARG;
  const int sys = kernel == OVS_ASM_NS ? OVS_SYS_NS : (kernel == OVS_ASM_NSVOF ? OVS_SYS_NSVOF : OVS_SYS_TEM);
  SysStore& S = c->sys[sys][prec];
  if (!S.vals || !S.rhs || !c->rec[prec] || !c->esum[prec]) return OVS_ERR_STATE;
  AsmArgs a;
  SumArgs sa;
  fill_args(c, prec, S, OVS_TENSOR_MAT | OVS_TENSOR_VEC, a, sa);
  int st;
  if ((st = dispatch_assemble(c, kernel, prec, a, sa))) return st;  // warm
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  for (int r = 0; r < reps; ++r)
    if ((st = dispatch_assemble(c, kernel, prec, a, sa, parts))) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float t = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&t, c->ev0, c->ev1));
  *ms = (double)t / reps;
  return OVS_OK;
}

// the assembly status of the pass (flags and CFL number) to the host, or to
// the page-locked slots of ovs_assemble_async
static int finish_status(ovs_ctx* c, double* cfl) {
  cudaStream_t s = c->stream;
  if (c->defer_status) {   // ovs_assemble_async: the status travels to a page-locked slot, read at the wait
    const int k = c->async_n++;
    OVS_CUDA_TRY(cudaMemcpyAsync(c->h_async_flags + 4 * k, c->flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
    OVS_CUDA_TRY(cudaMemcpyAsync(c->h_async_cfl + k, c->cfl_bits, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 s));
    return OVS_OK;
  }
  int hflags[4];
  unsigned long long hcfl = 0;
  OVS_CUDA_TRY(cudaMemcpyAsync(hflags, c->flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(&hcfl, c->cfl_bits, sizeof(hcfl), cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  if (cfl) {
    double v;
    memcpy(&v, &hcfl, sizeof(v));
    *cfl = v;
  }
  if (hflags[3]) return OVS_ERR_PATTERN;
  if (hflags[2]) return OVS_ERR_TIMEOUT;
  if (hflags[1]) return OVS_ERR_NONFINITE;
  if (hflags[0]) return OVS_WARN_NEG_DETJ;
  return OVS_OK;
}

// alpha-stage records of a pass (the record layout of the NS+VOF or the
// temperature routine)
static int alpha_stage(ovs_ctx* c, int prec, bool tem) {
  AlphaArgs aa;
  for (int f = 0; f < OVS_F_COUNT; ++f) aa.f[f] = c->field[f];
  aa.xg = c->field[OVS_F_XG];
  aa.rec = c->rec[prec];
  aa.N = c->N;
  aa.tem = tem;
  aa.almi = c->params.almi;
  aa.alfi = c->params.alfi;
  if (prec == OVS_FP64) alpha_records_kernel<double><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(aa);
  else alpha_records_kernel<float><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(aa);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// one pass of `kernel` (alpha stage, element pass, row pass, faces) with its
// flags and CFL number accumulated on the device (cleared by the caller)
static int assemble_pass(ovs_ctx* c, int kernel, int tensor_flag, int prec) {
  const int sys = kernel == OVS_ASM_NS ? OVS_SYS_NS : (kernel == OVS_ASM_NSVOF ? OVS_SYS_NSVOF : OVS_SYS_TEM);
  const size_t ts = prec == OVS_FP64 ? 8 : 4;
  SysStore& S = c->sys[sys][prec];
  int st;
  if ((st = ovs_ensure(&S.vals, ts * (size_t)c->nnz * ovs_sys_nv(sys)))) return st;
  if ((st = ovs_ensure(&S.rhs, ts * (size_t)c->N * ovs_sys_nf(sys)))) return st;
  if ((st = ovs_ensure(&c->rec[prec], ts * (size_t)c->N * REC))) return st;
  const size_t sw = c->nshl == 8 ? (size_t)HexLay<OVS_ASM_NSVOF>::SW : (size_t)Lay<OVS_ASM_NSVOF>::SW;
  if ((st = ovs_ensure(&c->esum[prec], ts * (size_t)c->E * sw))) return st;
  if ((st = alpha_stage(c, prec, kernel == OVS_ASM_TEM))) return st;
  AsmArgs a;
  SumArgs sa;
  fill_args(c, prec, S, tensor_flag, a, sa);
  if ((st = dispatch_assemble(c, kernel, prec, a, sa))) return st;
  if ((st = ovs_faces_assemble(c, kernel, prec, a.mat, a.vec))) return st;
  if (a.mat) S.have_mat = true;
  if (a.vec) S.have_rhs = true;
  return OVS_OK;
}

int ovs_assemble_impl(ovs_ctx* c, int kernel, int tensor_flag, int prec, double* cfl) {
  if (!c->have_pattern || !c->have_params) return OVS_ERR_STATE;
  if (c->nshl != 4 && c->nshl != 8) return OVS_ERR_ARG;
  if (kernel == OVS_ASM_QUENCH) {   // the NS+VOF pass, then the temperature pass; one status
    if (prec != OVS_FP64 && prec != OVS_FP32) return OVS_ERR_ARG;
    int st;
    OVS_CUDA_TRY(cudaMemsetAsync(c->flags, 0, sizeof(int) * 4, c->stream));
    OVS_CUDA_TRY(cudaMemsetAsync(c->cfl_bits, 0, sizeof(unsigned long long), c->stream));
    if ((st = assemble_pass(c, OVS_ASM_NSVOF, tensor_flag, prec))) return st;
    if ((st = assemble_pass(c, OVS_ASM_TEM, tensor_flag, prec))) return st;
    return finish_status(c, cfl);
  }
  if (c->nshl == 8 && kernel == OVS_ASM_NS) return OVS_ERR_ARG;
  if (kernel != OVS_ASM_NS && kernel != OVS_ASM_NSVOF && kernel != OVS_ASM_TEM) return OVS_ERR_ARG;
  if (prec != OVS_FP64 && prec != OVS_FP32) return OVS_ERR_ARG;
  int st;
  OVS_CUDA_TRY(cudaMemsetAsync(c->flags, 0, sizeof(int) * 4, c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(c->cfl_bits, 0, sizeof(unsigned long long), c->stream));
  if ((st = assemble_pass(c, kernel, tensor_flag, prec))) return st;
  return finish_status(c, cfl);
}

int ovs_residual_vjp_impl(ovs_ctx* c, int kernel, const double* cot_host, double* grad_host) {
  if (!c->have_pattern || !c->have_params) return OVS_ERR_STATE;
  if (c->nshl != 4) return OVS_ERR_ARG;   // the adjoint covers the tet routines
  if (c->face_flags_all) return OVS_ERR_STATE;   // face terms are not differentiated
  if (kernel != OVS_ASM_NSVOF && kernel != OVS_ASM_TEM) return OVS_ERR_ARG;
  if (!cot_host || !grad_host) return OVS_ERR_ARG;
  const int tem = kernel == OVS_ASM_TEM;
  const int nf = tem ? 1 : 5, NC = tem ? VjpMap<OVS_ASM_TEM>::NC : VjpMap<OVS_ASM_NSVOF>::NC;
  const size_t N = c->N, E = c->E;
  int st;
  if ((st = ovs_ensure(&c->rec[OVS_FP64], sizeof(double) * N * REC))) return st;
  if ((st = ovs_ensure((void**)&c->vjp_cot, sizeof(double) * N * 5))) return st;
  if ((st = ovs_ensure((void**)&c->vjp_ge, sizeof(double) * E * 4 * 13))) return st;
  if ((st = ovs_ensure((void**)&c->vjp_grad, sizeof(double) * N * OVS_VJP_COUNT))) return st;
  cudaStream_t s = c->stream;
  AlphaArgs aa;
  for (int f = 0; f < OVS_F_COUNT; ++f) aa.f[f] = c->field[f];
  aa.xg = c->field[OVS_F_XG];
  aa.rec = c->rec[OVS_FP64];
  aa.N = c->N;
  aa.tem = tem;
  aa.almi = c->params.almi;
  aa.alfi = c->params.alfi;
  alpha_records_kernel<double><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, s>>>(aa);
  ++c->launches;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->vjp_cot, cot_host, sizeof(double) * N * nf, cudaMemcpyHostToDevice, s));
  VjpArgs va;
  va.rec = reinterpret_cast<const double*>(c->rec[OVS_FP64]);
  va.ien = c->ien;
  va.elm_id = c->elm_id;
  va.ibc = c->ibc;
  va.cot = c->vjp_cot;
  va.ge = c->vjp_ge;
  va.E = c->E;
  va.N = c->N;
  va.p = c->params;
  const int eb = (int)((E + 127) / 128);
  if (tem) residual_vjp_kernel<OVS_ASM_TEM><<<eb, 128, 0, s>>>(va);
  else residual_vjp_kernel<OVS_ASM_NSVOF><<<eb, 128, 0, s>>>(va);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  VjpGatherArgs ga;
  ga.n2e_ptr = c->n2e_ptr;
  ga.n2e = c->n2e;
  ga.ge = c->vjp_ge;
  ga.grad = c->vjp_grad;
  ga.N = c->N;
  ga.NC = NC;
  for (int q = 0; q < NC; ++q) {
    const int fk = tem ? h_vjp_fac_tem[q] : h_vjp_fac_nsvof[q];
    ga.out[q] = tem ? h_vjp_out_tem[q] : h_vjp_out_nsvof[q];
    ga.fac[q] = fk == 0 ? 1.0 : (fk == 1 ? c->params.alfi : c->params.almi);
  }
  vjp_gather_kernel<<<ovs_grid(c->N, 128, 1 << 30), 128, 0, s>>>(ga);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaMemcpyAsync(grad_host, c->vjp_grad, sizeof(double) * N * OVS_VJP_COUNT, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  return OVS_OK;
}
