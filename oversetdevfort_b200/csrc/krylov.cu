// Block-CSR SpMV, diagonal (block-Jacobi) preconditioner and GMRES (sm_100a).
//
// Replaces SparseProdUP_3D / SparseProd_NS_conv / SparseProd_LS
// (src/SparseProd.f90:4-60,167-242,128-161) and SparseGMRES_up /
// SparseGMRES_ns_conv / SparseGMRES_tem (src/SparseGMRES_NS.f90:4-369,
// src/SparseGMRES_NS_conv.f:1-406, src/SparseGMRES_tem.f90:1-256).
//
// SpMV: a group of lanes owns one CSR row.  The slot values of a row are
// contiguous (24/16/1 per slot), so the lanes of a group read one 16-byte
// group each per slot and the whole row streams with full sectors; the x
// gathers hit L2.  The preconditioner (exact 3x3 inverse of the velocity
// diagonal block, reciprocal diagonal for p / phi / T) is applied to the row
// result before the store, so one pass produces P^-1 A x.
//
// GMRES: one Arnoldi cycle follows the reference step by step (left
// preconditioning, modified Gram-Schmidt with the reference's fused
// "project off j-1, dot with j" order, Givens rotations, exit rule
// |e(k+1)| <= tol |P^-1 b| and k >= kspace_min, back-substitution,
// sol += sum y_j v_j).  All scalars live on the device; every dot product is
// a fixed-grid, fixed-order FP64 reduction (last-block-done), so results are
// bit-identical from run to run.  The host only polls the "done" word once
// per batch of iterations.
#include "ovs_internal.cuh"

#include <cooperative_groups.h>
#include <math.h>
#include <string.h>

namespace cg = cooperative_groups;

namespace {

constexpr int SPMV_THREADS = 256;

template <typename T> __device__ __forceinline__ T ldm(const T* p) { return __ldcs(p); }

__device__ __forceinline__ void ld4(const float* p, float v[4]) {
  float4 q = __ldcs(reinterpret_cast<const float4*>(p));
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
  double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Accumulation precision of the SpMV: FP32 storage accumulates in FP32 on
// the mixed path (the inner solver of the refinement), FP64 otherwise.
// (FP64 accumulation and an FP64 work vector in Gram-Schmidt were measured on
// the 2.1M-node quench system: they converged in as many refinement cycles
// and ran slower, so the mixed path keeps everything in FP32 except the dots,
// Givens and the refinement residual.)
template <typename A, typename B, bool ACC64> struct AccT { using type = double; };
template <> struct AccT<float, float, false> { using type = float; };

// MODE 0: y = A x ; MODE 1: y = P^-1 A x ; MODE 2: y = b - A x
// Block systems: NG groups of 4 values per slot, one lane per group.
//   NS   (NG=4): groups rows u1,u2,u3,p over columns (u1,u2,u3,p)
//   NSVOF(NG=6): + row phi over (u1,u2,u3,phi), + column phi into (u1,u2,u3,p)
// The RPW = 32/NG rows of warp chunk `wglob` (all 32 lanes take part in
// the shuffles).
template <int NG, typename TM, typename TX, typename TY, int MODE, bool ACC64>
__device__ __forceinline__ void spmv_block_warp(long wglob, int N, const int* __restrict__ rowptr,
                                                const int* __restrict__ colidx, const TM* __restrict__ vals,
                                                const TX* __restrict__ x, TY* __restrict__ y,
                                                const TM* __restrict__ pre, const double* __restrict__ b) {
  using AT = typename AccT<TM, TX, ACC64>::type;
  constexpr int NV = 4 * NG;
  constexpr int RPW = 32 / NG;  // rows per warp
  const int lane = threadIdx.x & 31;
  const int sub = lane / NG;
  const int g = lane - sub * NG;
  const long rowl = wglob * RPW + sub;
  const bool active = sub < RPW && rowl < N;
  const int row = active ? (int)rowl : 0;
  // column fields read by this lane's 4 values
  int cf0, cf1, cf2, cf3;
  if (NG == 6 && g == 5) { cf0 = cf1 = cf2 = cf3 = 4; }
  else { cf0 = 0; cf1 = 1; cf2 = 2; cf3 = (NG == 6 && g == 4) ? 4 : 3; }
  const TX* x0 = x + (size_t)cf0 * N;
  const TX* x1 = x + (size_t)cf1 * N;
  const TX* x2 = x + (size_t)cf2 * N;
  const TX* x3 = x + (size_t)cf3 * N;
  AT a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  if (active) {
    const int s0 = __ldg(rowptr + row), s1 = __ldg(rowptr + row + 1);
    int s = s0;
    for (; s + 1 < s1; s += 2) {
      const int c0 = __ldg(colidx + s), c1 = __ldg(colidx + s + 1);
      TM v[4], w[4];
      ld4(vals + (size_t)s * NV + 4 * g, v);
      ld4(vals + (size_t)(s + 1) * NV + 4 * g, w);
      a0 += (AT)v[0] * (AT)__ldg(x0 + c0); a1 += (AT)v[1] * (AT)__ldg(x1 + c0);
      a2 += (AT)v[2] * (AT)__ldg(x2 + c0); a3 += (AT)v[3] * (AT)__ldg(x3 + c0);
      a0 += (AT)w[0] * (AT)__ldg(x0 + c1); a1 += (AT)w[1] * (AT)__ldg(x1 + c1);
      a2 += (AT)w[2] * (AT)__ldg(x2 + c1); a3 += (AT)w[3] * (AT)__ldg(x3 + c1);
    }
    if (s < s1) {
      const int c0 = __ldg(colidx + s);
      TM v[4];
      ld4(vals + (size_t)s * NV + 4 * g, v);
      a0 += (AT)v[0] * (AT)__ldg(x0 + c0); a1 += (AT)v[1] * (AT)__ldg(x1 + c0);
      a2 += (AT)v[2] * (AT)__ldg(x2 + c0); a3 += (AT)v[3] * (AT)__ldg(x3 + c0);
    }
  }
  const int base = sub * NG;
  AT yv;
  if (NG == 6) {
    // lane 5 of the group holds the phi-column contributions of rows u1,u2,u3,p
    const AT t0 = __shfl_sync(0xffffffffu, a0, (base + 5) & 31);
    const AT t1 = __shfl_sync(0xffffffffu, a1, (base + 5) & 31);
    const AT t2 = __shfl_sync(0xffffffffu, a2, (base + 5) & 31);
    const AT t3 = __shfl_sync(0xffffffffu, a3, (base + 5) & 31);
    const AT add = g == 0 ? t0 : (g == 1 ? t1 : (g == 2 ? t2 : (g == 3 ? t3 : (AT)0)));
    yv = ((a0 + a1) + (a2 + a3)) + add;
  } else {
    yv = (a0 + a1) + (a2 + a3);
  }
  const AT y0 = __shfl_sync(0xffffffffu, yv, base & 31);
  const AT y1 = __shfl_sync(0xffffffffu, yv, (base + 1) & 31);
  const AT y2 = __shfl_sync(0xffffffffu, yv, (base + 2) & 31);
  if (!active || g >= NG - (NG == 6 ? 1 : 0)) return;
  AT z = yv;
  if (MODE == 1) {
    if (g < 3) {
      const TM* B = pre + (size_t)row * 9 + 3 * g;
      z = (AT)B[0] * y0 + (AT)B[1] * y1 + (AT)B[2] * y2;
    } else if (g == 3) {
      z = yv * (AT)pre[(size_t)9 * N + row];
    } else {
      z = yv * (AT)pre[(size_t)10 * N + row];
    }
  } else if (MODE == 2) {
    z = (AT)b[(size_t)g * N + row] - yv;
  }
  y[(size_t)g * N + row] = (TY)z;
}

template <int NG, typename TM, typename TX, typename TY, int MODE, bool ACC64>
__global__ void __launch_bounds__(SPMV_THREADS)
spmv_block_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                  const TM* __restrict__ vals, const TX* __restrict__ x, TY* __restrict__ y,
                  const TM* __restrict__ pre, const double* __restrict__ b,
                  const int* __restrict__ done) {
  if (done && *done) return;
  const long wglob = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  spmv_block_warp<NG, TM, TX, TY, MODE, ACC64>(wglob, N, rowptr, colidx, vals, x, y, pre, b);
}

// scalar CSR (temperature): 8 lanes per row
template <typename TM, typename TX, typename TY, int MODE, bool ACC64>
__device__ __forceinline__ void spmv_scalar_warp(long wglob, int N, const int* __restrict__ rowptr,
                                                 const int* __restrict__ colidx, const TM* __restrict__ vals,
                                                 const TX* __restrict__ x, TY* __restrict__ y,
                                                 const TM* __restrict__ pre, const double* __restrict__ b) {
  using AT = typename AccT<TM, TX, ACC64>::type;
  const int lane = threadIdx.x & 31;
  const int sub = lane >> 3, k = lane & 7;
  const long rowl = wglob * 4 + sub;
  const bool active = rowl < N;
  const int row = active ? (int)rowl : 0;
  AT a = 0;
  if (active) {
    const int s0 = __ldg(rowptr + row), s1 = __ldg(rowptr + row + 1);
    for (int s = s0 + k; s < s1; s += 8) a += (AT)ldm(vals + s) * (AT)__ldg(x + __ldg(colidx + s));
  }
  a += __shfl_xor_sync(0xffffffffu, a, 4);
  a += __shfl_xor_sync(0xffffffffu, a, 2);
  a += __shfl_xor_sync(0xffffffffu, a, 1);
  if (!active || k != 0) return;
  AT z = a;
  if (MODE == 1) z = a * (AT)pre[row];
  else if (MODE == 2) z = (AT)b[row] - a;
  y[row] = (TY)z;
}

template <typename TM, typename TX, typename TY, int MODE, bool ACC64>
__global__ void __launch_bounds__(SPMV_THREADS)
spmv_scalar_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                   const TM* __restrict__ vals, const TX* __restrict__ x, TY* __restrict__ y,
                   const TM* __restrict__ pre, const double* __restrict__ b,
                   const int* __restrict__ done) {
  if (done && *done) return;
  const long wglob = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  spmv_scalar_warp<TM, TX, TY, MODE, ACC64>(wglob, N, rowptr, colidx, vals, x, y, pre, b);
}

template <typename TM, typename TX, typename TY, int MODE, bool ACC64 = true>
int launch_spmv(ovs_ctx* c, int sys, const TM* vals, const TX* x, TY* y, const TM* pre,
                const double* b, const int* done) {
  const int N = c->N;
  int rpw = sys == OVS_SYS_NS ? 8 : (sys == OVS_SYS_NSVOF ? 5 : 4);
  long warps = ((long)N + rpw - 1) / rpw;
  long blocks = (warps * 32 + SPMV_THREADS - 1) / SPMV_THREADS;
  if (sys == OVS_SYS_NS)
    {
      spmv_block_kernel<4, TM, TX, TY, MODE, ACC64><<<(int)blocks, SPMV_THREADS, 0, c->stream>>>(
          N, c->rowptr, c->colidx, vals, x, y, pre, b, done);
      ++c->launches;
    }
  else if (sys == OVS_SYS_NSVOF)
    {
      spmv_block_kernel<6, TM, TX, TY, MODE, ACC64><<<(int)blocks, SPMV_THREADS, 0, c->stream>>>(
          N, c->rowptr, c->colidx, vals, x, y, pre, b, done);
      ++c->launches;
    }
  else
    {
      spmv_scalar_kernel<TM, TX, TY, MODE, ACC64><<<(int)blocks, SPMV_THREADS, 0, c->stream>>>(
          N, c->rowptr, c->colidx, vals, x, y, pre, b, done);
      ++c->launches;
    }
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// ------------------------------------------------------ preconditioner
// Diagonal block extraction (scan of each row for the diagonal, taken from
// the pattern) and inversion: SparseGMRES_NS.f90:53-121 (u: 3x3 inverse by
// cofactors, p: 1/M or 1 if M == 0), SparseGMRES_NS_conv.f:54-139 (phi:
// 1/LS or 0 if LS == 0), SparseGMRES_tem.f90:38-58 (1/M or 1).
template <typename TM>
__global__ void precond_setup_kernel(int N, int sys, const int* __restrict__ diag,
                                     const TM* __restrict__ vals, TM* __restrict__ pre) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int d = diag[i];
  if (sys == OVS_SYS_TEM) {
    double m = d >= 0 ? (double)vals[d] : 0.0;
    pre[i] = (TM)(m != 0.0 ? 1.0 / m : 1.0);
    return;
  }
  const int nv = sys == OVS_SYS_NS ? 16 : 24;
  double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, m = 0.0, ls = 0.0;
  if (d >= 0) {
    const TM* v = vals + (size_t)d * nv;
    K[0] = v[0]; K[1] = v[1]; K[2] = v[2];
    K[3] = v[4]; K[4] = v[5]; K[5] = v[6];
    K[6] = v[8]; K[7] = v[9]; K[8] = v[10];
    m = v[15];
    if (sys == OVS_SYS_NSVOF) ls = v[19];
  }
  const double b11 = K[4] * K[8] - K[7] * K[5];
  const double b12 = K[7] * K[2] - K[1] * K[8];
  const double b13 = K[1] * K[5] - K[2] * K[4];
  const double tmp2 = b11 * K[0] + b12 * K[3] + b13 * K[6];
  const double t = 1.0 / tmp2;
  TM* B = pre + (size_t)i * 9;
  B[0] = (TM)(b11 * t); B[1] = (TM)(b12 * t); B[2] = (TM)(b13 * t);
  B[3] = (TM)((K[5] * K[6] - K[3] * K[8]) * t);
  B[4] = (TM)((K[0] * K[8] - K[6] * K[2]) * t);
  B[5] = (TM)((K[3] * K[2] - K[0] * K[5]) * t);
  B[6] = (TM)((K[3] * K[7] - K[4] * K[6]) * t);
  B[7] = (TM)((K[6] * K[1] - K[0] * K[7]) * t);
  B[8] = (TM)((K[0] * K[4] - K[1] * K[3]) * t);
  pre[(size_t)9 * N + i] = (TM)(m == 0.0 ? 1.0 : 1.0 / m);
  if (sys == OVS_SYS_NSVOF) pre[(size_t)10 * N + i] = (TM)(ls == 0.0 ? 0.0 : 1.0 / ls);
}

// ------------------------------------------------ deterministic reductions
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < nw; ++k) r += sh[k];
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// Finish a reduction: block partial -> gm->partials; the last block sums
// the partials in index order.  Returns true in thread 0 of the last block
// with the total in *total.
__device__ __forceinline__ bool finish_reduction(GmresDev* gm, double partial, double* total) {
  __shared__ double sh[32];
  __shared__ int is_last;
  if (threadIdx.x == 0) {
    gm->partials[blockIdx.x] = partial;
    __threadfence();
    const int t = atomicAdd(&gm->counter, 1);
    is_last = (t == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double v = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) v += __ldcg(gm->partials + k);
  const double s = block_sum(v, sh);
  if (threadIdx.x == 0) {
    gm->counter = 0;
    *total = s;
    return true;
  }
  return false;
}

template <typename TV> __device__ __forceinline__ double dv(TV v) { return (double)v; }

// generic dot of two vectors (FP64 accumulate), result to gm->scal[k]
template <typename TA, typename TB>
__global__ void __launch_bounds__(OVS_RED_THREADS)
dot_kernel(const TA* __restrict__ a, const TB* __restrict__ b, size_t n, GmresDev* gm, int k) {
  __shared__ double sh[32];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    s += dv(a[i]) * dv(b[i]);
  double part = block_sum(s, sh);
  double tot;
  if (finish_reduction(gm, part, &tot)) gm->scal[k] = tot;
}

// ---------------------------------------------------------------- GMRES
// v0 = P^-1 rhs (rhs FP64), ||v0||^2 -> unorm0, epsnrm, e(1)
template <typename TM, typename TV = double>
__global__ void __launch_bounds__(OVS_RED_THREADS)
gm_start_kernel(int N, int nf, int sys, const double* __restrict__ rhs, const TM* __restrict__ pre,
                TV* __restrict__ v0, double tol, GmresDev* gm) {  // v0: FP64 work vector
  __shared__ double sh[32];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)N;
       i += (size_t)gridDim.x * blockDim.x) {
    if (sys == OVS_SYS_TEM) {
      const double z = (double)pre[i] * rhs[i];
      v0[i] = (TV)z;
      s += z * z;
    } else {
      const double r0 = rhs[i], r1 = rhs[(size_t)N + i], r2 = rhs[2 * (size_t)N + i];
      const TM* B = pre + i * 9;
      const double z0 = (double)B[0] * r0 + (double)B[1] * r1 + (double)B[2] * r2;
      const double z1 = (double)B[3] * r0 + (double)B[4] * r1 + (double)B[5] * r2;
      const double z2 = (double)B[6] * r0 + (double)B[7] * r1 + (double)B[8] * r2;
      const double z3 = rhs[3 * (size_t)N + i] * (double)pre[(size_t)9 * N + i];
      v0[i] = (TV)z0; v0[(size_t)N + i] = (TV)z1; v0[2 * (size_t)N + i] = (TV)z2;
      v0[3 * (size_t)N + i] = (TV)z3;
      s += z0 * z0 + z1 * z1 + z2 * z2 + z3 * z3;
      if (nf == 5) {
        const double z4 = rhs[4 * (size_t)N + i] * (double)pre[(size_t)10 * N + i];
        v0[4 * (size_t)N + i] = (TV)z4;
        s += z4 * z4;
      }
    }
  }
  double part = block_sum(s, sh);
  double tot;
  if (finish_reduction(gm, part, &tot)) {
    const double un = sqrt(tot);
    gm->unorm0 = un;
    gm->epsnrm = tol * un;
    gm->e[0] = un;
    gm->iks = 0;
    gm->done = (un == 0.0) ? 1 : 0;
    gm->breakdown = (un == 0.0) ? 1 : 0;
    gm->converged = (un == 0.0) ? 1 : 0;
    gm->ercheck = un;
    gm->beta = 0.0;
  }
}

// Krylov vectors are stored with a padded leading dimension (multiple of
// 64 values) so every basis vector starts 256-byte aligned.  The vector
// being orthogonalized, w, is kept in FP64 whatever the basis precision, so
// the projections of Gram-Schmidt do not lose the small remainder to FP32
// rounding; only normalized vectors are rounded into the basis.
inline size_t basis_ld(size_t n) { return (n + 63) & ~(size_t)63; }

__device__ __forceinline__ void ld4v(const float* p, double v[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4v(const double* p, double v[4]) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4v(float* p, const double v[4]) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void st4v(double* p, const double v[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// v = w / d with d = unorm0 (first vector) or sqrt(beta) (later vectors):
// the normalization of SparseGMRES_NS.f90:159-160,291-294
template <typename TV, typename TW>
__global__ void __launch_bounds__(OVS_RED_THREADS)
gm_normalize_kernel(const TW* w, TV* v, size_t n, GmresDev* gm, int first) {
  if (gm->done && !first) return;
  const double d = first ? gm->unorm0 : sqrt(gm->beta);
  if (!(d != 0.0)) return;
  const size_t n4 = n >> 2, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (size_t q = t0; q < n4; q += stride) {
    double a[4];
    ld4v(w + 4 * q, a);
    a[0] /= d; a[1] /= d; a[2] /= d; a[3] /= d;
    st4v(v + 4 * q, a);
  }
  for (size_t i = 4 * n4 + t0; i < n; i += stride) v[i] = (TV)((double)w[i] / d);
}

// One modified Gram-Schmidt step j (1-based) of iteration k:
//   j >= 2: w -= beta * v_{j-1};  beta = <w, v_j>;  H(j,k) = beta
// (SparseGMRES_NS.f90:246-287); vj == nullptr means v_{k+1} = w itself.
template <typename TV, typename TW>
__global__ void __launch_bounds__(OVS_RED_THREADS)
gm_mgs_kernel(TW* __restrict__ w, const TV* __restrict__ vprev, const TV* __restrict__ vj, size_t n,
              GmresDev* gm, int j, int k) {
  __shared__ double sh[32];
  if (gm->done) return;
  const double beta = gm->beta;
  const size_t n4 = n >> 2, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  double s = 0.0;
  for (size_t q = t0; q < n4; q += stride) {
    double a[4], p[4];
    ld4v(w + 4 * q, a);
    if (j >= 2) {
      ld4v(vprev + 4 * q, p);
      a[0] = a[0] - beta * p[0]; a[1] = a[1] - beta * p[1];
      a[2] = a[2] - beta * p[2]; a[3] = a[3] - beta * p[3];
      st4v(w + 4 * q, a);
      if (sizeof(TW) == 4) ld4v(w + 4 * q, a);  // continue with the stored (rounded) values
    }
    if (vj) {
      ld4v(vj + 4 * q, p);
      s += a[0] * p[0] + a[1] * p[1] + a[2] * p[2] + a[3] * p[3];
    } else {
      s += a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    }
  }
  for (size_t i = 4 * n4 + t0; i < n; i += stride) {
    double a = (double)w[i];
    if (j >= 2) { a = a - beta * (double)vprev[i]; const TW ar = (TW)a; w[i] = ar; a = (double)ar; }
    s += a * (vj ? (double)vj[i] : a);
  }
  double part = block_sum(s, sh);
  double tot;
  if (finish_reduction(gm, part, &tot)) {
    gm->beta = tot;
    gm->H[(size_t)(k - 1) * (gm->kspace + 1) + (j - 1)] = tot;
  }
}

// H(k+1,k) = sqrt(beta), Givens rotations of column k, e update, exit test
// (SparseGMRES_NS.f90:289-327); one thread
__device__ void givens_step(GmresDev* gm, int k) {
  const int ld = gm->kspace + 1;
  double* Hk = gm->H + (size_t)(k - 1) * ld;
  const double unorm = sqrt(gm->beta);
  Hk[k] = unorm;
  for (int jk = 1; jk <= k - 1; ++jk) {
    const double tmp = gm->cs[jk - 1] * Hk[jk - 1] + gm->sn[jk - 1] * Hk[jk];
    Hk[jk] = -gm->sn[jk - 1] * Hk[jk - 1] + gm->cs[jk - 1] * Hk[jk];
    Hk[jk - 1] = tmp;
  }
  const double a = Hk[k - 1], b = Hk[k];
  const double tmp = sqrt(a * a + b * b);
  gm->cs[k - 1] = a / tmp;
  gm->sn[k - 1] = b / tmp;
  Hk[k - 1] = tmp;
  Hk[k] = 0.0;
  const double t2 = gm->cs[k - 1] * gm->e[k - 1] + gm->sn[k - 1] * gm->e[k];
  gm->e[k] = -gm->sn[k - 1] * gm->e[k - 1] + gm->cs[k - 1] * gm->e[k];
  gm->e[k - 1] = t2;
  const double er = fabs(gm->e[k]);
  gm->ercheck = er;
  gm->iks = k;
  const bool conv = (er <= gm->epsnrm) && (k >= gm->kmin);
  const bool brk = unorm == 0.0;  // exact breakdown; NaN propagates as in the reference
  if (conv || brk || k >= gm->kspace) {
    gm->done = 1;
    gm->converged = er <= gm->epsnrm;
    gm->breakdown = brk;
  }
}

__global__ void gm_givens_kernel(GmresDev* gm, int k) {
  if (gm->done) return;
  givens_step(gm, k);
}

// One Arnoldi iteration k in a single cooperative launch (all blocks
// co-resident): w = P^-1 A v_k into basis slot k, the k+1 modified
// Gram-Schmidt steps of the reference order with one grid-wide barrier
// each, the normalization and the Givens update.  The Gram-Schmidt partial
// sums are double buffered, so one barrier per step suffices; every block
// adds the partials in the same order, so all see the same beta, and the
// result does not depend on timing.
template <typename TM, typename TV, int SYS, bool ACC64>
__global__ void __launch_bounds__(256)
gm_arnoldi_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                  const TM* __restrict__ vals, const TM* __restrict__ pre, TV* V, size_t ld, size_t n,
                  int k, GmresDev* gm, double* part) {
  cg::grid_group grid = cg::this_grid();
  if (gm->done) return;
  __shared__ double sh[32];
  __shared__ double sbeta;
  const TV* vk = V + ld * (size_t)(k - 1);
  TV* w = V + ld * (size_t)k;
  // ---- w = P^-1 A v_k
  {
    constexpr int RPW = SYS == OVS_SYS_NS ? 8 : (SYS == OVS_SYS_NSVOF ? 5 : 4);
    const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
    const long nchunks = ((long)N + RPW - 1) / RPW;
    for (long c = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchunks; c += nwarps) {
      if constexpr (SYS == OVS_SYS_NS)
        spmv_block_warp<4, TM, TV, TV, 1, ACC64>(c, N, rowptr, colidx, vals, vk, w, pre, nullptr);
      else if constexpr (SYS == OVS_SYS_NSVOF)
        spmv_block_warp<6, TM, TV, TV, 1, ACC64>(c, N, rowptr, colidx, vals, vk, w, pre, nullptr);
      else
        spmv_scalar_warp<TM, TV, TV, 1, ACC64>(c, N, rowptr, colidx, vals, vk, w, pre, nullptr);
    }
  }
  grid.sync();
  // ---- modified Gram-Schmidt, SparseGMRES_NS.f90:246-287
  const size_t n4 = n >> 2, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int G = gridDim.x;
  double beta = 0.0;
  for (int j = 1; j <= k + 1; ++j) {
    const TV* vprev = j >= 2 ? V + ld * (size_t)(j - 2) : nullptr;
    const TV* vj = j <= k ? V + ld * (size_t)(j - 1) : nullptr;
    double sacc = 0.0;
    for (size_t q = t0; q < n4; q += stride) {
      double a[4], pv[4];
      ld4v(w + 4 * q, a);
      if (j >= 2) {
        ld4v(vprev + 4 * q, pv);
        a[0] = a[0] - beta * pv[0]; a[1] = a[1] - beta * pv[1];
        a[2] = a[2] - beta * pv[2]; a[3] = a[3] - beta * pv[3];
        st4v(w + 4 * q, a);
        if (sizeof(TV) == 4) ld4v(w + 4 * q, a);
      }
      if (vj) {
        ld4v(vj + 4 * q, pv);
        sacc += a[0] * pv[0] + a[1] * pv[1] + a[2] * pv[2] + a[3] * pv[3];
      } else {
        sacc += a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
      }
    }
    for (size_t i = 4 * n4 + t0; i < n; i += stride) {
      double a = (double)w[i];
      if (j >= 2) { a = a - beta * (double)vprev[i]; const TV ar = (TV)a; w[i] = ar; a = (double)ar; }
      sacc += a * (vj ? (double)vj[i] : a);
    }
    const double bp = block_sum(sacc, sh);
    double* pb = part + (size_t)(j & 1) * G;
    if (threadIdx.x == 0) pb[blockIdx.x] = bp;
    grid.sync();
    double v = 0.0;
    for (int b = threadIdx.x; b < G; b += blockDim.x) v += __ldcg(pb + b);
    const double tot = block_sum(v, sh);
    if (threadIdx.x == 0) sbeta = tot;
    __syncthreads();
    beta = sbeta;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      gm->H[(size_t)(k - 1) * (gm->kspace + 1) + (j - 1)] = beta;
      gm->beta = beta;
    }
    __syncthreads();
  }
  // ---- normalize (SparseGMRES_NS.f90:291-294) and the Givens update
  const double unorm = sqrt(beta);
  if (unorm != 0.0) {
    for (size_t q = t0; q < n4; q += stride) {
      double a[4];
      ld4v(w + 4 * q, a);
      a[0] /= unorm; a[1] /= unorm; a[2] /= unorm; a[3] /= unorm;
      st4v(w + 4 * q, a);
    }
    for (size_t i = 4 * n4 + t0; i < n; i += stride) w[i] = (TV)((double)w[i] / unorm);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) givens_step(gm, k);
}

// back-substitution (SparseGMRES_NS.f90:341-346); single thread
__global__ void gm_backsub_kernel(GmresDev* gm) {
  const int iks = gm->iks, ld = gm->kspace + 1;
  for (int jk = iks; jk >= 1; --jk) {
    const double y = gm->e[jk - 1] / gm->H[(size_t)(jk - 1) * ld + (jk - 1)];
    gm->y[jk - 1] = y;
    for (int lk = 1; lk <= jk - 1; ++lk) gm->e[lk - 1] = gm->e[lk - 1] - y * gm->H[(size_t)(jk - 1) * ld + (lk - 1)];
  }
}

// sol += sum_j y_j v_j (SparseGMRES_NS.f90:349-352)
template <typename TV>
__global__ void gm_update_kernel(double* __restrict__ sol, const TV* __restrict__ basis, size_t n, size_t ld,
                                 const GmresDev* __restrict__ gm) {
  const int iks = gm->iks;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double s = sol[i];
    for (int j = 0; j < iks; ++j) s = s + gm->y[j] * (double)basis[(size_t)j * ld + i];
    sol[i] = s;
  }
}

// elementwise helpers
template <typename TS, typename TD>
__global__ void convert_kernel(const TS* __restrict__ a, TD* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (TD)a[i];
}

// --------------------------------------------------------- host drivers
template <typename T> const T* as(const void* p) { return reinterpret_cast<const T*>(p); }

int ensure_basis(ovs_ctx* c, int prec, size_t bytes) {
  if (c->basis_bytes[prec] >= bytes) return OVS_OK;
  if (c->basis[prec]) cudaFree(c->basis[prec]);
  c->basis[prec] = nullptr;
  c->basis_bytes[prec] = 0;
  if (cudaMalloc(&c->basis[prec], bytes) != cudaSuccess) {
    cudaGetLastError();
    return OVS_ERR_NOMEM;
  }
  c->basis_bytes[prec] = bytes;
  return OVS_OK;
}

// One GMRES cycle on system `sys` with matrix/preconditioner precision TM
// and basis precision TV.  rhs and sol are FP64 device vectors (nf*N).
template <typename TM, typename TV, typename TW = double, bool ACC64 = true>
int gmres_cycle(ovs_ctx* c, int sys, const double* rhs, double* sol, double tol, int kspace,
                int kmin, ovs_gmres_info* info) {
  const int N = c->N, nf = ovs_sys_nf(sys);
  const size_t n = (size_t)N * nf;
  const int prec = sizeof(TM) == 8 ? OVS_FP64 : OVS_FP32;
  SysStore& S = c->sys[sys][prec];
  if (!S.vals || !S.binv) return OVS_ERR_STATE;
  if (kspace < 1 || kspace > OVS_MAX_KSPACE) return OVS_ERR_ARG;
  const int bprec = sizeof(TV) == 8 ? OVS_FP64 : OVS_FP32;
  const size_t ld = basis_ld(n);
  int st;
  if ((st = ensure_basis(c, bprec, sizeof(TV) * ld * (size_t)(kspace + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->wvec, sizeof(double) * basis_ld(5 * (size_t)N)))) return st;
  TV* V = reinterpret_cast<TV*>(c->basis[bprec]);
  // w: FP64 work vector, or (TW == TV) the next basis vector itself
  constexpr bool inplace = sizeof(TW) == sizeof(TV);
  double* wd = c->wvec;
  GmresDev* gm = c->gm;
  cudaStream_t s = c->stream;
  const TM* vals = as<TM>(S.vals);
  const TM* pre = as<TM>(S.binv);
  // set kspace/kmin and clear the Hessenberg matrix
  int km[2] = {kspace, kmin};
  OVS_CUDA_TRY(cudaMemcpyAsync(&gm->kspace, km, sizeof(km), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemsetAsync(gm->H, 0, sizeof(double) * (size_t)(kspace + 1) * kspace, s));
  OVS_CUDA_TRY(cudaMemsetAsync(gm->e, 0, sizeof(double) * (size_t)(kspace + 1), s));
  gm_start_kernel<TM, double><<<OVS_RED_BLOCKS, OVS_RED_THREADS, 0, s>>>(N, nf, sys, rhs, pre, wd, tol, gm);
  gm_normalize_kernel<TV, double><<<OVS_RED_BLOCKS, OVS_RED_THREADS, 0, s>>>(wd, V, n, gm, 1);
  c->launches += 2;
  OVS_CUDA_TRY(cudaGetLastError());
  // one cooperative launch per Arnoldi iteration
  void (*kern)(int, const int*, const int*, const TM*, const TM*, TV*, size_t, size_t, int, GmresDev*, double*);
  if (sys == OVS_SYS_NS) kern = gm_arnoldi_kernel<TM, TV, OVS_SYS_NS, ACC64>;
  else if (sys == OVS_SYS_NSVOF) kern = gm_arnoldi_kernel<TM, TV, OVS_SYS_NSVOF, ACC64>;
  else kern = gm_arnoldi_kernel<TM, TV, OVS_SYS_TEM, ACC64>;
  int per_sm = 0;
  OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
  if (per_sm < 1) return OVS_ERR_CUDA;
  int grid = per_sm * c->num_sms;
  if (grid > OVS_COOP_MAX_BLOCKS) grid = OVS_COOP_MAX_BLOCKS;
  if ((st = ovs_ensure((void**)&c->coop_part, sizeof(double) * 2 * OVS_COOP_MAX_BLOCKS))) return st;
  const int batch = N > 200000 ? 4 : 16;
  int k = 1;
  for (; k <= kspace;) {
    const int kend = (k + batch - 1 < kspace) ? k + batch - 1 : kspace;
    for (; k <= kend; ++k) {
      int Nn = N, kk = k;
      const int* rp = c->rowptr;
      const int* ci = c->colidx;
      TV* Vp = V;
      size_t ldv = ld, nn = n;
      double* part = c->coop_part;
      void* args[] = {&Nn, &rp, &ci, (void*)&vals, (void*)&pre, &Vp, &ldv, &nn, &kk, &gm, &part};
      OVS_CUDA_TRY(cudaLaunchCooperativeKernel((void*)kern, grid, 256, args, 0, s));
      ++c->launches;
    }
    OVS_CUDA_TRY(cudaMemcpyAsync(c->h_pinned, &gm->done, sizeof(int), cudaMemcpyDeviceToHost, s));
    OVS_CUDA_TRY(cudaStreamSynchronize(s));
    if (c->h_pinned[0]) break;
  }
  gm_backsub_kernel<<<1, 1, 0, s>>>(gm);
  ++c->launches;
  gm_update_kernel<TV><<<ovs_grid(n, 256, 4 * c->num_sms * 8), 256, 0, s>>>(sol, V, n, ld, gm);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  if (info) {
    GmresDev h;
    OVS_CUDA_TRY(cudaMemcpyAsync(&h, gm, offsetof(GmresDev, H), cudaMemcpyDeviceToHost, s));
    OVS_CUDA_TRY(cudaStreamSynchronize(s));
    info->iterations = h.iks;
    info->converged = h.converged;
    info->breakdown = h.breakdown;
    info->res0 = h.unorm0;
    info->ercheck = h.ercheck;
  }
  return OVS_OK;
}

int dot64(ovs_ctx* c, const double* a, const double* b, size_t n, double* out) {
  dot_kernel<double, double><<<OVS_RED_BLOCKS, OVS_RED_THREADS, 0, c->stream>>>(a, b, n, c->gm, 0);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaMemcpyAsync(c->h_pinned_d, c->gm->scal, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  *out = c->h_pinned_d[0];
  return OVS_OK;
}

}  // namespace

template <typename TV>
__global__ void fill_kernel(TV* __restrict__ p, size_t n, double v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = (TV)(v * (1.0 + 1e-3 * (double)(i % 97)));
}

// Time one Arnoldi iteration (k = 25 of a 50-vector cycle) or one
// preconditioned SpMV on the resident system.
template <typename TM, bool ACC64>
int profile_krylov_t(ovs_ctx* c, int what, int sys, int reps, double* ms) {
  const int prec = sizeof(TM) == 8 ? OVS_FP64 : OVS_FP32;
  SysStore& S = c->sys[sys][prec];
  if (!S.vals) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_precond_setup(c, sys, prec))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  const size_t ld = basis_ld(n);
  const int kspace = 50, k = 25;
  if ((st = ensure_basis(c, prec, sizeof(TM) * ld * (kspace + 1)))) return st;
  TM* V = reinterpret_cast<TM*>(c->basis[prec]);
  fill_kernel<TM><<<1184, 256, 0, c->stream>>>(V, ld * (kspace + 1), 1.0);
  GmresDev* gm = c->gm;
  int km[2] = {kspace, 1};
  OVS_CUDA_TRY(cudaMemcpyAsync(&gm->kspace, km, sizeof(km), cudaMemcpyHostToDevice, c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(&gm->done, 0, sizeof(int), c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(&gm->epsnrm, 0, sizeof(double), c->stream));
  const TM* vals = as<TM>(S.vals);
  const TM* pre = as<TM>(S.binv);
  void (*kern)(int, const int*, const int*, const TM*, const TM*, TM*, size_t, size_t, int, GmresDev*, double*);
  if (sys == OVS_SYS_NS) kern = gm_arnoldi_kernel<TM, TM, OVS_SYS_NS, ACC64>;
  else if (sys == OVS_SYS_NSVOF) kern = gm_arnoldi_kernel<TM, TM, OVS_SYS_NSVOF, ACC64>;
  else kern = gm_arnoldi_kernel<TM, TM, OVS_SYS_TEM, ACC64>;
  int per_sm = 0;
  OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
  int grid = per_sm * c->num_sms;
  if (grid > OVS_COOP_MAX_BLOCKS) grid = OVS_COOP_MAX_BLOCKS;
  if ((st = ovs_ensure((void**)&c->coop_part, sizeof(double) * 2 * OVS_COOP_MAX_BLOCKS))) return st;
  auto run = [&]() -> int {
    if (what == OVS_PROF_SPMV) {
      st = launch_spmv<TM, TM, TM, 1, ACC64>(c, sys, vals, V, V + ld, pre, nullptr, nullptr);
      return st;
    }
    int Nn = c->N, kk = k;
    const int* rp = c->rowptr;
    const int* ci = c->colidx;
    size_t ldv = ld, nn = n;
    double* part = c->coop_part;
    void* args[] = {&Nn, &rp, &ci, (void*)&vals, (void*)&pre, &V, &ldv, &nn, &kk, &gm, &part};
    OVS_CUDA_TRY(cudaLaunchCooperativeKernel((void*)kern, grid, 256, args, 0, c->stream));
    ++c->launches;
    return OVS_OK;
  };
  if ((st = run())) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  for (int r = 0; r < reps; ++r)
    if ((st = run())) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float t = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&t, c->ev0, c->ev1));
  *ms = (double)t / reps;
  return OVS_OK;
}

int ovs_profile_krylov(ovs_ctx* c, int what, int sys, int prec, int reps, double* ms) {
  if (prec == OVS_FP64) return profile_krylov_t<double, true>(c, what, sys, reps, ms);
  return profile_krylov_t<float, false>(c, what, sys, reps, ms);
}

int ovs_dot_impl(ovs_ctx* c, const double* a, const double* b, size_t n, double* out) {
  return dot64(c, a, b, n, out);
}

int ovs_precond_setup(ovs_ctx* c, int sys, int prec) {
  SysStore& S = c->sys[sys][prec];
  if (!S.vals) return OVS_ERR_STATE;
  const size_t ts = prec == OVS_FP64 ? 8 : 4;
  const size_t w = sys == OVS_SYS_TEM ? 1 : 11;
  int st;
  if ((st = ovs_ensure(&S.binv, ts * w * (size_t)c->N))) return st;
  if (prec == OVS_FP64)
    {
      precond_setup_kernel<double><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(
          c->N, sys, c->diag, as<double>(S.vals), reinterpret_cast<double*>(S.binv));
      ++c->launches;
    }
  else
    {
      precond_setup_kernel<float><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(
          c->N, sys, c->diag, as<float>(S.vals), reinterpret_cast<float*>(S.binv));
      ++c->launches;
    }
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// y = A x (dx, dy FP64 device vectors), plain product
int ovs_spmv_impl(ovs_ctx* c, int sys, int prec, const double* dx, double* dy) {
  SysStore& S = c->sys[sys][prec];
  if (!S.vals) return OVS_ERR_STATE;
  if (prec == OVS_FP64) return launch_spmv<double, double, double, 0>(c, sys, as<double>(S.vals), dx, dy, nullptr, nullptr, nullptr);
  return launch_spmv<float, double, double, 0>(c, sys, as<float>(S.vals), dx, dy, nullptr, nullptr, nullptr);
}

// Reference-semantics single cycle in FP64 (SparseGMRES_up / _ns_conv / _tem)
int ovs_gmres_ref_impl(ovs_ctx* c, int sys, double tol, int kspace, int kmin, double* dsol,
                       ovs_gmres_info* info) {
  SysStore& S = c->sys[sys][OVS_FP64];
  if (!S.vals || !S.rhs) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_precond_setup(c, sys, OVS_FP64))) return st;
  const double* rhs = reinterpret_cast<const double*>(S.rhs);
  if (sys == OVS_SYS_TEM) {
    // SparseGMRES_tem.f90:63-71: sol = 0 and return when ||rhs|| == 0
    double rr;
    if ((st = dot64(c, rhs, rhs, (size_t)c->N, &rr))) return st;
    if (rr == 0.0) {
      OVS_CUDA_TRY(cudaMemsetAsync(dsol, 0, sizeof(double) * c->N, c->stream));
      OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
      if (info) { memset(info, 0, sizeof(*info)); info->converged = 1; }
      return OVS_OK;
    }
  }
  st = gmres_cycle<double, double>(c, sys, rhs, dsol, tol, kspace, kmin, info);
  if (st) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

// Restarted / iteratively refined solve to a true FP64 relative residual.
int ovs_solve_impl(ovs_ctx* c, int sys, int mode, double rtol, int kspace, int max_cycles,
                   ovs_solve_info* info) {
  const int prec = mode == OVS_FP32 ? OVS_FP32 : OVS_FP64;
  SysStore& S = c->sys[sys][prec];
  if (!S.vals || !S.rhs) return OVS_ERR_STATE;
  const int N = c->N, nf = ovs_sys_nf(sys);
  const size_t n = (size_t)N * nf;
  int st;
  cudaStream_t s = c->stream;
  if ((st = ovs_ensure((void**)&c->sol[sys], sizeof(double) * 5 * (size_t)N))) return st;
  if ((st = ovs_ensure((void**)&c->work64, sizeof(double) * 10 * (size_t)N))) return st;
  double* x = c->sol[sys];
  double* b = c->work64;
  double* r = c->work64 + 5 * (size_t)N;
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, s));
  if ((st = ovs_precond_setup(c, sys, prec))) return st;
  if (prec == OVS_FP64) {
    OVS_CUDA_TRY(cudaMemcpyAsync(b, S.rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  } else {
    convert_kernel<float, double><<<ovs_grid(n, 256, 4096), 256, 0, s>>>(as<float>(S.rhs), b, n);
    ++c->launches;
  }
  OVS_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  double bb;
  if ((st = dot64(c, b, b, n, &bb))) return st;
  const double bnorm = sqrt(bb);
  double rel = bnorm > 0.0 ? 1.0 : 0.0;
  int cycles = 0, iters = 0;
  const double floor_tol = prec == OVS_FP32 ? 1e-6 : 1e-14;
  while (rel > rtol && cycles < max_cycles) {
    double tin = rtol / rel;
    if (tin < floor_tol) tin = floor_tol;
    if (tin > 0.5) tin = 0.5;
    ovs_gmres_info gi;
    if (prec == OVS_FP64) st = gmres_cycle<double, double, double, true>(c, sys, r, x, tin, kspace, 1, &gi);
    else st = gmres_cycle<float, float, float, false>(c, sys, r, x, tin, kspace, 1, &gi);
    if (st) return st;
    iters += gi.iterations;
    ++cycles;
    // r = b - A x in FP64 arithmetic
    if (prec == OVS_FP64) st = launch_spmv<double, double, double, 2>(c, sys, as<double>(S.vals), x, r, nullptr, b, nullptr);
    else st = launch_spmv<float, double, double, 2>(c, sys, as<float>(S.vals), x, r, nullptr, b, nullptr);
    if (st) return st;
    double rr;
    if ((st = dot64(c, r, r, n, &rr))) return st;
    rel = sqrt(rr) / bnorm;
    if (!(rel == rel)) break;
    if (gi.iterations == 0) break;
  }
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, s));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  if (info) {
    info->cycles = cycles;
    info->iterations = iters;
    info->converged = rel <= rtol;
    info->rel_residual = rel;
    info->seconds = ms * 1e-3;
  }
  return OVS_OK;
}
