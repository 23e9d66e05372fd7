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

#include <algorithm>
#include <vector>

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
// LIST: the warp chunks run over the row list rows[0, nrows) (local row
// indices; an index outside [0, N) is skipped) instead of rows 0..N-1;
// each listed row is computed exactly as in the full product.
template <int NG, typename TM, typename TX, typename TY, int MODE, bool ACC64, bool LIST = false>
__device__ __forceinline__ void spmv_block_warp(long wglob, int N, const int* __restrict__ rowptr,
                                                const int* __restrict__ colidx, const TM* __restrict__ vals,
                                                const TX* __restrict__ x, TY* __restrict__ y,
                                                const TM* __restrict__ pre, const double* __restrict__ b,
                                                const int* __restrict__ rows = nullptr, long nrows = 0) {
  using AT = typename AccT<TM, TX, ACC64>::type;
  constexpr int NV = 4 * NG;
  constexpr int RPW = 32 / NG;  // rows per warp
  const int lane = threadIdx.x & 31;
  const int sub = lane / NG;
  const int g = lane - sub * NG;
  const long rowl = wglob * RPW + sub;
  bool active;
  int row;
  if constexpr (LIST) {
    const int rl = (sub < RPW && rowl < nrows) ? __ldg(rows + rowl) : -1;
    active = rl >= 0 && rl < N;
    row = active ? rl : 0;
  } else {
    active = sub < RPW && rowl < N;
    row = active ? (int)rowl : 0;
  }
  // column fields read by this lane's 4 values
  int cf0, cf1, cf2, cf3;
  if (NG == 6 && g == 5) { cf0 = cf1 = cf2 = cf3 = 4; }
  else { cf0 = 0; cf1 = 1; cf2 = 2; cf3 = (NG == 6 && g == 4) ? 4 : 3; }
  AT a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  if (active) {
    const int s0 = __ldg(rowptr + row), s1 = __ldg(rowptr + row + 1);
    // lane g of the row gathers field g of x at the slot's column (NS+VOF:
    // u,v,w,p,phi in lanes 0-4) and the row's lanes exchange them by
    // shuffles: 4-5 gathers per slot instead of 4 per lane
    int s = s0;
    constexpr int NFX = NG == 6 ? 5 : 4;
    const unsigned gmask = ((1u << NG) - 1u) << (sub * NG);
    const int base = sub * NG;
    const TX* xg = x + (size_t)(g < NFX ? g : 0) * N;
    // FP32 values: 4 slots in flight per lane (measured 0.63 vs 0.72 ms at
    // 2.1M nodes); FP64 values already move 32 bytes per lane and slot, and
    // run faster with 2
    if constexpr (sizeof(TM) == 4) {
      for (; s + 3 < s1; s += 4) {
        const int c0 = __ldg(colidx + s), c1 = __ldg(colidx + s + 1), c2 = __ldg(colidx + s + 2),
                  c3 = __ldg(colidx + s + 3);
        TM v[4], w[4], y[4], z[4];
        ld4(vals + (size_t)s * NV + 4 * g, v);
        ld4(vals + (size_t)(s + 1) * NV + 4 * g, w);
        ld4(vals + (size_t)(s + 2) * NV + 4 * g, y);
        ld4(vals + (size_t)(s + 3) * NV + 4 * g, z);
        const AT f0 = (AT)__ldg(xg + c0), f1 = (AT)__ldg(xg + c1), f2 = (AT)__ldg(xg + c2), f3 = (AT)__ldg(xg + c3);
        a0 += (AT)v[0] * __shfl_sync(gmask, f0, base + cf0); a1 += (AT)v[1] * __shfl_sync(gmask, f0, base + cf1);
        a2 += (AT)v[2] * __shfl_sync(gmask, f0, base + cf2); a3 += (AT)v[3] * __shfl_sync(gmask, f0, base + cf3);
        a0 += (AT)w[0] * __shfl_sync(gmask, f1, base + cf0); a1 += (AT)w[1] * __shfl_sync(gmask, f1, base + cf1);
        a2 += (AT)w[2] * __shfl_sync(gmask, f1, base + cf2); a3 += (AT)w[3] * __shfl_sync(gmask, f1, base + cf3);
        a0 += (AT)y[0] * __shfl_sync(gmask, f2, base + cf0); a1 += (AT)y[1] * __shfl_sync(gmask, f2, base + cf1);
        a2 += (AT)y[2] * __shfl_sync(gmask, f2, base + cf2); a3 += (AT)y[3] * __shfl_sync(gmask, f2, base + cf3);
        a0 += (AT)z[0] * __shfl_sync(gmask, f3, base + cf0); a1 += (AT)z[1] * __shfl_sync(gmask, f3, base + cf1);
        a2 += (AT)z[2] * __shfl_sync(gmask, f3, base + cf2); a3 += (AT)z[3] * __shfl_sync(gmask, f3, base + cf3);
      }
    }
    for (; s + 1 < s1; s += 2) {
      const int c0 = __ldg(colidx + s), c1 = __ldg(colidx + s + 1);
      TM v[4], w[4];
      ld4(vals + (size_t)s * NV + 4 * g, v);
      ld4(vals + (size_t)(s + 1) * NV + 4 * g, w);
      const AT f0 = (AT)__ldg(xg + c0), f1 = (AT)__ldg(xg + c1);
      a0 += (AT)v[0] * __shfl_sync(gmask, f0, base + cf0); a1 += (AT)v[1] * __shfl_sync(gmask, f0, base + cf1);
      a2 += (AT)v[2] * __shfl_sync(gmask, f0, base + cf2); a3 += (AT)v[3] * __shfl_sync(gmask, f0, base + cf3);
      a0 += (AT)w[0] * __shfl_sync(gmask, f1, base + cf0); a1 += (AT)w[1] * __shfl_sync(gmask, f1, base + cf1);
      a2 += (AT)w[2] * __shfl_sync(gmask, f1, base + cf2); a3 += (AT)w[3] * __shfl_sync(gmask, f1, base + cf3);
    }
    if (s < s1) {
      const int c0 = __ldg(colidx + s);
      TM v[4];
      ld4(vals + (size_t)s * NV + 4 * g, v);
      const AT f0 = (AT)__ldg(xg + c0);
      a0 += (AT)v[0] * __shfl_sync(gmask, f0, base + cf0); a1 += (AT)v[1] * __shfl_sync(gmask, f0, base + cf1);
      a2 += (AT)v[2] * __shfl_sync(gmask, f0, base + cf2); a3 += (AT)v[3] * __shfl_sync(gmask, f0, base + cf3);
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

// the same product over a list of rows (a partition's interior or boundary
// rows, ovs_spmv_device_rows)
template <int NG, typename TM, typename TX, typename TY, int MODE>
__global__ void __launch_bounds__(SPMV_THREADS)
spmv_block_rows_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                       const TM* __restrict__ vals, const TX* __restrict__ x, TY* __restrict__ y,
                       const TM* __restrict__ pre, const int* __restrict__ rows, int nrows) {
  const long wglob = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  spmv_block_warp<NG, TM, TX, TY, MODE, true, true>(wglob, N, rowptr, colidx, vals, x, y, pre, nullptr, rows,
                                                     nrows);
}

// scalar CSR (temperature): 8 lanes per row
template <typename TM, typename TX, typename TY, int MODE, bool ACC64, bool LIST = false>
__device__ __forceinline__ void spmv_scalar_warp(long wglob, int N, const int* __restrict__ rowptr,
                                                 const int* __restrict__ colidx, const TM* __restrict__ vals,
                                                 const TX* __restrict__ x, TY* __restrict__ y,
                                                 const TM* __restrict__ pre, const double* __restrict__ b,
                                                 const int* __restrict__ rows = nullptr, long nrows = 0) {
  using AT = typename AccT<TM, TX, ACC64>::type;
  const int lane = threadIdx.x & 31;
  const int sub = lane >> 3, k = lane & 7;
  const long rowl = wglob * 4 + sub;
  bool active;
  int row;
  if constexpr (LIST) {
    const int rl = rowl < nrows ? __ldg(rows + rowl) : -1;
    active = rl >= 0 && rl < N;
    row = active ? rl : 0;
  } else {
    active = rowl < N;
    row = active ? (int)rowl : 0;
  }
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

template <typename TM, typename TX, typename TY, int MODE>
__global__ void __launch_bounds__(SPMV_THREADS)
spmv_scalar_rows_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                        const TM* __restrict__ vals, const TX* __restrict__ x, TY* __restrict__ y,
                        const TM* __restrict__ pre, const int* __restrict__ rows, int nrows) {
  const long wglob = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  spmv_scalar_warp<TM, TX, TY, MODE, true, true>(wglob, N, rowptr, colidx, vals, x, y, pre, nullptr, rows, nrows);
}

// y = A x or P^-1 A x (MODE 0 / 1) on the listed rows only (FP64 vectors,
// FP64 accumulation as in the full FP64-vector product)
template <typename TM, int MODE>
int launch_spmv_rows(ovs_ctx* c, int sys, const TM* vals, const double* x, double* y, const TM* pre,
                     const int* rows, int nrows) {
  if (nrows <= 0) return OVS_OK;
  const int N = c->N;
  int rpw = sys == OVS_SYS_NS ? 8 : (sys == OVS_SYS_NSVOF ? 5 : 4);
  long warps = ((long)nrows + rpw - 1) / rpw;
  long blocks = (warps * 32 + SPMV_THREADS - 1) / SPMV_THREADS;
  if (sys == OVS_SYS_NS)
    spmv_block_rows_kernel<4, TM, double, double, MODE><<<(int)blocks, SPMV_THREADS, 0, c->stream>>>(
        N, c->rowptr, c->colidx, vals, x, y, pre, rows, nrows);
  else if (sys == OVS_SYS_NSVOF)
    spmv_block_rows_kernel<6, TM, double, double, MODE><<<(int)blocks, SPMV_THREADS, 0, c->stream>>>(
        N, c->rowptr, c->colidx, vals, x, y, pre, rows, nrows);
  else
    spmv_scalar_rows_kernel<TM, double, double, MODE><<<(int)blocks, SPMV_THREADS, 0, c->stream>>>(
        N, c->rowptr, c->colidx, vals, x, y, pre, rows, nrows);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
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
                TV* __restrict__ v0, double tol, GmresDev* gm, int raw) {  // v0: FP64 work vector
  __shared__ double sh[32];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)N;
       i += (size_t)gridDim.x * blockDim.x) {
    if (raw) {   // rhs is already preconditioned
      for (int f = 0; f < nf; ++f) {
        const double z = rhs[(size_t)f * N + i];
        v0[(size_t)f * N + i] = (TV)z;
        s += z * z;
      }
    } else if (sys == OVS_SYS_TEM) {
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
  if (tmp == 0.0) {
    // column k of H is zero (P^-1 A v_k has no component outside
    // v_1..v_{k-1}): the rotation would be 0/0 and the reference carries NaN
    // on; the cycle ends with the solution of the first k-1 columns
    gm->iks = k - 1;
    gm->ercheck = fabs(gm->e[k - 1]);
    gm->done = 1;
    gm->converged = gm->ercheck <= gm->epsnrm;
    gm->breakdown = 1;
    return;
  }
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

// Sizes of the on-chip Gram-Schmidt kernel (gm_mgs_onchip_kernel below):
// 512 threads (16 warps); each warp owns the TMEM lanes of its quarter
// (warp % 4) and a quarter of the 512 columns (warp / 4), so every thread
// holds 128 32-bit columns: 32 groups of 4 FP32 values, or 16 groups of 4
// FP64 values split into low and high words.
constexpr int ONCHIP_THREADS = 512;
constexpr int TMEM_COLS = 512;
constexpr int TMEM_COLS_PER_THREAD = 128;
template <typename TV> struct TmemGeom {
  static constexpr int words = (int)(sizeof(TV) / 4);              // columns per value
  static constexpr int gpp = 16 / (4 * words);                     // groups per 16-column piece
  static constexpr int pieces = TMEM_COLS_PER_THREAD / 16;         // pieces per thread
  static constexpr int groups = pieces * gpp;                      // groups per thread
  static constexpr int cap = 4 * groups * ONCHIP_THREADS;          // values per block
};

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
__device__ __forceinline__ void tmem_st16(uint32_t addr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15, %16};\n"
      :
      : "r"(addr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// group gi of a 16-column piece <-> 4 values
__device__ __forceinline__ void unpack_group(const uint32_t (&r)[16], int gi, float*, double a[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) a[e] = (double)__uint_as_float(r[4 * gi + e]);
}
__device__ __forceinline__ void unpack_group(const uint32_t (&r)[16], int gi, double*, double a[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) a[e] = __hiloint2double((int)r[8 * gi + 2 * e + 1], (int)r[8 * gi + 2 * e]);
}
__device__ __forceinline__ void pack_group(uint32_t (&r)[16], int gi, float*, const double a[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) r[4 * gi + e] = __float_as_uint((float)a[e]);
}
__device__ __forceinline__ void pack_group(uint32_t (&r)[16], int gi, double*, const double a[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    r[8 * gi + 2 * e] = (uint32_t)__double2loint(a[e]);
    r[8 * gi + 2 * e + 1] = (uint32_t)__double2hiint(a[e]);
  }
}

// The on-chip kernel indexes 32-bit within its block's chunk, from base
// pointers at the chunk start.  ld4m loads the group at local index li (a
// multiple of 4) or, when !ok, the chunk's first group; the load itself is
// unconditional so a thread keeps several in flight.  Values at or beyond
// the chunk end nl, and all four when !ok, come back as zero.  The group
// stays in the storage type until it is used.
template <typename TV> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { struct type { double x, y, z, w; }; };
template <typename TV>
__device__ __forceinline__ typename Vec4<TV>::type ld4m(const TV* p, int li, int nl, bool ok) {
  typename Vec4<TV>::type v;
  const TV* q = p + (ok ? li : 0);
  if constexpr (sizeof(TV) == 4) {
    v = *reinterpret_cast<const float4*>(q);
  } else {
    const double2 a = reinterpret_cast<const double2*>(q)[0], b = reinterpret_cast<const double2*>(q)[1];
    v.x = a.x; v.y = a.y; v.z = b.x; v.w = b.y;
  }
  if (!ok || li + 4 > nl) {
    if (!ok || li >= nl) v.x = 0;
    if (!ok || li + 1 >= nl) v.y = 0;
    if (!ok || li + 2 >= nl) v.z = 0;
    if (!ok || li + 3 >= nl) v.w = 0;
  }
  return v;
}
template <typename TV>
__device__ __forceinline__ void st4l(TV* p, int li, int nl, const double v[4]) {
  if (li + 4 <= nl) { st4v(p + li, v); return; }
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (li + q < nl) p[li + q] = (TV)v[q];
}
template <typename V4> __device__ __forceinline__ void widen(const V4& v, double a[4]) {
  a[0] = (double)v.x; a[1] = (double)v.y; a[2] = (double)v.z; a[3] = (double)v.w;
}
// Gram-Schmidt step on one group: a -= beta * p (rounded to TV), dot term
template <typename TV, typename V4>
__device__ __forceinline__ double mgs_apply(double a[4], const V4& p, const V4& y, double beta, bool sub,
                                            bool self) {
  if (sub) {
    double pv[4];
    widen(p, pv);
#pragma unroll
    for (int q = 0; q < 4; ++q) a[q] = (double)(TV)(a[q] - beta * pv[q]);
  }
  if (self) return a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
  double yv[4];
  widen(y, yv);
  return a[0] * yv[0] + a[1] * yv[1] + a[2] * yv[2] + a[3] * yv[3];
}

// FP32 basis: the update w -= beta * v_{j-1} runs in FP32 (one FMA with
// beta rounded to FP32; w is stored in FP32 either way) and only the dot
// product is formed in FP64: the products of two FP32 values are exact in
// FP64 and are summed there.  Two conversions per value instead of five.
__device__ __forceinline__ double mgs_apply_f(float a[4], const float4& p, const float4& y, float bf, bool sub,
                                              bool self) {
  if (sub) {
    a[0] = fmaf(-bf, p.x, a[0]); a[1] = fmaf(-bf, p.y, a[1]);
    a[2] = fmaf(-bf, p.z, a[2]); a[3] = fmaf(-bf, p.w, a[3]);
  }
  const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3];
  if (self) return a0 * a0 + a1 * a1 + a2 * a2 + a3 * a3;
  return a0 * (double)y.x + a1 * (double)y.y + a2 * (double)y.z + a3 * (double)y.w;
}

// The chunk of w owned by a block is cut into pieces of 16 columns per
// thread: piece p holds groups p*gpp .. p*gpp+gpp-1 of every thread, group g
// of thread t at local index 4*(g*512 + t), so each load instruction of a
// warp covers contiguous memory.  Pieces 0..7 live in tensor memory, the
// next `spieces` in dynamic shared memory (one 32 KB slot each), the rest
// stay in global memory (w's own basis slot).
template <typename TV> struct PieceLoads {
  typename Vec4<TV>::type p[TmemGeom<TV>::gpp], y[TmemGeom<TV>::gpp];
};
template <typename TV> struct PieceGeom {
  static constexpr int values = 4 * TmemGeom<TV>::gpp * ONCHIP_THREADS;   // values per piece
  static constexpr int bytes = values * (int)sizeof(TV);                   // 32 KB
};
__device__ __forceinline__ int piece_li(int p, int gi, int gpp) {
  return 4 * ((p * gpp + gi) * ONCHIP_THREADS + (int)threadIdx.x);
}

// Global loads of v_{j-1} (pp, null in step 1) and v_j (yp, null in step
// k+1) for one piece, all issued before any is used.
template <typename TV>
__device__ __forceinline__ void issue_piece(PieceLoads<TV>& L, const TV* pp, const TV* yp, int p, int nl) {
  using Geo = TmemGeom<TV>;
#pragma unroll
  for (int gi = 0; gi < Geo::gpp; ++gi) {
    const int li = piece_li(p, gi, Geo::gpp);
    const bool ok = li < nl;
    if (pp) L.p[gi] = ld4m(pp, li, nl, ok);
    if (yp) L.y[gi] = ld4m(yp, li, nl, ok);
  }
}

// One Gram-Schmidt step on group gi of a piece whose w values are in r
// (the 16 columns of the piece, as stored in tensor memory).
template <typename TV>
__device__ __forceinline__ double step_group(uint32_t (&r)[16], int gi, const PieceLoads<TV>& L, double beta,
                                             bool sub, bool self) {
  if constexpr (sizeof(TV) == 4) {
    float f[4] = {__uint_as_float(r[4 * gi]), __uint_as_float(r[4 * gi + 1]), __uint_as_float(r[4 * gi + 2]),
                  __uint_as_float(r[4 * gi + 3])};
    const double s = mgs_apply_f(f, L.p[gi], L.y[gi], (float)beta, sub, self);
#pragma unroll
    for (int e = 0; e < 4; ++e) r[4 * gi + e] = __float_as_uint(f[e]);
    return s;
  } else {
    double a[4];
    unpack_group(r, gi, (TV*)nullptr, a);
    const double s = mgs_apply<TV>(a, L.p[gi], L.y[gi], beta, sub, self);
    pack_group(r, gi, (TV*)nullptr, a);
    return s;
  }
}

// the piece's 16 columns from / to shared or global memory
template <typename TV>
__device__ __forceinline__ void mem_to_cols(const TV* base, int p, int nl, bool global, uint32_t (&r)[16]) {
  using Geo = TmemGeom<TV>;
#pragma unroll
  for (int gi = 0; gi < Geo::gpp; ++gi) {
    const int li = piece_li(p, gi, Geo::gpp);
    double a[4];
    if (global) widen(ld4m(base, li, nl, li < nl), a);
    else ld4v(base + 4 * (gi * ONCHIP_THREADS + (int)threadIdx.x), a);
    pack_group(r, gi, (TV*)nullptr, a);
  }
}
template <typename TV>
__device__ __forceinline__ void cols_to_mem(TV* base, int p, int nl, bool global, const uint32_t (&r)[16]) {
  using Geo = TmemGeom<TV>;
#pragma unroll
  for (int gi = 0; gi < Geo::gpp; ++gi) {
    const int li = piece_li(p, gi, Geo::gpp);
    double a[4];
    unpack_group(r, gi, (TV*)nullptr, a);
    if (global) { if (li < nl) st4l(base, li, nl, a); }
    else st4v(base + 4 * (gi * ONCHIP_THREADS + (int)threadIdx.x), a);
  }
}

// Gram-Schmidt of one Arnoldi iteration with w held on chip (w = P^-1 A v_k
// already written to basis slot k by the SpMV launch before it).  One block
// of 512 threads per SM; block b owns a contiguous chunk of w (a multiple of
// 4 values) and keeps it, for all k+1 steps, in tensor memory (all 512
// columns of the SM, used as plain storage), then in dynamic shared memory;
// only what does not fit there stays in global memory.  Each step then
// streams v_{j-1} and v_j alone, two pieces at a time with all their loads
// in flight together.  The steps, their order and the fixed-order reductions
// follow gm_arnoldi_kernel (FP32 basis: see mgs_apply_f); entries at and
// beyond n are never touched.  Every block allocates its tensor memory after
// the done test and frees it on the one exit path below.
template <typename TV>
__global__ void __launch_bounds__(ONCHIP_THREADS, 1)
gm_mgs_onchip_kernel(TV* V, size_t ld, size_t n, int k, GmresDev* gm, double* part, size_t chunk, int spieces) {
  using Geo = TmemGeom<TV>;
  using PG = PieceGeom<TV>;
  cg::grid_group grid = cg::this_grid();
  if (gm->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TV* ws = reinterpret_cast<TV*>(smem_raw);
  __shared__ double sh[32];
  __shared__ double sbeta;
  __shared__ uint32_t tmem_base_sh;
  const int G = gridDim.x, b = blockIdx.x, t = threadIdx.x, wid = t >> 5;
  if (wid == 0) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&tmem_base_sh);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base_sh;
  // this warp's lanes (quarter wid % 4) and columns (slot wid / 4)
  const uint32_t taddr = tbase + ((uint32_t)(32 * (wid & 3)) << 16) + (uint32_t)(TMEM_COLS_PER_THREAD * (wid >> 2));
  const size_t c0 = (size_t)b * chunk;
  const int nl = c0 < n ? (int)((c0 + chunk < n ? c0 + chunk : n) - c0) : 0;   // values of this chunk
  const int np = (nl + PG::values - 1) / PG::values;                            // pieces of this chunk
  const int ponchip = Geo::pieces + spieces;                                    // pieces held on chip
  TV* wb = V + ld * (size_t)k + c0;
  // w into tensor and shared memory
#pragma unroll 1
  for (int p = 0; p < np && p < ponchip; ++p) {
    uint32_t r[16];
    mem_to_cols(wb, p, nl, true, r);
    if (p < Geo::pieces) tmem_st16(taddr + 16 * p, r);
    else cols_to_mem(ws + (size_t)(p - Geo::pieces) * PG::values, p, nl, false, r);
  }
  tmem_wait_st();
  double beta = 0.0;
  PieceLoads<TV> L0, L1;
  for (int j = 1; j <= k + 1; ++j) {
    const bool sub = j >= 2, self = j == k + 1;
    const TV* pp = sub ? V + ld * (size_t)(j - 2) + c0 : nullptr;
    const TV* yp = self ? nullptr : V + ld * (size_t)(j - 1) + c0;
    double sacc = 0.0;
#pragma unroll 1
    for (int p0 = 0; p0 < np; p0 += 2) {
      issue_piece(L0, pp, yp, p0, nl);
      if (p0 + 1 < np) issue_piece(L1, pp, yp, p0 + 1, nl);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int p = p0 + h;
        if (p >= np) break;
        const PieceLoads<TV>& L = h ? L1 : L0;
        uint32_t r[16];
        const bool in_tmem = p < Geo::pieces, in_smem = !in_tmem && p < ponchip;
        TV* sbase = ws + (size_t)(p - Geo::pieces) * PG::values;
        if (in_tmem) {
          tmem_ld16(taddr + 16 * p, r);
          tmem_wait_ld();
        } else {
          mem_to_cols(in_smem ? sbase : wb, p, nl, !in_smem, r);
        }
#pragma unroll
        for (int gi = 0; gi < Geo::gpp; ++gi) sacc += step_group<TV>(r, gi, L, beta, sub, self);
        if (sub) {
          if (in_tmem) tmem_st16(taddr + 16 * p, r);
          else cols_to_mem(in_smem ? sbase : wb, p, nl, !in_smem, r);
        }
      }
    }
    tmem_wait_st();
    const double bp = block_sum(sacc, sh);
    double* pb = part + (size_t)(j & 1) * G;
    if (t == 0) pb[b] = bp;
    grid.sync();
    // every block adds the partials in the same order (lane-strided, then a
    // fixed butterfly; lane 0's value is used), so all see the same beta
    if (t < 32) {
      double v = 0.0;
      for (int q = t; q < G; q += 32) v += __ldcg(pb + q);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (t == 0) sbeta = v;
    }
    __syncthreads();
    beta = sbeta;
    if (b == 0 && t == 0) {
      gm->H[(size_t)(k - 1) * (gm->kspace + 1) + (j - 1)] = beta;
      gm->beta = beta;
    }
  }
  // normalize into basis slot k (SparseGMRES_NS.f90:291-294), Givens update
  const double unorm = sqrt(beta);
  const double d = unorm != 0.0 ? unorm : 1.0;
#pragma unroll 1
  for (int p = 0; p < np; ++p) {
    uint32_t r[16];
    const bool in_tmem = p < Geo::pieces, in_smem = !in_tmem && p < ponchip;
    if (in_tmem) {
      tmem_ld16(taddr + 16 * p, r);
      tmem_wait_ld();
    } else {
      mem_to_cols(in_smem ? ws + (size_t)(p - Geo::pieces) * PG::values : wb, p, nl, !in_smem, r);
    }
#pragma unroll
    for (int gi = 0; gi < Geo::gpp; ++gi) {
      const int li = piece_li(p, gi, Geo::gpp);
      double a[4];
      unpack_group(r, gi, (TV*)nullptr, a);
      a[0] /= d; a[1] /= d; a[2] /= d; a[3] /= d;
      if (li < nl) st4l(wb, li, nl, a);
    }
  }
  // release the tensor memory (every access to it has completed above)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (wid == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TMEM_COLS));
  if (b == 0 && t == 0) givens_step(gm, k);
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

// Launch plan of one Arnoldi iteration.  Default: the preconditioned SpMV
// as an ordinary launch, then gm_mgs_onchip_kernel (one 512-thread block
// per SM, cooperative).  fused = 1 (environment OVS_ARNOLDI_FUSED=1, or when
// the on-chip kernel cannot be made co-resident): gm_arnoldi_kernel alone.
struct ArnoldiPlan {
  bool fused = false;
  int grid = 0;
  size_t chunk = 0, smem_bytes = 0;
  int spieces = 0;
};

template <typename TM, typename TV, bool ACC64>
using ArnoldiKern = void (*)(int, const int*, const int*, const TM*, const TM*, TV*, size_t, size_t, int,
                             GmresDev*, double*);

template <typename TM, typename TV, bool ACC64>
ArnoldiKern<TM, TV, ACC64> fused_kernel(int sys) {
  if (sys == OVS_SYS_NS) return gm_arnoldi_kernel<TM, TV, OVS_SYS_NS, ACC64>;
  if (sys == OVS_SYS_NSVOF) return gm_arnoldi_kernel<TM, TV, OVS_SYS_NSVOF, ACC64>;
  return gm_arnoldi_kernel<TM, TV, OVS_SYS_TEM, ACC64>;
}

template <typename TM, typename TV, bool ACC64>
int plan_arnoldi(ovs_ctx* c, int sys, size_t n, bool want_fused, ArnoldiPlan* pl) {
  int st;
  if ((st = ovs_ensure((void**)&c->coop_part, sizeof(double) * 2 * OVS_COOP_MAX_BLOCKS))) return st;
  pl->fused = want_fused;
  if (!want_fused) {
    const int G = c->num_sms;
    const size_t chunk = ((n + G - 1) / G + 3) & ~(size_t)3;
    const size_t rcap = (size_t)TmemGeom<TV>::cap;
    int optin = 0;
    OVS_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    const size_t pv = PieceGeom<TV>::values, pbytes = PieceGeom<TV>::bytes;
    const size_t max_sp = optin > 2048 ? (size_t)(optin - 2048) / pbytes : 0;   // room for static smem
    const size_t want = chunk > rcap ? (chunk - rcap + pv - 1) / pv : 0;
    const size_t sp = want < max_sp ? want : max_sp;
    // The kernel takes all 512 tensor-memory columns of its SM, so two of
    // its blocks must never share an SM (the second allocation would wait
    // for the first block, which waits for it in grid.sync): request more
    // than half of the SM's shared memory and require exactly one block.
    const size_t min_bytes = 118784;
    const size_t bytes = sp * pbytes > min_bytes ? sp * pbytes : min_bytes;
    auto kern = gm_mgs_onchip_kernel<TV>;
    if ((size_t)optin >= bytes + 512 && chunk < ((size_t)1 << 30)) {
      OVS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
      int per_sm = 0;
      OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ONCHIP_THREADS, bytes));
      if (per_sm == 1) {
        pl->grid = G;
        pl->chunk = chunk;
        pl->spieces = (int)sp;
        pl->smem_bytes = bytes;
        return OVS_OK;
      }
    }
    pl->fused = true;
  }
  int per_sm = 0;
  OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_kernel<TM, TV, ACC64>(sys), 256, 0));
  if (per_sm < 1) return OVS_ERR_CUDA;
  pl->grid = per_sm * c->num_sms;
  if (pl->grid > OVS_COOP_MAX_BLOCKS) pl->grid = OVS_COOP_MAX_BLOCKS;
  return OVS_OK;
}

// Arnoldi iteration k (1-based) on basis V (leading dimension ld, n values)
template <typename TM, typename TV, bool ACC64>
int launch_arnoldi(ovs_ctx* c, int sys, const ArnoldiPlan& pl, const TM* vals, const TM* pre, TV* V, size_t ld,
                   size_t n, int k) {
  GmresDev* gm = c->gm;
  double* part = c->coop_part;
  if (pl.fused) {
    int Nn = c->N, kk = k;
    const int* rp = c->rowptr;
    const int* ci = c->colidx;
    size_t ldv = ld, nn = n;
    void* args[] = {&Nn, &rp, &ci, (void*)&vals, (void*)&pre, &V, &ldv, &nn, &kk, &gm, &part};
    OVS_CUDA_TRY(cudaLaunchCooperativeKernel((void*)fused_kernel<TM, TV, ACC64>(sys), pl.grid, 256, args, 0,
                                             c->stream));
    ++c->launches;
    return OVS_OK;
  }
  int st = launch_spmv<TM, TV, TV, 1, ACC64>(c, sys, vals, V + ld * (size_t)(k - 1), V + ld * (size_t)k, pre,
                                               nullptr, &gm->done);
  if (st) return st;
  int kk = k;
  size_t ldv = ld, nn = n, ch = pl.chunk;
  int sp = pl.spieces;
  void* args[] = {&V, &ldv, &nn, &kk, &gm, &part, &ch, &sp};
  OVS_CUDA_TRY(cudaLaunchCooperativeKernel((void*)gm_mgs_onchip_kernel<TV>, pl.grid, ONCHIP_THREADS, args,
                                           pl.smem_bytes, c->stream));
  ++c->launches;
  return OVS_OK;
}

// One GMRES cycle on system `sys` with matrix/preconditioner precision TM
// and basis precision TV.  rhs and sol are FP64 device vectors (nf*N).
// rhs_pre: rhs is P^-1 times the right-hand side already (the cycle then
// solves P^-1 A x = rhs)
template <typename TM, typename TV, bool ACC64 = true>
int gmres_cycle(ovs_ctx* c, int sys, const double* rhs, double* sol, double tol, int kspace,
                int kmin, ovs_gmres_info* info, bool rhs_pre = false) {
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
  // v_1 = P^-1 rhs / ||P^-1 rhs|| through the FP64 work vector; later
  // vectors are orthogonalized in place in their basis slot
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
  gm_start_kernel<TM, double><<<OVS_RED_BLOCKS, OVS_RED_THREADS, 0, s>>>(N, nf, sys, rhs, pre, wd, tol, gm,
                                                                         rhs_pre ? 1 : 0);
  gm_normalize_kernel<TV, double><<<OVS_RED_BLOCKS, OVS_RED_THREADS, 0, s>>>(wd, V, n, gm, 1);
  c->launches += 2;
  OVS_CUDA_TRY(cudaGetLastError());
  // one Arnoldi iteration per step (see ArnoldiPlan)
  ArnoldiPlan pl;
  if ((st = plan_arnoldi<TM, TV, ACC64>(c, sys, n, c->arnoldi_fused, &pl))) return st;
  const int batch = N > 200000 ? 4 : 16;
  int k = 1;
  for (; k <= kspace;) {
    const int kend = (k + batch - 1 < kspace) ? k + batch - 1 : kspace;
    for (; k <= kend; ++k)
      if ((st = launch_arnoldi<TM, TV, ACC64>(c, sys, pl, vals, pre, V, ld, n, k))) return st;
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
  ++c->launches;
  GmresDev* gm = c->gm;
  int km[2] = {kspace, 1};
  OVS_CUDA_TRY(cudaMemcpyAsync(&gm->kspace, km, sizeof(km), cudaMemcpyHostToDevice, c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(&gm->done, 0, sizeof(int), c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(&gm->epsnrm, 0, sizeof(double), c->stream));
  const TM* vals = as<TM>(S.vals);
  const TM* pre = as<TM>(S.binv);
  ArnoldiPlan pl;
  if ((st = plan_arnoldi<TM, TM, ACC64>(c, sys, n, what == OVS_PROF_ARNOLDI_FUSED, &pl))) return st;
  auto run = [&]() -> int {
    if (what == OVS_PROF_SPMV) {
      st = launch_spmv<TM, TM, TM, 1, ACC64>(c, sys, vals, V, V + ld, pre, nullptr, nullptr);
      return st;
    }
    return launch_arnoldi<TM, TM, ACC64>(c, sys, pl, vals, pre, V, ld, n, k);
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

// y = P^-1 x with the block-diagonal preconditioner in `pre` (the layout of
// precond_setup_kernel: 3x3 velocity inverses, then 1/M and 1/LS per node;
// one value per node for the temperature system)
template <typename TM>
__global__ void precond_apply_kernel(int N, int sys, const TM* __restrict__ pre, const double* __restrict__ x,
                                     double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const size_t n = N;
  if (sys == OVS_SYS_TEM) { y[i] = (double)pre[i] * x[i]; return; }
  const TM* B = pre + (size_t)i * 9;
  const double x0 = x[i], x1 = x[n + i], x2 = x[2 * n + i];
  for (int g = 0; g < 3; ++g)
    y[g * n + i] = (double)B[3 * g] * x0 + (double)B[3 * g + 1] * x1 + (double)B[3 * g + 2] * x2;
  y[3 * n + i] = x[3 * n + i] * (double)pre[9 * n + i];
  if (sys == OVS_SYS_NSVOF) y[4 * n + i] = x[4 * n + i] * (double)pre[10 * n + i];
}

int ovs_precond_apply_impl(ovs_ctx* c, int sys, int prec, const double* dx, double* dy) {
  SysStore& S = c->sys[sys][prec];
  if (!S.binv) return OVS_ERR_STATE;
  if (prec == OVS_FP64)
    precond_apply_kernel<double><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(c->N, sys, as<double>(S.binv), dx, dy);
  else
    precond_apply_kernel<float><<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(c->N, sys, as<float>(S.binv), dx, dy);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// y = P^-1 A x (dx, dy FP64 device vectors), preconditioned product
int ovs_spmv_pre_impl(ovs_ctx* c, int sys, int prec, const double* dx, double* dy) {
  SysStore& S = c->sys[sys][prec];
  if (!S.vals || !S.binv) return OVS_ERR_STATE;
  if (prec == OVS_FP64)
    return launch_spmv<double, double, double, 1>(c, sys, as<double>(S.vals), dx, dy, as<double>(S.binv), nullptr, nullptr);
  return launch_spmv<float, double, double, 1>(c, sys, as<float>(S.vals), dx, dy, as<float>(S.binv), nullptr, nullptr);
}

// the same products on a list of rows (device int array, local indices)
int ovs_spmv_rows_impl(ovs_ctx* c, int sys, int prec, bool precond, const double* dx, double* dy, const int* rows,
                       int nrows) {
  SysStore& S = c->sys[sys][prec];
  if (!S.vals || (precond && !S.binv)) return OVS_ERR_STATE;
  if (prec == OVS_FP64) {
    if (precond) return launch_spmv_rows<double, 1>(c, sys, as<double>(S.vals), dx, dy, as<double>(S.binv), rows, nrows);
    return launch_spmv_rows<double, 0>(c, sys, as<double>(S.vals), dx, dy, nullptr, rows, nrows);
  }
  if (precond) return launch_spmv_rows<float, 1>(c, sys, as<float>(S.vals), dx, dy, as<float>(S.binv), rows, nrows);
  return launch_spmv_rows<float, 0>(c, sys, as<float>(S.vals), dx, dy, nullptr, rows, nrows);
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

// The FP32 matrix of `sys` := the FP32 rounding of its FP64 matrix (queued
// on the context stream).
int ovs_round_impl(ovs_ctx* c, int sys) {
  SysStore& S = c->sys[sys][OVS_FP64];
  if (!S.vals) return OVS_ERR_STATE;
  SysStore& S32 = c->sys[sys][OVS_FP32];
  const size_t nv = (size_t)c->nnz * ovs_sys_nv(sys);
  int st;
  if ((st = ovs_ensure(&S32.vals, sizeof(float) * nv))) return st;
  convert_kernel<double, float><<<ovs_grid(nv, 256, 16 * c->num_sms), 256, 0, c->stream>>>(
      as<double>(S.vals), reinterpret_cast<float*>(S32.vals), nv);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  S32.have_mat = true;
  return OVS_OK;
}

// y = y + a x and y = a x over n values (y FP64)
template <typename TX>
__global__ void axpy64_kernel(double* __restrict__ y, const TX* __restrict__ x, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] += a * (double)x[i];
}
__global__ void scale64_kernel(double* __restrict__ y, const double* __restrict__ x, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = a * x[i];
}

// OVS_MIXED with a flexible Krylov outer (FGMRES(m), Saad 1993): the outer
// iteration runs in FP64 on the FP64 system, and each of its directions is
// preconditioned by one FP32 GMRES cycle on the FP32 rounding of the matrix
// (z_j ~ A^-1 v_j), so the corrections of successive inner cycles are
// combined by a least-squares fit instead of added one after another.  The
// outer basis V (m + 1 vectors) and the preconditioned directions Z (m) are
// FP64; the outer Gram-Schmidt is modified Gram-Schmidt with FP64 dots.
// After m directions, or when the outer residual estimate reaches rtol, x
// is updated and the true residual b - A x recomputed with the FP64 matrix.
// x, r, b: FP64 device vectors (r = b - A x on entry); cycles counts inner
// cycles (max_cycles bounds them), iters inner iterations.
static int solve_flexible(ovs_ctx* c, int sys, double rtol, int kspace, int max_cycles, int m, double* x,
                          double* r, const double* b, double bnorm, int& cycles, int& iters, double& rel) {
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  cudaStream_t s = c->stream;
  SysStore& S = c->sys[sys][OVS_FP64];
  const int gr = ovs_grid(n, 256, 8 * c->num_sms);
  // V (m + 1 FP64 vectors) and Z (m FP32 vectors: a direction rounded to
  // FP32 before its product is taken is as good a direction, and A z_j is
  // formed from the rounded z_j), kept by the context between solves
  const size_t need = sizeof(double) * n * ((size_t)m + 1) + sizeof(float) * n * (size_t)m;
  if (c->fg_bytes < need) {
    if (c->fg_buf) cudaFree(c->fg_buf);
    c->fg_buf = nullptr;
    c->fg_bytes = 0;
    if (cudaMalloc(&c->fg_buf, need) != cudaSuccess) {
      cudaGetLastError();
      c->fg_buf = nullptr;
      return OVS_ERR_NOMEM;
    }
    c->fg_bytes = need;
  }
  double* V = reinterpret_cast<double*>(c->fg_buf);
  float* Z = reinterpret_cast<float*>(V + n * ((size_t)m + 1));
  double* zw = r;   // the inner cycle's FP64 correction, in the residual's storage until the update
  std::vector<double> H((size_t)(m + 1) * m), g(m + 1), cs(m), sn(m), y(m);
  int st = OVS_OK;
  if ((st = ovs_precond_setup(c, sys, OVS_FP64))) return st;
  while (rel > rtol && cycles < max_cycles) {
    // the outer iteration minimizes the preconditioned residual P^-1 (b - A x)
    // (the block-Jacobi scaling balances the fields, whose raw residuals
    // differ by orders of magnitude); v_1 = P^-1 r / |P^-1 r|
    if ((st = ovs_precond_apply_impl(c, sys, OVS_FP64, r, V))) break;
    double vv;
    if ((st = dot64(c, V, V, n, &vv))) break;
    const double beta = sqrt(vv);
    if (!(beta > 0.0)) break;
    scale64_kernel<<<gr, 256, 0, s>>>(V, V, 1.0 / beta, n);
    ++c->launches;
    const double target = 0.5 * beta * rtol / rel;   // the reduction the true residual still needs
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    bool stop = false;
    for (; j < m && !stop && cycles < max_cycles; ++j) {
      double* vj = V + n * (size_t)j;
      float* zj = Z + n * (size_t)j;
      double* w = V + n * (size_t)(j + 1);
      OVS_CUDA_TRY(cudaMemsetAsync(zw, 0, sizeof(double) * n, s));
      double tin = target / fabs(g[j]);
      if (tin < 1e-6) tin = 1e-6;
      if (tin > 0.5) tin = 0.5;
      ovs_gmres_info gi;
      if ((st = gmres_cycle<float, float, false>(c, sys, vj, zw, tin, kspace, 1, &gi, true))) break;
      iters += gi.iterations;
      ++cycles;
      convert_kernel<double, float><<<gr, 256, 0, s>>>(zw, zj, n);
      ++c->launches;
      if ((st = launch_spmv<double, float, double, 1>(c, sys, as<double>(S.vals), zj, w, as<double>(S.binv),
                                                        nullptr, nullptr)))
        break;
      for (int i = 0; i <= j; ++i) {
        double h;
        if ((st = dot64(c, w, V + n * (size_t)i, n, &h))) break;
        H[(size_t)j * (m + 1) + i] = h;
        axpy64_kernel<<<gr, 256, 0, s>>>(w, V + n * (size_t)i, -h, n);
        ++c->launches;
      }
      if (st) break;
      double ww;
      if ((st = dot64(c, w, w, n, &ww))) break;
      const double hn = sqrt(ww);
      H[(size_t)j * (m + 1) + j + 1] = hn;
      if (hn > 0.0) {
        scale64_kernel<<<gr, 256, 0, s>>>(w, w, 1.0 / hn, n);
        ++c->launches;
      }
      // Givens rotations of column j
      double* hc = &H[(size_t)j * (m + 1)];
      for (int i = 0; i < j; ++i) {
        const double t = cs[i] * hc[i] + sn[i] * hc[i + 1];
        hc[i + 1] = -sn[i] * hc[i] + cs[i] * hc[i + 1];
        hc[i] = t;
      }
      const double den = sqrt(hc[j] * hc[j] + hc[j + 1] * hc[j + 1]);
      if (den == 0.0) { stop = true; break; }   // a zero column: the directions so far span the solution
      cs[j] = hc[j] / den;
      sn[j] = hc[j + 1] / den;
      hc[j] = den;
      hc[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (!(hn > 0.0) || fabs(g[j + 1]) <= target) stop = true;
    }
    if (st) break;
    // x += Z y with H y = g (upper triangular, j x j)
    for (int i = j - 1; i >= 0; --i) {
      double t = g[i];
      for (int k = i + 1; k < j; ++k) t -= H[(size_t)k * (m + 1) + i] * y[k];
      y[i] = H[(size_t)i * (m + 1) + i] != 0.0 ? t / H[(size_t)i * (m + 1) + i] : 0.0;
    }
    for (int i = 0; i < j; ++i) {
      axpy64_kernel<<<gr, 256, 0, s>>>(x, Z + n * (size_t)i, y[i], n);
      ++c->launches;
    }
    // (zw, the residual's storage, is rewritten with the true residual next)
    // the true residual with the FP64 matrix
    if ((st = launch_spmv<double, double, double, 2>(c, sys, as<double>(S.vals), x, r, nullptr, b, nullptr))) break;
    double rr;
    if ((st = dot64(c, r, r, n, &rr))) break;
    rel = sqrt(rr) / bnorm;
    if (!(rel == rel) || j == 0) break;
  }
  OVS_CUDA_TRY(cudaGetLastError());
  return st;
}

// Restarted / iteratively refined solve to a true FP64 relative residual.
// `outer` is the system whose residual b - A x is driven to rtol (matrix and
// right-hand side of that precision, FP64 arithmetic), `inner` the matrix
// precision of the GMRES cycles that compute the corrections:
//   OVS_FP64  outer FP64, inner FP64 (restarted GMRES);
//   OVS_MIXED outer FP64, inner FP32 = the rounding of the FP64 matrix;
//   OVS_FP32  outer FP32, inner FP32 (the FP32-assembled system).
int ovs_solve_impl(ovs_ctx* c, int sys, int mode, double rtol, int kspace, int max_cycles,
                   ovs_solve_info* info) {
  const int outer = mode == OVS_FP32 ? OVS_FP32 : OVS_FP64;
  const int prec = mode == OVS_FP64 ? OVS_FP64 : OVS_FP32;   // inner
  SysStore& S = c->sys[sys][outer];
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
  // the inner operator of OVS_MIXED: FP32 rounding of the FP64 matrix values
  if (mode == OVS_MIXED && (st = ovs_round_impl(c, sys))) return st;
  if ((st = ovs_precond_setup(c, sys, prec))) return st;
  if (outer == OVS_FP64) {
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
  if (mode == OVS_MIXED && c->mixed_outer > 0 && rel > rtol) {
    if ((st = solve_flexible(c, sys, rtol, kspace, max_cycles, c->mixed_outer, x, r, b, bnorm, cycles, iters, rel)))
      return st;
  }
  while (rel > rtol && cycles < max_cycles) {
    double tin = rtol / rel;
    if (tin < floor_tol) tin = floor_tol;
    if (tin > 0.5) tin = 0.5;
    ovs_gmres_info gi;
    if (prec == OVS_FP64) st = gmres_cycle<double, double, true>(c, sys, r, x, tin, kspace, 1, &gi);
    else st = gmres_cycle<float, float, false>(c, sys, r, x, tin, kspace, 1, &gi);
    if (st) return st;
    iters += gi.iterations;
    ++cycles;
    // r = b - A x in FP64 arithmetic, with the outer system's matrix
    if (outer == OVS_FP64) st = launch_spmv<double, double, double, 2>(c, sys, as<double>(S.vals), x, r, nullptr, b, nullptr);
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

// ------------------------------------------------------ transposed solve
// Slot of (j, i) for every slot (i, j): the pattern of a finite-element
// matrix is symmetric, so row j holds column i; a missing entry flags an
// error instead.
__global__ void transpose_map_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                     int* __restrict__ tmap, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    const int j = colidx[k];
    int lo = rowptr[j], hi = rowptr[j + 1];
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (colidx[mid] > i) hi = mid; else lo = mid;
    }
    if (colidx[lo] != i) { atomicOr(err, 1); tmap[k] = k; }
    else tmap[k] = lo;
  }
}

__global__ void gather_vals_kernel(const double* __restrict__ v, const int* __restrict__ tmap,
                                   double* __restrict__ vt, size_t nnz) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nnz; k += (size_t)gridDim.x * blockDim.x)
    vt[k] = v[tmap[k]];
}

// A^T x = rhs for the scalar temperature system: the transposed values
// stand in for the system's values during one reference-semantics cycle;
// the diagonal, and so the Jacobi preconditioner, is the same.
int ovs_gmres_transposed_impl(ovs_ctx* c, int sys, const double* drhs, double tol, int kspace, int kmin,
                              double* dsol, ovs_gmres_info* info) {
  if (sys != OVS_SYS_TEM) return OVS_ERR_ARG;
  SysStore& S = c->sys[sys][OVS_FP64];
  if (!S.vals) return OVS_ERR_STATE;
  int st;
  cudaStream_t s = c->stream;
  const size_t nnz = c->nnz;
  if (!c->tmap) {
    if ((st = ovs_ensure((void**)&c->tmap, sizeof(int) * (nnz > 0 ? nnz : 1)))) return st;
    OVS_CUDA_TRY(cudaMemsetAsync(c->flags, 0, sizeof(int) * 4, s));
    transpose_map_kernel<<<ovs_grid(c->N, 128, 1 << 30), 128, 0, s>>>(c->N, c->rowptr, c->colidx, c->tmap,
                                                                      c->flags + 2);
    ++c->launches;
    int herr = 0;
    OVS_CUDA_TRY(cudaMemcpyAsync(&herr, c->flags + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    OVS_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) { cudaFree(c->tmap); c->tmap = nullptr; return OVS_ERR_PATTERN; }
  }
  if ((st = ovs_ensure(&c->vals_t, sizeof(double) * (nnz > 0 ? nnz : 1)))) return st;
  gather_vals_kernel<<<4 * c->num_sms, 256, 0, s>>>(reinterpret_cast<const double*>(S.vals), c->tmap,
                                                    reinterpret_cast<double*>(c->vals_t), nnz);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  if ((st = ovs_precond_setup(c, sys, OVS_FP64))) return st;
  double rr;
  if ((st = dot64(c, drhs, drhs, (size_t)c->N, &rr))) return st;
  if (rr == 0.0) {   // SparseGMRES_tem.f90:63-71
    OVS_CUDA_TRY(cudaMemsetAsync(dsol, 0, sizeof(double) * c->N, s));
    OVS_CUDA_TRY(cudaStreamSynchronize(s));
    if (info) { memset(info, 0, sizeof(*info)); info->converged = 1; }
    return OVS_OK;
  }
  void* saved = S.vals;
  S.vals = c->vals_t;
  st = gmres_cycle<double, double>(c, sys, drhs, dsol, tol, kspace, kmin, info);
  S.vals = saved;
  if (st) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  return OVS_OK;
}
