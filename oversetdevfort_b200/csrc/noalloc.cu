// Allocation-free variant of the temperature-system GMRES cycle.
//
// Some callers cannot allocate device memory at solve time: codes that run
// inside a framework whose memory pool owns all device memory (a cudaMalloc
// behind its back fragments the pool or is forbidden by policy), time-critical
// loops that cannot afford the device-wide synchronization cudaMalloc and
// cudaFree imply, and plug-in hosts that only allow allocation during
// initialization.  ovs_gmres_tem_noalloc serves them: the caller passes
// device buffers for the matrix, right-hand side and solution, and every
// temporary the solver needs (Krylov basis, Jacobi preconditioner,
// Hessenberg matrix, rotations) lives in one file-scope __device__ array of
// fixed size that is part of the loaded library.
//
// The solver is one kernel with a single 1024-thread block that runs the
// whole cycle (SpMV, modified Gram-Schmidt, Givens, back-substitution,
// update) with block-level reductions, so it needs no grid-wide scratch and
// no host round trips.  It is meant for small systems (at most
// OVS_NOALLOC_MAX_N unknowns).
#include "ovs_internal.cuh"

#include <mutex>

namespace {

constexpr int NA_THREADS = 1024;
constexpr int NA_LDH = OVS_NOALLOC_MAX_KSPACE + 1;

// Scratch layout (doubles): Hessenberg (MAX_KSPACE+1) x MAX_KSPACE, e, cs,
// sn, y, 8 scalars, then the preconditioner (MAX_N) and the Krylov basis
// (MAX_KSPACE+1) x MAX_N.
constexpr size_t NA_H = 0;
constexpr size_t NA_E = NA_H + (size_t)NA_LDH * OVS_NOALLOC_MAX_KSPACE;
constexpr size_t NA_CS = NA_E + NA_LDH;
constexpr size_t NA_SN = NA_CS + OVS_NOALLOC_MAX_KSPACE;
constexpr size_t NA_Y = NA_SN + OVS_NOALLOC_MAX_KSPACE;
constexpr size_t NA_SCAL = NA_Y + OVS_NOALLOC_MAX_KSPACE;
constexpr size_t NA_PINV = (NA_SCAL + 8 + 31) & ~(size_t)31;
constexpr size_t NA_V = NA_PINV + OVS_NOALLOC_MAX_N;
constexpr size_t NA_TOTAL = NA_V + (size_t)(OVS_NOALLOC_MAX_KSPACE + 1) * OVS_NOALLOC_MAX_N;
static_assert(NA_TOTAL * sizeof(double) <= OVS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the array");

// The scratch array: allocated with the module, one instance per device that
// loads the library, kept until the process exits.  Every call shares it.
static __device__ __align__(256) double g_noalloc_scratch[OVS_NOALLOC_SCRATCH_BYTES / sizeof(double)];

__device__ __forceinline__ double na_block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
    sh[32] = r;
  }
  __syncthreads();
  return sh[32];  // same value in every thread
}

// One cycle with the semantics of SparseGMRES_tem (src/SparseGMRES_tem.f90):
// sol = 0 when ||rhs|| = 0; Jacobi preconditioner 1/M_ii (1 when M_ii = 0);
// left preconditioning; modified Gram-Schmidt in the reference order; exit
// when |e(k+1)| <= tol |P^-1 rhs| and k >= kspace_min; sol += sum y_j v_j.
__global__ void __launch_bounds__(NA_THREADS)
gmres_tem_single_cta(int n, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                     const double* __restrict__ vals, const double* __restrict__ rhs, double* __restrict__ sol,
                     double tol, int kspace, int kmin, double* __restrict__ S, int* __restrict__ info_i,
                     double* __restrict__ info_d) {
  __shared__ double sh[33];
  __shared__ int s_done;
  double* H = S + NA_H;
  double* e = S + NA_E;
  double* cs = S + NA_CS;
  double* sn = S + NA_SN;
  double* y = S + NA_Y;
  double* pinv = S + NA_PINV;
  double* V = S + NA_V;
  const size_t ldv = OVS_NOALLOC_MAX_N;
  const int t = threadIdx.x;
  // the scratch keeps the previous call's values: clear what must start at 0
  for (int i = t; i < NA_LDH * OVS_NOALLOC_MAX_KSPACE; i += NA_THREADS) H[i] = 0.0;
  for (int i = t; i < NA_LDH; i += NA_THREADS) e[i] = 0.0;
  if (t == 0) s_done = 0;
  double rr = 0.0;
  for (int i = t; i < n; i += NA_THREADS) rr += rhs[i] * rhs[i];
  rr = na_block_sum(rr, sh);
  if (rr == 0.0) {
    for (int i = t; i < n; i += NA_THREADS) sol[i] = 0.0;
    if (t == 0) { info_i[0] = 0; info_i[1] = 1; info_i[2] = 0; info_d[0] = 0.0; info_d[1] = 0.0; }
    return;
  }
  // Jacobi preconditioner (last diagonal match of the row, as the reference's scan)
  for (int i = t; i < n; i += NA_THREADS) {
    double m = 0.0;
    for (int s = rowptr[i]; s < rowptr[i + 1]; ++s)
      if (colidx[s] == i) m = vals[s];
    pinv[i] = (m != 0.0) ? 1.0 / m : 1.0;
  }
  __syncthreads();
  double un = 0.0;
  for (int i = t; i < n; i += NA_THREADS) {
    const double z = pinv[i] * rhs[i];
    V[i] = z;
    un += z * z;
  }
  un = sqrt(na_block_sum(un, sh));
  const double epsnrm = tol * un;
  if (t == 0) e[0] = un;
  const double uninv = 1.0 / un;                   // unorm = 1/unorm; u = u*unorm
  for (int i = t; i < n; i += NA_THREADS) V[i] = V[i] * uninv;
  __syncthreads();
  int iks = 0;
  double ercheck = un;
  int breakdown = 0;
  for (int k = 1; k <= kspace; ++k) {
    double* w = V + ldv * (size_t)k;
    const double* vk = V + ldv * (size_t)(k - 1);
    for (int i = t; i < n; i += NA_THREADS) {     // w = P^-1 A v_k
      double a = 0.0;
      for (int s = rowptr[i]; s < rowptr[i + 1]; ++s) a = a + vals[s] * vk[colidx[s]];
      w[i] = a * pinv[i];
    }
    __syncthreads();
    double beta = 0.0;
    for (int j = 1; j <= k + 1; ++j) {            // modified Gram-Schmidt
      const double* vj = V + ldv * (size_t)(j - 1);
      const double* vp = j >= 2 ? V + ldv * (size_t)(j - 2) : nullptr;
      double sacc = 0.0;
      for (int i = t; i < n; i += NA_THREADS) {
        double a = w[i];
        if (j >= 2) { a = a - beta * vp[i]; w[i] = a; }
        sacc += a * vj[i];
      }
      beta = na_block_sum(sacc, sh);
      if (t == 0) H[(size_t)(k - 1) * NA_LDH + (j - 1)] = beta;
    }
    const double unorm = sqrt(beta);
    if (unorm != 0.0) {
      const double uinv = 1.0 / unorm;
      for (int i = t; i < n; i += NA_THREADS) w[i] = w[i] * uinv;
    }
    if (t == 0) {                                  // Givens update and exit test
      double* Hk = H + (size_t)(k - 1) * NA_LDH;
      Hk[k] = unorm;
      for (int jk = 1; jk <= k - 1; ++jk) {
        const double tmp = cs[jk - 1] * Hk[jk - 1] + sn[jk - 1] * Hk[jk];
        Hk[jk] = -sn[jk - 1] * Hk[jk - 1] + cs[jk - 1] * Hk[jk];
        Hk[jk - 1] = tmp;
      }
      const double a = Hk[k - 1], b = Hk[k];
      const double tmp = sqrt(a * a + b * b);
      if (tmp == 0.0) {
        // column k of H is zero: P^-1 A v_k lies in the span of v_1..v_{k-1}
        // with no component of its own, the rotation is 0/0 (the reference
        // would carry NaN on).  The cycle ends with the solution of the
        // first k-1 columns.
        s_done = 3;
      } else {
        const double tmp1 = 1.0 / tmp;
        cs[k - 1] = a * tmp1;
        sn[k - 1] = b * tmp1;
        Hk[k - 1] = tmp;
        Hk[k] = 0.0;
        const double t2 = cs[k - 1] * e[k - 1] + sn[k - 1] * e[k];
        e[k] = -sn[k - 1] * e[k - 1] + cs[k - 1] * e[k];
        e[k - 1] = t2;
        const double er = fabs(e[k]);
        S[NA_SCAL] = er;
        if ((er <= epsnrm && k >= kmin) || unorm == 0.0) s_done = (unorm == 0.0) ? 2 : 1;
      }
    }
    __syncthreads();
    if (s_done == 3) { breakdown = 1; break; }
    iks = k;
    ercheck = S[NA_SCAL];
    if (s_done) { breakdown = s_done == 2; break; }
  }
  if (t == 0) {                                    // back-substitution
    for (int jk = iks; jk >= 1; --jk) {
      const double yj = e[jk - 1] / H[(size_t)(jk - 1) * NA_LDH + (jk - 1)];
      y[jk - 1] = yj;
      for (int lk = 1; lk <= jk - 1; ++lk) e[lk - 1] = e[lk - 1] - yj * H[(size_t)(jk - 1) * NA_LDH + (lk - 1)];
    }
  }
  __syncthreads();
  for (int i = t; i < n; i += NA_THREADS) {
    double s = sol[i];
    for (int j = 0; j < iks; ++j) s = s + y[j] * V[ldv * (size_t)j + i];
    sol[i] = s;
  }
  if (t == 0) {
    info_i[0] = iks;
    info_i[1] = ercheck <= epsnrm;
    info_i[2] = breakdown;
    info_d[0] = un;
    info_d[1] = ercheck;
  }
}

// device address of the scratch array, looked up once per device
std::mutex g_na_mutex;
double* g_na_ptr[64] = {nullptr};

}  // namespace

extern "C" int ovs_gmres_tem_noalloc(int n, const int* rowptr, const int* colidx, const double* vals,
                                     const double* rhs, double* sol, double tol, int kspace, int kspace_min,
                                     void* stream, ovs_gmres_info* info) {
  if (n < 1 || !rowptr || !colidx || !vals || !rhs || !sol) return OVS_ERR_ARG;
  if (n > OVS_NOALLOC_MAX_N || kspace < 1 || kspace > OVS_NOALLOC_MAX_KSPACE) return OVS_ERR_ARG;
  int dev = 0;
  OVS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return OVS_ERR_ARG;
  double* S = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
      // In host code g_noalloc_scratch names a host-side shadow, not device
      // memory; the kernel must get the device address.
      void* p = nullptr;
      OVS_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      g_na_ptr[dev] = static_cast<double*>(p);
    }
    S = g_na_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* info_i = reinterpret_cast<int*>(S + NA_SCAL + 2);
  double* info_d = S + NA_SCAL + 4;
  // an error left pending by an earlier call of the caller's is not this
  // launch's: clear it so the check below sees this launch alone
  (void)cudaGetLastError();
  gmres_tem_single_cta<<<1, NA_THREADS, 0, s>>>(n, rowptr, colidx, vals, rhs, sol, tol, kspace, kspace_min, S,
                                                info_i, info_d);
  OVS_CUDA_TRY(cudaGetLastError());
  int hi[3] = {0, 0, 0};
  double hd[2] = {0.0, 0.0};
  OVS_CUDA_TRY(cudaMemcpyAsync(hi, info_i, sizeof(hi), cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(hd, info_d, sizeof(hd), cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  if (info) {
    info->iterations = hi[0];
    info->converged = hi[1];
    info->breakdown = hi[2];
    info->reserved = 0;
    info->res0 = hd[0];
    info->ercheck = hd[1];
  }
  return OVS_OK;
}
