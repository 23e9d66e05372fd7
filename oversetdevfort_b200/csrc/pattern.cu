// CSR sparsity pattern and node->element map (replaces genSparStruc/Asadj,
// src/genSparStruc.f90:4-105, and the per-element slot lookups of
// SparseMatLoc_3D, src/FillSparseMat.f90:4-28).
//
// The reference builds, per node, the unique list of nodes that share an
// element and sorts every row ascending.  The sorted unique set does not
// depend on the visit order, so it is built here row-parallel: one thread per
// node walks its elements (node->element map), inserts their nodes into a
// small sorted array and emits the row.  Two passes (count, scan, fill) keep
// the output layout identical to the reference's col/row arrays.
#include "ovs_internal.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <vector>

#include <math.h>

namespace {

// ------------------------------------------------ spatial order of the rows
// Per block: min and max of each coordinate (N x 3 column-major xg).
__global__ void bbox_kernel(const double* __restrict__ xg, int N, double* __restrict__ out) {
  __shared__ double sh[6][256];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      const double v = xg[(size_t)d * N + i];
      lo[d] = fmin(lo[d], v);
      hi[d] = fmax(hi[d], v);
    }
  for (int d = 0; d < 3; ++d) { sh[d][threadIdx.x] = lo[d]; sh[3 + d][threadIdx.x] = hi[d]; }
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int d = 0; d < 3; ++d) {
        sh[d][threadIdx.x] = fmin(sh[d][threadIdx.x], sh[d][threadIdx.x + o]);
        sh[3 + d][threadIdx.x] = fmax(sh[3 + d][threadIdx.x], sh[3 + d][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) out[(size_t)blockIdx.x * 6 + threadIdx.x] = sh[threadIdx.x][0];
}

// 21 bits of each quantized coordinate interleaved into a 63-bit Morton key
__device__ __forceinline__ unsigned long long spread21(unsigned v) {
  unsigned long long x = v & 0x1fffffULL;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

__global__ void morton_kernel(const double* __restrict__ xg, int N, double x0, double y0, double z0, double sx,
                              double sy, double sz, unsigned long long* __restrict__ key, int* __restrict__ id) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double q[3] = {(xg[i] - x0) * sx, (xg[(size_t)N + i] - y0) * sy, (xg[2 * (size_t)N + i] - z0) * sz};
  unsigned u[3];
  for (int d = 0; d < 3; ++d) u[d] = (unsigned)fmin(fmax(q[d], 0.0), 2097151.0);
  key[i] = spread21(u[0]) | (spread21(u[1]) << 1) | (spread21(u[2]) << 2);
  id[i] = i;
}

constexpr int SCAN_T = 1024;

// ---------------------------------------------------------------- scans
__global__ void scan_block_kernel(const int* __restrict__ in, int* __restrict__ out,
                                  int* __restrict__ block_sums, int n) {
  __shared__ int wsum[32];
  int i = blockIdx.x * SCAN_T + threadIdx.x;
  int v = (i < n) ? in[i] : 0;
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  int excl = x - v + (w > 0 ? wsum[w - 1] : 0);
  if (i < n) out[i] = excl;
  if (threadIdx.x == SCAN_T - 1) block_sums[blockIdx.x] = excl + v;
}

__global__ void scan_add_kernel(int* __restrict__ out, const int* __restrict__ offs, int n) {
  int i = blockIdx.x * SCAN_T + threadIdx.x;
  if (i < n && blockIdx.x > 0) out[i] += offs[blockIdx.x];
}

// exclusive scan of n ints (n may be large); tmp needs >= 2*ceil(n/1024)+2 ints;
// *launches counts the kernels it launches
int exclusive_scan(const int* in, int* out, int n, int* tmp, cudaStream_t s, long long* launches) {
  int nb = (n + SCAN_T - 1) / SCAN_T;
  int* sums = tmp;
  int* sums_scan = tmp + nb + 1;
  scan_block_kernel<<<nb, SCAN_T, 0, s>>>(in, out, sums, n);
  ++*launches;
  if (nb > 1) {
    int nb2 = (nb + SCAN_T - 1) / SCAN_T;
    if (nb2 > 1) {
      // second level recursion (n up to 2^30)
      int* tmp2 = sums_scan + nb + 1;
      int st = exclusive_scan(sums, sums_scan, nb, tmp2, s, launches);
      if (st) return st;
    } else {
      int* dummy = sums_scan + nb + 1;
      scan_block_kernel<<<1, SCAN_T, 0, s>>>(sums, sums_scan, dummy, nb);
      ++*launches;
    }
    scan_add_kernel<<<nb, SCAN_T, 0, s>>>(out, sums_scan, n);
    ++*launches;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : OVS_ERR_CUDA;
}

// ------------------------------------------------------ node -> element map
__global__ void count_n2e_kernel(const int* __restrict__ ien, int E, int nshl,
                                 int N, int* __restrict__ cnt, int* __restrict__ bad) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)E * nshl) return;
  int node = ien[t];
  if (node < 0 || node >= N) { atomicAdd(bad, 1); return; }
  atomicAdd(&cnt[node], 1);
}

__global__ void fill_n2e_kernel(const int* __restrict__ ien, int E, int nshl, int N,
                                int* __restrict__ cursor, int* __restrict__ n2e) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)E * nshl) return;
  int node = ien[t];
  if (node < 0 || node >= N) return;
  int e = (int)(t / nshl), a = (int)(t % nshl);
  int pos = atomicAdd(&cursor[node], 1);
  n2e[pos] = (e << 3) | a;
}

// sort every node's element list by element id (insertion sort; lists are short)
__global__ void sort_n2e_kernel(const int* __restrict__ ptr, int* __restrict__ n2e, int N,
                                int* __restrict__ max_elem) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int b = ptr[i], e = ptr[i + 1];
  for (int k = b + 1; k < e; ++k) {
    int v = n2e[k];
    int j = k - 1;
    while (j >= b && n2e[j] > v) { n2e[j + 1] = n2e[j]; --j; }
    n2e[j + 1] = v;
  }
  atomicMax(max_elem, e - b);
}

// Collect the sorted unique neighbour list of node i into buf (local memory).
__device__ int collect_row(int i, const int* __restrict__ ien, int nshl,
                           const int* __restrict__ ptr, const int* __restrict__ n2e,
                           int* buf) {
  int len = 0;
  for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
    int e = n2e[k] >> 3;
    for (int a = 0; a < nshl; ++a) {
      int nd = ien[(size_t)e * nshl + a];
      // binary search for nd in buf[0,len)
      int lo = 0, hi = len;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (buf[mid] < nd) lo = mid + 1; else hi = mid;
      }
      if (lo < len && buf[lo] == nd) continue;
      if (len >= OVS_MAX_DEG) return -1;
      for (int t = len; t > lo; --t) buf[t] = buf[t - 1];
      buf[lo] = nd;
      ++len;
    }
  }
  return len;
}

__global__ void row_len_kernel(const int* __restrict__ ien, int nshl, int N,
                               const int* __restrict__ ptr, const int* __restrict__ n2e,
                               int* __restrict__ rowlen, int* __restrict__ flags,
                               int* __restrict__ max_deg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int buf[OVS_MAX_DEG];
  int len = collect_row(i, ien, nshl, ptr, n2e, buf);
  if (len < 0) { atomicOr(flags, 1); len = 0; }
  rowlen[i] = len;
  atomicMax(max_deg, len);
}

__global__ void row_fill_kernel(const int* __restrict__ ien, int nshl, int N,
                                const int* __restrict__ ptr, const int* __restrict__ n2e,
                                const int* __restrict__ rowptr, int* __restrict__ colidx,
                                int* __restrict__ diag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int buf[OVS_MAX_DEG];
  int len = collect_row(i, ien, nshl, ptr, n2e, buf);
  int base = rowptr[i];
  int d = -1;
  for (int k = 0; k < len; ++k) {
    colidx[base + k] = buf[k];
    if (buf[k] == i) d = base + k;
  }
  diag[i] = d;
}

// Slot map: for node-to-element entry k of row A (element e, sorted by
// element), the slots in A's column list of e's 4 nodes, one byte each
// (rows have at most OVS_MAX_DEG <= 255 columns).  The assembly row pass
// reads it instead of searching the row for every element block.
__global__ void slot_map_kernel(const int* __restrict__ ien, int N, const int* __restrict__ n2e_ptr,
                                const int* __restrict__ n2e, const int* __restrict__ rowptr,
                                const int* __restrict__ colidx, unsigned* __restrict__ n2s) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= N) return;
  const int rp = rowptr[A], deg = rowptr[A + 1] - rp;
  for (int k = n2e_ptr[A]; k < n2e_ptr[A + 1]; ++k) {
    const int4 nd = reinterpret_cast<const int4*>(ien)[n2e[k] >> 3];
    const int nodes[4] = {nd.x, nd.y, nd.z, nd.w};
    unsigned packed = 0;
    for (int b = 0; b < 4; ++b) {
      int lo = 0, hi = deg;   // last index with colidx <= node (SparseMatLoc_3D)
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (colidx[rp + mid] > nodes[b]) hi = mid; else lo = mid;
      }
      packed |= (unsigned)lo << (8 * b);
    }
    n2s[k] = packed;
  }
}

// The same for hexahedra: 8 slots, bytes 0-3 in the first word and 4-7 in
// the second.
__global__ void slot_map8_kernel(const int* __restrict__ ien, int N, const int* __restrict__ n2e_ptr,
                                 const int* __restrict__ n2e, const int* __restrict__ rowptr,
                                 const int* __restrict__ colidx, uint2* __restrict__ n2s) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= N) return;
  const int rp = rowptr[A], deg = rowptr[A + 1] - rp;
  for (int k = n2e_ptr[A]; k < n2e_ptr[A + 1]; ++k) {
    const int* nodes = ien + 8 * (size_t)(n2e[k] >> 3);
    unsigned w[2] = {0u, 0u};
    for (int b = 0; b < 8; ++b) {
      int lo = 0, hi = deg;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (colidx[rp + mid] > nodes[b]) hi = mid; else lo = mid;
      }
      w[b >> 2] |= (unsigned)lo << (8 * (b & 3));
    }
    n2s[k] = make_uint2(w[0], w[1]);
  }
}

// Global 1-based CSR slot k(e, a, b) of every element entry, from the slot
// map: the n2e entry (e, a) of row A = IEN(e, a) holds the in-row offsets of
// the element's nodes, so k = rowptr[A] + offset_b + 1.  Every (e, a) occurs
// exactly once in the node-to-element lists.  lmap is (E, nshl, nshl)
// column-major, the index order of FillSparseMat_3D's (a, b) loops.
__global__ void slot_export_kernel(int N, int E, int nshl, const int* __restrict__ n2e_ptr,
                                   const int* __restrict__ n2e, const unsigned* __restrict__ n2s,
                                   const int* __restrict__ rowptr, int* __restrict__ lmap) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= N) return;
  const int rp1 = rowptr[A] + 1;
  const int words = nshl == 8 ? 2 : 1;
  for (int k = n2e_ptr[A]; k < n2e_ptr[A + 1]; ++k) {
    const int e = n2e[k] >> 3, a = n2e[k] & 7;
    for (int b = 0; b < nshl; ++b) {
      const unsigned w = n2s[(size_t)k * words + (b >> 2)];
      const int off = (int)((w >> (8 * (b & 3))) & 0xffu);
      lmap[(size_t)e + (size_t)E * ((size_t)a + (size_t)nshl * b)] = rp1 + off;
    }
  }
}

__global__ void to_one_based_kernel(const int* __restrict__ in, int* __restrict__ out, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] + 1;
}

}  // namespace

int ovs_pattern_to_host(ovs_ctx* c, int* col, int* row) {
  cudaStream_t s = c->stream;
  size_t n1 = (size_t)c->N + 1, n2 = (size_t)c->nnz;
  int* tmp = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * (n1 > n2 ? n1 : n2), s));
  to_one_based_kernel<<<ovs_grid(n1, 256, 1 << 30), 256, 0, s>>>(c->rowptr, tmp, n1);
  ++c->launches;
  OVS_CUDA_TRY(cudaMemcpyAsync(col, tmp, sizeof(int) * n1, cudaMemcpyDeviceToHost, s));
  if (row && n2) {
    to_one_based_kernel<<<ovs_grid(n2, 256, 1 << 30), 256, 0, s>>>(c->colidx, tmp, n2);
    ++c->launches;
    OVS_CUDA_TRY(cudaMemcpyAsync(row, tmp, sizeof(int) * n2, cudaMemcpyDeviceToHost, s));
  }
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  return OVS_OK;
}

int ovs_slot_map_to_host(ovs_ctx* c, int* lmap) {
  cudaStream_t s = c->stream;
  const size_t n = (size_t)c->E * c->nshl * c->nshl;
  int* tmp = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * (n > 0 ? n : 1), s));
  slot_export_kernel<<<ovs_grid(c->N, 128, 1 << 30), 128, 0, s>>>(c->N, c->E, c->nshl, c->n2e_ptr, c->n2e,
                                                                 c->n2s, c->rowptr, tmp);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  if (n) OVS_CUDA_TRY(cudaMemcpyAsync(lmap, tmp, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  return OVS_OK;
}

// c->row_order: the nodes sorted by the Morton key of their coordinates,
// the order in which the assembly's row pass visits the rows (each row's
// result does not depend on the order).  Rows that share an element then
// run close together in time and the element's summary is reused from L2.
static int build_row_order(ovs_ctx* c) {
  cudaStream_t s = c->stream;
  const int N = c->N;
  const double* xg = c->field[OVS_F_XG];
  if (!xg || N < 2) return OVS_OK;
  int st;
  if ((st = ovs_ensure((void**)&c->row_order, sizeof(int) * N))) return st;
  const int nb = ovs_grid(N, 256, 4 * c->num_sms);
  double* part = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&part, sizeof(double) * 6 * nb, s));
  bbox_kernel<<<nb, 256, 0, s>>>(xg, N, part);
  ++c->launches;
  std::vector<double> h((size_t)6 * nb);
  OVS_CUDA_TRY(cudaMemcpyAsync(h.data(), part, sizeof(double) * 6 * nb, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  OVS_CUDA_TRY(cudaFreeAsync(part, s));
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int b = 0; b < nb; ++b)
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], h[(size_t)b * 6 + d]);
      hi[d] = fmax(hi[d], h[(size_t)b * 6 + 3 + d]);
    }
  double sc[3];
  for (int d = 0; d < 3; ++d) sc[d] = hi[d] > lo[d] ? 2097151.0 / (hi[d] - lo[d]) : 0.0;
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  int* id0 = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&k0, sizeof(unsigned long long) * N, s));
  OVS_CUDA_TRY(cudaMallocAsync(&k1, sizeof(unsigned long long) * N, s));
  OVS_CUDA_TRY(cudaMallocAsync(&id0, sizeof(int) * N, s));
  morton_kernel<<<ovs_grid(N, 256, 1 << 30), 256, 0, s>>>(xg, N, lo[0], lo[1], lo[2], sc[0], sc[1], sc[2], k0, id0);
  ++c->launches;
  size_t tbytes = 0;
  OVS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tbytes, k0, k1, id0, c->row_order, N, 0, 63, s));
  void* tmp = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, tbytes > 0 ? tbytes : 16, s));
  OVS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tbytes, k0, k1, id0, c->row_order, N, 0, 63, s));
  c->launches += 4;   // the radix sort's passes (counted approximately)
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaFreeAsync(k0, s));
  OVS_CUDA_TRY(cudaFreeAsync(k1, s));
  OVS_CUDA_TRY(cudaFreeAsync(id0, s));
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// the row pass's row records, in its processing order (row_order[t], or t):
// {A, rowptr[A], n2e_ptr[A], deg | sd << 8 | ne << 16} with sd the slot of
// the diagonal entry in the row, one 16-byte load per row
__global__ void row_rec_kernel(const int* order, const int* rowptr, const int* n2e_ptr, const int* diag, int N,
                               int4* rec) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  const int A = order ? order[t] : t;
  const int rp = rowptr[A], ep = n2e_ptr[A], deg = rowptr[A + 1] - rp;
  const int sd = diag[A] >= rp ? diag[A] - rp : 0;
  rec[t] = make_int4(A, rp, ep, deg | (sd << 8) | ((n2e_ptr[A + 1] - ep) << 16));
}

static int build_row_rec(ovs_ctx* c) {
  const int N = c->N;
  if (N < 1) return OVS_OK;
  // the record packs the degree and the diagonal slot in 8 bits each
  // (OVS_MAX_DEG <= 255) and the element count in 15
  if (c->max_deg > 0xff || c->max_elem > 0x7fff) return OVS_ERR_PATTERN;
  int st;
  if ((st = ovs_ensure((void**)&c->row_rec, sizeof(int4) * (size_t)N))) return st;
  row_rec_kernel<<<ovs_grid(N, 256, 1 << 30), 256, 0, c->stream>>>(c->row_order, c->rowptr, c->n2e_ptr, c->diag,
                                                                   N, c->row_rec);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// Contribution lists of the off-diagonal entries (tets), the gather row
// pass's input: for entry (A, B), B != A, the elements holding both nodes in
// ascending element order, each as (e << 4) | (la << 2) | b with
// A = ien[e][la], B = ien[e][b]; cptr[k]..cptr[k+1] delimits entry k's list
// (diagonal entries have none: every element of the row adds to them).
// One thread per row, the row's entries counted / filled in n2e order.
__global__ void contrib_count_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ n2e_ptr,
                                     const int* __restrict__ n2e, const unsigned* __restrict__ n2s,
                                     int* __restrict__ cnt) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= N) return;
  const int rp = rowptr[A];
  for (int k = n2e_ptr[A]; k < n2e_ptr[A + 1]; ++k) {
    const int la = n2e[k] & 7;
    const unsigned w = n2s[k];
    for (int b = 0; b < 4; ++b)
      if (b != la) ++cnt[rp + ((w >> (8 * b)) & 0xffu)];
  }
}

__global__ void contrib_fill_kernel(int N, const int* __restrict__ rowptr, const int* __restrict__ n2e_ptr,
                                    const int* __restrict__ n2e, const unsigned* __restrict__ n2s,
                                    int* __restrict__ cursor, int* __restrict__ list) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= N) return;
  const int rp = rowptr[A];
  for (int k = n2e_ptr[A]; k < n2e_ptr[A + 1]; ++k) {
    const int e = n2e[k] >> 3, la = n2e[k] & 7;
    const unsigned w = n2s[k];
    for (int b = 0; b < 4; ++b)
      if (b != la) list[cursor[rp + ((w >> (8 * b)) & 0xffu)]++] = (e << 4) | (la << 2) | b;
  }
}

static int build_contrib(ovs_ctx* c) {
  cudaStream_t s = c->stream;
  const int N = c->N, nnz = c->nnz;
  if (c->nshl != 4 || N < 1 || nnz < 1) return OVS_OK;
  if (c->E >= (1 << 27)) return OVS_OK;   // (e << 4) must fit an int: the chunked row pass serves
  const size_t ents = (size_t)12 * c->E;  // 3 off-diagonal blocks per element row
  int st;
  if ((st = ovs_ensure((void**)&c->cptr, sizeof(int) * ((size_t)nnz + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->clist, sizeof(int) * (ents > 0 ? ents : 1)))) return st;
  int *cnt = nullptr, *tmp = nullptr;
  const int nb = (nnz + 1 + SCAN_T - 1) / SCAN_T;
  OVS_CUDA_TRY(cudaMallocAsync(&cnt, sizeof(int) * ((size_t)nnz + 1), s));
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * (4 * (size_t)nb + 64), s));
  OVS_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)nnz + 1), s));
  contrib_count_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(N, c->rowptr, c->n2e_ptr, c->n2e, c->n2s, cnt);
  ++c->launches;
  if ((st = exclusive_scan(cnt, c->cptr, nnz + 1, tmp, s, &c->launches))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(cnt, c->cptr, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToDevice, s));
  contrib_fill_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(N, c->rowptr, c->n2e_ptr, c->n2e, c->n2s, cnt,
                                                                c->clist);
  ++c->launches;
  OVS_CUDA_TRY(cudaFreeAsync(cnt, s));
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// Row tiles of the tiled row pass, built on the host from the row records,
// the node-to-element lists and the contribution lists: consecutive rows of
// the row order (Morton order of the nodes, so a tile is a compact cluster
// of nodes) are added to a tile while its distinct elements stay within
// maxe and its rows within 16.  For every row entry the element is
// renumbered to its place in the tile's element list (n2e_loc, clist_loc).
// A row with more than maxe elements takes no tile (big_rec lists them for
// the gather pass).
int ovs_tiles_build(ovs_ctx* c, int maxe) {
  constexpr int RMAX = 16;
  cudaStream_t s = c->stream;
  const int N = c->N, E = c->E;
  if (c->nshl != 4 || !c->cptr || !c->row_rec || N < 1) return OVS_ERR_STATE;
  if (maxe < 4 || maxe > 4000) return OVS_ERR_ARG;
  if (c->tile_maxe == maxe && c->tile_rptr) return OVS_OK;
  void** olds[] = {(void**)&c->tile_rptr, (void**)&c->tile_rows, (void**)&c->tile_eptr, (void**)&c->tile_elems,
                   (void**)&c->n2e_loc, (void**)&c->clist_loc, (void**)&c->big_rec};
  for (void** q : olds) {
    if (*q) cudaFree(*q);
    *q = nullptr;
  }
  c->ntiles = c->nbig = c->tile_maxe = 0;
  const size_t EN = (size_t)E * 4, NC = (size_t)12 * E, nnz = (size_t)c->nnz;
  std::vector<int4> rec(N);
  std::vector<int> n2e(EN), cptr(nnz + 1), clist(NC > 0 ? NC : 1);
  OVS_CUDA_TRY(cudaMemcpyAsync(rec.data(), c->row_rec, sizeof(int4) * N, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(n2e.data(), c->n2e, sizeof(int) * EN, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(cptr.data(), c->cptr, sizeof(int) * (nnz + 1), cudaMemcpyDeviceToHost, s));
  if (NC) OVS_CUDA_TRY(cudaMemcpyAsync(clist.data(), c->clist, sizeof(int) * NC, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<int> stamp(E, -1), loc(E, 0), trptr{0}, trows, teptr{0}, telems;
  std::vector<uint16_t> n2e_loc(EN, 0), clist_loc(NC > 0 ? NC : 1, 0);
  std::vector<int4> big;
  trows.reserve(N);
  telems.reserve((size_t)N * 20);
  int tile = 0, cnt = 0, rows = 0;
  for (int t = 0; t < N; ++t) {
    const int4 r = rec[t];
    const int rp = r.y, ep = r.z, deg = r.w & 0xff, sd = (r.w >> 8) & 0xff, ne = r.w >> 16;
    if (ne > maxe) {
      big.push_back(r);
      continue;
    }
    int nnew = 0;
    for (int j = 0; j < ne; ++j) nnew += stamp[n2e[ep + j] >> 3] != tile;
    if (rows > 0 && (cnt + nnew > maxe || rows >= RMAX)) {   // close the tile
      trptr.push_back((int)trows.size());
      teptr.push_back((int)telems.size());
      ++tile;
      cnt = rows = 0;
    }
    for (int j = 0; j < ne; ++j) {
      const int e = n2e[ep + j] >> 3, la = n2e[ep + j] & 7;
      if (stamp[e] != tile) {
        stamp[e] = tile;
        loc[e] = cnt++;
        telems.push_back(e);
      }
      n2e_loc[ep + j] = (uint16_t)((loc[e] << 2) | la);
    }
    for (int q = 0; q < deg; ++q) {
      if (q == sd) continue;
      for (int k = cptr[rp + q]; k < cptr[rp + q + 1]; ++k)
        clist_loc[k] = (uint16_t)((loc[clist[k] >> 4] << 4) | (clist[k] & 15));
    }
    trows.push_back(t);
    ++rows;
  }
  if (rows > 0) {
    trptr.push_back((int)trows.size());
    teptr.push_back((int)telems.size());
    ++tile;
  }
  int st;
  const int nt = tile;
  if ((st = ovs_ensure((void**)&c->tile_rptr, sizeof(int) * (nt + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->tile_rows, sizeof(int) * (trows.size() + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->tile_eptr, sizeof(int) * (nt + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->tile_elems, sizeof(int) * (telems.size() + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->n2e_loc, sizeof(uint16_t) * EN))) return st;
  if ((st = ovs_ensure((void**)&c->clist_loc, sizeof(uint16_t) * clist_loc.size()))) return st;
  if ((st = ovs_ensure((void**)&c->big_rec, sizeof(int4) * (big.size() + 1)))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->tile_rptr, trptr.data(), sizeof(int) * (nt + 1), cudaMemcpyHostToDevice, s));
  if (!trows.empty())
    OVS_CUDA_TRY(cudaMemcpyAsync(c->tile_rows, trows.data(), sizeof(int) * trows.size(), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->tile_eptr, teptr.data(), sizeof(int) * (nt + 1), cudaMemcpyHostToDevice, s));
  if (!telems.empty())
    OVS_CUDA_TRY(
        cudaMemcpyAsync(c->tile_elems, telems.data(), sizeof(int) * telems.size(), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->n2e_loc, n2e_loc.data(), sizeof(uint16_t) * EN, cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(c->clist_loc, clist_loc.data(), sizeof(uint16_t) * clist_loc.size(),
                               cudaMemcpyHostToDevice, s));
  if (!big.empty())
    OVS_CUDA_TRY(cudaMemcpyAsync(c->big_rec, big.data(), sizeof(int4) * big.size(), cudaMemcpyHostToDevice, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  c->ntiles = nt;
  c->nbig = (int)big.size();
  c->tile_maxe = maxe;
  return OVS_OK;
}

int ovs_pattern_build(ovs_ctx* c) {
  cudaStream_t s = c->stream;
  const int N = c->N, E = c->E, nshl = c->nshl;
  const size_t EN = (size_t)E * nshl;
  int st;
  if ((st = ovs_ensure((void**)&c->n2e_ptr, sizeof(int) * (N + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->n2e, sizeof(int) * EN))) return st;
  if ((st = ovs_ensure((void**)&c->rowptr, sizeof(int) * (N + 1)))) return st;
  if ((st = ovs_ensure((void**)&c->diag, sizeof(int) * N))) return st;
  int *cnt = nullptr, *tmp = nullptr, *stats = nullptr;
  const int nb = (N + 1 + SCAN_T - 1) / SCAN_T;
  const size_t tmp_ints = 4 * (size_t)nb + 64;
  OVS_CUDA_TRY(cudaMallocAsync(&cnt, sizeof(int) * (N + 1), s));
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * tmp_ints, s));
  OVS_CUDA_TRY(cudaMallocAsync(&stats, sizeof(int) * 8, s));
  OVS_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * (N + 1), s));
  OVS_CUDA_TRY(cudaMemsetAsync(stats, 0, sizeof(int) * 8, s));
  // stats: [0] bad node ids, [1] row overflow, [2] max elements per node, [3] max degree
  count_n2e_kernel<<<ovs_grid(EN, 256, 1 << 30), 256, 0, s>>>(c->ien, E, nshl, N, cnt, stats + 0);
  ++c->launches;
  if ((st = exclusive_scan(cnt, c->n2e_ptr, N + 1, tmp, s, &c->launches))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(cnt, c->n2e_ptr, sizeof(int) * N, cudaMemcpyDeviceToDevice, s));
  fill_n2e_kernel<<<ovs_grid(EN, 256, 1 << 30), 256, 0, s>>>(c->ien, E, nshl, N, cnt, c->n2e);
  sort_n2e_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(c->n2e_ptr, c->n2e, N, stats + 2);
  row_len_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(c->ien, nshl, N, c->n2e_ptr, c->n2e,
                                                           cnt, stats + 1, stats + 3);
  c->launches += 3;
  OVS_CUDA_TRY(cudaMemsetAsync(cnt + N, 0, sizeof(int), s));
  if ((st = exclusive_scan(cnt, c->rowptr, N + 1, tmp, s, &c->launches))) return st;
  int h[8];
  OVS_CUDA_TRY(cudaMemcpyAsync(h, stats, sizeof(int) * 8, cudaMemcpyDeviceToHost, s));
  int nnz = 0;
  OVS_CUDA_TRY(cudaMemcpyAsync(&nnz, c->rowptr + N, sizeof(int), cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  if (h[0] != 0) { cudaFreeAsync(cnt, s); cudaFreeAsync(tmp, s); cudaFreeAsync(stats, s); return OVS_ERR_ARG; }
  if (h[1] != 0) { cudaFreeAsync(cnt, s); cudaFreeAsync(tmp, s); cudaFreeAsync(stats, s); return OVS_ERR_PATTERN; }
  c->max_elem = h[2];
  if (c->tmap) { cudaFree(c->tmap); c->tmap = nullptr; }   // transpose map of an earlier pattern
  c->max_deg = h[3];
  c->nnz = nnz;
  if ((st = ovs_ensure((void**)&c->colidx, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)))) return st;
  row_fill_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(c->ien, nshl, N, c->n2e_ptr, c->n2e,
                                                            c->rowptr, c->colidx, c->diag);
  ++c->launches;
  if (nshl == 8) {
    if ((st = ovs_ensure((void**)&c->n2s, 2 * sizeof(unsigned) * (size_t)(EN > 0 ? EN : 1)))) return st;
    slot_map8_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(c->ien, N, c->n2e_ptr, c->n2e, c->rowptr,
                                                               c->colidx, reinterpret_cast<uint2*>(c->n2s));
    ++c->launches;
  }
  if (nshl == 4) {
    if ((st = ovs_ensure((void**)&c->n2s, sizeof(unsigned) * (size_t)(EN > 0 ? EN : 1)))) return st;
    slot_map_kernel<<<ovs_grid(N, 128, 1 << 30), 128, 0, s>>>(c->ien, N, c->n2e_ptr, c->n2e, c->rowptr,
                                                              c->colidx, c->n2s);
    ++c->launches;
  }
  OVS_CUDA_TRY(cudaFreeAsync(cnt, s));
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaFreeAsync(stats, s));
  if ((st = build_row_order(c))) return st;
  if ((st = build_row_rec(c))) return st;
  if ((st = build_contrib(c))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  OVS_CUDA_TRY(cudaGetLastError());
  c->have_pattern = true;
  return OVS_OK;
}
