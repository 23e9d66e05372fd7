// C ABI of the library (include/ovs.h): context, mesh/state transfer,
// reference-layout conversions, Newton update and residual norms.
#include <chrono>
#include <cstdlib>
#include "ovs_internal.cuh"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static thread_local char g_last_error[512] = {0};

void ovs_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", cudaGetErrorName(e), what, file, line);
}

int ovs_ensure(void** p, size_t bytes) {
  if (*p) return OVS_OK;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return OVS_ERR_NOMEM;
  }
  return OVS_OK;
}

int ovs_activate(ovs_ctx* c) {
  OVS_CUDA_TRY(cudaSetDevice(c->device));
  return OVS_OK;
}

namespace {

inline int field_width(int f) { return f <= OVS_F_ACGMOLD ? 3 : 1; }

__global__ void ien_pack_kernel(const int* __restrict__ ien_cm, int E, int nshl, int* __restrict__ out,
                                int* __restrict__ bad) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)E * nshl) return;
  int e = (int)(t / nshl), a = (int)(t % nshl);
  int v = ien_cm[(size_t)a * E + e] - 1;
  out[t] = v;
  // an element must not repeat a node
  for (int b = 0; b < a; ++b)
    if (ien_cm[(size_t)b * E + e] - 1 == v) atomicOr(bad, 1);
}

__global__ void ibc_pack_kernel(const int* __restrict__ ibc, int N, int nibc, uint8_t* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  unsigned m = 0;
  for (int d = 0; d < nibc && d < 8; ++d)
    if (ibc[(size_t)d * N + i] == 1) m |= 1u << d;
  out[i] = (uint8_t)m;
}

// reference block <-> internal slot position (see assemble.cu)
__constant__ int c_pos_k11[9] = {0, 1, 2, 4, 5, 6, 8, 9, 10};
__constant__ int c_pos_g[3] = {3, 7, 11};
__constant__ int c_pos_d[3] = {12, 13, 14};
__constant__ int c_pos_lsu[3] = {16, 17, 18};
__constant__ int c_pos_uls[3] = {20, 21, 22};

__device__ int block_pos(int block, int t) {
  switch (block) {
    case OVS_BLK_K11: return c_pos_k11[t];
    case OVS_BLK_G: return c_pos_g[t];
    case OVS_BLK_D1: return c_pos_d[t];
    case OVS_BLK_M: return 15;
    case OVS_BLK_LS: return 19;
    case OVS_BLK_LSU: return c_pos_lsu[t];
    case OVS_BLK_ULS: return c_pos_uls[t];
    case OVS_BLK_PLS: return 23;
    default: return 0;
  }
}

template <typename T>
__global__ void block_get_kernel(const T* __restrict__ vals, int nv, int block, int w, size_t nnz,
                                 double* __restrict__ out) {
  size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= nnz * w) return;
  size_t k = q / w;
  int t = (int)(q - k * w);
  out[q] = (double)vals[k * nv + block_pos(block, t)];
}

template <typename T>
__global__ void block_set_kernel(T* __restrict__ vals, int nv, int block, int w, size_t nnz,
                                 const double* __restrict__ in) {
  size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= nnz * w) return;
  size_t k = q / w;
  int t = (int)(q - k * w);
  vals[k * nv + block_pos(block, t)] = (T)in[q];
}

__global__ void fill_int_kernel(int* __restrict__ p, size_t n, int v) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

template <typename TS, typename TD>
__global__ void copy_convert_kernel(const TS* __restrict__ a, TD* __restrict__ b, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (TD)a[i];
}

// predictor of a time step (src/driver.f90:83-85): ug = ugold,
// acg = (gami - 1)/gami acgold (pg = pgold is the identity here: the old
// pressure is the pressure left by the previous step)
__global__ void predictor_kernel(size_t n3, double c, const double* __restrict__ ugold, const double* __restrict__ acgold,
                                 double* __restrict__ ug, double* __restrict__ acg) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    ug[i] = ugold[i];
    acg[i] = c * acgold[i];
  }
}

// Newton update, src/solveFlow.f90:99-104,139-140
__global__ void newton_update_kernel(int N, int sys, double gdt, double agdt, const double* __restrict__ sol,
                                     double* acg, double* ug, double* pg, double* rphig, double* phig,
                                     double* rtg, double* tg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (sys == OVS_SYS_TEM) {
    rtg[i] = rtg[i] + sol[i];
    tg[i] = tg[i] + gdt * sol[i];
    return;
  }
  for (int d = 0; d < 3; ++d) {
    size_t k = i + (size_t)N * d;
    acg[k] = acg[k] + sol[k];
    ug[k] = ug[k] + gdt * sol[k];
  }
  pg[i] = pg[i] + agdt * sol[3 * (size_t)N + i];
  if (sys == OVS_SYS_NSVOF) {
    rphig[i] = rphig[i] + sol[4 * (size_t)N + i];
    phig[i] = phig[i] + gdt * sol[4 * (size_t)N + i];
  }
}

int upload_double(ovs_ctx* c, double** dst, const double* host, size_t n) {
  double* d = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&d, sizeof(double) * n, c->stream));
  OVS_CUDA_TRY(cudaMemcpyAsync(d, host, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  *dst = d;
  return OVS_OK;
}

}  // namespace

extern "C" {

int ovs_version(void) { return 10000; }

const char* ovs_status_string(int status) {
  switch (status) {
    case OVS_OK: return "ok";
    case OVS_WARN_NEG_DETJ: return "warning: element with non-positive Jacobian determinant";
    case OVS_ERR_ARG: return "invalid argument";
    case OVS_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA error";
    case OVS_ERR_NOMEM: return "device allocation failed";
    case OVS_ERR_STATE: return "call order: required data not yet provided";
    case OVS_ERR_NONFINITE: return "non-finite value in an assembled residual";
    case OVS_ERR_PATTERN: return "a node has more CSR neighbours than supported";
    case OVS_ERR_NODEVICE: return "no CUDA device";
    case OVS_ERR_TIMEOUT: return "timed out waiting for the device";
    default: return "unknown status";
  }
}

int ovs_params_genalpha(double rhoinf, ovs_params* p) {
  if (!p) return OVS_ERR_ARG;
  if (rhoinf < 0.0 || rhoinf > 1.0) {
    p->almi = 1.0; p->alfi = 1.0; p->gami = 1.0; p->beti = 1.0;
  } else {
    p->almi = (3.0 - rhoinf) / (1.0 + rhoinf) / 2.0;
    p->alfi = 1.0 / (1.0 + rhoinf);
    p->gami = 0.5 + p->almi - p->alfi;
    p->beti = 0.25 * (1.0 + p->almi - p->alfi) * (1.0 + p->almi - p->alfi);
  }
  return OVS_OK;
}

namespace {
// Everything ovs_create allocates; on an error the caller destroys the
// partly built context (ovs_destroy frees whatever is non-null).
int create_resources(ovs_ctx* c, const ovs_dims* dims) {
  OVS_CUDA_TRY(cudaGetDevice(&c->device));
  OVS_CUDA_TRY(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
  {
    const char* e = getenv("OVS_ARNOLDI_FUSED");
    c->arnoldi_fused = e && e[0] == '1';
    const char* h = getenv("OVS_HEX_TC");
    c->hex_tc = h && h[0] == '1';
    const char* rs = getenv("OVS_ROWS_STAGED");
    if (rs) c->rows_staged = rs[0] != '0';
    const char* es = getenv("OVS_ELEM_SMEM");
    if (es) c->elem_smem = es[0] != '0';
    const char* rg = getenv("OVS_ROWS_GATHER");
    if (rg) c->rows_gather = rg[0] != '0';
    const char* mo = getenv("OVS_MIXED_OUTER");
    if (mo && atoi(mo) >= 0 && atoi(mo) <= 200) c->mixed_outer = atoi(mo);
    const char* rt = getenv("OVS_ROWS_TILED");
    if (rt) c->rows_tiled = rt[0] != '0';
    const char* te = getenv("OVS_TILE_ELEMS");
    if (te && atoi(te) >= 4 && atoi(te) <= 4000) c->tile_elems_opt = atoi(te);
  }
  c->N = dims->nnode;
  c->E = dims->nelem;
  c->nshl = dims->nshl;
  OVS_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  OVS_CUDA_TRY(cudaEventCreate(&c->ev0));
  OVS_CUDA_TRY(cudaEventCreate(&c->ev1));
  int st;
  const size_t N = c->N;
  for (int f = 0; f < OVS_F_COUNT; ++f) {
    if ((st = ovs_ensure((void**)&c->field[f], sizeof(double) * N * field_width(f)))) return st;
    OVS_CUDA_TRY(cudaMemsetAsync(c->field[f], 0, sizeof(double) * N * field_width(f), c->stream));
  }
  if ((st = ovs_ensure((void**)&c->ien, sizeof(int) * (size_t)c->E * c->nshl)) ||
      (st = ovs_ensure((void**)&c->elm_id, sizeof(int) * (size_t)c->E)) ||
      (st = ovs_ensure((void**)&c->ibc, N)) ||
      (st = ovs_ensure((void**)&c->gm, sizeof(GmresDev))) ||
      (st = ovs_ensure((void**)&c->flags, sizeof(int) * 4)) ||
      (st = ovs_ensure((void**)&c->cfl_bits, sizeof(unsigned long long))))
    return st;
  OVS_CUDA_TRY(cudaMemsetAsync(c->ibc, 0, N, c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(c->gm, 0, sizeof(GmresDev), c->stream));
  OVS_CUDA_TRY(cudaMallocHost(&c->h_pinned, sizeof(int) * 16));
  OVS_CUDA_TRY(cudaMallocHost(&c->h_pinned_d, sizeof(double) * 16));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}
}  // namespace

int ovs_create(ovs_ctx** out, const ovs_dims* dims) {
  if (!out || !dims) return OVS_ERR_ARG;
  *out = nullptr;
  if (dims->nnode <= 0 || dims->nelem <= 0 || (dims->nshl != 4 && dims->nshl != 8)) return OVS_ERR_ARG;
  if ((long)dims->nelem * dims->nshl >= (1L << 31) || dims->nelem >= (1 << 28)) return OVS_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return OVS_ERR_NODEVICE; }
  if (dims->device >= ndev) return OVS_ERR_ARG;
  if (dims->device >= 0) OVS_CUDA_TRY(cudaSetDevice(dims->device));
  ovs_ctx* c = new ovs_ctx();
  if (dims->device >= 0) c->device = dims->device;
  const int st = create_resources(c, dims);
  if (st) {
    ovs_destroy(c);
    return st;
  }
  *out = c;
  return OVS_OK;
}

int ovs_destroy(ovs_ctx* c) {
  if (!c) return OVS_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  ovs_faces_free(c);
  ovs_bcs_free(c);
  ovs_streaming_free(c);
  if (c->hex_kbuf) cudaFree(c->hex_kbuf);
  if (c->hex_w) cudaFree(c->hex_w);
  void* ptrs[] = {c->ien, c->elm_id, c->ibc, c->rowptr, c->colidx, c->diag, c->n2e_ptr, c->n2e, c->n2s, c->row_order, c->row_rec, c->cptr, c->clist, c->tile_rptr, c->tile_rows,
                  c->tile_eptr, c->tile_elems, c->n2e_loc, c->clist_loc, c->big_rec, c->fg_buf, c->tmap, c->vals_t, c->vjp_cot, c->vjp_ge, c->vjp_grad,
                  c->rec[0], c->rec[1], c->esum[0], c->esum[1], c->gm, c->basis[0], c->basis[1], c->work64, c->work32, c->wvec, c->coop_part,
                  c->flags, c->cfl_bits};
  for (void* p : ptrs) if (p) cudaFree(p);
  for (int f = 0; f < OVS_F_COUNT; ++f) if (c->field[f]) cudaFree(c->field[f]);
  for (int s = 0; s < 4; ++s) {
    if (c->sol[s]) cudaFree(c->sol[s]);
    for (int p = 0; p < 2; ++p) {
      SysStore& S = c->sys[s][p];
      if (S.vals) cudaFree(S.vals);
      if (S.rhs) cudaFree(S.rhs);
      if (S.binv) cudaFree(S.binv);
    }
  }
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->h_pinned_d) cudaFreeHost(c->h_pinned_d);
  if (c->h_async_flags) cudaFreeHost(c->h_async_flags);
  if (c->h_async_cfl) cudaFreeHost(c->h_async_cfl);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  cudaGetLastError();
  delete c;
  return OVS_OK;
}

int ovs_synchronize(ovs_ctx* c) {
  if (!c) return OVS_ERR_ARG;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_get_stream(ovs_ctx* c, void** stream) {
  if (!c || !stream) return OVS_ERR_ARG;
  *stream = (void*)c->stream;
  return OVS_OK;
}

int ovs_upload_mesh(ovs_ctx* c, const double* xg, const int* ien, const int* elm_id) {
  if (!c || !ien) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  cudaStream_t s = c->stream;
  const size_t EN = (size_t)c->E * c->nshl;
  if (xg) OVS_CUDA_TRY(cudaMemcpyAsync(c->field[OVS_F_XG], xg, sizeof(double) * 3 * (size_t)c->N, cudaMemcpyHostToDevice, s));
  int *tmp = nullptr, *bad = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * EN, s));
  OVS_CUDA_TRY(cudaMallocAsync(&bad, sizeof(int), s));
  OVS_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
  OVS_CUDA_TRY(cudaMemcpyAsync(tmp, ien, sizeof(int) * EN, cudaMemcpyHostToDevice, s));
  ien_pack_kernel<<<ovs_grid(EN, 256, 1 << 30), 256, 0, s>>>(tmp, c->E, c->nshl, c->ien, bad);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  if (elm_id) {
    OVS_CUDA_TRY(cudaMemcpyAsync(c->elm_id, elm_id, sizeof(int) * (size_t)c->E, cudaMemcpyHostToDevice, s));
  } else {
    fill_int_kernel<<<ovs_grid(c->E, 256, 1 << 30), 256, 0, s>>>(c->elm_id, (size_t)c->E, 102);
    ++c->launches;
  }
  int hbad = 0;
  OVS_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaFreeAsync(bad, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  if (hbad) return OVS_ERR_ARG;
  c->have_mesh = true;
  c->have_pattern = false;
  return OVS_OK;
}


int ovs_build_pattern(ovs_ctx* c, int* icnt) {
  if (!c) return OVS_ERR_ARG;
  if (!c->have_mesh) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ovs_pattern_build(c))) return st;
  if (icnt) *icnt = c->nnz;
  return OVS_OK;
}

int ovs_get_pattern(ovs_ctx* c, int* col, int* row) {
  if (!c || !col) return OVS_ERR_ARG;
  if (!c->have_pattern) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  return ovs_pattern_to_host(c, col, row);
}

int ovs_get_slot_map(ovs_ctx* c, int* lmap) {
  if (!c || !lmap) return OVS_ERR_ARG;
  if (!c->have_pattern || !c->n2s) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  return ovs_slot_map_to_host(c, lmap);
}

int ovs_gen_spar_struc(int nnode, int nelem, int nshl, const int* ien, int* col, int* row, int* icnt) {
  if (!ien || !col || !icnt) return OVS_ERR_ARG;
  ovs_dims d = {nnode, nelem, nshl, 0};
  ovs_ctx* c = nullptr;
  int st = ovs_create(&c, &d);
  if (st) return st;
  if ((st = ovs_upload_mesh(c, nullptr, ien, nullptr)) || (st = ovs_build_pattern(c, nullptr))) {
    ovs_destroy(c);
    return st;
  }
  if (row && *icnt < c->nnz) { *icnt = c->nnz; ovs_destroy(c); return OVS_ERR_ARG; }
  *icnt = c->nnz;
  st = ovs_pattern_to_host(c, col, row);
  ovs_destroy(c);
  return st;
}

int ovs_set_params(ovs_ctx* c, const ovs_params* p) {
  if (!c || !p) return OVS_ERR_ARG;
  if (!(p->delt > 0.0)) return OVS_ERR_ARG;
  c->params = *p;
  c->have_params = true;
  return OVS_OK;
}

int ovs_set_ibc(ovs_ctx* c, const int* ibc, int nibc) {
  if (!c || !ibc || nibc < 1) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  cudaStream_t s = c->stream;
  int* tmp = nullptr;
  const size_t n = (size_t)c->N * nibc;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * n, s));
  OVS_CUDA_TRY(cudaMemcpyAsync(tmp, ibc, sizeof(int) * n, cudaMemcpyHostToDevice, s));
  ibc_pack_kernel<<<ovs_grid(c->N, 256, 1 << 30), 256, 0, s>>>(tmp, c->N, nibc, c->ibc);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  return OVS_OK;
}

int ovs_set_option(ovs_ctx* c, int option, int value) {
  if (!c) return OVS_ERR_ARG;
  switch (option) {
    case OVS_OPT_HEX_TC: c->hex_tc = value != 0; return OVS_OK;
    case OVS_OPT_ROWS_STAGED: c->rows_staged = value != 0; return OVS_OK;
    case OVS_OPT_ELEM_SMEM: c->elem_smem = value < 0 ? -1 : (value != 0); return OVS_OK;
    case OVS_OPT_ROWS_GATHER: c->rows_gather = value != 0; return OVS_OK;
    case OVS_OPT_ROWS_TILED: c->rows_tiled = value != 0; return OVS_OK;
    case OVS_OPT_MIXED_OUTER:
      if (value < 0 || value > 200) return OVS_ERR_ARG;
      c->mixed_outer = value;
      return OVS_OK;
    case OVS_OPT_TILE_ELEMS:
      if (value < 4 || value > 4000) return OVS_ERR_ARG;
      c->tile_elems_opt = value;
      return OVS_OK;
    case OVS_OPT_ARNOLDI_FUSED: c->arnoldi_fused = value != 0; return OVS_OK;
    default: return OVS_ERR_ARG;
  }
}

int ovs_set_faces(ovs_ctx* c, int nface, const int* f2e, const int* face_or, const int* flags,
                  const double* hconv, const double* tinf) {
  if (!c) return OVS_ERR_ARG;
  return ovs_faces_set_impl(c, nface, f2e, face_or, flags, hconv, tinf);
}

int ovs_set_field(ovs_ctx* c, int field, const double* host) {
  if (!c || !host || field < 0 || field >= OVS_F_COUNT) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->field[field], host, sizeof(double) * (size_t)c->N * field_width(field),
                               cudaMemcpyHostToDevice, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_get_field(ovs_ctx* c, int field, double* host) {
  if (!c || !host || field < 0 || field >= OVS_F_COUNT) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(host, c->field[field], sizeof(double) * (size_t)c->N * field_width(field),
                               cudaMemcpyDeviceToHost, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_assemble(ovs_ctx* c, int kernel, int tensor_flag, int precision, double* cfl) {
  if (!c) return OVS_ERR_ARG;
  if ((tensor_flag & (OVS_TENSOR_VEC | OVS_TENSOR_MAT)) == 0) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  st = ovs_assemble_impl(c, kernel, tensor_flag, precision, cfl);
  if (st < 0) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  return st;
}

int ovs_assemble_async(ovs_ctx* c, int kernel, int tensor_flag, int precision) {
  if (!c) return OVS_ERR_ARG;
  if ((tensor_flag & (OVS_TENSOR_VEC | OVS_TENSOR_MAT)) == 0) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if (c->async_n >= OVS_ASYNC_SLOTS) return OVS_ERR_STATE;   // ovs_assemble_wait first
  if (!c->h_async_flags) {
    OVS_CUDA_TRY(cudaMallocHost(&c->h_async_flags, sizeof(int) * 4 * OVS_ASYNC_SLOTS));
    OVS_CUDA_TRY(cudaMallocHost(&c->h_async_cfl, sizeof(unsigned long long) * OVS_ASYNC_SLOTS));
  }
  c->defer_status = true;
  st = ovs_assemble_impl(c, kernel, tensor_flag, precision, nullptr);
  c->defer_status = false;
  return st;
}

int ovs_assemble_wait(ovs_ctx* c, double* cfl) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  int err = OVS_OK, warn = OVS_OK;
  double mx = 0.0;
  for (int k = 0; k < c->async_n; ++k) {   // the status ovs_assemble would have returned, per pass
    const int* f = c->h_async_flags + 4 * k;
    const int s1 = f[3] ? OVS_ERR_PATTERN : f[2] ? OVS_ERR_TIMEOUT : f[1] ? OVS_ERR_NONFINITE : OVS_OK;
    if (s1 && !err) err = s1;
    if (f[0]) warn = OVS_WARN_NEG_DETJ;
    double v;
    memcpy(&v, c->h_async_cfl + k, sizeof(v));
    if (v > mx) mx = v;
  }
  c->async_n = 0;
  if (cfl) *cfl = mx;
  return err ? err : warn;
}

static int sys_ok(ovs_ctx* c, int sys, int prec) {
  if (!c) return 0;
  if (sys != OVS_SYS_NS && sys != OVS_SYS_NSVOF && sys != OVS_SYS_TEM) return 0;
  if (prec != OVS_FP64 && prec != OVS_FP32) return 0;
  return 1;
}

int ovs_get_rhs(ovs_ctx* c, int sys, int prec, double* rhs) {
  if (!sys_ok(c, sys, prec) || !rhs) return OVS_ERR_ARG;
  SysStore& S = c->sys[sys][prec];
  if (!S.rhs) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  if (prec == OVS_FP64) {
    OVS_CUDA_TRY(cudaMemcpyAsync(rhs, S.rhs, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  } else {
    // through the context's FP64 read-back buffer of this system (no
    // allocation per call), after any asynchronous read-back still using it
    if ((st = ovs_ensure((void**)&c->rhs_out[sys], sizeof(double) * n))) return st;
    if (c->ev_rhs_out[sys]) OVS_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_rhs_out[sys], 0));
    double* tmp = c->rhs_out[sys];
    copy_convert_kernel<float, double><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>((const float*)S.rhs, tmp, n);
    ++c->launches;
    OVS_CUDA_TRY(cudaMemcpyAsync(rhs, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  }
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_set_rhs(ovs_ctx* c, int sys, int prec, const double* rhs) {
  if (!sys_ok(c, sys, prec) || !rhs) return OVS_ERR_ARG;
  SysStore& S = c->sys[sys][prec];
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  const size_t ts = prec == OVS_FP64 ? 8 : 4;
  if ((st = ovs_ensure(&S.rhs, ts * n))) return st;
  double* tmp = nullptr;
  if ((st = upload_double(c, &tmp, rhs, n))) return st;
  if (prec == OVS_FP64)
    {
      copy_convert_kernel<double, double><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>(tmp, (double*)S.rhs, n);
      ++c->launches;
    }
  else
    {
      copy_convert_kernel<double, float><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>(tmp, (float*)S.rhs, n);
      ++c->launches;
    }
  OVS_CUDA_TRY(cudaFreeAsync(tmp, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  S.have_rhs = true;
  return OVS_OK;
}

static int block_width(int sys, int block) {
  if (sys == OVS_SYS_TEM) return block == OVS_BLK_TEM ? 1 : 0;
  switch (block) {
    case OVS_BLK_K11: return 9;
    case OVS_BLK_G: case OVS_BLK_D1: return 3;
    case OVS_BLK_M: return 1;
    case OVS_BLK_LS: case OVS_BLK_PLS: return sys == OVS_SYS_NSVOF ? 1 : 0;
    case OVS_BLK_LSU: case OVS_BLK_ULS: return sys == OVS_SYS_NSVOF ? 3 : 0;
    default: return 0;
  }
}

int ovs_get_lhs_block(ovs_ctx* c, int sys, int prec, int block, double* out) {
  if (!sys_ok(c, sys, prec) || !out) return OVS_ERR_ARG;
  const int w = block_width(sys, block);
  if (!w) return OVS_ERR_ARG;
  SysStore& S = c->sys[sys][prec];
  if (!S.vals) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->nnz * w;
  double* tmp = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(double) * (n ? n : 1), c->stream));
  const int nv = ovs_sys_nv(sys);
  const int bl = sys == OVS_SYS_TEM ? -1 : block;
  if (prec == OVS_FP64)
    {
      block_get_kernel<double><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>((const double*)S.vals, nv, bl, w, c->nnz, tmp);
      ++c->launches;
    }
  else
    {
      block_get_kernel<float><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>((const float*)S.vals, nv, bl, w, c->nnz, tmp);
      ++c->launches;
    }
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaMemcpyAsync(out, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  OVS_CUDA_TRY(cudaFreeAsync(tmp, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_set_lhs_block(ovs_ctx* c, int sys, int prec, int block, const double* in) {
  if (!sys_ok(c, sys, prec) || !in) return OVS_ERR_ARG;
  if (!c->have_pattern) return OVS_ERR_STATE;
  const int w = block_width(sys, block);
  if (!w) return OVS_ERR_ARG;
  SysStore& S = c->sys[sys][prec];
  int st;
  if ((st = ovs_activate(c))) return st;
  const int nv = ovs_sys_nv(sys);
  const size_t ts = prec == OVS_FP64 ? 8 : 4;
  if (!S.vals) {
    if ((st = ovs_ensure(&S.vals, ts * (size_t)c->nnz * nv))) return st;
    OVS_CUDA_TRY(cudaMemsetAsync(S.vals, 0, ts * (size_t)c->nnz * nv, c->stream));
  }
  const size_t n = (size_t)c->nnz * w;
  double* tmp = nullptr;
  if ((st = upload_double(c, &tmp, in, n))) return st;
  const int bl = sys == OVS_SYS_TEM ? -1 : block;
  if (prec == OVS_FP64)
    {
      block_set_kernel<double><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>((double*)S.vals, nv, bl, w, c->nnz, tmp);
      ++c->launches;
    }
  else
    {
      block_set_kernel<float><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>((float*)S.vals, nv, bl, w, c->nnz, tmp);
      ++c->launches;
    }
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaFreeAsync(tmp, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  S.have_mat = true;
  return OVS_OK;
}

int ovs_spmv(ovs_ctx* c, int sys, int prec, const double* x, double* y) {
  if (!sys_ok(c, sys, prec) || !x || !y) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  double *dx = nullptr, *dy = nullptr;
  if ((st = upload_double(c, &dx, x, n))) return st;
  OVS_CUDA_TRY(cudaMallocAsync(&dy, sizeof(double) * n, c->stream));
  st = ovs_spmv_impl(c, sys, prec, dx, dy);
  if (!st) OVS_CUDA_TRY(cudaMemcpyAsync(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  cudaFreeAsync(dx, c->stream);
  cudaFreeAsync(dy, c->stream);
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return st;
}

int ovs_build_precond(ovs_ctx* c, int sys, int prec) {
  if (!sys_ok(c, sys, prec)) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ovs_precond_setup(c, sys, prec))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_spmv_device(ovs_ctx* c, int sys, int prec, int flags, const double* dx, double* dy) {
  if (!sys_ok(c, sys, prec) || !dx || !dy || (flags & ~OVS_SPMV_PRECOND)) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  st = (flags & OVS_SPMV_PRECOND) ? ovs_spmv_pre_impl(c, sys, prec, dx, dy) : ovs_spmv_impl(c, sys, prec, dx, dy);
  if (st) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_spmv_device_rows(ovs_ctx* c, int sys, int prec, int flags, const double* dx, double* dy,
                         const int* drows, int nrows) {
  if (!sys_ok(c, sys, prec) || !dx || !dy || (flags & ~OVS_SPMV_PRECOND) || nrows < 0 || (nrows > 0 && !drows))
    return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ovs_spmv_rows_impl(c, sys, prec, (flags & OVS_SPMV_PRECOND) != 0, dx, dy, drows, nrows))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_precond_device(ovs_ctx* c, int sys, int prec, const double* dx, double* dy) {
  if (!sys_ok(c, sys, prec) || !dx || !dy) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ovs_precond_apply_impl(c, sys, prec, dx, dy))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_gmres(ovs_ctx* c, int sys, double tol, int kspace, int kspace_min, double* sol, ovs_gmres_info* info) {
  if (!sys_ok(c, sys, OVS_FP64) || !sol) return OVS_ERR_ARG;
  if (kspace < 1 || kspace > OVS_MAX_KSPACE) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  if ((st = ovs_ensure((void**)&c->sol[sys], sizeof(double) * 5 * (size_t)c->N))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->sol[sys], sol, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  ovs_gmres_info gi;
  memset(&gi, 0, sizeof(gi));
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  st = ovs_gmres_ref_impl(c, sys, tol, kspace, kspace_min, c->sol[sys], &gi);
  if (st) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  {
    float ms = 0.f;
    OVS_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
  }
  OVS_CUDA_TRY(cudaMemcpyAsync(sol, c->sol[sys], sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (info) *info = gi;
  return OVS_OK;
}

int ovs_solve(ovs_ctx* c, int sys, int mode, double rtol, int kspace, int max_cycles, double* sol,
              ovs_solve_info* info) {
  if (mode != OVS_FP64 && mode != OVS_FP32 && mode != OVS_MIXED) return OVS_ERR_ARG;
  if (!sys_ok(c, sys, mode == OVS_FP32 ? OVS_FP32 : OVS_FP64)) return OVS_ERR_ARG;
  if (kspace < 1 || kspace > OVS_MAX_KSPACE || max_cycles < 1 || !(rtol > 0.0)) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  ovs_solve_info si;
  memset(&si, 0, sizeof(si));
  if ((st = ovs_solve_impl(c, sys, mode, rtol, kspace, max_cycles, &si))) return st;
  c->last_ms = si.seconds * 1e3;
  if (sol) {
    const size_t n = (size_t)c->N * ovs_sys_nf(sys);
    OVS_CUDA_TRY(cudaMemcpyAsync(sol, c->sol[sys], sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  if (info) *info = si;
  return OVS_OK;
}

int ovs_round_matrix(ovs_ctx* c, int sys) {
  if (!sys_ok(c, sys, OVS_FP64)) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c)) || (st = ovs_round_impl(c, sys))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_newton_update(ovs_ctx* c, int sys) {
  if (!sys_ok(c, sys, OVS_FP64)) return OVS_ERR_ARG;
  if (!c->sol[sys] || !c->have_params) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  const ovs_params& p = c->params;
  newton_update_kernel<<<ovs_grid(c->N, 256, 1 << 30), 256, 0, c->stream>>>(
      c->N, sys, p.gami * p.delt, p.alfi * p.gami * p.delt, c->sol[sys], c->field[OVS_F_ACG], c->field[OVS_F_UG],
      c->field[OVS_F_PG], c->field[OVS_F_RPHIG], c->field[OVS_F_PHIG], c->field[OVS_F_RTG], c->field[OVS_F_TG]);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_set_solution(ovs_ctx* c, int sys, const double* sol) {
  if (!sys_ok(c, sys, OVS_FP64) || !sol) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  if ((st = ovs_ensure((void**)&c->sol[sys], sizeof(double) * 5 * (size_t)c->N))) return st;
  // host or device source: the unified address space tells them apart
  OVS_CUDA_TRY(cudaMemcpyAsync(c->sol[sys], sol, sizeof(double) * n, cudaMemcpyDefault, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_residual_norms(ovs_ctx* c, int prec, double r[4]) {
  if (!c || !r || (prec != OVS_FP64 && prec != OVS_FP32)) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  r[0] = r[1] = r[2] = r[3] = 0.0;
  const size_t N = c->N;
  // momentum/continuity/VOF from the NS+VOF system if assembled, else NS
  int fs = c->sys[OVS_SYS_NSVOF][prec].rhs ? OVS_SYS_NSVOF : (c->sys[OVS_SYS_NS][prec].rhs ? OVS_SYS_NS : 0);
  double* tmp = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(double) * 5 * N, c->stream));
  auto sumsq = [&](int sys, int f0, int nf, double* out) -> int {
    const size_t n = N * nf;
    if (prec == OVS_FP64)
      {
        copy_convert_kernel<double, double><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>(
            (const double*)c->sys[sys][prec].rhs + N * f0, tmp, n);
        ++c->launches;
      }
    else
      {
        copy_convert_kernel<float, double><<<ovs_grid(n, 256, 1 << 30), 256, 0, c->stream>>>(
            (const float*)c->sys[sys][prec].rhs + N * f0, tmp, n);
        ++c->launches;
      }
    return ovs_dot_impl(c, tmp, tmp, n, out);
  };
  if (fs) {
    if ((st = sumsq(fs, 0, 3, &r[0]))) return st;
    if ((st = sumsq(fs, 3, 1, &r[1]))) return st;
    if (fs == OVS_SYS_NSVOF && (st = sumsq(fs, 4, 1, &r[2]))) return st;
  }
  if (c->sys[OVS_SYS_TEM][prec].rhs && (st = sumsq(OVS_SYS_TEM, 0, 1, &r[3]))) return st;
  OVS_CUDA_TRY(cudaFreeAsync(tmp, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_profile(ovs_ctx* c, int what, int system, int precision, int reps, double* avg_ms) {
  if (!c || !avg_ms || reps < 1 || (precision != OVS_FP64 && precision != OVS_FP32)) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if (what == OVS_PROF_ASSEMBLE) return ovs_profile_assemble(c, system, precision, reps, avg_ms, 3);
  if (what == OVS_PROF_ASSEMBLE_ELEMENTS) return ovs_profile_assemble(c, system, precision, reps, avg_ms, 1);
  if (what == OVS_PROF_ASSEMBLE_ROWS) return ovs_profile_assemble(c, system, precision, reps, avg_ms, 2);
  if (what != OVS_PROF_SPMV && what != OVS_PROF_ARNOLDI && what != OVS_PROF_ARNOLDI_FUSED) return OVS_ERR_ARG;
  if (!sys_ok(c, system, precision)) return OVS_ERR_ARG;
  return ovs_profile_krylov(c, what, system, precision, reps, avg_ms);
}

// FMA throughput of the device in T (float or double): 8 independent chains
// per thread, 4 blocks of 256 threads per SM; the compute-side roofline
// denominators of the assembly kernels (their work is FP32 or FP64
// arithmetic on the CUDA cores).
extern "C++" {
template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T* out, int iters, T seed) {
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + (T)1e-7 * (T)threadIdx.x + (T)k;
  const T m = (T)1.0000001, b = (T)1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, b);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

template <typename T>
static int measure_fma_peak(ovs_ctx* c, int iters, double* tflops) {
  int st;
  if ((st = ovs_activate(c))) return st;
  const int blocks = 4 * c->num_sms;
  T* out = nullptr;
  OVS_CUDA_TRY(cudaMallocAsync(&out, sizeof(T) * blocks, c->stream));
  for (int w = 0; w < 3; ++w) fma_peak_kernel<T><<<blocks, 256, 0, c->stream>>>(out, iters, (T)1);
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  const int reps = 10;
  for (int r = 0; r < reps; ++r) fma_peak_kernel<T><<<blocks, 256, 0, c->stream>>>(out, iters, (T)1);
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  c->launches += 3 + reps;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  OVS_CUDA_TRY(cudaFreeAsync(out, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const double flops = 2.0 * 8.0 * iters * 256.0 * blocks * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return OVS_OK;
}
}  // extern "C++"

int ovs_measure_fp32_peak(ovs_ctx* c, double* tflops) {
  if (!c || !tflops) return OVS_ERR_ARG;
  return measure_fma_peak<float>(c, 1 << 14, tflops);
}

int ovs_measure_fp64_peak(ovs_ctx* c, double* tflops) {
  if (!c || !tflops) return OVS_ERR_ARG;
  return measure_fma_peak<double>(c, 1 << 13, tflops);
}

int ovs_launch_count(ovs_ctx* c, long long* n) {
  if (!c || !n) return OVS_ERR_ARG;
  *n = c->launches;
  return OVS_OK;
}

int ovs_last_device_ms(ovs_ctx* c, double* ms) {
  if (!c || !ms) return OVS_ERR_ARG;
  *ms = c->last_ms;
  return OVS_OK;
}

int ovs_host_alloc(void** p, size_t bytes) {
  if (!p) return OVS_ERR_ARG;
  OVS_CUDA_TRY(cudaMallocHost(p, bytes ? bytes : 16));
  return OVS_OK;
}

int ovs_host_free(void* p) {
  if (p) OVS_CUDA_TRY(cudaFreeHost(p));
  return OVS_OK;
}


int ovs_residual_vjp(ovs_ctx* c, int kernel, const double* cot, double* grad) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  if ((st = ovs_residual_vjp_impl(c, kernel, cot, grad))) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  return OVS_OK;
}

int ovs_gmres_transposed(ovs_ctx* c, int sys, const double* rhs, double tol, int kspace, int kspace_min,
                         double* sol, ovs_gmres_info* info) {
  if (!c || sys != OVS_SYS_TEM || !rhs || !sol) return OVS_ERR_ARG;
  if (!sys_ok(c, sys, OVS_FP64)) return OVS_ERR_ARG;
  if (kspace < 1 || kspace > OVS_MAX_KSPACE) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  const size_t n = (size_t)c->N;
  if ((st = ovs_ensure((void**)&c->sol[sys], sizeof(double) * 5 * n))) return st;
  if ((st = ovs_ensure((void**)&c->work64, sizeof(double) * 15 * n))) return st;
  OVS_CUDA_TRY(cudaMemcpyAsync(c->work64, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  OVS_CUDA_TRY(cudaMemsetAsync(c->sol[sys], 0, sizeof(double) * n, c->stream));
  ovs_gmres_info gi;
  memset(&gi, 0, sizeof(gi));
  OVS_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  if ((st = ovs_gmres_transposed_impl(c, sys, c->work64, tol, kspace, kspace_min, c->sol[sys], &gi))) return st;
  OVS_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  OVS_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  OVS_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  OVS_CUDA_TRY(cudaMemcpyAsync(sol, c->sol[sys], sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (info) *info = gi;
  return OVS_OK;
}


// solmultiphasethermofluid_stag (src/solveFlow.f90:4-164) on the context
int ovs_quench_newton(ovs_ctx* c, const ovs_newton_opts* o, ovs_newton_info* info) {
  if (!c || !o || (o->mode != OVS_FP64 && o->mode != OVS_FP32 && o->mode != OVS_MIXED) || o->newton_max < 0)
    return OVS_ERR_ARG;
  if (o->kspace < 1 || o->kspace > OVS_MAX_KSPACE || o->max_cycles < 1) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  const auto t0 = std::chrono::steady_clock::now();
  const int prec = o->mode == OVS_FP32 ? OVS_FP32 : OVS_FP64;   // assembly and residual precision
  ovs_newton_info ni;
  memset(&ni, 0, sizeof(ni));
  auto check = [&](const double* r) {   // check_convergence, all three field groups
    int all = 1;
    for (int k = 0; k < 4; ++k) {
      ni.field_converged[k] = (r[k] < o->utol[k] * ni.residual0[k]) || (r[k] < o->atol[k]);
      all &= ni.field_converged[k];
    }
    return all;
  };
  auto solve = [&](int sys, double tol, int* its) -> int {
    const size_t n = (size_t)c->N * ovs_sys_nf(sys);
    int s2;
    if (o->mode == OVS_FP64) {
      if ((s2 = ovs_ensure((void**)&c->sol[sys], sizeof(double) * 5 * (size_t)c->N))) return s2;
      OVS_CUDA_TRY(cudaMemsetAsync(c->sol[sys], 0, sizeof(double) * n, c->stream));
      ovs_gmres_info gi;
      memset(&gi, 0, sizeof(gi));
      if ((s2 = ovs_gmres_ref_impl(c, sys, tol, o->kspace, o->kspace_min, c->sol[sys], &gi))) return s2;
      *its += gi.iterations;
    } else {
      ovs_solve_info si;
      memset(&si, 0, sizeof(si));
      if ((s2 = ovs_solve_impl(c, sys, o->mode, tol, o->kspace, o->max_cycles, &si))) return s2;
      *its += si.iterations;
    }
    return ovs_newton_update(c, sys);
  };
  const int vec = OVS_TENSOR_VEC, both = OVS_TENSOR_MAT | OVS_TENSOR_VEC;
  auto vec_all = [&]() -> int {
    int s2;
    if ((s2 = ovs_assemble_impl(c, OVS_ASM_NSVOF, vec, prec, nullptr)) < 0) return s2;
    if ((s2 = ovs_assemble_impl(c, OVS_ASM_TEM, vec, prec, nullptr)) < 0) return s2;
    return OVS_OK;
  };
  // setBCs_NSVOF + setBCs_Tem before the first residual and at the top of
  // every Newton iteration (src/solveFlow.f90:35-36, :58-60), when registered
  auto bcs = [&]() -> int { return c->have_bcs ? ovs_apply_bcs_impl(c, 3) : OVS_OK; };
  if ((st = bcs())) return st;
  if ((st = vec_all())) return st;
  if ((st = ovs_residual_norms(c, prec, ni.residual0))) return st;
  memcpy(ni.residual, ni.residual0, sizeof(ni.residual));
  ni.converged = check(ni.residual);
  for (int it = 1; it <= o->newton_max; ++it) {
    if ((st = bcs())) return st;
    if ((st = ovs_assemble_impl(c, OVS_ASM_NSVOF, both, prec, nullptr)) < 0) return st;
    if ((st = solve(OVS_SYS_NSVOF, o->tol_ns, &ni.krylov_iterations_ns))) return st;
    if (o->solve_tem) {
      if ((st = ovs_assemble_impl(c, OVS_ASM_TEM, both, prec, nullptr)) < 0) return st;
      if ((st = solve(OVS_SYS_TEM, o->tol_tem, &ni.krylov_iterations_tem))) return st;
    }
    if ((st = vec_all())) return st;
    if ((st = ovs_residual_norms(c, prec, ni.residual))) return st;
    ni.iterations = it;
    ni.converged = check(ni.residual);
    if (ni.converged) break;
  }
  ni.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (info) *info = ni;
  return OVS_OK;
}


// The time loop of the reference driver around solmultiphasethermofluid_stag
// (src/driver.f90:70-100): predictor, the Newton loop (one Newton iteration
// and no temperature solve while istep <= 1 / istep == 0, solveFlow.f90:50-54,
// :109), then the old values the driver updates (:95-100: ug, acg, dg, ugm,
// acgm; pg is its own old value here).  The driver does not update phigold,
// rphigold, Tgold, rTgold; update_vof_tem_old = 1 updates them too.
// The driver's predictor (src/driver.f90:83-85; pg = pgold is the identity
// here, as pgold = pg closes every step): ug = ugold,
// acg = (gami - 1)/gami acgold, on the context stream.
static int launch_predictor(ovs_ctx* c) {
  const size_t N = c->N;
  const double gami = c->params.gami;
  predictor_kernel<<<ovs_grid(3 * N, 256, 1 << 30), 256, 0, c->stream>>>(
      3 * N, (gami - 1.0) / gami, c->field[OVS_F_UGOLD], c->field[OVS_F_ACGOLD], c->field[OVS_F_UG], c->field[OVS_F_ACG]);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}

// The old values the driver updates after a step (src/driver.f90:98-103),
// queued on the context stream; update_vof_tem_old also copies phig, rphig,
// Tg and rTg, which the driver leaves alone.
static int copy_old_values(ovs_ctx* c, int update_vof_tem_old) {
  const size_t N = c->N;
  const int pairs3[][2] = {{OVS_F_UG, OVS_F_UGOLD}, {OVS_F_ACG, OVS_F_ACGOLD}, {OVS_F_DG, OVS_F_DGOLD},
                           {OVS_F_UGM, OVS_F_UGMOLD}, {OVS_F_ACGM, OVS_F_ACGMOLD}};
  for (auto& pr : pairs3)
    OVS_CUDA_TRY(cudaMemcpyAsync(c->field[pr[1]], c->field[pr[0]], sizeof(double) * 3 * N,
                                 cudaMemcpyDeviceToDevice, c->stream));
  if (update_vof_tem_old) {
    const int pairs1[][2] = {{OVS_F_PHIG, OVS_F_PHIGOLD}, {OVS_F_RPHIG, OVS_F_RPHIGOLD}, {OVS_F_TG, OVS_F_TGOLD},
                             {OVS_F_RTG, OVS_F_RTGOLD}};
    for (auto& pr : pairs1)
      OVS_CUDA_TRY(cudaMemcpyAsync(c->field[pr[1]], c->field[pr[0]], sizeof(double) * N,
                                   cudaMemcpyDeviceToDevice, c->stream));
  }
  return OVS_OK;
}

int ovs_predictor(ovs_ctx* c) {
  if (!c) return OVS_ERR_ARG;
  if (!c->have_params) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c)) || (st = launch_predictor(c))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_commit_old(ovs_ctx* c, int update_vof_tem_old) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c)) || (st = copy_old_values(c, update_vof_tem_old))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_quench_time_steps(ovs_ctx* c, int first_step, int nsteps, const ovs_newton_opts* o,
                          int update_vof_tem_old, ovs_newton_info* last, int* krylov_total) {
  if (!c || !o || nsteps < 0) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  int kt = 0;
  for (int s = 0; s < nsteps; ++s) {
    const int istep = first_step + s;
    if ((st = launch_predictor(c))) return st;
    ovs_newton_opts os = *o;
    if (istep <= 1) os.newton_max = 1;
    os.solve_tem = o->solve_tem && istep > 0;
    ovs_newton_info ni;
    if ((st = ovs_quench_newton(c, &os, &ni))) return st;
    kt += ni.krylov_iterations_ns + ni.krylov_iterations_tem;
    if ((st = copy_old_values(c, update_vof_tem_old))) return st;
    OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (last) *last = ni;
  }
  if (krylov_total) *krylov_total = kt;
  return OVS_OK;
}

}  // extern "C"
