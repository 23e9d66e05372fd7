// Boundary-condition producers of the quench Newton routine on the device:
// setBCs_NSVOF (src/setBCs.f90:172-244) and setBCs_Tem (:248-278).
//
// The reference reads the *Type tables by FACE_ID and the *Valu tables by
// boundary number (src/setBCs.f90:212-216, :230-234, :266-268); both are
// kept.  Boundaries are applied in order, one launch each, so a node shared
// by two boundaries (an edge of the box) ends with the later boundary's
// values, as in the reference's loop.  The acceleration-like updates
//   acg = ((ug - ugold) Dtgl + (gami - 1) acgold) / gami
// use explicitly rounded operations so they match a plain sequential
// evaluation bit for bit.
#include "ovs_internal.cuh"

#include <algorithm>
#include <vector>

namespace {

constexpr uint8_t PHIB = 16, TB = 32;

__global__ void bc_reset_kernel(int N, const uint8_t* __restrict__ n101, uint8_t* __restrict__ ibc, int which) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (which & 1) ibc[i] = (n101 && n101[i]) ? (uint8_t)0x1F : (uint8_t)0;   // IBC = 0; NodeID 101: IBC(1:5) = 1
  else ibc[i] = (uint8_t)(ibc[i] & ~TB);                                     // IBC(:, 6) = 0
}

__device__ inline double rate(double v, double vold, double rold, double dtgl, double gami) {
  const double a = __dmul_rn(__dsub_rn(v, vold), dtgl);
  const double b = __dmul_rn(__dsub_rn(gami, 1.0), rold);
  return __ddiv_rn(__dadd_rn(a, b), gami);
}

struct BcArgs {
  BcBound b;
  const int* nodes;
  double* f[OVS_F_COUNT];
  uint8_t* ibc;
  int N, which;
  double dtgl, gami;
};

__global__ void bc_apply_kernel(const BcArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.b.n) return;
  const int k = a.nodes[a.b.off + j];
  const size_t N = a.N;
  uint8_t m = a.ibc[k];
  if (a.which & 1) {
    for (int d = 0; d < 3; ++d)
      if (a.b.ut[d] == 1) {
        const size_t i = k + N * d;
        m |= (uint8_t)(1u << d);
        a.f[OVS_F_UG][i] = a.b.uv[d];
        a.f[OVS_F_ACG][i] = rate(a.b.uv[d], a.f[OVS_F_UGOLD][i], a.f[OVS_F_ACGOLD][i], a.dtgl, a.gami);
      }
    if (a.b.pt == 1) {
      m |= PHIB;
      a.f[OVS_F_PHIG][k] = a.b.pv;
      a.f[OVS_F_RPHIG][k] = rate(a.b.pv, a.f[OVS_F_PHIGOLD][k], a.f[OVS_F_RPHIGOLD][k], a.dtgl, a.gami);
    }
  }
  if ((a.which & 2) && a.b.tt == 1) {
    m |= TB;
    a.f[OVS_F_TG][k] = a.b.tv;
    a.f[OVS_F_RTG][k] = rate(a.b.tv, a.f[OVS_F_TGOLD][k], a.f[OVS_F_RTGOLD][k], a.dtgl, a.gami);
  }
  a.ibc[k] = m;
}

__global__ void ibc_unpack_kernel(const uint8_t* __restrict__ ibc, int N, int nibc, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int d = 0; d < nibc; ++d) out[(size_t)d * N + i] = (d < 8 && (ibc[i] >> d) & 1) ? 1 : 0;
}

}  // namespace

void ovs_bcs_free(ovs_ctx* c) {
  if (c->bc_nodes) cudaFree(c->bc_nodes);
  if (c->bc_n101) cudaFree(c->bc_n101);
  c->bc_nodes = nullptr;
  c->bc_n101 = nullptr;
  c->bc_bounds.clear();
  c->have_bcs = false;
}

namespace {
// The checks of a setBCs input for a mesh of N nodes: FACE_IDs index the
// *Type tables, offsets ascend from 0, node ids lie in 1..N and are
// distinct within a boundary (one writer per node per launch).  Fills the
// per-boundary records (types read by FACE_ID, values by boundary number)
// and the 0-based node ids when the outputs are given.
int validate_bc_spec(const ovs_bc_spec* sp, int N, std::vector<BcBound>* bbo, std::vector<int>* nodeso) {
  const int nb = sp->nbound, nt = sp->ntype;
  if (nb < 0 || nt < 0 || (nb > 0 && (!sp->face_id || !sp->bnode_ptr))) return OVS_ERR_ARG;
  if (nb > 0 && (!sp->bcug_type || !sp->bcug_valu || !sp->bcphig_type || !sp->bcphig_valu ||
                 !sp->bctg_type || !sp->bctg_valu))
    return OVS_ERR_ARG;
  std::vector<BcBound> bb(nb);
  const int total = nb > 0 ? sp->bnode_ptr[nb] : 0;
  if (nb > 0 && (sp->bnode_ptr[0] != 0 || total < 0 || (total > 0 && !sp->bnodes))) return OVS_ERR_ARG;
  for (int b = 0; b < nb; ++b) {
    const int fid = sp->face_id[b];
    if (fid < 1 || fid > nt) return OVS_ERR_ARG;   // the *Type tables are read by FACE_ID
    const int o0 = sp->bnode_ptr[b], o1 = sp->bnode_ptr[b + 1];
    if (o0 < 0 || o1 < o0 || o1 > total) return OVS_ERR_ARG;
    BcBound& r = bb[b];
    r.off = o0;
    r.n = o1 - o0;
    for (int d = 0; d < 3; ++d) {
      r.ut[d] = sp->bcug_type[(fid - 1) + (size_t)nt * d];
      r.uv[d] = sp->bcug_valu[b + (size_t)nb * d];
    }
    r.pt = sp->bcphig_type[fid - 1];
    r.pv = sp->bcphig_valu[b];
    r.tt = sp->bctg_type[fid - 1];
    r.tv = sp->bctg_valu[b];
  }
  std::vector<int> nodes(total);
  for (int k = 0; k < total; ++k) {
    if (sp->bnodes[k] < 1 || sp->bnodes[k] > N) return OVS_ERR_ARG;
    nodes[k] = sp->bnodes[k] - 1;
  }
  for (int b = 0; b < nb; ++b) {   // BNODES of one boundary are distinct (one writer per node per launch)
    std::vector<int> v(nodes.begin() + bb[b].off, nodes.begin() + bb[b].off + bb[b].n);
    std::sort(v.begin(), v.end());
    if (std::adjacent_find(v.begin(), v.end()) != v.end()) return OVS_ERR_ARG;
  }
  if (bbo) *bbo = std::move(bb);
  if (nodeso) *nodeso = std::move(nodes);
  return OVS_OK;
}
}  // namespace

int ovs_check_bc_spec(const ovs_bc_spec* sp, int nnode) {
  if (!sp || nnode <= 0) return OVS_ERR_ARG;
  return validate_bc_spec(sp, nnode, nullptr, nullptr);
}

int ovs_set_bc_spec(ovs_ctx* c, const ovs_bc_spec* sp) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (!sp) { ovs_bcs_free(c); return OVS_OK; }
  std::vector<BcBound> bb;
  std::vector<int> nodes;
  if ((st = validate_bc_spec(sp, c->N, &bb, &nodes))) return st;
  const int total = (int)nodes.size();
  ovs_bcs_free(c);
  cudaStream_t s = c->stream;
  if (total > 0) {
    if ((st = ovs_ensure((void**)&c->bc_nodes, sizeof(int) * total))) return st;
    OVS_CUDA_TRY(cudaMemcpyAsync(c->bc_nodes, nodes.data(), sizeof(int) * total, cudaMemcpyHostToDevice, s));
  }
  if (sp->node_id) {
    std::vector<uint8_t> h(c->N);
    for (int i = 0; i < c->N; ++i) h[i] = sp->node_id[i] == 101 ? 1 : 0;
    if ((st = ovs_ensure((void**)&c->bc_n101, c->N))) return st;
    OVS_CUDA_TRY(cudaMemcpyAsync(c->bc_n101, h.data(), c->N, cudaMemcpyHostToDevice, s));
  }
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  c->bc_bounds = bb;
  c->have_bcs = true;
  return OVS_OK;
}

int ovs_apply_bcs_impl(ovs_ctx* c, int which) {
  if (!c->have_bcs || !c->have_params) return OVS_ERR_STATE;
  if (which < 1 || which > 3) return OVS_ERR_ARG;
  cudaStream_t s = c->stream;
  bc_reset_kernel<<<ovs_grid(c->N, 256, 1 << 30), 256, 0, s>>>(c->N, c->bc_n101, c->ibc, which);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  BcArgs a;
  for (int f = 0; f < OVS_F_COUNT; ++f) a.f[f] = c->field[f];
  a.nodes = c->bc_nodes;
  a.ibc = c->ibc;
  a.N = c->N;
  a.which = which;
  a.dtgl = 1.0 / c->params.delt;   // Dtgl, src/param.f90:488
  a.gami = c->params.gami;
  for (const BcBound& b : c->bc_bounds) {
    if (b.n == 0) continue;
    a.b = b;
    bc_apply_kernel<<<ovs_grid(b.n, 128, 1 << 30), 128, 0, s>>>(a);
    ++c->launches;
    OVS_CUDA_TRY(cudaGetLastError());
  }
  return OVS_OK;
}

int ovs_apply_bcs(ovs_ctx* c, int which) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ovs_apply_bcs_impl(c, which))) return st;
  OVS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return OVS_OK;
}

int ovs_get_ibc(ovs_ctx* c, int* ibc, int nibc) {
  if (!c || !ibc || nibc < 1) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  cudaStream_t s = c->stream;
  int* tmp = nullptr;
  const size_t n = (size_t)c->N * nibc;
  OVS_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(int) * n, s));
  ibc_unpack_kernel<<<ovs_grid(c->N, 256, 1 << 30), 256, 0, s>>>(c->ibc, c->N, nibc, tmp);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaMemcpyAsync(ibc, tmp, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  OVS_CUDA_TRY(cudaFreeAsync(tmp, s));
  OVS_CUDA_TRY(cudaStreamSynchronize(s));
  return OVS_OK;
}
