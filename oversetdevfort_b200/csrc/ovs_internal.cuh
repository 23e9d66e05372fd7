// Internal declarations of the B200 hot-path library (not part of the ABI).
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/ovs.h"

#define OVS_MAX_DEG 128        // longest CSR row supported (27*nshl hex bound = 216 not needed)
#define OVS_MAX_KSPACE 400     // largest Krylov space
#define OVS_ASYNC_SLOTS 16     // assembly passes ovs_assemble_async queues before a wait
#define OVS_RED_BLOCKS 592     // fixed grid of every deterministic reduction (4 x 148 SMs)
#define OVS_RED_THREADS 256
#define OVS_COOP_MAX_BLOCKS 4096  // largest cooperative grid of the Arnoldi kernel

#define OVS_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) {                                 \
      ovs_set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
      return OVS_ERR_CUDA;                                   \
    }                                                        \
  } while (0)

void ovs_set_last_cuda_error(cudaError_t e, const char* what, const char* file,
                             int line);

// number of field components per node of each system
static inline int ovs_sys_nf(int sys) {
  return sys == OVS_SYS_NS ? 4 : (sys == OVS_SYS_NSVOF ? 5 : 1);
}
// matrix values stored per CSR slot
static inline int ovs_sys_nv(int sys) {
  return sys == OVS_SYS_NS ? 16 : (sys == OVS_SYS_NSVOF ? 24 : 1);
}

// Device-side GMRES bookkeeping (one per context, FP64 throughout).
struct GmresDev {
  double beta;        // result of the latest Gram-Schmidt dot
  double epsnrm;      // tol * |P^-1 b|
  double unorm0;      // |P^-1 b|
  double ercheck;
  int iks;            // iterations completed
  int done;           // cycle finished (converged, breakdown or kspace)
  int breakdown;
  int converged;
  int kspace, kmin;
  int counter;        // last-block-done counter of the reductions
  int pad;
  double H[(OVS_MAX_KSPACE + 1) * OVS_MAX_KSPACE];  // column-major (kspace+1) x kspace
  double e[OVS_MAX_KSPACE + 1];
  double cs[OVS_MAX_KSPACE], sn[OVS_MAX_KSPACE];
  double y[OVS_MAX_KSPACE];
  double partials[OVS_RED_BLOCKS];
  double scal[8];     // misc scalar results (norms)
};

// one boundary of setBCs_NSVOF / setBCs_Tem with its types (read by FACE_ID)
// and values (read by boundary number) resolved on the host
struct BcBound {
  int off = 0, n = 0;        // node range in bc_nodes
  int ut[3] = {0, 0, 0};     // BCugType(FACE_ID, d)
  double uv[3] = {0, 0, 0};  // BCugValu(b, d)
  int pt = 0, tt = 0;        // BCphigType(FACE_ID), BCTgType(FACE_ID)
  double pv = 0, tv = 0;     // BCphigValu(b), BCTgValu(b)
};

struct SysStore {
  void* vals = nullptr;   // nnz * nv values (internal slot layout)
  void* rhs = nullptr;    // nf * N, field-major
  void* binv = nullptr;   // preconditioner: N*9 (+N pinv +N lsinv), same precision
  bool have_mat = false, have_rhs = false;
};

struct ovs_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int N = 0, E = 0, nshl = 0;
  // mesh
  int* ien = nullptr;        // E*nshl, element-major, 0-based
  int* elm_id = nullptr;     // E
  uint8_t* ibc = nullptr;    // N bit masks (bit d <=> IBC(:,d+1) == 1)
  // pattern
  int* rowptr = nullptr;     // N+1, 0-based
  int* colidx = nullptr;     // nnz
  int* diag = nullptr;       // N: slot of the diagonal entry
  int* n2e_ptr = nullptr;    // N+1
  int* n2e = nullptr;        // nshl*E: (element << 3) | local index, sorted by element
  int* tmap = nullptr;       // nnz: slot of (j, i) for slot (i, j), transposed solves
  void* vals_t = nullptr;    // transposed FP64 values of the temperature system
  double* vjp_cot = nullptr; // residual VJP work: cotangent, element terms, nodal result
  double* vjp_ge = nullptr;
  double* vjp_grad = nullptr;
  int* row_order = nullptr;  // N: rows in Morton order of the node coordinates (the row pass's order)
  int4* row_rec = nullptr;   // N: per row in that order {A, rowptr[A], n2e_ptr[A], deg | sd << 8 | ne << 16}
  int* cptr = nullptr;       // nnz + 1: off-diagonal contribution lists (tets), offsets into clist
  int* clist = nullptr;      // 12 E entries (e << 4) | (la << 2) | b, ascending element per entry
  // row tiles of the tiled row pass (tets; built at the first assembly that
  // takes that pass, ovs_tiles_build): runs of consecutive rows of row_rec
  // whose elements, at most tile_maxe of them, are staged in one CTA's
  // shared memory
  int ntiles = 0, nbig = 0, tile_maxe = 0;
  int* tile_rptr = nullptr;  // ntiles + 1: offsets into tile_rows
  int* tile_rows = nullptr;  // row positions t (into row_rec) of each tile
  int* tile_eptr = nullptr;  // ntiles + 1: offsets into tile_elems
  int* tile_elems = nullptr; // the tile's elements, in first-use order
  uint16_t* n2e_loc = nullptr;   // per n2e entry: (tile-local element << 2) | la
  uint16_t* clist_loc = nullptr; // per clist entry: (tile-local element << 4) | (la << 2) | b
  int4* big_rec = nullptr;   // nbig row records of rows with more than tile_maxe elements
  unsigned* n2s = nullptr;   // nshl*E entries: slots of the element's nodes in the row, one byte each
                             // (one word per entry for tets, two for hexahedra)
  int nnz = 0;
  int max_deg = 0, max_elem = 0;
  // boundary faces of the face assemblies (ovs_set_faces)
  int nface = 0, nfnode = 0, face_flags_all = 0;
  int* face_e = nullptr;      // nface owning elements, 0-based
  int* face_info = nullptr;   // nface: (FACE_OR - 1) | flags << 2
  double* face_h = nullptr;   // nface pairs (h, T_inf)
  int* fnode = nullptr;       // nfnode nodes touched by a face element, ascending
  int* fnode_ptr = nullptr;   // nfnode + 1
  int* fnode_ent = nullptr;   // 4 nface entries (face << 2) | local node, ascending face per node
  void* fbuf[2] = {nullptr, nullptr};   // per-face element arrays, per precision
  // streaming time steps (streaming.cu): staged field buffers, copy streams
  double* stage[OVS_F_COUNT] = {};
  unsigned staged_mask = 0;
  double* rhs_out[4] = {};                // FP64 read-back buffer per system
  cudaStream_t up_stream = nullptr, up_stream2 = nullptr, down_stream = nullptr;
  cudaEvent_t ev_staged = nullptr, ev_staged2 = nullptr, ev_commit = nullptr, ev_rhs_ready = nullptr;
  cudaEvent_t ev_rhs_out[4] = {};         // the last read-back of rhs_out[sys] done
  // hex tensor-core pass (FP32 NS+VOF): off unless OVS_HEX_TC=1 or OVS_OPT_HEX_TC
  int hex_tc = 0;
  // tet row pass: element summaries staged through shared memory by
  // asynchronous copies (1, default) or read by every lane from global memory
  int rows_staged = 1;
  // FP64 element pass: node records in registers (0) or shared memory (1);
  // -1 (default): shared memory for NS+VOF, registers for the others, the
  // faster of the two measured for each
  int elem_smem = -1;
  // OVS_MIXED: FGMRES(m) outer over FP32 inner cycles (m = mixed_outer > 0,
  // default 30) or the restarted refinement (0)
  int mixed_outer = 30;
  void* fg_buf = nullptr;    // the flexible outer's basis and directions
  size_t fg_bytes = 0;
  // tet row pass: lanes gather whole blocks by the contribution lists (1,
  // default) or the chunked pass reduces element blocks in shared memory (0)
  int rows_gather = 1;
  // tet row pass: rows in CTA tiles with their element summaries staged in
  // shared memory by bulk copies (1; default 0, measured slower than the
  // gather pass), the element budget per tile
  int rows_tiled = 0;
  int tile_elems_opt = 96;
  void* hex_kbuf = nullptr;              // E x 64 x 24 block values
  float* hex_w = nullptr;                // W hi + lo, canonical layout
  // boundary-condition producers (ovs_set_bc_spec)
  bool have_bcs = false;
  int* bc_nodes = nullptr;               // BNODES of all boundaries, 0-based
  uint8_t* bc_n101 = nullptr;            // NodeID == 101 per node (or null)
  std::vector<BcBound> bc_bounds;        // in NBOUND order
  // nodal state (FP64, reference layout)
  double* field[OVS_F_COUNT] = {};
  // alpha-stage node records (16 values per node), per precision
  void* rec[2] = {nullptr, nullptr};
  // per-element summaries of the element pass, per precision
  void* esum[2] = {nullptr, nullptr};
  // systems [sys][prec]
  SysStore sys[4][2];
  // last solution of each system (FP64, field-major)
  double* sol[4] = {};
  // GMRES / solve workspace
  GmresDev* gm = nullptr;
  void* basis[2] = {nullptr, nullptr};   // Krylov basis per precision
  size_t basis_bytes[2] = {0, 0};
  double* work64 = nullptr;              // 3 vectors of 5N doubles (b, r, x)
  float* work32 = nullptr;               // 1 vector of 5N floats
  double* wvec = nullptr;                // FP64 vector under orthogonalization
  double* coop_part = nullptr;           // partial sums of the cooperative Arnoldi kernels
  bool arnoldi_fused = false;            // one-launch Arnoldi variant (env OVS_ARNOLDI_FUSED=1)
  // status words: [0] negative DetJ count, [1] non-finite flag, [3] face column missing from a row
  int* flags = nullptr;
  unsigned long long* cfl_bits = nullptr;
  // pinned host mirror
  int* h_pinned = nullptr;
  double* h_pinned_d = nullptr;
  // ovs_assemble_async: status words and CFL bits of the queued passes, read
  // by ovs_assemble_wait (page-locked, OVS_ASYNC_SLOTS entries)
  bool defer_status = false;
  int async_n = 0;
  int* h_async_flags = nullptr;
  unsigned long long* h_async_cfl = nullptr;
  ovs_params params{};
  bool have_mesh = false, have_pattern = false, have_params = false;
  long long launches = 0;                // kernels launched by this context
  double last_ms = 0.0;                  // device time of the last top-level call
};

// ------------------------------------------------------------ helpers
int ovs_ensure(void** p, size_t bytes);
int ovs_tiles_build(ovs_ctx* c, int maxe);
int ovs_activate(ovs_ctx* c);

// pattern.cu
int ovs_pattern_build(ovs_ctx* c);
int ovs_pattern_to_host(ovs_ctx* c, int* col, int* row);
int ovs_slot_map_to_host(ovs_ctx* c, int* lmap);

// assemble.cu
int ovs_assemble_impl(ovs_ctx* c, int kernel, int tensor_flag, int prec,
                      double* cfl);

// assemble.cu: W operand and block buffer of the hex tensor-core pass
int hex_tc_prepare(ovs_ctx* c);

// streaming.cu
void ovs_streaming_free(ovs_ctx* c);

// faces.cu
int ovs_faces_set_impl(ovs_ctx* c, int nface, const int* f2e, const int* face_or, const int* flags,
                       const double* hconv, const double* tinf);
int ovs_faces_assemble(ovs_ctx* c, int kernel, int prec, int mat, int vec);
void ovs_faces_free(ovs_ctx* c);

// bcs.cu
int ovs_apply_bcs_impl(ovs_ctx* c, int which);
void ovs_bcs_free(ovs_ctx* c);

// spmv.cu / gmres.cu
int ovs_precond_setup(ovs_ctx* c, int sys, int prec);
int ovs_spmv_impl(ovs_ctx* c, int sys, int prec, const double* dx,
                  double* dy);
int ovs_spmv_pre_impl(ovs_ctx* c, int sys, int prec, const double* dx, double* dy);
int ovs_spmv_rows_impl(ovs_ctx* c, int sys, int prec, bool precond, const double* dx, double* dy, const int* rows,
                       int nrows);
int ovs_precond_apply_impl(ovs_ctx* c, int sys, int prec, const double* dx, double* dy);
int ovs_gmres_ref_impl(ovs_ctx* c, int sys, double tol, int kspace, int kmin,
                       double* dsol, ovs_gmres_info* info);
int ovs_solve_impl(ovs_ctx* c, int sys, int mode, double rtol, int kspace,
                   int max_cycles, ovs_solve_info* info);
int ovs_round_impl(ovs_ctx* c, int sys);
int ovs_update_impl(ovs_ctx* c, int sys);
int ovs_resnorm_impl(ovs_ctx* c, int prec, double r[4]);
int ovs_dot_impl(ovs_ctx* c, const double* a, const double* b, size_t n,
                 double* out);
int ovs_profile_assemble(ovs_ctx* c, int kernel, int prec, int reps, double* ms, int parts);
int ovs_residual_vjp_impl(ovs_ctx* c, int kernel, const double* cot_host, double* grad_host);
int ovs_gmres_transposed_impl(ovs_ctx* c, int sys, const double* drhs, double tol, int kspace, int kmin,
                              double* dsol, ovs_gmres_info* info);
int ovs_profile_krylov(ovs_ctx* c, int what, int sys, int prec, int reps, double* ms);

// launch geometry helper
static inline int ovs_grid(size_t n, int threads, int cap) {
  size_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > (size_t)cap) g = cap;
  return (int)g;
}
