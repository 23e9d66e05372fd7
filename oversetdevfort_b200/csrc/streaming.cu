// Streaming time steps: the host fields of the next assembly are copied on
// an upload stream into a second device buffer per field while the current
// assembly runs, and the residual of the current one is copied out on a
// download stream while the next one runs.  The device's copy engines and
// its SMs then work at the same time; every copy is still one call of the
// caller's step.  (The reference's Newton drivers push the state to the
// assembly and read the residual back every iteration,
// src/solveFlow.f90:39-40, 71-72, 116-117, 148-149.)
#include "ovs_internal.cuh"

namespace {

inline int field_width_s(int f) { return f <= OVS_F_ACGMOLD ? 3 : 1; }

template <typename TI, typename TO>
__global__ void convert_kernel(const TI* __restrict__ in, TO* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (TO)in[i];
}

int ensure_copy_streams(ovs_ctx* c) {
  if (!c->up_stream) {
    OVS_CUDA_TRY(cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking));
    OVS_CUDA_TRY(cudaStreamCreateWithFlags(&c->up_stream2, cudaStreamNonBlocking));
    OVS_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_staged2, cudaEventDisableTiming));
    OVS_CUDA_TRY(cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking));
    OVS_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_staged, cudaEventDisableTiming));
    OVS_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_commit, cudaEventDisableTiming));
    OVS_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_rhs_ready, cudaEventDisableTiming));
    for (int s = 0; s < 4; ++s) OVS_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_rhs_out[s], cudaEventDisableTiming));
    // nothing has used the staging buffers yet
    OVS_CUDA_TRY(cudaEventRecord(c->ev_commit, c->stream));
    for (int s = 0; s < 4; ++s) OVS_CUDA_TRY(cudaEventRecord(c->ev_rhs_out[s], c->down_stream));
  }
  return OVS_OK;
}

}  // namespace

void ovs_streaming_free(ovs_ctx* c) {
  for (int f = 0; f < OVS_F_COUNT; ++f)
    if (c->stage[f]) { cudaFree(c->stage[f]); c->stage[f] = nullptr; }
  for (int s = 0; s < 4; ++s)
    if (c->rhs_out[s]) { cudaFree(c->rhs_out[s]); c->rhs_out[s] = nullptr; }
  if (c->up_stream) cudaStreamDestroy(c->up_stream);
  if (c->up_stream2) cudaStreamDestroy(c->up_stream2);
  if (c->down_stream) cudaStreamDestroy(c->down_stream);
  cudaEvent_t evs[] = {c->ev_staged, c->ev_staged2, c->ev_commit, c->ev_rhs_ready,
                       c->ev_rhs_out[0], c->ev_rhs_out[1], c->ev_rhs_out[2], c->ev_rhs_out[3]};
  for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
  c->up_stream = c->up_stream2 = c->down_stream = nullptr;
  c->ev_staged = c->ev_staged2 = c->ev_commit = c->ev_rhs_ready = nullptr;
  for (int s = 0; s < 4; ++s) c->ev_rhs_out[s] = nullptr;
  c->staged_mask = 0;
}

int ovs_stage_fields(ovs_ctx* c, int nfields, const int* ids, const double* const* host) {
  if (!c || nfields < 0 || (nfields > 0 && (!ids || !host))) return OVS_ERR_ARG;
  for (int k = 0; k < nfields; ++k)
    if (ids[k] < 0 || ids[k] >= OVS_F_COUNT || !host[k]) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ensure_copy_streams(c))) return st;
  // the staging buffers held the fields of earlier steps: wait until the
  // work committed before now has stopped reading them
  OVS_CUDA_TRY(cudaStreamWaitEvent(c->up_stream, c->ev_commit, 0));
  OVS_CUDA_TRY(cudaStreamWaitEvent(c->up_stream2, c->ev_commit, 0));
  // the copies alternate between two upload streams (two copy engines)
  for (int k = 0; k < nfields; ++k) {
    const int f = ids[k];
    const size_t bytes = sizeof(double) * (size_t)c->N * field_width_s(f);
    if ((st = ovs_ensure((void**)&c->stage[f], bytes))) return st;
    OVS_CUDA_TRY(cudaMemcpyAsync(c->stage[f], host[k], bytes, cudaMemcpyHostToDevice,
                                 (k & 1) ? c->up_stream2 : c->up_stream));
    c->staged_mask |= 1u << f;
  }
  OVS_CUDA_TRY(cudaEventRecord(c->ev_staged, c->up_stream));
  OVS_CUDA_TRY(cudaEventRecord(c->ev_staged2, c->up_stream2));
  return OVS_OK;
}

int ovs_commit_staged(ovs_ctx* c) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if (!c->up_stream || !c->staged_mask) return OVS_ERR_STATE;
  OVS_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_staged, 0));
  OVS_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_staged2, 0));
  for (int f = 0; f < OVS_F_COUNT; ++f)
    if (c->staged_mask & (1u << f)) {
      double* t = c->field[f];
      c->field[f] = c->stage[f];
      c->stage[f] = t;
    }
  c->staged_mask = 0;
  // later staging into the buffers just retired waits for what is queued now
  OVS_CUDA_TRY(cudaEventRecord(c->ev_commit, c->stream));
  return OVS_OK;
}

int ovs_get_rhs_async(ovs_ctx* c, int sys, int prec, double* host) {
  if (!c || !host || sys < OVS_SYS_NS || sys > OVS_SYS_TEM || (prec != OVS_FP64 && prec != OVS_FP32))
    return OVS_ERR_ARG;
  SysStore& S = c->sys[sys][prec];
  if (!S.rhs) return OVS_ERR_STATE;
  int st;
  if ((st = ovs_activate(c))) return st;
  if ((st = ensure_copy_streams(c))) return st;
  const size_t n = (size_t)c->N * ovs_sys_nf(sys);
  if ((st = ovs_ensure((void**)&c->rhs_out[sys], sizeof(double) * n))) return st;
  // the previous read-back of this system's buffer must be done before it
  // is rewritten (each system has its own buffer and event: the read-back
  // of one system does not hold up the conversion of another)
  OVS_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_rhs_out[sys], 0));
  if (prec == OVS_FP64)
    convert_kernel<double, double><<<ovs_grid(n, 256, 4 * c->num_sms * 8), 256, 0, c->stream>>>(
        reinterpret_cast<const double*>(S.rhs), c->rhs_out[sys], n);
  else
    convert_kernel<float, double><<<ovs_grid(n, 256, 4 * c->num_sms * 8), 256, 0, c->stream>>>(
        reinterpret_cast<const float*>(S.rhs), c->rhs_out[sys], n);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  OVS_CUDA_TRY(cudaEventRecord(c->ev_rhs_ready, c->stream));
  OVS_CUDA_TRY(cudaStreamWaitEvent(c->down_stream, c->ev_rhs_ready, 0));
  OVS_CUDA_TRY(cudaMemcpyAsync(host, c->rhs_out[sys], sizeof(double) * n, cudaMemcpyDeviceToHost, c->down_stream));
  OVS_CUDA_TRY(cudaEventRecord(c->ev_rhs_out[sys], c->down_stream));
  return OVS_OK;
}

int ovs_sync_copies(ovs_ctx* c) {
  if (!c) return OVS_ERR_ARG;
  int st;
  if ((st = ovs_activate(c))) return st;
  if (c->up_stream) OVS_CUDA_TRY(cudaStreamSynchronize(c->up_stream));
  if (c->up_stream2) OVS_CUDA_TRY(cudaStreamSynchronize(c->up_stream2));
  if (c->down_stream) OVS_CUDA_TRY(cudaStreamSynchronize(c->down_stream));
  return OVS_OK;
}
