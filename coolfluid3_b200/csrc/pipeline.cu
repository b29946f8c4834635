// pipeline.cu -- host-buffer inputs and outputs that overlap with the
// assembly (no counterpart in the reference, whose fields are host tables
// that its CPU assembly reads in place).
//
// A caller that holds each step's fields in (pinned) host memory and wants
// each step's RHS back -- a parameter sweep over states of one mesh, or a
// driver that keeps its fields on the host -- would otherwise pay the
// host-to-device copy, the assembly and the device-to-host copy one after the
// other.  These entry points split the transfer from its use:
//   ufem_ns_stage_state   copies the fields into one of two device staging
//                         buffers on a copy stream (returns at once);
//   ufem_ns_commit_state  unpacks the oldest staged buffer into the live fields
//                         on the compute stream, after its copy has landed;
//   ufem_ns_fetch_rhs     copies the assembled RHS into one of two device
//                         output buffers on the compute stream and reads it
//                         back on the copy stream.
// So step k+1's upload and step k-1's read-back run on the copy engines while
// step k is assembled.  Events order the streams; a staging buffer is not
// overwritten before its commit has read it, an output buffer not before its
// read-back has finished.

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "internal.h"

namespace ufem {
namespace {

int pipe_alloc(double** p, size_t count, const char* what) {
  DeviceLock lk(device_mutex());
  const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(double));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(UFEM_ERR_NOMEM, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
  }
  return UFEM_OK;
}

void pipe_free(double*& p) {
  DeviceLock lk(device_mutex());
  if (p) cudaFree(p);
  p = nullptr;
}

// One thread per node: staged rows (up | lin | nu) -> the padded node records,
// the same values ufem_ns_upload_state writes.
__global__ void commit_unpack_kernel(int64_t N, int d, int neq, const double* __restrict__ buf,
                                     double* __restrict__ state, double* __restrict__ uadv,
                                     double* __restrict__ hist, double* __restrict__ nu) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double* up = buf + i * neq;
  const double* lin = buf + N * neq + i * 4 * d;
  for (int k = 0; k < 4; ++k) {
    state[4 * i + k] = k < neq ? up[k] : 0.0;
    uadv[4 * i + k] = k < d ? lin[k] : 0.0;
    hist[4 * i + k] = k < d ? lin[d + k] : 0.0;
    hist[4 * (N + i) + k] = k < d ? lin[2 * d + k] : 0.0;
    hist[4 * (2 * N + i) + k] = k < d ? lin[3 * d + k] : 0.0;
  }
  nu[i] = buf[N * (neq + 4 * d) + i];
}

int ensure_pipe(ufem_ns_handle* h) {
  StagePipe& p = h->pipe;
  if (p.buf[0]) return UFEM_OK;
  const size_t in = size_t(h->N) * (h->neq + 4 * h->dim + 1);
  int rc;
  for (int j = 0; j < 2; ++j) {
    if ((rc = pipe_alloc(&p.buf[j], in, "staging")) || (rc = pipe_alloc(&p.out[j], size_t(h->nrows), "rhs output")))
      return rc;
    cudaEvent_t* evs[4] = {&p.staged[j], &p.consumed[j], &p.out_ready[j], &p.out_free[j]};
    for (cudaEvent_t* e : evs)
      if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess)
        return set_error(UFEM_ERR_CUDA, "cudaEventCreate failed");
  }
  return UFEM_OK;
}

}  // namespace

void free_stage_pipe(ufem_ns_handle* h) {
  StagePipe& p = h->pipe;
  for (int j = 0; j < 2; ++j) {
    pipe_free(p.buf[j]);
    pipe_free(p.out[j]);
    cudaEvent_t* evs[4] = {&p.staged[j], &p.consumed[j], &p.out_ready[j], &p.out_free[j]};
    for (cudaEvent_t* e : evs)
      if (*e) cudaEventDestroy(*e);
  }
  p = StagePipe();
}

}  // namespace ufem

using namespace ufem;

extern "C" {

int ufem_ns_stage_state(ufem_ns_handle* h, const double* up, const double* lin, const double* nu,
                        void* copy_stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!up || !lin || !nu) return set_error(UFEM_ERR_ARG, "up, lin and nu are required");
  int rc;
  if ((rc = ensure_pipe(h))) return rc;
  StagePipe& p = h->pipe;
  if (p.npending == 2) return set_error(UFEM_ERR_STATE, "two staged states are waiting for ufem_ns_commit_state");
  cudaStream_t s = static_cast<cudaStream_t>(copy_stream);
  const int j = p.next;
  const int64_t N = h->N;
  const int d = h->dim, neq = h->neq;
  if (p.consumed_rec[j]) UFEM_CUDA_TRY(cudaStreamWaitEvent(s, p.consumed[j], 0));
  double* b = p.buf[j];
  UFEM_CUDA_TRY(cudaMemcpyAsync(b, up, size_t(N) * neq * 8, cudaMemcpyHostToDevice, s));
  UFEM_CUDA_TRY(cudaMemcpyAsync(b + N * neq, lin, size_t(N) * 4 * d * 8, cudaMemcpyHostToDevice, s));
  UFEM_CUDA_TRY(cudaMemcpyAsync(b + N * (neq + 4 * d), nu, size_t(N) * 8, cudaMemcpyHostToDevice, s));
  UFEM_CUDA_TRY(cudaEventRecord(p.staged[j], s));
  p.pending[p.npending++] = j;
  p.next = 1 - j;
  return UFEM_OK;
}

int ufem_ns_commit_state(ufem_ns_handle* h, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  StagePipe& p = h->pipe;
  if (p.npending == 0) return set_error(UFEM_ERR_STATE, "no staged state to commit (ufem_ns_stage_state first)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int j = p.pending[0];
  p.pending[0] = p.pending[1];
  --p.npending;
  UFEM_CUDA_TRY(cudaStreamWaitEvent(s, p.staged[j], 0));
  commit_unpack_kernel<<<unsigned((h->N + 255) / 256), 256, 0, s>>>(h->N, h->dim, h->neq, p.buf[j], h->d_state,
                                                                    h->d_uadv, h->d_hist, h->d_nu);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaEventRecord(p.consumed[j], s));
  p.consumed_rec[j] = true;
  h->state_set = true;
  return UFEM_OK;
}

int ufem_ns_fetch_rhs(ufem_ns_handle* h, double* rhs, void* stream, void* copy_stream) {
  if (!h || !rhs) return set_error(UFEM_ERR_ARG, "NULL argument");
  int rc;
  if ((rc = ensure_pipe(h))) return rc;
  StagePipe& p = h->pipe;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStream_t c = static_cast<cudaStream_t>(copy_stream);
  const int j = p.out_next;
  if (p.out_free_rec[j]) UFEM_CUDA_TRY(cudaStreamWaitEvent(s, p.out_free[j], 0));
  UFEM_CUDA_TRY(cudaMemcpyAsync(p.out[j], h->d_rhs, size_t(h->nrows) * 8, cudaMemcpyDeviceToDevice, s));
  UFEM_CUDA_TRY(cudaEventRecord(p.out_ready[j], s));
  UFEM_CUDA_TRY(cudaStreamWaitEvent(c, p.out_ready[j], 0));
  UFEM_CUDA_TRY(cudaMemcpyAsync(rhs, p.out[j], size_t(h->nrows) * 8, cudaMemcpyDeviceToHost, c));
  UFEM_CUDA_TRY(cudaEventRecord(p.out_free[j], c));
  p.out_free_rec[j] = true;
  p.out_next = 1 - j;
  return UFEM_OK;
}

}  // extern "C"
