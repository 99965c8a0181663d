// athb_slab.cu -- device-buffer pieces of the slab decomposition (one grid
// split along x2 over several contexts, athena_cuda_b200/decomp.py).
//
// The exchange of an iteration stays on the GPU: the 4 boundary rows of all
// 11 planes are packed into one contiguous device buffer by a kernel, carried
// to the neighbour's own receive buffer (NCCL send/recv between GPUs, or a
// cudaMemcpyAsync into a CUDA-IPC mapping of the neighbour's buffer), and
// unpacked into the ghost rows by a kernel; the running CFL maximum leaves
// and re-enters the step state as a device word, so the all-reduce of 1/dt
// runs on device memory too (NCCL, or a max over the ranks' words read
// through IPC mappings).  No host copy of rows or of dt per iteration.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>

#include "athb_internal.h"
#include "step_kernels.cuh"

using namespace athb;

#define CUDA_TRY(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return athb_fail(ATHB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                              \
  } while (0)

namespace {

// the rectangle rows [j0, j0+nj) x columns [i0, i0+ni) of the 11 planes <->
// buf laid out [plane][row][column]
__global__ void __launch_bounds__(kThreads) k_rect_pack(const double* __restrict__ s, long long ps, int pitch, int i0,
                                                       int ni, int j0, int nj, double* __restrict__ buf) {
  const long long per = (long long)nj * ni, n = per * NSTATE;
  for (long long t = blockIdx.x * (long long)kThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kThreads) {
    const int p = (int)(t / per);
    const long long r = t - p * per;
    const int j = (int)(r / ni), i = (int)(r - (long long)j * ni);
    buf[t] = s[p * ps + (long long)(j0 + j) * pitch + i0 + i];
  }
}

__global__ void __launch_bounds__(kThreads) k_rect_unpack(double* __restrict__ s, long long ps, int pitch, int i0,
                                                         int ni, int j0, int nj, const double* __restrict__ buf) {
  const long long per = (long long)nj * ni, n = per * NSTATE;
  for (long long t = blockIdx.x * (long long)kThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kThreads) {
    const int p = (int)(t / per);
    const long long r = t - p * per;
    const int j = (int)(r / ni), i = (int)(r - (long long)j * ni);
    s[p * ps + (long long)(j0 + j) * pitch + i0 + i] = buf[t];
  }
}

// the running maximum of 1/dt as a device word (the all-reduce operand)
__global__ void k_get_max_dti(const StepState* st, unsigned long long* out) { *out = st->max_dti_bits; }

// the maximum over n words (the all-reduced value, or every rank's word)
__global__ void k_set_max_dti_n(StepState* st, const unsigned long long* bits, int n) {
  unsigned long long m = 0ull;
  for (int k = 0; k < n; k++) m = bits[k] > m ? bits[k] : m;
  st->max_dti_bits = m;
}

int grid_of(long long n) {
  const long long b = (n + kThreads - 1) / kThreads;
  return (int)(b < 148LL * 8 ? (b < 1 ? 1 : b) : 148LL * 8);
}

int rect_ok(const athb_ctx* c, int i0, int ni, int j0, int nj) {
  return i0 >= 0 && ni >= 1 && i0 + ni <= c->sx && j0 >= 0 && nj >= 1 && j0 + nj <= c->sy;
}

}  // namespace

extern "C" int athb_rect_pack(athb_ctx* c, int i0, int ni, int j0, int nj, double* dev) {
  if (!c || !dev || !rect_ok(c, i0, ni, j0, nj)) return athb_fail(ATHB_ERR_ARG, "bad rectangle");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  k_rect_pack<<<grid_of((long long)ni * nj * NSTATE), kThreads, 0, c->stream>>>(c->state[c->cur], c->ps, c->pitch,
                                                                                i0, ni, j0, nj, dev);
  CUDA_TRY(cudaGetLastError());
  return ATHB_OK;
}

extern "C" int athb_rect_unpack(athb_ctx* c, int i0, int ni, int j0, int nj, const double* dev) {
  if (!c || !dev || !rect_ok(c, i0, ni, j0, nj)) return athb_fail(ATHB_ERR_ARG, "bad rectangle");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  k_rect_unpack<<<grid_of((long long)ni * nj * NSTATE), kThreads, 0, c->stream>>>(c->state[c->cur], c->ps, c->pitch,
                                                                                  i0, ni, j0, nj, dev);
  CUDA_TRY(cudaGetLastError());
  return ATHB_OK;
}

extern "C" int athb_rows_pack(athb_ctx* c, int j0, int nrows, double* dev) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  return athb_rect_pack(c, 0, c->sx, j0, nrows, dev);
}

extern "C" int athb_rows_unpack(athb_ctx* c, int j0, int nrows, const double* dev) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  return athb_rect_unpack(c, 0, c->sx, j0, nrows, dev);
}

extern "C" int athb_max_dti_bits_device(athb_ctx* c, unsigned long long* dev) {
  if (!c || !dev) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  k_get_max_dti<<<1, 1, 0, c->stream>>>(c->st, dev);
  CUDA_TRY(cudaGetLastError());
  return ATHB_OK;
}

extern "C" int athb_finish_step_device(athb_ctx* c, const unsigned long long* dev_bits, int n, int after_step) {
  if (!c || !dev_bits || n < 1) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  k_set_max_dti_n<<<1, 1, 0, c->stream>>>(c->st, dev_bits, n);
  k_finalize<<<1, 1, 0, c->stream>>>(c->st, c->dx1, c->dx2, after_step ? 1 : 0);
  CUDA_TRY(cudaGetLastError());
  if (after_step) c->cur ^= 1;
  return ATHB_OK;
}

// ---- device buffers shared between processes (CUDA IPC) -------------------
extern "C" void* athb_device_alloc(athb_ctx* c, unsigned long long bytes) {
  if (!c || bytes == 0) return nullptr;
  if (cudaSetDevice(c->cfg.device) != cudaSuccess) return nullptr;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  if (cudaMemset(p, 0, bytes) != cudaSuccess) {
    cudaFree(p);
    return nullptr;
  }
  return p;
}

extern "C" void athb_device_free(athb_ctx* c, void* p) {
  if (!c || !p) return;
  cudaSetDevice(c->cfg.device);
  cudaFree(p);
}

extern "C" int athb_ipc_handle(athb_ctx* c, void* dev, unsigned char handle[64]) {
  if (!c || !dev || !handle) return athb_fail(ATHB_ERR_ARG, "null argument");
  static_assert(sizeof(cudaIpcMemHandle_t) == 64, "IPC handle size");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  cudaIpcMemHandle_t h;
  CUDA_TRY(cudaIpcGetMemHandle(&h, dev));
  memcpy(handle, &h, sizeof h);
  return ATHB_OK;
}

extern "C" int athb_ipc_open(athb_ctx* c, const unsigned char handle[64], void** dev) {
  if (!c || !handle || !dev) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  cudaIpcMemHandle_t h;
  memcpy(&h, handle, sizeof h);
  *dev = nullptr;
  CUDA_TRY(cudaIpcOpenMemHandle(dev, h, cudaIpcMemLazyEnablePeerAccess));
  return ATHB_OK;
}

extern "C" int athb_ipc_close(athb_ctx* c, void* dev) {
  if (!c || !dev) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  CUDA_TRY(cudaIpcCloseMemHandle(dev));
  return ATHB_OK;
}

// One copy on the context's stream between device buffers (its own, or a
// neighbour's reached through an IPC mapping): plain peer stores.
extern "C" int athb_copy_async(athb_ctx* c, void* dst, const void* src, unsigned long long bytes) {
  if (!c || !dst || !src) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
  return ATHB_OK;
}
