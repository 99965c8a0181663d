// athb_noalloc.cu -- one integrate_2d step on caller-owned device buffers that
// allocates no memory at all.
//
// The regular paths allocate their face scratch with cudaMalloc when a context
// is created.  Some callers cannot do that: code that runs while a CUDA graph
// is being captured (cudaMalloc is not a capturable operation), coupling codes
// that reserve the whole device memory budget up front and hand out only
// pre-allocated buffers, and real-time loops that must not pay an allocation.
// For them this entry point keeps its scratch in a file-scope __device__ array
// of fixed size, which exists on every GPU that loads the library from load
// time until the process exits (kNoAllocDoubles doubles below, ~2.4 MB).
//
// Limits and rules (also in include/athena_b200.h):
//  * grids with (Nx1+8)*(Nx2+8) <= kNoAllocCells (64 x 64 interior, or any
//    other shape of at most that many cells); larger grids are rejected;
//  * every call uses the same array, so calls that overlap on the GPU (on two
//    streams, or from two host threads) race and corrupt each other; the
//    array keeps the last call's contents, and the step state in it is reset
//    at the start of every call;
//  * the device address of the array is looked up (cudaGetSymbolAddress) on
//    the first call made on each device, with that device current; make that
//    first call before any stream capture;
//  * the step runs on the current device, which must be cfg->device;
//  * no non-finite check: a NaN or negative-pressure step is not reported
//    (the regular paths report it through athb_status / athb_run).
#include <cuda_runtime.h>

#include <mutex>

#include "athb_internal.h"
#include "step_kernels.cuh"

using namespace athb;

namespace {

constexpr int kNoAllocCells = 72 * 72;          // (Nx1+8) * (Nx2+8) at most
constexpr int kStateDoubles = 32;               // StepState slot, 256-byte aligned planes after it
constexpr long long kNoAllocDoubles = kStateDoubles + (long long)NSCRATCH * kNoAllocCells;
constexpr int kMaxDevices = 64;

static_assert(sizeof(StepState) <= kStateDoubles * sizeof(double), "StepState slot too small");

// The scratch of athb_integrate_noalloc: a StepState slot, then NSCRATCH
// planes of kNoAllocCells doubles.
__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// Reset the step state held in the array and derive the dt factors.
__global__ void k_noalloc_begin(StepState* st, double dt, double dx1, double dx2) {
  StepState s;
  s.time = 0.0; s.tlim = 0.0; s.cour_no = 0.0;
  s.nstep = 0; s.nlim = -1; s.done = 0; s.flags = 0; s.max_dti_bits = 0ull;
  s.tpause = 0.0; s.has_pause = 0;
  s.dt = dt;
  s.dt_new = dt;
  s.dtodx1 = dt / dx1;
  s.dtodx2 = dt / dx2;
  s.hdtodx1 = 0.5 * s.dtodx1;
  s.hdtodx2 = 0.5 * s.dtodx2;
  s.hdt = 0.5 * dt;
  *st = s;
}

int scratch_address(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices) return athb_fail(ATHB_ERR_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return athb_fail(ATHB_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return ATHB_OK;
}

int blocks_of(long long n) { return (int)((n + kThreads - 1) / kThreads); }

}  // namespace

extern "C" int athb_integrate_noalloc(const athb_config* cfg, const double* d_in, double* d_out, double dt,
                                      void* stream) {
  if (!cfg || !d_in || !d_out) return athb_fail(ATHB_ERR_ARG, "null argument");
  if (d_in == d_out) return athb_fail(ATHB_ERR_ARG, "d_in and d_out must be different buffers");
  int rc = athb_ctx_validate(cfg);
  if (rc) return rc;
  const int nx1 = cfg->nx1, nx2 = cfg->nx2;
  const int sx = nx1 + 2 * kNghost, sy = nx2 + 2 * kNghost;
  if ((long long)sx * sy > kNoAllocCells)
    return athb_fail(ATHB_ERR_ARG,
                     "athb_integrate_noalloc: grid %d x %d needs %lld cells with ghosts, the fixed scratch holds "
                     "%d ((Nx1+8)*(Nx2+8) <= %d, e.g. 64 x 64)",
                     nx1, nx2, (long long)sx * sy, kNoAllocCells, kNoAllocCells);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  // The step runs on the calling thread's current device (no cudaSetDevice
  // here: switching devices is the caller's business mid-capture); a config
  // naming another device is a caller error, not a silent redirect.
  if (cfg->device != dev)
    return athb_fail(ATHB_ERR_ARG,
                     "athb_integrate_noalloc: cfg->device is %d but the current device is %d (make the "
                     "device current with cudaSetDevice before the call)",
                     cfg->device, dev);
  double* scratch = nullptr;
  rc = scratch_address(dev, &scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // State planes (caller) and scratch planes (fixed array) share one plane
  // stride, sx * sy <= kNoAllocCells, as the kernels index both with it.
  GridArgs gs;
  gs.in = d_in;
  gs.out = d_out;
  gs.st = reinterpret_cast<StepState*>(scratch);
  gs.scr = scratch + kStateDoubles;
  gs.ps = (long long)sx * sy;
  gs.pitch = sx;
  gs.is = kNghost; gs.ie = nx1 + kNghost - 1; gs.js = kNghost; gs.je = nx2 + kNghost - 1;
  gs.ly = 4;
  gs.dx1 = (cfg->x1max - cfg->x1min) / (double)nx1;
  gs.dx2 = (cfg->x2max - cfg->x2min) / (double)nx2;
  gs.eos = Eos{cfg->gamma, cfg->gamma - 1.0, cfg->gamma - 2.0};
  gs.bc[0] = cfg->bc_ix1; gs.bc[1] = cfg->bc_ox1; gs.bc[2] = cfg->bc_ix2; gs.bc[3] = cfg->bc_ox2;

  k_noalloc_begin<<<1, 1, 0, s>>>(gs.st, dt, gs.dx1, gs.dx2);

  const PredictGeom pg = make_predict_geom(nx1, nx2, gs.ly);
  if (cfg->flux == ATHB_FLUX_HLLE) k_predict<kFluxHlle><<<pg.nx_blocks + pg.ny_blocks, kThreads, 0, s>>>(gs, pg);
  else k_predict<kFluxRoe><<<pg.nx_blocks + pg.ny_blocks, kThreads, 0, s>>>(gs, pg);
  k_emf<<<blocks_of((long long)(nx1 + 3) * (nx2 + 3)), kThreads, 0, s>>>(gs, gs.is - 1, gs.js - 1, nx1 + 3, nx2 + 3,
                                                                           S_FX, S_FY);
  CorrectGeom cg;
  cg.xw = nx1 + 1; cg.xn = nx2 + 3;
  cg.yw = nx1 + 3; cg.yn = nx2 + 1;
  cg.ew = nx1 + 3; cg.en = nx2 + 3;
  cg.xb = blocks_of((long long)cg.xw * cg.xn);
  cg.yb = blocks_of((long long)cg.yw * cg.yn);
  cg.eb = blocks_of((long long)cg.ew * cg.en);
  if (cfg->flux == ATHB_FLUX_HLLE) k_correct<kFluxHlle><<<cg.xb + cg.yb + cg.eb, kThreads, 0, s>>>(gs, cg);
  else k_correct<kFluxRoe><<<cg.xb + cg.yb + cg.eb, kThreads, 0, s>>>(gs, cg);
  k_emf<<<blocks_of((long long)(nx1 + 1) * (nx2 + 1)), kThreads, 0, s>>>(gs, gs.is, gs.js, nx1 + 1, nx2 + 1, S_FX2,
                                                                           S_FY2);
  const int n = nx1 * nx2;
  k_update<<<blocks_of(n), kThreads, 0, s>>>(gs, nx1, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "athb_integrate_noalloc launch: %s", cudaGetErrorString(e));
  return ATHB_OK;
}
