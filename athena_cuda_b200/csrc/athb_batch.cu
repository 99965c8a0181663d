// athb_batch.cu -- many independent grids of uneven size, each with its own
// dt and end time, advanced by ONE persistent kernel launch per step.
//
// The persistent kernel walks six phases (predict, half-step corner EMF,
// correct, full-step corner EMF, update + CFL, ghost fill + finalize); in each
// phase the blocks of the launch take the (instance, block) work items of all
// active instances round-robin, and a grid-wide barrier separates the phases.
// The per-item work is the very device code of the single-grid kernels, so
// every instance is bit-identical to a single-grid run of the same problem.
//
// * Instances keep their own StepState (dt, time, nstep, done) and their own
//   buffer parity (cur[k]); an instance that reached its end time is skipped.
// * The finalize of instance k (time += dt, dt rule, tlim clamp, parity flip)
//   runs in the block that completes k's last ghost item (a per-instance
//   countdown), so it needs no extra barrier.
// * The grid barrier is a generation counter with a bounded spin: a block that
//   waits longer than kBarrierSpins sets the batch error flag and proceeds,
//   so a failure ends the launch instead of hanging the GPU.  The launch is
//   cooperative, so all its blocks are co-resident.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "athb_internal.h"
#include "step_kernels.cuh"

using namespace athb;

namespace {

constexpr int kPhases = 6;
constexpr long long kBarrierSpins = 20000000;  // x ~64 ns sleep: ~1-2 s
constexpr int kBatchMinBlocks = 3;  // as k_predict: 168 registers per thread

struct InstGeom {
  GridArgs g;  // g.in = state[0], g.out = state[1]
  PredictGeom pg;
  CorrectGeom cg;
  int nx1, nx2, sx, sy, nframe;
};

struct BarrierState {
  unsigned int count;
  unsigned int gen;
};

struct BatchDev {
  const InstGeom* inst;
  StepState* st;
  int* cur;
  unsigned int* ghost_left;
  const int* off;  // kPhases x (n+1) prefix sums of work items of the active instances
  const int* ids;  // active instance ids; ids[n] = number active
  int n;
  BarrierState* bar;
  int* err;
};

__device__ __forceinline__ int item_count(const InstGeom& I, int ph) {
  switch (ph) {
  case 0: return I.pg.nx_blocks + I.pg.ny_blocks;
  case 1: return (int)(((long long)(I.nx1 + 3) * (I.nx2 + 3) + kThreads - 1) / kThreads);
  case 2: return I.cg.xb + I.cg.yb + I.cg.eb;
  case 3: return (int)(((long long)(I.nx1 + 1) * (I.nx2 + 1) + kThreads - 1) / kThreads);
  case 4: return (int)(((long long)I.nx1 * I.nx2 + kThreads - 1) / kThreads);
  default: return (I.nframe + kThreads - 1) / kThreads;
  }
}

__device__ void grid_barrier(const BatchDev& B) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &B.bar->gen;
    const unsigned int gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&B.bar->count, 1u) + 1u;
    if (arrived == gridDim.x) {
      B.bar->count = 0u;
      __threadfence();
      atomicAdd(&B.bar->gen, 1u);
    } else {
      long long spins = 0;
      while (*vgen == gen) {
        __nanosleep(64);
        if (++spins > kBarrierSpins) { atomicExch(B.err, 1); break; }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <int FLUX>
__global__ void __launch_bounds__(kThreads, kBatchMinBlocks) k_batch_step(BatchDev B) {
  // the current work item's instance data, loaded once per item by thread 0
  __shared__ InstGeom s_I;
  __shared__ int s_k, s_b, s_skip;
  const int na = B.ids[B.n];
  for (int ph = 0; ph < kPhases; ph++) {
    const int* off = B.off + ph * (B.n + 1);
    const int total = off[na];
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
      __syncthreads();  // the previous item is finished with s_I
      if (threadIdx.x == 0) {
        int lo = 0, hi = na;  // off[lo] <= w < off[hi]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (off[mid] <= w) lo = mid; else hi = mid;
        }
        const int id = B.ids[lo];
        s_k = id;
        s_b = w - off[lo];
        s_skip = *(volatile int*)&B.st[id].done;
        if (!s_skip) {
          s_I = B.inst[id];
          if (B.cur[id]) {  // the state lives in the second buffer
            const double* a = s_I.g.in;
            s_I.g.in = s_I.g.out;
            s_I.g.out = const_cast<double*>(a);
          }
        }
      }
      __syncthreads();
      if (s_skip) continue;  // instance has reached its end time
      const int k = s_k, b = s_b;
      const InstGeom& I = s_I;
      const GridArgs& g = I.g;
      const int t = b * kThreads + threadIdx.x;
      switch (ph) {
      case 0: predict_block<FLUX>(g, I.pg, b); break;
      case 1: emf_item(g, g.is - 1, g.js - 1, I.nx1 + 3, I.nx2 + 3, S_FX, S_FY, t); break;
      case 2: correct_block<FLUX>(g, I.cg, b); break;
      case 3: emf_item(g, g.is, g.js, I.nx1 + 1, I.nx2 + 1, S_FX2, S_FY2, t); break;
      case 4:
        block_max_to(update_cell(g, I.nx1, I.nx1 * I.nx2, t), &g.st->max_dti_bits, &g.st->flags);
        break;
      default: {
        ghost_item(g, I.sx, I.sy, I.nframe, 3, 3, t);
        __syncthreads();
        if (threadIdx.x == 0) {
          __threadfence();
          if (atomicSub(&B.ghost_left[k], 1u) == 1u) {
            // last ghost item of instance k: end of its step
            __threadfence();
            B.ghost_left[k] = (unsigned int)item_count(I, kPhases - 1);
            finalize_state(B.st[k], g.dx1, g.dx2, 1);
            B.cur[k] ^= 1;
            __threadfence();
          }
        }
        break;
      }
      }
    }
    if (ph < kPhases - 1) grid_barrier(B);
  }
}

}  // namespace

struct athb_batch {
  int n = 0;
  int flux = ATHB_FLUX_ROE;
  int device = 0;
  std::vector<athb_config> cfg;
  std::vector<InstGeom> geom;  // host copy
  std::vector<int> ly;         // y-march segment length per instance
  double* pool = nullptr;
  StepState* st = nullptr;
  int* cur = nullptr;
  unsigned int* ghost_left = nullptr;
  int* off = nullptr;
  int* ids = nullptr;
  std::vector<int> active;     // ids of the instances in the work tables
  InstGeom* dgeom = nullptr;
  BarrierState* bar = nullptr;
  int* err = nullptr;
  cudaStream_t stream = nullptr;
  int grid = 0;            // persistent blocks
  cudaGraphExec_t graph = nullptr;
  bool graph_tried = false;
};

#define CUDA_TRY(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return athb_fail(ATHB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                               \
  } while (0)

static int pick_ly(int nx1, int nx2) {
  long long ly = ((long long)(nx1 + 4) * (nx2 + 3)) / (148LL * 512);
  return (int)std::max(4LL, std::min(64LL, ly));
}

// Geometry of instance k (same rules as the single-grid launcher).
static InstGeom make_geom(const athb_config& c, int ly, double* state0, double* state1, double* scr,
                          StepState* st) {
  InstGeom I;
  memset(&I, 0, sizeof I);
  const int sx = c.nx1 + 2 * kNghost, sy = c.nx2 + 2 * kNghost;
  const int pitch = (sx + 15) & ~15;
  GridArgs& g = I.g;
  g.in = state0; g.out = state1; g.scr = scr; g.st = st;
  g.ps = (long long)pitch * sy; g.pitch = pitch;
  g.is = kNghost; g.ie = c.nx1 + kNghost - 1; g.js = kNghost; g.je = c.nx2 + kNghost - 1;
  g.ly = ly;
  g.dx1 = (c.x1max - c.x1min) / (double)c.nx1;
  g.dx2 = (c.x2max - c.x2min) / (double)c.nx2;
  g.eos = Eos{c.gamma, c.gamma - 1.0, c.gamma - 2.0};
  g.bc[0] = c.bc_ix1; g.bc[1] = c.bc_ox1; g.bc[2] = c.bc_ix2; g.bc[3] = c.bc_ox2;
  const int nx1 = c.nx1, nx2 = c.nx2;
  I.pg.xseg = (nx1 + 3 + kXFacesPerWarp - 1) / kXFacesPerWarp;
  I.pg.xrowblk = (nx2 + 4 + kXRowsPerBlock - 1) / kXRowsPerBlock;
  I.pg.nx_blocks = I.pg.xseg * I.pg.xrowblk;
  I.pg.ycolblk = (nx1 + 4 + kThreads - 1) / kThreads;
  I.pg.yseg = (nx2 + 3 + ly - 1) / ly;
  I.pg.ny_blocks = I.pg.ycolblk * I.pg.yseg;
  I.cg.xw = nx1 + 1; I.cg.xn = nx2 + 3;
  I.cg.yw = nx1 + 3; I.cg.yn = nx2 + 1;
  I.cg.ew = nx1 + 3; I.cg.en = nx2 + 3;
  auto bf = [](long long n) { return (int)((n + kThreads - 1) / kThreads); };
  I.cg.xb = bf((long long)I.cg.xw * I.cg.xn);
  I.cg.yb = bf((long long)I.cg.yw * I.cg.yn);
  I.cg.eb = bf((long long)I.cg.ew * I.cg.en);
  I.nx1 = nx1; I.nx2 = nx2; I.sx = sx; I.sy = sy;
  I.nframe = g.js * sx + (sy - g.je - 1) * sx + nx2 * 2 * g.is;
  return I;
}

static int host_items(const InstGeom& I, int ph) {
  auto bf = [](long long n) { return (int)((n + kThreads - 1) / kThreads); };
  switch (ph) {
  case 0: return I.pg.nx_blocks + I.pg.ny_blocks;
  case 1: return bf((long long)(I.nx1 + 3) * (I.nx2 + 3));
  case 2: return I.cg.xb + I.cg.yb + I.cg.eb;
  case 3: return bf((long long)(I.nx1 + 1) * (I.nx2 + 1));
  case 4: return bf((long long)I.nx1 * I.nx2);
  default: return bf(I.nframe);
  }
}

static void release(athb_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->pool); cudaFree(b->st); cudaFree(b->cur); cudaFree(b->ghost_left); cudaFree(b->off);
  cudaFree(b->ids);
  cudaFree(b->dgeom); cudaFree(b->bar); cudaFree(b->err);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// Work-item tables over the active instances (b->active).  The graph reads
// the tables through fixed device pointers, so it stays valid.
static int upload_work(athb_batch* b) {
  const int n = b->n, na = (int)b->active.size();
  std::vector<int> off((size_t)kPhases * (n + 1), 0);
  for (int ph = 0; ph < kPhases; ph++) {
    int acc = 0;
    for (int a = 0; a < na; a++) {
      off[(size_t)ph * (n + 1) + a] = acc;
      acc += host_items(b->geom[b->active[a]], ph);
    }
    off[(size_t)ph * (n + 1) + na] = acc;
  }
  std::vector<int> ids(n + 1, 0);
  for (int a = 0; a < na; a++) ids[a] = b->active[a];
  ids[n] = na;
  CUDA_TRY(cudaMemcpyAsync(b->off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaMemcpyAsync(b->ids, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return ATHB_OK;
}

// (Re)build the device geometry and work-item tables from cfg/ly.
static int upload_tables(athb_batch* b) {
  const int n = b->n;
  std::vector<unsigned int> gl(n);
  for (int k = 0; k < n; k++) gl[k] = (unsigned int)host_items(b->geom[k], kPhases - 1);
  CUDA_TRY(cudaMemcpyAsync(b->dgeom, b->geom.data(), n * sizeof(InstGeom), cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaMemcpyAsync(b->ghost_left, gl.data(), n * sizeof(unsigned int), cudaMemcpyHostToDevice, b->stream));
  if (b->active.empty()) {
    b->active.resize(n);
    for (int k = 0; k < n; k++) b->active[k] = k;
  }
  return upload_work(b);
}

extern "C" int athb_batch_create(int n, const athb_config* cfgs, athb_batch** out) {
  if (!out || n < 1 || !cfgs) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  *out = nullptr;
  for (int k = 0; k < n; k++) {
    int rc = athb_ctx_validate(&cfgs[k]);
    if (rc) return rc;
    if (cfgs[k].flux != cfgs[0].flux || cfgs[k].device != cfgs[0].device)
      return athb_fail(ATHB_ERR_ARG, "all instances of a batch share flux and device");
  }
  athb_batch* b = new athb_batch();
  b->n = n;
  b->flux = cfgs[0].flux;
  b->device = cfgs[0].device;
  b->cfg.assign(cfgs, cfgs + n);
  b->ly.resize(n);
  for (int k = 0; k < n; k++) b->ly[k] = pick_ly(cfgs[k].nx1, cfgs[k].nx2);
  // one pool: per instance two state buffers and the scratch planes
  std::vector<size_t> base(n);
  size_t total = 0;
  for (int k = 0; k < n; k++) {
    const int sx = cfgs[k].nx1 + 2 * kNghost, sy = cfgs[k].nx2 + 2 * kNghost;
    const size_t ps = (size_t)((sx + 15) & ~15) * sy;
    base[k] = total;
    total += ps * (2 * NSTATE + NSCRATCH);
    total = (total + 31) & ~(size_t)31;  // 256-byte alignment
  }
  cudaError_t e = cudaSetDevice(b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&b->pool, total * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->st, n * sizeof(StepState));
  if (e == cudaSuccess) e = cudaMalloc(&b->cur, n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->ghost_left, n * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&b->off, (size_t)kPhases * (n + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->ids, (size_t)(n + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->dgeom, n * sizeof(InstGeom));
  if (e == cudaSuccess) e = cudaMalloc(&b->bar, sizeof(BarrierState));
  if (e == cudaSuccess) e = cudaMalloc(&b->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->pool, 0, total * sizeof(double), b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->cur, 0, n * sizeof(int), b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->bar, 0, sizeof(BarrierState), b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->err, 0, sizeof(int), b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->st, 0, n * sizeof(StepState), b->stream);
  if (e != cudaSuccess) {
    release(b);
    return athb_fail(e == cudaErrorMemoryAllocation ? ATHB_ERR_NOMEM : ATHB_ERR_CUDA, "athb_batch_create: %s",
                     cudaGetErrorString(e));
  }
  b->geom.resize(n);
  for (int k = 0; k < n; k++) {
    const int sx = cfgs[k].nx1 + 2 * kNghost, sy = cfgs[k].nx2 + 2 * kNghost;
    const size_t ps = (size_t)((sx + 15) & ~15) * sy;
    double* p = b->pool + base[k];
    b->geom[k] = make_geom(cfgs[k], b->ly[k], p, p + ps * NSTATE, p + 2 * ps * NSTATE, b->st + k);
  }
  int rc = upload_tables(b);
  if (rc) { release(b); return rc; }
  // persistent grid: co-resident blocks on every SM
  int sms = 0, per_sm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  if (b->flux == ATHB_FLUX_HLLE)
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_step<kFluxHlle>, kThreads, 0));
  else
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_step<kFluxRoe>, kThreads, 0));
  b->grid = sms * std::max(1, per_sm);
  *out = b;
  return ATHB_OK;
}

extern "C" void athb_batch_destroy(athb_batch* b) { release(b); }

extern "C" int athb_batch_size(const athb_batch* b) { return b ? b->n : 0; }

// Per-size-class y-march segment lengths (set by the autotuner).
extern "C" int athb_batch_set_ly(athb_batch* b, int k, int ly) {
  if (!b || k < 0 || k >= b->n || ly < 1) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  b->ly[k] = ly;
  InstGeom& I = b->geom[k];
  const double* s0 = I.g.in;
  b->geom[k] = make_geom(b->cfg[k], ly, const_cast<double*>(s0), I.g.out, I.g.scr, I.g.st);
  return ATHB_OK;
}
extern "C" int athb_batch_commit(athb_batch* b) {
  if (!b) return athb_fail(ATHB_ERR_ARG, "null batch");
  return upload_tables(b);
}
extern "C" int athb_batch_set_grid(athb_batch* b, int blocks) {
  if (!b || blocks < 1) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  int sms = 0, per_sm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  if (b->flux == ATHB_FLUX_HLLE)
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_step<kFluxHlle>, kThreads, 0));
  else
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_step<kFluxRoe>, kThreads, 0));
  if (blocks > sms * per_sm) return athb_fail(ATHB_ERR_ARG, "more blocks than can be co-resident");
  b->grid = blocks;
  return ATHB_OK;
}

// Load instance k's state (host SoA planes, as athb_upload) and its clock.
extern "C" int athb_batch_upload(athb_batch* b, int k, const double* planes, double dt, double time, int nstep) {
  if (!b || k < 0 || k >= b->n || !planes) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  const InstGeom& I = b->geom[k];
  int cur = 0;
  CUDA_TRY(cudaMemcpy(&cur, b->cur + k, sizeof(int), cudaMemcpyDeviceToHost));
  double* dst = cur ? I.g.out : const_cast<double*>(I.g.in);
  CUDA_TRY(cudaMemcpy2DAsync(dst, sizeof(double) * I.g.pitch, planes, sizeof(double) * I.sx,
                             sizeof(double) * I.sx, (size_t)I.sy * NSTATE, cudaMemcpyHostToDevice, b->stream));
  StepState h{};
  const athb_config& c = b->cfg[k];
  h.dt = dt; h.time = time; h.tlim = c.tlim; h.cour_no = c.cour_no; h.nstep = nstep; h.nlim = c.nlim;
  h.done = !((time < c.tlim) && (c.nlim < 0 || nstep < c.nlim));
  h.dtodx1 = dt / I.g.dx1; h.dtodx2 = dt / I.g.dx2;
  h.hdtodx1 = 0.5 * h.dtodx1; h.hdtodx2 = 0.5 * h.dtodx2; h.hdt = 0.5 * dt;
  CUDA_TRY(cudaMemcpyAsync(b->st + k, &h, sizeof h, cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return ATHB_OK;
}

extern "C" int athb_batch_download(athb_batch* b, int k, double* planes, double* dt, double* time, int* nstep) {
  if (!b || k < 0 || k >= b->n) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  const InstGeom& I = b->geom[k];
  int cur = 0;
  CUDA_TRY(cudaMemcpyAsync(&cur, b->cur + k, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  const double* src = cur ? I.g.out : I.g.in;
  if (planes)
    CUDA_TRY(cudaMemcpy2DAsync(planes, sizeof(double) * I.sx, src, sizeof(double) * I.g.pitch,
                               sizeof(double) * I.sx, (size_t)I.sy * NSTATE, cudaMemcpyDeviceToHost, b->stream));
  StepState h;
  CUDA_TRY(cudaMemcpyAsync(&h, b->st + k, sizeof h, cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (dt) *dt = h.dt;
  if (time) *time = h.time;
  if (nstep) *nstep = h.nstep;
  return ATHB_OK;
}

// set_bvals + first new_dt of every instance (src/main.c:139-149), with the
// single-grid kernels.
extern "C" int athb_batch_prepare(athb_batch* b) {
  if (!b) return athb_fail(ATHB_ERR_ARG, "null batch");
  CUDA_TRY(cudaSetDevice(b->device));
  std::vector<int> cur(b->n);
  CUDA_TRY(cudaMemcpy(cur.data(), b->cur, b->n * sizeof(int), cudaMemcpyDeviceToHost));
  for (int k = 0; k < b->n; k++) {
    const InstGeom& I = b->geom[k];
    GridArgs g = I.g;
    if (cur[k]) { const double* a = g.in; g.in = g.out; g.out = const_cast<double*>(a); }
    GridArgs gg = g;  // ghost fill writes the current buffer
    gg.out = const_cast<double*>(g.in);
    k_ghost<<<(I.nframe + kThreads - 1) / kThreads, kThreads, 0, b->stream>>>(gg, I.sx, I.sy, I.nframe, 3, 3);
    const int ncell = I.nx1 * I.nx2;
    k_cfl<<<(ncell + kThreads - 1) / kThreads, kThreads, 0, b->stream>>>(g, I.nx1, ncell);
    k_finalize<<<1, 1, 0, b->stream>>>(b->st + k, g.dx1, g.dx2, 0);
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return ATHB_OK;
}

static int launch_step(athb_batch* b) {
  BatchDev D;
  D.inst = b->dgeom; D.st = b->st; D.cur = b->cur; D.ghost_left = b->ghost_left; D.off = b->off;
  D.ids = b->ids;
  D.n = b->n; D.bar = b->bar; D.err = b->err;
  void* args[] = {&D};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(b->grid);
  cfg.blockDim = dim3(kThreads);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (b->flux == ATHB_FLUX_HLLE)
    CUDA_TRY(cudaLaunchKernelExC(&cfg, (const void*)k_batch_step<kFluxHlle>, args));
  else
    CUDA_TRY(cudaLaunchKernelExC(&cfg, (const void*)k_batch_step<kFluxRoe>, args));
  return ATHB_OK;
}

// Launch nsteps persistent steps (one cooperative launch each; captured in a
// CUDA graph when the driver allows it) without synchronising.
extern "C" int athb_batch_run_async(athb_batch* b, int nsteps) {
  if (!b || nsteps < 0) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  if (!b->graph && !b->graph_tried) {
    b->graph_tried = true;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      int rc = launch_step(b);
      cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
      if (rc == ATHB_OK && e == cudaSuccess && graph) {
        if (cudaGraphInstantiate(&b->graph, graph, 0) != cudaSuccess) b->graph = nullptr;
      }
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
    }
  }
  for (int s = 0; s < nsteps; s++) {
    if (b->graph) CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
    else { int rc = launch_step(b); if (rc) return rc; }
  }
  return ATHB_OK;
}

// Run until every instance is done (or max_steps launches).  Launches as
// many steps as the earliest-finishing active instance still needs, then
// re-reads the clocks; instances that finished are dropped from the work
// tables.  Returns the number of launches.
extern "C" int athb_batch_run(athb_batch* b, int max_steps, int* launches) {
  if (!b) return athb_fail(ATHB_ERR_ARG, "null batch");
  CUDA_TRY(cudaSetDevice(b->device));
  std::vector<StepState> h(b->n);
  int done_launches = 0;
  for (;;) {
    CUDA_TRY(cudaMemcpyAsync(h.data(), b->st, b->n * sizeof(StepState), cudaMemcpyDeviceToHost, b->stream));
    int err = 0;
    CUDA_TRY(cudaMemcpyAsync(&err, b->err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (err) {
      if (launches) *launches = done_launches;
      return athb_fail(ATHB_ERR_STATE, "batch grid barrier timed out");
    }
    std::vector<int> act;
    long long want = -1;
    for (int k = 0; k < b->n; k++) {
      if (h[k].flags) {
        if (launches) *launches = done_launches;
        return athb_fail(ATHB_ERR_STATE, "instance %d: non-finite CFL rate", k);
      }
      if (h[k].done) continue;
      act.push_back(k);
      const double est = (h[k].tlim - h[k].time) / h[k].dt;
      long long need = est < 1.0 ? 1 : (long long)std::ceil(est);
      if (h[k].nlim >= 0) need = std::min<long long>(need, std::max(1, h[k].nlim - h[k].nstep));
      want = want < 0 ? need : std::min(want, need);
    }
    if (act.empty() || done_launches >= max_steps) break;
    if (act != b->active) {
      b->active = act;
      int rc = upload_work(b);
      if (rc) return rc;
    }
    want = std::min<long long>(want, max_steps - done_launches);
    int rc = athb_batch_run_async(b, (int)want);
    if (rc) return rc;
    done_launches += (int)want;
  }
  if (launches) *launches = done_launches;
  return ATHB_OK;
}

extern "C" int athb_batch_synchronize(athb_batch* b) {
  if (!b) return athb_fail(ATHB_ERR_ARG, "null batch");
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  int err = 0;
  CUDA_TRY(cudaMemcpy(&err, b->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return athb_fail(ATHB_ERR_STATE, "batch grid barrier timed out");
  return ATHB_OK;
}

extern "C" void* athb_batch_stream(athb_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" int athb_batch_grid(const athb_batch* b) { return b ? b->grid : 0; }
