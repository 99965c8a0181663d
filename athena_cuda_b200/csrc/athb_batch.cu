// athb_batch.cu -- many independent grids of uneven size, each with its own
// dt and end time, advanced together: one launch per phase of the step for
// all instances (the default), or ONE persistent kernel launch per step.
//
// The persistent kernel walks six phases (predict, half-step corner EMF,
// correct, full-step corner EMF, update + CFL, ghost fill + finalize); in each
// phase the blocks of the launch take the (instance, block) work items of all
// active instances from a shared counter, and a grid-wide barrier separates
// the phases.
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
constexpr int kPhasedGraphMinSteps = 32;
constexpr int kRing256Bytes = 4 * 7 * 256 * (int)sizeof(double);   // predictor ring of 256-thread units
constexpr long long kBarrierSpins = 20000000;  // x ~64 ns sleep: ~1-2 s
constexpr int kBatchMinBlocks = 3;  // as k_predict: 168 registers per thread

struct InstGeom {
  GridArgs g;  // g.in = state[0], g.out = state[1]
  PredictGeom pg;
  CorrectGeom cg;
  int nx1, nx2, sx, sy, nframe;
  int nt;      // threads per work unit (the block size of the phase launches)
  int pad;
};

struct BarrierState {
  unsigned int count;
  unsigned int gen;
};

// Units of work: the 128-thread blocks of the single-grid kernels.  The work
// map has kSegs segments: the predictor's role-Y units of every active
// instance, then its role-X units (so every long column march of the phase
// is handed out before any short row segment and the phase ends on short
// work), then one segment per later phase.  A work item is a chunk of up to
// chunk_of(seg) consecutive units of one instance; item w of segment s is
// wmap[mbase[s] + w].  Chunks amortise the per-item cost (ticket, lookup,
// barriers) over several units; short units take longer chunks.
constexpr int kSegs = kPhases + 1;
enum Seg { kSegPredictY = 0, kSegPredictX, kSegEmfHalf, kSegCorrect, kSegEmfFull, kSegUpdate, kSegGhost };
__host__ __device__ constexpr int seg_first(int ph) { return ph == 0 ? 0 : ph + 1; }  // phase -> first segment
__host__ __device__ constexpr int chunk_of(int seg) {
  return seg == kSegPredictY ? 1 : seg == kSegPredictX || seg == kSegCorrect ? 2
       : seg == kSegEmfHalf || seg == kSegEmfFull ? 8 : 4;
}

struct __align__(16) WorkItem {
  int id, b0, nb, pad;
};

struct BatchDev {
  const InstGeom* inst;
  StepState* st;
  int* cur;
  unsigned int* ghost_left;
  const int* mbase;     // kSegs + 1: start of each segment's items in wmap
  const WorkItem* wmap;
  unsigned int* tick;   // kPhases work counters (dynamic item assignment)
  int n;
  BarrierState* bar;
  int* err;
  unsigned long long* timing;  // optional: ns spent per phase, accumulated by block 0
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Units of instance I in map segment seg.
__host__ __device__ inline int item_count(const InstGeom& I, int seg) {
  const int nt = I.nt;
  auto bf = [nt](long long n) { return (int)((n + nt - 1) / nt); };
  switch (seg) {
  case kSegPredictY: return I.pg.ny_blocks;
  case kSegPredictX: return I.pg.nx_blocks;
  case kSegEmfHalf: return bf((long long)(I.nx1 + 3) * (I.nx2 + 3));
  case kSegCorrect: return I.cg.xb + I.cg.yb + I.cg.eb;
  case kSegEmfFull: return bf((long long)(I.nx1 + 1) * (I.nx2 + 1));
  case kSegUpdate: return bf((long long)I.nx1 * I.nx2);
  default: return bf(I.nframe);
  }
}

// Wait until `blocks` blocks have arrived.  A block that waits longer than
// `spins` polls gives up: it sets *err and carries on, so a launch whose
// blocks cannot all arrive ends with an error status instead of a hang.
__device__ void grid_barrier_n(BarrierState* bar, int* err, unsigned int blocks, long long spins) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &bar->gen;
    const unsigned int gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&bar->count, 1u) + 1u;
    if (arrived == blocks) {
      bar->count = 0u;
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      long long n = 0;
      while (*vgen == gen) {
        __nanosleep(64);
        if (++n > spins) { atomicExch(err, 1); break; }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

__device__ void grid_barrier(const BatchDev& B) { grid_barrier_n(B.bar, B.err, gridDim.x, kBarrierSpins); }

// Self-test of the bounded wait: one block waits for two at a barrier.
__global__ void k_barrier_selftest(BarrierState* bar, int* err, long long spins) {
  grid_barrier_n(bar, err, 2u, spins);
}

// Copy instance k's geometry into shared memory (all threads), with the
// state buffers swapped when its current state is in the second buffer.
__device__ __forceinline__ void load_geom(const BatchDev& B, InstGeom& s_I, int k, int cur) {
  constexpr int kWords = (int)(sizeof(InstGeom) / sizeof(unsigned long long));
  static_assert(sizeof(InstGeom) % sizeof(unsigned long long) == 0, "InstGeom copy granularity");
  static_assert(kWords <= 64, "InstGeom copy width (the smallest block has 64 threads)");
  if (threadIdx.x < kWords)
    reinterpret_cast<unsigned long long*>(&s_I)[threadIdx.x] =
        reinterpret_cast<const unsigned long long*>(&B.inst[k])[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0 && cur) {
    const double* a = s_I.g.in;
    s_I.g.in = s_I.g.out;
    s_I.g.out = const_cast<double*>(a);
  }
  __syncthreads();
}

// Units b0 .. b0+nb-1 of phase ph of instance k (geometry I), NT threads
// per unit (the block size).
template <int FLUX, int NT>
__device__ __forceinline__ void run_chunk(const BatchDev& B, int ph, int k, int b0, int nb, const InstGeom& I) {
  const GridArgs& g = I.g;
  switch (ph) {
  case 0:
    for (int u = 0; u < nb; u++) predict_block<FLUX, false, NT>(g, I.pg, b0 + u);
    break;
  case 1:
    for (int u = 0; u < nb; u++)
      emf_item(g, g.is - 1, g.js - 1, I.nx1 + 3, I.nx2 + 3, S_FX, S_FY, (b0 + u) * NT + threadIdx.x);
    break;
  case 2:
    for (int u = 0; u < nb; u++) correct_block<FLUX, NT>(g, I.cg, b0 + u);
    break;
  case 3:
    for (int u = 0; u < nb; u++)
      emf_item(g, g.is, g.js, I.nx1 + 1, I.nx2 + 1, S_FX2, S_FY2, (b0 + u) * NT + threadIdx.x);
    break;
  case 4: {
    // the CFL rate max over the chunk, then one block reduction (max is
    // order-independent, so dt is the single-grid value)
    double m = 0.0;
    bool bad = false;
    for (int u = 0; u < nb; u++) {
      const double v = update_cell(g, I.nx1, I.nx1 * I.nx2, (b0 + u) * NT + threadIdx.x);
      if (!(v >= 0.0) || isinf(v)) bad = true;
      else m = fmax(m, v);
    }
    if (bad) atomicOr(&g.st->flags, kErrNonFinite);
    block_max_to<NT>(m, &g.st->max_dti_bits, &g.st->flags);
    break;
  }
  default: {
    for (int u = 0; u < nb; u++) ghost_item(g, I.sx, I.sy, I.nframe, 3, 3, (b0 + u) * NT + threadIdx.x);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicSub(&B.ghost_left[k], (unsigned int)nb) == (unsigned int)nb) {
        // last ghost unit of instance k: end of its step
        __threadfence();
        B.ghost_left[k] = (unsigned int)item_count(I, kSegGhost);
        finalize_state(B.st[k], g.dx1, g.dx2, 1);
        B.cur[k] ^= 1;
        __threadfence();
      }
    }
    break;
  }
  }
}

// The persistent kernel: all six phases of a step, grid barriers between
// them.  In each phase a block takes its items from the phase's counter
// (dynamic assignment, so long and short items balance as under the hardware
// block scheduler) one item ahead: the ticket of the next item is requested
// when an item starts and read when it ends.
template <int FLUX>
__global__ void __launch_bounds__(kThreads, kBatchMinBlocks) k_batch_step(BatchDev B) {
  // the current work item's instance data, loaded when the instance changes
  __shared__ InstGeom s_I;
  __shared__ int s_k, s_b, s_nb, s_skip, s_load, s_w;
  unsigned long long t_phase = (B.timing && blockIdx.x == 0 && threadIdx.x == 0) ? global_ns() : 0ull;
  int k_prev = -1;  // instance held in s_I
  int cur_prev = -1;
  for (int ph = 0; ph < kPhases; ph++) {
    const int base = B.mbase[seg_first(ph)];
    const int total = B.mbase[seg_first(ph + 1)] - base;
    unsigned int* tick = B.tick + ph;
    if (threadIdx.x == 0) {
      // every block is past the previous phase: its counter is free again
      if (blockIdx.x == 0) B.tick[ph == 0 ? kPhases - 1 : ph - 1] = 0u;
      s_w = (int)atomicAdd(tick, 1u);
    }
    __syncthreads();
    int w = s_w;
    while (w < total) {
      unsigned int nxt = 0u;
      if (threadIdx.x == 0) {
        nxt = atomicAdd(tick, 1u);
        const WorkItem it = B.wmap[base + w];
        s_k = it.id;
        s_b = it.b0;
        s_nb = it.nb;
        s_skip = *(volatile int*)&B.st[it.id].done;
        const int cur = s_skip ? 0 : *(volatile int*)&B.cur[it.id];
        s_load = (!s_skip && (it.id != k_prev || cur != cur_prev)) ? (cur + 1) : 0;
      }
      __syncthreads();  // S1: the item is known (and every thread has read s_w)
      if (s_skip) {
        k_prev = -1;  // instance has reached its end time
      } else {
        if (s_load) {
          load_geom(B, s_I, s_k, s_load - 1);
          k_prev = s_k;
          cur_prev = s_load - 1;
        }
        run_chunk<FLUX, kThreads>(B, ph, s_k, s_b, s_nb, s_I);
      }
      if (threadIdx.x == 0) s_w = (int)nxt;
      __syncthreads();  // S2: the item is finished with s_I; the next ticket is visible
      w = s_w;
    }
    if (ph < kPhases - 1) grid_barrier(B);
    if (B.timing && blockIdx.x == 0 && threadIdx.x == 0) {
      const unsigned long long now = global_ns();
      atomicAdd(&B.timing[ph], now - t_phase);
      t_phase = now;
    }
  }
}

// Phased execution: one launch per phase, one work item per block (the
// hardware block scheduler balances), each phase with the register budget of
// its single-grid kernel.
// The register budget per thread stays that of the 128-thread single-grid
// kernels where the block size allows it (64 threads: twice the blocks).
template <int PH, int NT>
struct PhaseBlocks {
  static constexpr int at128 = PH == 0 ? kPredictMinBlocks : PH == 2 ? kCorrectMinBlocks : 1;
  static constexpr int value = at128 * kThreads / NT > 0 ? at128 * kThreads / NT : 1;
};

template <int FLUX, int PH, int NT>
__global__ void __launch_bounds__(NT, (PhaseBlocks<PH, NT>::value)) k_batch_phase(BatchDev B) {
  __shared__ InstGeom s_I;
  __shared__ int s_k, s_b, s_nb, s_cur;
  const int base = B.mbase[seg_first(PH)];
  if ((int)blockIdx.x >= B.mbase[seg_first(PH + 1)] - base) return;
  if (threadIdx.x == 0) {
    const WorkItem it = B.wmap[base + blockIdx.x];
    s_k = it.id;
    s_b = it.b0;
    s_nb = it.nb;
    s_cur = B.st[it.id].done ? -1 : B.cur[it.id];
  }
  __syncthreads();
  if (s_cur < 0) return;  // instance has reached its end time
  load_geom(B, s_I, s_k, s_cur);
  run_chunk<FLUX, NT>(B, PH, s_k, s_b, s_nb, s_I);
}

// Phase timing of the phased mode: the time since the previous stamp, added
// to timing[ph] (ph < 0 only sets the stamp); timing[kPhases] holds it.
__global__ void k_stamp(unsigned long long* timing, int ph) {
  const unsigned long long now = global_ns();
  if (ph >= 0) timing[ph] += now - timing[kPhases];
  timing[kPhases] = now;
}

// wmap of the active instances: block (a, seg) writes the chunks of active
// slot a in segment seg.  Role-X units follow the role-Y units in the
// predictor's block numbering (predict_block).
__global__ void k_build_map(const InstGeom* inst, const int* off, const int* mbase, const int* ids, int n,
                            WorkItem* wmap) {
  const int a = blockIdx.x, seg = blockIdx.y;
  if (a >= ids[n]) return;
  const int* o = off + seg * (n + 1);
  const int i0 = o[a], i1 = o[a + 1];
  const int id = ids[a];
  const int units = item_count(inst[id], seg), r = chunk_of(seg);
  const int first = seg == kSegPredictX ? inst[id].pg.ny_blocks : 0;
  WorkItem* m = wmap + mbase[seg];
  for (int w = i0 + threadIdx.x; w < i1; w += blockDim.x) {
    const int u = (w - i0) * r;
    m[w] = WorkItem{id, first + u, min(r, units - u), 0};
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
  int* off = nullptr;           // kSegs x (n+1) item prefix sums, then mbase (kSegs+1)
  WorkItem* wmap = nullptr;     // item -> (instance, block), built on the device
  size_t wmap_cap = 0;
  unsigned int* tick = nullptr; // kPhases work counters
  int* ids = nullptr;
  std::vector<int> active;     // ids of the instances in the work tables
  InstGeom* dgeom = nullptr;
  BarrierState* bar = nullptr;
  int* err = nullptr;
  unsigned long long* timing = nullptr;  // per-phase ns (when enabled), then a stamp
  bool timing_on = false;
  int mode = ATHB_BATCH_PHASED;
  int nt = kThreads;           // threads per work unit (phased mode: 64, 128 or 256)
  int phase_total[kPhases] = {0, 0, 0, 0, 0, 0};  // work items per phase (active set)
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
static InstGeom make_geom(const athb_config& c, int ly, int nt, double* state0, double* state1, double* scr,
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
  I.nt = nt;
  I.pg = make_predict_geom(nx1, nx2, ly, nt);
  I.cg.xw = nx1 + 1; I.cg.xn = nx2 + 3;
  I.cg.yw = nx1 + 3; I.cg.yn = nx2 + 1;
  I.cg.ew = nx1 + 3; I.cg.en = nx2 + 3;
  auto bf = [nt](long long n) { return (int)((n + nt - 1) / nt); };
  I.cg.xb = bf((long long)I.cg.xw * I.cg.xn);
  I.cg.yb = bf((long long)I.cg.yw * I.cg.yn);
  I.cg.eb = bf((long long)I.cg.ew * I.cg.en);
  I.nx1 = nx1; I.nx2 = nx2; I.sx = sx; I.sy = sy;
  I.nframe = g.js * sx + (sy - g.je - 1) * sx + nx2 * 2 * g.is;
  return I;
}

static int host_chunks(const InstGeom& I, int seg) {
  return (item_count(I, seg) + chunk_of(seg) - 1) / chunk_of(seg);
}

static void release(athb_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->pool); cudaFree(b->st); cudaFree(b->cur); cudaFree(b->ghost_left); cudaFree(b->off);
  cudaFree(b->ids); cudaFree(b->wmap); cudaFree(b->tick);
  cudaFree(b->dgeom); cudaFree(b->bar); cudaFree(b->err); cudaFree(b->timing);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// The captured step launches; it is captured again on the next run.
static void drop_graph(athb_batch* b) {
  if (b->graph) {
    cudaStreamSynchronize(b->stream);
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->graph_tried = false;
}

// Work-item tables over the active instances (b->active).  The graph reads
// the tables through fixed device pointers, so it stays valid.
static int upload_work(athb_batch* b) {
  const int n = b->n, na = (int)b->active.size();
  std::vector<int> off((size_t)kSegs * (n + 1) + kSegs + 1, 0);
  int* mbase = off.data() + (size_t)kSegs * (n + 1);
  for (int seg = 0; seg < kSegs; seg++) {
    int acc = 0;
    for (int a = 0; a < na; a++) {
      off[(size_t)seg * (n + 1) + a] = acc;
      acc += host_chunks(b->geom[b->active[a]], seg);
    }
    off[(size_t)seg * (n + 1) + na] = acc;
    mbase[seg + 1] = mbase[seg] + acc;
  }
  for (int ph = 0; ph < kPhases; ph++) b->phase_total[ph] = mbase[seg_first(ph + 1)] - mbase[seg_first(ph)];
  if ((size_t)mbase[kSegs] > b->wmap_cap)
    return athb_fail(ATHB_ERR_STATE, "work map capacity %zu < %d items", b->wmap_cap, mbase[kSegs]);
  std::vector<int> ids(n + 1, 0);
  for (int a = 0; a < na; a++) ids[a] = b->active[a];
  ids[n] = na;
  CUDA_TRY(cudaMemcpyAsync(b->off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaMemcpyAsync(b->ids, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  if (na > 0) {
    k_build_map<<<dim3(na, kSegs), kThreads, 0, b->stream>>>(b->dgeom, b->off, b->off + (size_t)kSegs * (n + 1),
                                                                b->ids, n, b->wmap);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  // the phased step's graph holds the phase grid sizes of the old tables
  if (b->mode == ATHB_BATCH_PHASED) drop_graph(b);
  return ATHB_OK;
}

// (Re)build the device geometry and work-item tables from cfg/ly.
static int upload_tables(athb_batch* b) {
  const int n = b->n;
  std::vector<unsigned int> gl(n);
  for (int k = 0; k < n; k++) gl[k] = (unsigned int)item_count(b->geom[k], kSegGhost);
  CUDA_TRY(cudaMemcpyAsync(b->dgeom, b->geom.data(), n * sizeof(InstGeom), cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaMemcpyAsync(b->ghost_left, gl.data(), n * sizeof(unsigned int), cudaMemcpyHostToDevice, b->stream));
  if (b->active.empty()) {
    b->active.resize(n);
    for (int k = 0; k < n; k++) b->active[k] = k;
  }
  size_t items = 0;  // every instance active: the largest map
  for (int k = 0; k < n; k++)
    for (int seg = 0; seg < kSegs; seg++) items += (size_t)host_chunks(b->geom[k], seg);
  if (items > b->wmap_cap) {
    drop_graph(b);
    cudaFree(b->wmap);
    b->wmap = nullptr;
    b->wmap_cap = 0;
    CUDA_TRY(cudaMalloc(&b->wmap, items * sizeof(WorkItem)));
    b->wmap_cap = items;
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
  if (e == cudaSuccess) e = cudaMalloc(&b->off, ((size_t)kSegs * (n + 1) + kSegs + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->tick, kPhases * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->tick, 0, kPhases * sizeof(unsigned int), b->stream);
  if (e == cudaSuccess) e = cudaMalloc(&b->ids, (size_t)(n + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->dgeom, n * sizeof(InstGeom));
  if (e == cudaSuccess) e = cudaMalloc(&b->bar, sizeof(BarrierState));
  if (e == cudaSuccess) e = cudaMalloc(&b->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->timing, (kPhases + 1) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->timing, 0, (kPhases + 1) * sizeof(unsigned long long), b->stream);
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
    b->geom[k] = make_geom(cfgs[k], b->ly[k], b->nt, p, p + ps * NSTATE, p + 2 * ps * NSTATE, b->st + k);
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
  b->geom[k] = make_geom(b->cfg[k], ly, b->nt, const_cast<double*>(s0), I.g.out, I.g.scr, I.g.st);
  return ATHB_OK;
}

// Threads per work unit of the phased launches (64, 128 or 256), applied to
// every instance by athb_batch_commit.  The persistent kernel keeps 128.
extern "C" int athb_batch_set_threads(athb_batch* b, int nt) {
  if (!b || (nt != 64 && nt != 128 && nt != 256)) return athb_fail(ATHB_ERR_ARG, "threads per unit: 64, 128 or 256");
  if (nt != kThreads && b->mode != ATHB_BATCH_PHASED)
    return athb_fail(ATHB_ERR_ARG, "the persistent mode runs 128-thread units");
  if (nt == 256) {
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaFuncSetAttribute(k_batch_phase<kFluxRoe, 0, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kRing256Bytes));
    CUDA_TRY(cudaFuncSetAttribute(k_batch_phase<kFluxHlle, 0, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kRing256Bytes));
  }
  b->nt = nt;
  for (int k = 0; k < b->n; k++) {
    InstGeom& I = b->geom[k];
    b->geom[k] = make_geom(b->cfg[k], b->ly[k], nt, const_cast<double*>(I.g.in), I.g.out, I.g.scr, I.g.st);
  }
  return ATHB_OK;
}
extern "C" int athb_batch_threads(const athb_batch* b) { return b ? b->nt : -1; }
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

// Instance k's clock (dt as the reference Grid holds it; the next step takes
// it after the tlim clamp, src/main.c:230-232).
static int set_inst_clock(athb_batch* b, int k, double dt, double time, int nstep) {
  const InstGeom& I = b->geom[k];
  const athb_config& c = b->cfg[k];
  StepState h{};
  h.time = time; h.tlim = c.tlim; h.cour_no = c.cour_no; h.nstep = nstep; h.nlim = c.nlim;
  h.done = !((time < c.tlim) && (c.nlim < 0 || nstep < c.nlim));
  h.dt_new = dt;
  h.dt = (!h.done && (h.tlim - time) < dt) ? (h.tlim - time) : dt;
  h.dtodx1 = h.dt / I.g.dx1; h.dtodx2 = h.dt / I.g.dx2;
  h.hdtodx1 = 0.5 * h.dtodx1; h.hdtodx2 = 0.5 * h.dtodx2; h.hdt = 0.5 * h.dt;
  CUDA_TRY(cudaMemcpyAsync(b->st + k, &h, sizeof h, cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return ATHB_OK;
}

// The buffer holding instance k's current state.
static int inst_state(athb_batch* b, int k, double** state) {
  const InstGeom& I = b->geom[k];
  int cur = 0;
  CUDA_TRY(cudaMemcpy(&cur, b->cur + k, sizeof(int), cudaMemcpyDeviceToHost));
  *state = cur ? I.g.out : const_cast<double*>(I.g.in);
  return ATHB_OK;
}

// Load instance k's state (host SoA planes, as athb_upload) and its clock.
extern "C" int athb_batch_upload(athb_batch* b, int k, const double* planes, double dt, double time, int nstep) {
  if (!b || k < 0 || k >= b->n || !planes) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  const InstGeom& I = b->geom[k];
  double* dst = nullptr;
  int rc = inst_state(b, k, &dst);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpy2DAsync(dst, sizeof(double) * I.g.pitch, planes, sizeof(double) * I.sx,
                             sizeof(double) * I.sx, (size_t)I.sy * NSTATE, cudaMemcpyHostToDevice, b->stream));
  return set_inst_clock(b, k, dt, time, nstep);
}

// Instance k's initial condition formed on the GPU (built-in "blast" and
// "field_loop", as athb_generate); clock reset.  Other problems: upload.
extern "C" int athb_batch_generate(athb_batch* b, int k, const char* name, const athb_params* p) {
  if (!b || k < 0 || k >= b->n || !name || !p) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  const int kind = athb_builtin_problem(name);
  if (kind == kProblemNone)
    return athb_fail(ATHB_ERR_NOTFOUND, "problem \"%s\" has no device generator (use athb_batch_upload)", name);
  const InstGeom& I = b->geom[k];
  double* dst = nullptr;
  int rc = inst_state(b, k, &dst);
  if (rc) return rc;
  rc = athb_generate_device_into(kind, p, dst, I.g.scr + (size_t)S_EMF * I.g.ps, I.g.ps, I.g.pitch, b->cfg[k],
                                 b->stream);
  if (rc) return rc;
  return set_inst_clock(b, k, 0.0, 0.0, 0);
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
  if (dt) *dt = h.dt_new;
  if (time) *time = h.time;
  if (nstep) *nstep = h.nstep;
  return ATHB_OK;
}

// set_bvals + first new_dt of every instance (src/main.c:139-149), with the
// single-grid kernels.
extern "C" int athb_batch_prepare(athb_batch* b) {
  if (!b) return athb_fail(ATHB_ERR_ARG, "null batch");
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaMemsetAsync(b->tick, 0, kPhases * sizeof(unsigned int), b->stream));
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

static BatchDev batch_dev(const athb_batch* b) {
  BatchDev D;
  D.inst = b->dgeom; D.st = b->st; D.cur = b->cur; D.ghost_left = b->ghost_left;
  D.mbase = b->off + (size_t)kSegs * (b->n + 1);
  D.wmap = b->wmap;
  D.tick = b->tick;
  D.n = b->n; D.bar = b->bar; D.err = b->err;
  D.timing = b->timing_on ? b->timing : nullptr;
  return D;
}

template <int FLUX, int PH>
static cudaError_t launch_phase(const athb_batch* b, const BatchDev& D) {
  if (b->phase_total[PH] > 0) {
    if (b->nt == 64) k_batch_phase<FLUX, PH, 64><<<b->phase_total[PH], 64, 0, b->stream>>>(D);
    else if (b->nt == 256)   // the predictor's role-Y ring in dynamic shared memory (see predict_y)
      k_batch_phase<FLUX, PH, 256><<<b->phase_total[PH], 256, PH == 0 ? kRing256Bytes : 0, b->stream>>>(D);
    else k_batch_phase<FLUX, PH, kThreads><<<b->phase_total[PH], kThreads, 0, b->stream>>>(D);
  }
  if (b->timing_on) k_stamp<<<1, 1, 0, b->stream>>>(b->timing, PH);
  return cudaGetLastError();
}

template <int FLUX>
static int launch_phases(const athb_batch* b) {
  const BatchDev D = batch_dev(b);
  if (b->timing_on) k_stamp<<<1, 1, 0, b->stream>>>(b->timing, -1);
  CUDA_TRY((launch_phase<FLUX, 0>(b, D)));
  CUDA_TRY((launch_phase<FLUX, 1>(b, D)));
  CUDA_TRY((launch_phase<FLUX, 2>(b, D)));
  CUDA_TRY((launch_phase<FLUX, 3>(b, D)));
  CUDA_TRY((launch_phase<FLUX, 4>(b, D)));
  CUDA_TRY((launch_phase<FLUX, 5>(b, D)));
  return ATHB_OK;
}

static int launch_step(athb_batch* b) {
  if (b->mode == ATHB_BATCH_PHASED)
    return b->flux == ATHB_FLUX_HLLE ? launch_phases<kFluxHlle>(b) : launch_phases<kFluxRoe>(b);
  BatchDev D = batch_dev(b);
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

// Launch nsteps steps without synchronising: one step (persistent: one
// cooperative launch; phased: six launches) captured in a CUDA graph when
// CUDA accepts the capture, then one graph launch per step.  The phased graph
// is captured again whenever the work tables change (instances finishing),
// and only for calls of at least kPhasedGraphMinSteps steps.
extern "C" int athb_batch_run_async(athb_batch* b, int nsteps) {
  if (!b || nsteps < 0) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  // a phased graph is only worth capturing for a run of steps long enough to
  // amortise it (its phase sizes change whenever an instance finishes)
  const bool capture = b->mode == ATHB_BATCH_PERSISTENT || nsteps >= kPhasedGraphMinSteps;
  if (capture && !b->graph && !b->graph_tried) {
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

// Per-phase timing of the persistent kernel (block 0's view: each phase ends
// at the grid barrier): enable, then read ns accumulated per phase.
extern "C" int athb_batch_timing(athb_batch* b, int enable, double* ms_out) {
  if (!b) return athb_fail(ATHB_ERR_ARG, "null batch");
  if (ms_out) {
    unsigned long long t[kPhases];
    CUDA_TRY(cudaMemcpyAsync(t, b->timing, sizeof t, cudaMemcpyDeviceToHost, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (int k = 0; k < kPhases; k++) ms_out[k] = 1e-6 * (double)t[k];
  }
  if (enable >= 0 && (enable != 0) != b->timing_on) {
    b->timing_on = enable != 0;
    CUDA_TRY(cudaMemsetAsync(b->timing, 0, (kPhases + 1) * sizeof(unsigned long long), b->stream));
    drop_graph(b);
  }
  return ATHB_OK;
}

extern "C" int athb_batch_grid(const athb_batch* b) { return b ? b->grid : 0; }

// The failure path of the batch's grid barrier, on purpose: a single block
// waits at a barrier for two, gives up after `spins` polls (~64 ns each),
// records the time-out and returns; the device stays usable.  *timed_out is
// 1 when the wait ran out (the expected outcome).
extern "C" int athb_batch_selftest_barrier(int device, long long spins, int* timed_out) {
  if (!timed_out || spins < 1) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(device));
  BarrierState* bar = nullptr;
  int* err = nullptr;
  CUDA_TRY(cudaMalloc(&bar, sizeof(BarrierState)));
  cudaError_t e = cudaMalloc(&err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(bar, 0, sizeof(BarrierState));
  if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(int));
  if (e == cudaSuccess) {
    k_barrier_selftest<<<1, kThreads>>>(bar, err, spins);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(bar);
  cudaFree(err);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "barrier self-test: %s", cudaGetErrorString(e));
  *timed_out = h;
  return ATHB_OK;
}

// Execution mode: ATHB_BATCH_PERSISTENT (one cooperative launch per step) or
// ATHB_BATCH_PHASED (one launch per phase).  Results are identical.
extern "C" int athb_batch_set_mode(athb_batch* b, int mode) {
  if (!b || (mode != ATHB_BATCH_PERSISTENT && mode != ATHB_BATCH_PHASED))
    return athb_fail(ATHB_ERR_ARG, "bad arguments");
  if (mode == ATHB_BATCH_PERSISTENT && b->nt != kThreads)
    return athb_fail(ATHB_ERR_ARG, "the persistent mode runs 128-thread units (athb_batch_set_threads)");
  CUDA_TRY(cudaSetDevice(b->device));
  b->mode = mode;
  drop_graph(b);
  return ATHB_OK;
}
extern "C" int athb_batch_mode(const athb_batch* b) { return b ? b->mode : -1; }
