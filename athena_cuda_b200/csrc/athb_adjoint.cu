// athb_adjoint.cu -- the tangent-linear model and the adjoint of the main
// loop on the GPU: the sm_100a executor of adjoint_driver.cuh and the C ABI
// (athb_tlm_run, athb_adjoint_gradient).
//
// Every stage is one launch of a per-item kernel over its range on the
// context's stream; reductions (the CFL max with the cell that attains it,
// the adjoint of dt, the objective) are two-pass and deterministic: a fixed
// assignment of items to blocks, a fixed tree inside a block, blocks summed
// in order by one thread.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <vector>

#include "adjoint_driver.cuh"
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

constexpr int kItemThreads = 128;
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;   // 2 per SM of a B200

// Resident 128-thread blocks per SM each stage kernel is compiled for (the
// register cap = 65536 / (128 x blocks)); 1 leaves the compiler its choice.
#ifndef ATHB_ADJ_MINB_PLM
#define ATHB_ADJ_MINB_PLM 1
#endif
#ifndef ATHB_ADJ_MINB_RIE
#define ATHB_ADJ_MINB_RIE 1
#endif
#ifndef ATHB_ADJ_MINB_COR
#define ATHB_ADJ_MINB_COR 1
#endif
template <class F> struct ItemMinBlocks { static constexpr int value = 1; };
template <int STAGE, int FLUX> struct ItemMinBlocks<AdjFn<STAGE, FLUX>> {
  static constexpr int value = (STAGE == R_PLMX || STAGE == R_PLMY)   ? ATHB_ADJ_MINB_PLM
                               : (STAGE == R_RIEX || STAGE == R_RIEY) ? ATHB_ADJ_MINB_RIE
                               : (STAGE == R_CORX || STAGE == R_CORY) ? ATHB_ADJ_MINB_COR
                                                                      : 1;
};

template <class F>
__global__ void __launch_bounds__(kItemThreads, ItemMinBlocks<F>::value) k_items(GenRange r, long long n, F f) {
  const long long t = (long long)blockIdx.x * kItemThreads + threadIdx.x;
  if (t >= n) return;
  int j, i;
  range_item(r, t, j, i);
  f(j, i);
}

template <class F>
__global__ void k_single(F f) { f(); }

__global__ void __launch_bounds__(kRedThreads) k_argmax_part(const double* p, GenRange r, int pitch, long long n,
                                                             MaxLoc* part) {
  __shared__ double sm[kRedThreads];
  __shared__ long long sa[kRedThreads];
  double m = -INFINITY;
  long long arg = LLONG_MAX;
  for (long long t = (long long)blockIdx.x * kRedThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kRedThreads) {
    int j, i;
    range_item(r, t, j, i);
    const long long o = (long long)j * pitch + i;
    const double v = p[o];
    if (v > m || (v == m && o < arg)) { m = v; arg = o; }
  }
  sm[threadIdx.x] = m;
  sa[threadIdx.x] = arg;
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double m2 = sm[threadIdx.x + s];
      const long long a2 = sa[threadIdx.x + s];
      if (m2 > sm[threadIdx.x] || (m2 == sm[threadIdx.x] && a2 < sa[threadIdx.x])) {
        sm[threadIdx.x] = m2;
        sa[threadIdx.x] = a2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[blockIdx.x].m = sm[0]; part[blockIdx.x].arg = sa[0]; }
}

// one block: the partials folded by a fixed tree (max, then lowest index)
__global__ void __launch_bounds__(kRedThreads) k_argmax_final(const MaxLoc* part, int nb, long long first,
                                                              MaxLoc* out) {
  __shared__ double sm[kRedThreads];
  __shared__ long long sa[kRedThreads];
  double m = -INFINITY;
  long long arg = LLONG_MAX;
  for (int b = threadIdx.x; b < nb; b += kRedThreads)
    if (part[b].m > m || (part[b].m == m && part[b].arg < arg)) { m = part[b].m; arg = part[b].arg; }
  sm[threadIdx.x] = m;
  sa[threadIdx.x] = arg;
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double m2 = sm[threadIdx.x + s];
      const long long a2 = sa[threadIdx.x + s];
      if (m2 > sm[threadIdx.x] || (m2 == sm[threadIdx.x] && a2 < sa[threadIdx.x])) {
        sm[threadIdx.x] = m2;
        sa[threadIdx.x] = a2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out->m = sm[0];
    out->arg = sa[0] == LLONG_MAX ? first : sa[0];   // no comparable value (NaN everywhere): keep the index valid
  }
}

__global__ void __launch_bounds__(kRedThreads) k_sum_part(const double* p, GenRange r, int pitch, long long n,
                                                          double* part) {
  __shared__ double sm[kRedThreads];
  double s = 0.0;
  for (long long t = (long long)blockIdx.x * kRedThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kRedThreads) {
    int j, i;
    range_item(r, t, j, i);
    s += p[(long long)j * pitch + i];
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int k = kRedThreads / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sm[threadIdx.x] += sm[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// one block: the partials summed by a fixed tree
__global__ void __launch_bounds__(kRedThreads) k_sum_final(const double* part, int nb, double* out) {
  __shared__ double sm[kRedThreads];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += kRedThreads) s += part[b];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int k = kRedThreads / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sm[threadIdx.x] += sm[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}

// StepState of the fast kernels from the step's factors
struct SetStFn {
  StepState* st;
  const StepCoef<double>* cf;
  __device__ void operator()() const {
    st->dt = cf->dt; st->dt_new = cf->dt;
    st->dtodx1 = cf->dtodx1; st->dtodx2 = cf->dtodx2;
    st->hdtodx1 = cf->hdtodx1; st->hdtodx2 = cf->hdtodx2; st->hdt = cf->hdt;
    st->done = 0;
    st->max_dti_bits = 0ull;
  }
};

}  // namespace

// Device blocks kept between adjoint calls: (pointer, bytes), unused by the
// call in flight.
struct athb_adj_cache {
  std::vector<std::pair<void*, size_t>> blocks;
};

namespace {

void* cache_take(athb_adj_cache* c, size_t b) {
  for (auto it = c->blocks.begin(); it != c->blocks.end(); ++it)
    if (it->second == b) {
      void* p = it->first;
      c->blocks.erase(it);
      return p;
    }
  return nullptr;
}
void cache_put(athb_adj_cache* c, void* p, size_t b) { c->blocks.emplace_back(p, b); }
// free every cached block; true if there were any
bool cache_drop_all(athb_adj_cache* c) {
  const bool any = !c->blocks.empty();
  for (auto& bl : c->blocks) cudaFree(bl.first);
  c->blocks.clear();
  return any;
}
size_t cache_bytes(const athb_adj_cache* c) {
  size_t n = 0;
  for (auto& bl : c->blocks) n += bl.second;
  return n;
}

struct GpuExec {
  cudaStream_t s = nullptr;
  StepState* st = nullptr;     // StepState of the fast kernels
  cudaError_t err = cudaSuccess;
  double* red = nullptr;       // reduction partials
  MaxLoc* redm = nullptr;
  std::vector<std::pair<void*, size_t>> owned;
  size_t bytes = 0;

  void note(cudaError_t e) { if (e != cudaSuccess && err == cudaSuccess) err = e; }
  bool ok() {
    note(cudaGetLastError());
    return err == cudaSuccess;
  }
  static int blocks(long long n, int threads) { return (int)((n + threads - 1) / threads); }

  template <class F> void items(const GenRange& r, const F& f) {
    const long long n = range_count(r);
    if (n <= 0 || err != cudaSuccess) return;
    k_items<F><<<blocks(n, kItemThreads), kItemThreads, 0, s>>>(r, n, f);
  }
  template <class F> void single(const F& f) {
    if (err != cudaSuccess) return;
    k_single<F><<<1, 1, 0, s>>>(f);
  }
  int red_blocks(long long n) const { return (int)std::max(1LL, std::min((long long)kRedBlocks, (n + kRedThreads - 1) / kRedThreads)); }
  void argmax(const double* p, const GenRange& r, int pitch, MaxLoc* out) {
    const long long n = range_count(r);
    if (err != cudaSuccess) return;
    const int nb = red_blocks(n);
    k_argmax_part<<<nb, kRedThreads, 0, s>>>(p, r, pitch, n, redm);
    k_argmax_final<<<1, kRedThreads, 0, s>>>(redm, nb, (long long)r.j0 * pitch + r.i0, out);
  }
  void sum(const double* p, const GenRange& r, int pitch, double* out) {
    const long long n = range_count(r);
    if (err != cudaSuccess) return;
    const int nb = red_blocks(n);
    k_sum_part<<<nb, kRedThreads, 0, s>>>(p, r, pitch, n, red);
    k_sum_final<<<1, kRedThreads, 0, s>>>(red, nb, out);
  }
  // One plain step on the fast kernels (step_kernels.cuh); taped: the
  // predictor also keeps its face states and the half-step emf is saved.
  template <int FLUX, class D> void forward_step(D& d, int cur, bool taped) {
    if (err != cudaSuccess) return;
    const LoopGeom& G = d.G;
    single(SetStFn{st, d.cf});
    GridArgs g;
    g.in = d.S[cur];
    g.out = d.S[cur ^ 1];
    g.scr = d.tape;
    g.st = st;
    g.ps = G.ps;
    g.pitch = G.pitch;
    g.is = G.is; g.ie = G.ie; g.js = G.js; g.je = G.je;
    g.ly = G.ly;
    g.dx1 = G.dx1; g.dx2 = G.dx2;
    g.eos = G.eos;
    for (int k = 0; k < 4; k++) g.bc[k] = G.bc[k];
    const int nx1 = G.nx1, nx2 = G.nx2;
    const PredictGeom pg = make_predict_geom(nx1, nx2, G.ly);
    if (taped) k_predict<FLUX, true><<<pg.nx_blocks + pg.ny_blocks, kThreads, 0, s>>>(g, pg);
    else k_predict<FLUX, false><<<pg.nx_blocks + pg.ny_blocks, kThreads, 0, s>>>(g, pg);
    k_emf<<<blocks((long long)(nx1 + 3) * (nx2 + 3), kThreads), kThreads, 0, s>>>(g, G.is - 1, G.js - 1, nx1 + 3,
                                                                                   nx2 + 3, S_FX, S_FY);
    if (taped) copy(d.tape + (size_t)T_EMF0 * G.ps, d.tape + (size_t)S_EMF * G.ps, (size_t)G.ps);
    CorrectGeom cgm;
    cgm.xw = nx1 + 1; cgm.xn = nx2 + 3;
    cgm.yw = nx1 + 3; cgm.yn = nx2 + 1;
    cgm.ew = nx1 + 3; cgm.en = nx2 + 3;
    cgm.xb = blocks((long long)cgm.xw * cgm.xn, kThreads);
    cgm.yb = blocks((long long)cgm.yw * cgm.yn, kThreads);
    cgm.eb = blocks((long long)cgm.ew * cgm.en, kThreads);
    k_correct<FLUX><<<cgm.xb + cgm.yb + cgm.eb, kThreads, 0, s>>>(g, cgm);
    k_emf<<<blocks((long long)(nx1 + 1) * (nx2 + 1), kThreads), kThreads, 0, s>>>(g, G.is, G.js, nx1 + 1, nx2 + 1,
                                                                                   S_FX2, S_FY2);
    const int n = nx1 * nx2;
    k_update<<<blocks(n, kThreads), kThreads, 0, s>>>(g, nx1, n);
    const int nframe = G.js * G.sx + (G.sy - G.je - 1) * G.sx + nx2 * 2 * G.is;
    GridArgs gg = g;
    gg.in = d.S[cur ^ 1];
    k_ghost<<<blocks(nframe, kThreads), kThreads, 0, s>>>(gg, G.sx, G.sy, nframe, 3, 3);
    d.cfl(d.pd(d.S[cur ^ 1]), d.pd(d.tape + (size_t)G_DTI * G.ps));
  }

  // With a cache (athb_adjoint_keep_workspace on) a block of the same size
  // left by the previous call is reused, released blocks go back to the
  // cache, and a failed cudaMalloc first gives the unused cached blocks back.
  athb_adj_cache* cache = nullptr;
  void* alloc_bytes(size_t b) {
    void* p = nullptr;
    if (err != cudaSuccess) return nullptr;
    b = b ? b : 8;
    if (cache && (p = cache_take(cache, b)) != nullptr) {
      owned.emplace_back(p, b);
      bytes += b;
      return p;
    }
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaErrorMemoryAllocation && cache && cache_drop_all(cache)) {
      (void)cudaGetLastError();
      e = cudaMalloc(&p, b);
    }
    note(e);
    if (e == cudaSuccess) { owned.emplace_back(p, b); bytes += b; }
    return e == cudaSuccess ? p : nullptr;
  }
  double* alloc(size_t n) { return (double*)alloc_bytes(n * sizeof(double)); }
  void release_bytes(void* p) {
    if (!p) return;
    size_t b = 0;
    for (auto it = owned.begin(); it != owned.end(); ++it)
      if (it->first == p) { b = it->second; owned.erase(it); break; }
    if (cache && b) cache_put(cache, p, b);
    else cudaFree(p);
  }
  void release(double* p) { release_bytes(p); }
  void zero(double* p, size_t n) { if (err == cudaSuccess) note(cudaMemsetAsync(p, 0, n * sizeof(double), s)); }
  void zero_bytes(void* p, size_t b) { if (err == cudaSuccess) note(cudaMemsetAsync(p, 0, b, s)); }
  void copy(double* d, const double* src, size_t n) {
    if (err == cudaSuccess) note(cudaMemcpyAsync(d, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  void to_host(void* d, const void* src, size_t b) {
    if (err != cudaSuccess) return;
    note(cudaMemcpyAsync(d, src, b, cudaMemcpyDeviceToHost, s));
    note(cudaStreamSynchronize(s));
  }
  ~GpuExec() {
    for (auto& o : owned) {
      if (cache) cache_put(cache, o.first, o.second);
      else cudaFree(o.first);
    }
  }
};

LoopGeom geom_of(const athb_ctx* c) {
  LoopGeom G;
  G.nx1 = c->cfg.nx1; G.nx2 = c->cfg.nx2;
  G.sx = c->sx; G.sy = c->sy;
  G.pitch = c->pitch;
  G.ly = c->ly;
  G.ps = c->ps;
  G.is = c->is; G.ie = c->ie; G.js = c->js; G.je = c->je;
  G.dx1 = c->dx1; G.dx2 = c->dx2;
  G.cour = c->cfg.cour_no;
  G.tlim = c->cfg.tlim;
  G.eos = Eos{c->cfg.gamma, c->cfg.gamma - 1.0, c->cfg.gamma - 2.0};
  G.flux = c->cfg.flux;
  G.bc[0] = c->cfg.bc_ix1; G.bc[1] = c->cfg.bc_ox1; G.bc[2] = c->cfg.bc_ix2; G.bc[3] = c->cfg.bc_ox2;
  return G;
}

// host planes (unpadded rows of sx) <-> device planes (rows of pitch)
cudaError_t planes_h2d(const athb_ctx* c, double* dev, const double* host, cudaStream_t s) {
  return cudaMemcpy2DAsync(dev, sizeof(double) * c->pitch, host, sizeof(double) * c->sx, sizeof(double) * c->sx,
                           (size_t)c->sy * NSTATE, cudaMemcpyHostToDevice, s);
}
cudaError_t planes_d2h(const athb_ctx* c, double* host, const double* dev, cudaStream_t s) {
  return cudaMemcpy2DAsync(host, sizeof(double) * c->sx, dev, sizeof(double) * c->pitch, sizeof(double) * c->sx,
                           (size_t)c->sy * NSTATE, cudaMemcpyDeviceToHost, s);
}

int finish(GpuExec& x, const char* what) {
  if (!x.ok())
    return athb_fail(x.err == cudaErrorMemoryAllocation ? ATHB_ERR_NOMEM : ATHB_ERR_CUDA, "%s: %s", what,
                     cudaGetErrorString(x.err));
  return ATHB_OK;
}

// Zero the ghost entries of a host direction: only the cells a step writes
// are independent inputs (the ghosts are set_bvals of them).
void interior_only(const athb_ctx* c, std::vector<double>& d) {
  for (int p = 0; p < NSTATE; p++)
    for (int j = 0; j < c->sy; j++)
      for (int i = 0; i < c->sx; i++) {
        bool keep = j >= c->js && j <= c->je && i >= c->is && i <= c->ie;
        if (p == P_B1I) keep = j >= c->js && j <= c->je && i >= c->is && i <= c->ie + 1;
        if (p == P_B2I) keep = j >= c->js && j <= c->je + 1 && i >= c->is && i <= c->ie;
        if (!keep) d[((size_t)p * c->sy + j) * c->sx + i] = 0.0;
      }
}

}  // namespace

extern "C" int athb_tlm_run(athb_ctx* ctx, int nsteps, const double* dstate0, double* J, double* dJ,
                            double* dstate_out) {
  if (!ctx || !dstate0 || nsteps < 0) return athb_fail(ATHB_ERR_ARG, "athb_tlm_run: bad arguments");
  CUDA_TRY(cudaSetDevice(ctx->cfg.device));
  GpuExec x;
  x.s = ctx->stream;
  x.cache = ctx->adj_keep ? ctx->adj_cache : nullptr;
  AdjointDriver<GpuExec> d(x, geom_of(ctx));
  x.red = x.alloc(kRedBlocks);
  x.redm = (MaxLoc*)x.alloc_bytes(sizeof(MaxLoc) * kRedBlocks);
  x.st = (StepState*)x.alloc_bytes(sizeof(StepState));
  if (d.setup(nsteps, true)) return finish(x, "athb_tlm_run: allocation");
  std::vector<double> h((size_t)NSTATE * ctx->sy * ctx->sx);
  std::copy(dstate0, dstate0 + h.size(), h.begin());
  interior_only(ctx, h);
  x.copy(d.S[0], ctx->state[ctx->cur], d.state_doubles());
  x.note(planes_h2d(ctx, d.dS[0], h.data(), x.s));
  int cur = 0;
  if (ctx->cfg.flux == ATHB_FLUX_HLLE) d.tlm<kFluxHlle>(nsteps, cur); else d.tlm<kFluxRoe>(nsteps, cur);
  AdjScal sc{};
  x.to_host(&sc, d.sc, sizeof sc);
  if (dstate_out) {
    x.note(planes_d2h(ctx, dstate_out, d.dS[cur], x.s));
    x.note(cudaStreamSynchronize(x.s));
  }
  int rc = finish(x, "athb_tlm_run");
  if (rc) return rc;
  if (J) *J = sc.J;
  if (dJ) *dJ = sc.dJ;
  return ATHB_OK;
}

namespace {

int adjoint_impl(athb_ctx* ctx, int nsteps, long long snapshot_bytes, const double* seed_host, double* J,
                 double* grad, athb_adjoint_stats* stats) {
  if (!ctx || nsteps < 0) return athb_fail(ATHB_ERR_ARG, "athb_adjoint_gradient: bad arguments");
  CUDA_TRY(cudaSetDevice(ctx->cfg.device));
  const auto t0 = std::chrono::steady_clock::now();
  GpuExec x;
  x.s = ctx->stream;
  x.cache = ctx->adj_keep ? ctx->adj_cache : nullptr;
  AdjointDriver<GpuExec> d(x, geom_of(ctx));
  x.red = x.alloc(kRedBlocks);
  x.redm = (MaxLoc*)x.alloc_bytes(sizeof(MaxLoc) * kRedBlocks);
  x.st = (StepState*)x.alloc_bytes(sizeof(StepState));
  if (d.setup(nsteps, false)) return finish(x, "athb_adjoint_gradient: workspace");
  if (seed_host) {   // the cotangent of S^N, on the entries a step writes
    std::vector<double> h((size_t)NSTATE * ctx->sy * ctx->sx);
    std::copy(seed_host, seed_host + h.size(), h.begin());
    interior_only(ctx, h);
    double* dseed = x.alloc(d.state_doubles());
    if (!x.ok()) return finish(x, "athb_adjoint_vjp: seed");
    x.zero(dseed, d.state_doubles());
    x.note(planes_h2d(ctx, dseed, h.data(), x.s));
    x.note(cudaStreamSynchronize(x.s));   // h is freed at the end of this block
    d.seed = dseed;
  }
  // snapshot slots: as many as the budget allows, at most one per step
  const size_t sbytes = sizeof(double) * d.state_doubles();
  long long budget = snapshot_bytes;
  if (budget <= 0) {
    size_t fr = 0, tot = 0;
    CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    if (x.cache) fr += cache_bytes(x.cache);   // kept blocks are this call's to reuse
    budget = (long long)(0.85 * (double)fr) - (1LL << 30);   // keep 1 GiB of headroom
  }
  const size_t tbytes = sizeof(double) * d.tape_doubles();
  const bool tape_mode = (double)budget >= (double)(nsteps + 1) * (double)sbytes + (double)nsteps * (double)tbytes;
  long long ns = std::min<long long>((long long)nsteps + 1, budget / (long long)sbytes);
  if (ns < 1) return athb_fail(ATHB_ERR_NOMEM, "athb_adjoint_gradient: no room for one state snapshot (%zu bytes)", sbytes);
  d.nslot = (int)ns;
  if (tape_mode && nsteps > 0) d.tapes = x.alloc((size_t)nsteps * d.tape_doubles());
  d.slots = x.alloc((size_t)d.nslot * d.state_doubles());
  if (!x.ok()) return finish(x, "athb_adjoint_gradient: snapshots");
  x.copy(d.S[0], ctx->state[ctx->cur], d.state_doubles());
  int lc = 0, steps = 0;
  if (ctx->cfg.flux == ATHB_FLUX_HLLE) d.adjoint<kFluxHlle>(nsteps, lc, steps); else d.adjoint<kFluxRoe>(nsteps, lc, steps);
  AdjScal sc{};
  x.to_host(&sc, d.sc, sizeof sc);
  if (grad) {
    x.note(planes_d2h(ctx, grad, d.lam[lc], x.s));
    x.note(cudaStreamSynchronize(x.s));
  }
  int rc = finish(x, "athb_adjoint_gradient");
  if (rc) return rc;
  if (sc.nonfinite) return athb_fail(ATHB_ERR_STATE, "athb_adjoint_gradient: non-finite adjoint of dt");
  if (J) *J = sc.J;
  if (stats) {
    stats->steps = steps;
    stats->snapshots = d.nslot;
    stats->advances = d.advances;
    stats->taped = d.taped;
    stats->workspace_bytes = (long long)x.bytes;
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    stats->tape_mode = d.tapes != nullptr;
  }
  return ATHB_OK;
}

}  // namespace

extern "C" int athb_adjoint_gradient(athb_ctx* ctx, int nsteps, long long snapshot_bytes, double* J, double* grad,
                                     athb_adjoint_stats* stats) {
  return adjoint_impl(ctx, nsteps, snapshot_bytes, nullptr, J, grad, stats);
}

extern "C" int athb_adjoint_vjp(athb_ctx* ctx, int nsteps, long long snapshot_bytes, const double* seed, double* J,
                                double* grad, athb_adjoint_stats* stats) {
  if (!seed) return athb_fail(ATHB_ERR_ARG, "athb_adjoint_vjp: null seed");
  return adjoint_impl(ctx, nsteps, snapshot_bytes, seed, J, grad, stats);
}

// Keep (on != 0) the adjoint's device workspace between calls on this
// context, or free it now (on == 0).
extern "C" int athb_adjoint_keep_workspace(athb_ctx* ctx, int on) {
  if (!ctx) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(ctx->cfg.device));
  if (on) {
    if (!ctx->adj_cache) ctx->adj_cache = new athb_adj_cache;
    ctx->adj_keep = 1;
  } else {
    athb_adjoint_cache_free(ctx);
  }
  return ATHB_OK;
}

void athb_adjoint_cache_free(athb_ctx* c) {
  if (!c || !c->adj_cache) return;
  cudaSetDevice(c->cfg.device);
  cudaStreamSynchronize(c->stream);
  cache_drop_all(c->adj_cache);
  delete c->adj_cache;
  c->adj_cache = nullptr;
  c->adj_keep = 0;
}
