// athb_core.cu -- device-resident context, step launch sequence, CUDA-graph
// loop and the athb_* C ABI of libathena_b200.so.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "athb_internal.h"
#include "step_kernels.cuh"

using namespace athb;

// ---------------------------------------------------------------------------
// error reporting
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

int athb_fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CUDA_TRY(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return athb_fail(ATHB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                              \
  } while (0)

extern "C" const char* athb_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* athb_error_string(int code) {
  switch (code) {
  case ATHB_OK: return "ok";
  case ATHB_ERR_ARG: return "invalid argument";
  case ATHB_ERR_CUDA: return "CUDA error";
  case ATHB_ERR_STATE: return "non-finite state";
  case ATHB_ERR_PARSE: return "parameter error";
  case ATHB_ERR_NOMEM: return "out of memory";
  case ATHB_ERR_NOTFOUND: return "not found";
  default: return "unknown error";
  }
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
static GridArgs grid_args(const athb_ctx* c, int from) {
  GridArgs g;
  g.in = c->state[from];
  g.out = c->state[from ^ 1];
  g.scr = c->scr;
  g.st = c->st;
  g.ps = c->ps;
  g.pitch = c->pitch;
  g.is = c->is; g.ie = c->ie; g.js = c->js; g.je = c->je;
  g.ly = c->ly;
  g.dx1 = c->dx1; g.dx2 = c->dx2;
  g.eos = Eos{c->cfg.gamma, c->cfg.gamma - 1.0, c->cfg.gamma - 2.0};
  g.bc[0] = c->cfg.bc_ix1; g.bc[1] = c->cfg.bc_ox1; g.bc[2] = c->cfg.bc_ix2; g.bc[3] = c->cfg.bc_ox2;
  return g;
}

static int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

static bool valid_bc(int b) { return b == BC_REFLECT || b == BC_OUTFLOW || b == BC_PERIODIC; }

int athb_ctx_validate(const athb_config* cfg) {
  if (!cfg) return athb_fail(ATHB_ERR_ARG, "null config");
  if (cfg->nx1 < 4 || cfg->nx2 < 4)
    return athb_fail(ATHB_ERR_ARG, "grid must have Nx1 >= 4 and Nx2 >= 4 (got %d x %d)", cfg->nx1, cfg->nx2);
  if ((long long)(cfg->nx1 + 8) * (cfg->nx2 + 8) > (1LL << 30))
    return athb_fail(ATHB_ERR_ARG, "grid too large (%d x %d)", cfg->nx1, cfg->nx2);
  if (!(cfg->x1max >= cfg->x1min) || !(cfg->x2max >= cfg->x2min))
    return athb_fail(ATHB_ERR_ARG, "x1max < x1min or x2max < x2min");
  if (!valid_bc(cfg->bc_ix1) || !valid_bc(cfg->bc_ox1) || !valid_bc(cfg->bc_ix2) || !valid_bc(cfg->bc_ox2))
    return athb_fail(ATHB_ERR_ARG, "boundary flags must be 1 (reflect), 2 (outflow) or 4 (periodic)");
  if (cfg->flux != ATHB_FLUX_ROE && cfg->flux != ATHB_FLUX_HLLE)
    return athb_fail(ATHB_ERR_ARG, "unknown flux %d", cfg->flux);
  if (!(cfg->gamma > 1.0)) return athb_fail(ATHB_ERR_ARG, "gamma must be > 1");
  return ATHB_OK;
}

extern "C" int athb_create(const athb_config* cfg, athb_ctx** out) {
  if (!out) return athb_fail(ATHB_ERR_ARG, "null output pointer");
  *out = nullptr;
  int rc = athb_ctx_validate(cfg);
  if (rc) return rc;
  athb_ctx* c = new (std::nothrow) athb_ctx();
  if (!c) return athb_fail(ATHB_ERR_NOMEM, "context allocation failed");
  c->cfg = *cfg;
  c->sx = cfg->nx1 + 2 * kNghost;
  c->sy = cfg->nx2 + 2 * kNghost;
  c->pitch = (c->sx + 15) & ~15;
  c->ps = (long long)c->pitch * c->sy;
  c->is = kNghost; c->ie = cfg->nx1 + kNghost - 1;
  c->js = kNghost; c->je = cfg->nx2 + kNghost - 1;
  // src/init_grid.c: dx = (xmax - xmin)/Nx, x_0 = xmin, disp = -nghost
  c->dx1 = (cfg->x1max - cfg->x1min) / (double)cfg->nx1;
  c->dx2 = (cfg->x2max - cfg->x2min) / (double)cfg->nx2;
  c->x1_0 = cfg->x1min; c->x2_0 = cfg->x2min;
  {
    // rows per column march: short marches on small grids, where the step
    // is latency-bound and more threads shorten it (64^2 and 128^2 run
    // fastest at 1, 200x300 at 2-3), else enough marches for ~512 threads
    // per SM (measured on B200, blast and field loop)
    const long long cf = (long long)(cfg->nx1 + 4) * (cfg->nx2 + 3);
    c->ly = cf < 40000 ? 1 : cf < 100000 ? 2 : (int)std::max(4LL, std::min(64LL, cf / (148LL * 512)));
  }
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  const size_t state_bytes = sizeof(double) * (size_t)c->ps * NSTATE;
  const size_t scr_bytes = sizeof(double) * (size_t)c->ps * NSCRATCH;
  if (e == cudaSuccess) e = cudaMalloc(&c->state[0], state_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->state[1], state_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->scr, scr_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->st, sizeof(StepState));
  if (e == cudaSuccess) e = cudaMemsetAsync(c->state[0], 0, state_bytes, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->state[1], 0, state_bytes, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->scr, 0, scr_bytes, c->stream);
  if (e == cudaSuccess) {
    StepState h{};
    h.tlim = cfg->tlim;
    h.cour_no = cfg->cour_no;
    h.nlim = cfg->nlim;
    e = cudaMemcpyAsync(c->st, &h, sizeof h, cudaMemcpyHostToDevice, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    athb_destroy(c);
    return athb_fail(e == cudaErrorMemoryAllocation ? ATHB_ERR_NOMEM : ATHB_ERR_CUDA,
                     "athb_create: %s", cudaGetErrorString(e));
  }
  *out = c;
  return ATHB_OK;
}

static void drop_graphs(athb_ctx* c) {
  for (int k = 0; k < 2; k++)
    if (c->graph[k]) { cudaGraphExecDestroy(c->graph[k]); c->graph[k] = nullptr; }
}

extern "C" void athb_destroy(athb_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->cfg.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  cudaFree(c->state[0]);
  cudaFree(c->state[1]);
  cudaFree(c->scr);
  cudaFree(c->st);
  cudaFree(c->aos);
  cudaFree(c->cpaw_soln);
  athb_adjoint_cache_free(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" int athb_shape(const athb_ctx* c, int* sx, int* sy) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  if (sx) *sx = c->sx;
  if (sy) *sy = c->sy;
  return ATHB_OK;
}

extern "C" void* athb_stream(athb_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" void* athb_host_alloc(unsigned long long bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}
extern "C" void athb_host_free(void* p) { if (p) cudaFreeHost(p); }

// ---------------------------------------------------------------------------
// state transfer
// ---------------------------------------------------------------------------
int athb_set_clock(athb_ctx* c, double dt, double time, int nstep) {
  StepState h{};
  h.time = time;
  h.tlim = c->cfg.tlim;
  h.cour_no = c->cfg.cour_no;
  h.nstep = nstep;
  h.nlim = c->cfg.nlim;
  h.done = !((time < c->cfg.tlim) && (c->cfg.nlim < 0 || nstep < c->cfg.nlim));
  // dt as the reference Grid holds it; the next step takes it after the tlim
  // clamp (src/main.c:230-232)
  h.dt_new = dt;
  h.dt = (!h.done && (h.tlim - time) < dt) ? (h.tlim - time) : dt;
  h.dtodx1 = h.dt / c->dx1;
  h.dtodx2 = h.dt / c->dx2;
  h.hdtodx1 = 0.5 * h.dtodx1;
  h.hdtodx2 = 0.5 * h.dtodx2;
  h.hdt = 0.5 * h.dt;
  CUDA_TRY(cudaMemcpyAsync(c->st, &h, sizeof h, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}

int athb_read_clock(athb_ctx* c, StepState* h) {
  CUDA_TRY(cudaMemcpyAsync(h, c->st, sizeof *h, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}

extern "C" int athb_upload(athb_ctx* c, const double* planes, double dt, double time, int nstep) {
  if (!c || !planes) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  CUDA_TRY(cudaMemcpy2DAsync(c->state[c->cur], sizeof(double) * c->pitch, planes,
                             sizeof(double) * c->sx, sizeof(double) * c->sx,
                             (size_t)c->sy * NSTATE, cudaMemcpyHostToDevice, c->stream));
  return athb_set_clock(c, dt, time, nstep);
}

extern "C" int athb_download(athb_ctx* c, double* planes, double* dt, double* time, int* nstep) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  if (planes)
    CUDA_TRY(cudaMemcpy2DAsync(planes, sizeof(double) * c->sx, c->state[c->cur],
                               sizeof(double) * c->pitch, sizeof(double) * c->sx,
                               (size_t)c->sy * NSTATE, cudaMemcpyDeviceToHost, c->stream));
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  if (dt) *dt = h.dt_new;
  if (time) *time = h.time;
  if (nstep) *nstep = h.nstep;
  return ATHB_OK;
}

// ---------------------------------------------------------------------------
// launch sequences
// ---------------------------------------------------------------------------
int athb_launch_ghost_phase(athb_ctx* c, int buf, int mode, int sides) {
  GridArgs g = grid_args(c, buf ^ 1);  // out = buf
  const int nframe = c->js * c->sx + (c->sy - c->je - 1) * c->sx + c->cfg.nx2 * 2 * c->is;
  k_ghost<<<blocks_for(nframe), kThreads, 0, c->stream>>>(g, c->sx, c->sy, nframe, mode, sides);
  CUDA_TRY(cudaGetLastError());
  return ATHB_OK;
}

int athb_launch_ghost(athb_ctx* c, int buf) { return athb_launch_ghost_phase(c, buf, 3, 3); }

int athb_launch_set_dt(athb_ctx* c, double dt) {
  k_set_dt<<<1, 1, 0, c->stream>>>(c->st, dt, c->dx1, c->dx2);
  CUDA_TRY(cudaGetLastError());
  return ATHB_OK;
}

int athb_launch_cfl(athb_ctx* c, int buf) {
  GridArgs g = grid_args(c, buf);
  const int n = c->cfg.nx1 * c->cfg.nx2;
  k_cfl<<<blocks_for(n), kThreads, 0, c->stream>>>(g, c->cfg.nx1, n);
  CUDA_TRY(cudaGetLastError());
  return ATHB_OK;
}

// The integrator proper: reads state[from], writes the interior of state[from^1].
// With ev != nullptr, events ev[0..5] bracket the five kernels.
int athb_launch_integrate_split(athb_ctx* c, int from, cudaEvent_t* ev) {
#define MARK(k) do { if (ev) CUDA_TRY(cudaEventRecord(ev[k], c->stream)); } while (0)
  GridArgs g = grid_args(c, from);
  const int nx1 = c->cfg.nx1, nx2 = c->cfg.nx2;
  const PredictGeom pg = make_predict_geom(nx1, nx2, c->ly);
  const bool hlle = c->cfg.flux == ATHB_FLUX_HLLE;
  MARK(0);
  if (hlle)
    k_predict<kFluxHlle><<<pg.nx_blocks + pg.ny_blocks, kThreads, 0, c->stream>>>(g, pg);
  else
    k_predict<kFluxRoe><<<pg.nx_blocks + pg.ny_blocks, kThreads, 0, c->stream>>>(g, pg);
  CUDA_TRY(cudaGetLastError());

  MARK(1);
  k_emf<<<blocks_for((long long)(nx1 + 3) * (nx2 + 3)), kThreads, 0, c->stream>>>(
      g, c->is - 1, c->js - 1, nx1 + 3, nx2 + 3, S_FX, S_FY);
  CUDA_TRY(cudaGetLastError());

  CorrectGeom cg;
  cg.xw = nx1 + 1; cg.xn = nx2 + 3;
  cg.yw = nx1 + 3; cg.yn = nx2 + 1;
  cg.ew = nx1 + 3; cg.en = nx2 + 3;
  cg.xb = blocks_for((long long)cg.xw * cg.xn);
  cg.yb = blocks_for((long long)cg.yw * cg.yn);
  cg.eb = blocks_for((long long)cg.ew * cg.en);
  MARK(2);
  if (hlle)
    k_correct<kFluxHlle><<<cg.xb + cg.yb + cg.eb, kThreads, 0, c->stream>>>(g, cg);
  else
    k_correct<kFluxRoe><<<cg.xb + cg.yb + cg.eb, kThreads, 0, c->stream>>>(g, cg);
  CUDA_TRY(cudaGetLastError());

  MARK(3);
  k_emf<<<blocks_for((long long)(nx1 + 1) * (nx2 + 1)), kThreads, 0, c->stream>>>(
      g, c->is, c->js, nx1 + 1, nx2 + 1, S_FX2, S_FY2);
  CUDA_TRY(cudaGetLastError());

  MARK(4);
  const int n = nx1 * nx2;
  k_update<<<blocks_for(n), kThreads, 0, c->stream>>>(g, nx1, n);
  CUDA_TRY(cudaGetLastError());
  MARK(5);
  return ATHB_OK;
#undef MARK
}

int athb_launch_integrate(athb_ctx* c, int from) { return athb_launch_integrate_split(c, from, nullptr); }

// Per-kernel timing of the loop step (CUDA events on the context's stream
// between consecutive launches).  Kernel order: predict, emf(half), correct,
// emf(full), update, finalize, ghost.
extern "C" int athb_profile_steps(athb_ctx* c, int nsteps, double* ms_out) {
  if (!c || nsteps < 1 || !ms_out) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  constexpr int K = 7;
  std::vector<cudaEvent_t> ev((size_t)nsteps * (K + 1));
  for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
  for (int k = 0; k < K; k++) ms_out[k] = 0.0;
  int rc = ATHB_OK;
  for (int s = 0; s < nsteps && rc == ATHB_OK; s++) {
    cudaEvent_t* e = &ev[(size_t)s * (K + 1)];
    const int from = c->cur;
    GridArgs g = grid_args(c, from);
    const int nx1 = c->cfg.nx1, nx2 = c->cfg.nx2;
    rc = athb_launch_integrate_split(c, from, e);
    if (rc) break;
    k_finalize<<<1, 1, 0, c->stream>>>(c->st, c->dx1, c->dx2, 1);
    CUDA_TRY(cudaEventRecord(e[6], c->stream));
    rc = athb_launch_ghost(c, from ^ 1);
    CUDA_TRY(cudaEventRecord(e[7], c->stream));
    c->cur ^= 1;
    (void)g; (void)nx1; (void)nx2;
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int s = 0; s < nsteps && rc == ATHB_OK; s++) {
    cudaEvent_t* e = &ev[(size_t)s * (K + 1)];
    for (int k = 0; k < K; k++) {
      float ms = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms, e[k], e[k + 1]));
      ms_out[k] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < K; k++) ms_out[k] /= nsteps;
  return rc;
}

// One iteration of the reference main loop (src/main.c:229-307) on the device.
static int launch_loop_step(athb_ctx* c, int from) {
  int rc = athb_launch_integrate(c, from);
  if (rc) return rc;
  k_finalize<<<1, 1, 0, c->stream>>>(c->st, c->dx1, c->dx2, 1);
  CUDA_TRY(cudaGetLastError());
  return athb_launch_ghost(c, from ^ 1);
}

static int build_graph(athb_ctx* c, int from) {
  cudaGraph_t graph = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = launch_loop_step(c, from);
  if (rc == ATHB_OK) rc = launch_loop_step(c, from ^ 1);
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->graph[from], graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  return ATHB_OK;
}

extern "C" int athb_run_async(athb_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  int left = nsteps;
  while (left >= 2) {
    if (!c->graph[c->cur]) { int rc = build_graph(c, c->cur); if (rc) return rc; }
    CUDA_TRY(cudaGraphLaunch(c->graph[c->cur], c->stream));
    left -= 2;  // two steps: the state returns to the same buffer
  }
  if (left == 1) {
    int rc = launch_loop_step(c, c->cur);
    if (rc) return rc;
    c->cur ^= 1;
  }
  return ATHB_OK;
}

extern "C" int athb_synchronize(athb_ctx* c) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}

extern "C" int athb_status(athb_ctx* c, double* time, double* dt, int* nstep, int* done) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  if (time) *time = h.time;
  if (dt) *dt = h.dt_new;
  if (nstep) *nstep = h.nstep;
  if (done) *done = h.done;
  if (h.flags & kErrNonFinite)
    return athb_fail(ATHB_ERR_STATE, "non-finite or negative CFL rate at step %d", h.nstep);
  return ATHB_OK;
}

// Launches as many steps as the clock says remain (dt can grow at most 2x per
// step, so (tlim - time)/dt does not overshoot the end by more than the nlim
// bound allows), then re-reads the clock, until done or nsteps launched.
extern "C" int athb_run(athb_ctx* c, int nsteps, int* steps_done) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  const int start = h.nstep;
  long long launched = 0;
  while (!h.done && launched < nsteps) {
    const double tend = h.has_pause ? std::min(h.tlim, h.tpause) : h.tlim;
    double est = (tend - h.time) / h.dt;
    long long want = est < 1.0 ? 1 : (long long)std::ceil(est);
    if (h.nlim >= 0) want = std::min<long long>(want, std::max(1, h.nlim - h.nstep));
    want = std::min<long long>(want, nsteps - launched);
    rc = athb_run_async(c, (int)want);
    if (rc) return rc;
    launched += want;
    rc = athb_read_clock(c, &h);
    if (rc) return rc;
    if (h.flags & kErrNonFinite) break;
  }
  int nstep = 0;
  rc = athb_status(c, nullptr, nullptr, &nstep, nullptr);
  if (steps_done) *steps_done = nstep - start;
  return rc;
}

// Pause the loop at the first step that starts at time >= tpause (on != 0),
// or run freely (on == 0).  athb_status then reports done = 2.
extern "C" int athb_set_pause(athb_ctx* c, double tpause, int on) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  k_set_pause<<<1, 1, 0, c->stream>>>(c->st, tpause, on ? 1 : 0);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}

extern "C" int athb_set_bvals(athb_ctx* c) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  int rc = athb_launch_ghost(c, c->cur);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}

extern "C" int athb_new_dt(athb_ctx* c, double* dt) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  int rc = athb_launch_cfl(c, c->cur);
  if (rc) return rc;
  k_finalize<<<1, 1, 0, c->stream>>>(c->st, c->dx1, c->dx2, 0);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return athb_status(c, nullptr, dt, nullptr, nullptr);
}

// Tuning: rows per y-sweep march segment (any value >= 1 gives the same
// results; it only changes the work decomposition).
extern "C" int athb_set_ly(athb_ctx* c, int ly) {
  if (!c || ly < 1) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  c->ly = ly;
  drop_graphs(c);
  return ATHB_OK;
}

extern "C" int athb_get_ly(const athb_ctx* c) { return c ? c->ly : 0; }

extern "C" int athb_grid_info_of(const athb_ctx* c, athb_grid_info* g) {
  if (!c || !g) return athb_fail(ATHB_ERR_ARG, "null argument");
  g->nx1 = c->cfg.nx1; g->nx2 = c->cfg.nx2; g->sx = c->sx; g->sy = c->sy;
  g->is = c->is; g->ie = c->ie; g->js = c->js; g->je = c->je;
  g->dx1 = c->dx1; g->dx2 = c->dx2; g->x1_0 = c->x1_0; g->x2_0 = c->x2_0;
  g->idisp = -c->is; g->jdisp = -c->js;
  g->gamma = c->cfg.gamma; g->gamma_1 = c->cfg.gamma - 1.0; g->gamma_2 = c->cfg.gamma - 2.0;
  return ATHB_OK;
}

// ---------------------------------------------------------------------------
// FP64 issue-rate probe: every thread runs 8 independent chains of dependent
// DADD/DMUL pairs; 2 operations per pair.  All accesses stay in registers;
// one store per thread keeps the work alive.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fp64_probe(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      x[k] = __dadd_rn(x[k], a);
      x[k] = __dmul_rn(x[k], b);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

extern "C" int athb_fp64_peak(int device, double* ops_per_s) {
  if (!ops_per_s) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(device));
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  double* out = nullptr;
  CUDA_TRY(cudaMalloc(&out, sizeof(double) * blocks * threads));
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 6; rep++) {
    CUDA_TRY(cudaEventRecord(e0));
    k_fp64_probe<<<blocks, threads>>>(out, iters, 1.0000001, 0.9999999);
    CUDA_TRY(cudaEventRecord(e1));
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    const double ops = 2.0 * 8.0 * iters * (double)blocks * threads;
    if (rep > 0 && ms > 0.f) best = std::max(best, ops / (ms * 1e-3));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *ops_per_s = best;
  return ATHB_OK;
}

// ---------------------------------------------------------------------------
// Diagnostics of the resident state (interior cells): volume integrals of
// d, E, the magnetic energy (B1c^2+B2c^2+B3c^2)/2 and of Bp2 = B1c^2+B2c^2
// (the field-loop output expression, src/field_loop.c:167-171), and the
// maxima of |div B| from the face fields (the CT invariant) and of |J3|
// (src/field_loop.c:161-165).  Two deterministic passes: per-block partials
// into the scratch planes (free between steps), then one block sums them in
// a fixed order, so a result is the same on every run.
// ---------------------------------------------------------------------------
namespace {
constexpr int kDiag = 6;  // mass, energy, emag, bp2, max|divB|, max|J3|

__global__ void __launch_bounds__(kThreads) k_diag_partial(GridArgs g, int nx1, int ncell, double* part) {
  const int t = blockIdx.x * kThreads + threadIdx.x;
  double v[kDiag] = {0, 0, 0, 0, 0, 0};
  if (t < ncell) {
    const int j = g.js + t / nx1, i = g.is + t % nx1;
    const long long ps = g.ps, o = off(g, j, i), P = g.pitch;
    const double* s = g.in;
    const double dv = g.dx1 * g.dx2;
    const double b1 = s[P_B1C * ps + o], b2 = s[P_B2C * ps + o], b3 = s[P_B3C * ps + o];
    v[0] = s[P_D * ps + o] * dv;
    v[1] = s[P_E * ps + o] * dv;
    v[2] = 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) * dv;
    v[3] = (b1 * b1 + b2 * b2) * dv;
    v[4] = fabs((s[P_B1I * ps + o + 1] - s[P_B1I * ps + o]) / g.dx1 +
                (s[P_B2I * ps + o + P] - s[P_B2I * ps + o]) / g.dx2);
    v[5] = fabs((s[P_B2I * ps + o] - s[P_B2I * ps + o - 1]) / g.dx1 -
                (s[P_B1I * ps + o] - s[P_B1I * ps + o - P]) / g.dx2);
  }
  __shared__ double red[kThreads / 32][kDiag];
#pragma unroll
  for (int k = 0; k < kDiag; k++) {
    double x = v[k];
    for (int d = 16; d > 0; d >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, d);
      x = k < 4 ? x + y : fmax(x, y);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < kDiag) {
    const int k = threadIdx.x;
    double x = red[0][k];
    for (int w = 1; w < kThreads / 32; w++) x = k < 4 ? x + red[w][k] : fmax(x, red[w][k]);
    part[(size_t)blockIdx.x * kDiag + k] = x;
  }
}

__global__ void k_diag_final(const double* part, int nblocks, double* out) {
  if (threadIdx.x < kDiag) {
    const int k = threadIdx.x;
    double x = 0.0;
    for (int b = 0; b < nblocks; b++) x = k < 4 ? x + part[(size_t)b * kDiag + k] : fmax(x, part[(size_t)b * kDiag + k]);
    out[k] = x;
  }
}
}  // namespace

extern "C" int athb_diagnostics(athb_ctx* c, double out[6]) {
  if (!c || !out) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  GridArgs g = grid_args(c, c->cur);
  const int n = c->cfg.nx1 * c->cfg.nx2;
  const int nb = blocks_for(n);
  double* part = c->scr;                   // scratch planes are free between steps
  double* res = c->scr + (size_t)nb * kDiag;
  if ((size_t)(nb + 1) * kDiag > (size_t)c->ps * NSCRATCH) return athb_fail(ATHB_ERR_ARG, "grid too small");
  k_diag_partial<<<nb, kThreads, 0, c->stream>>>(g, c->cfg.nx1, n, part);
  k_diag_final<<<1, 32, 0, c->stream>>>(part, nb, res);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(out, res, kDiag * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}

// ---------------------------------------------------------------------------
// Pieces of a main-loop iteration for callers that split a grid over several
// contexts (a slab decomposition along x2, one context per GPU): the step of
// the local interior, the local and the imposed CFL maximum, the ghost fill
// by direction and side, and row transfers for the exchange of the
// inter-slab ghost rows.
// ---------------------------------------------------------------------------
namespace {
__global__ void k_set_max_dti(StepState* st, unsigned long long bits) { st->max_dti_bits = bits; }
}  // namespace

// Cell sizes and origin of the local grid (a slab takes the global grid's dx
// exactly, which (x2max - x2min) / Nx2 of the slab need not reproduce).
extern "C" int athb_set_geometry(athb_ctx* c, double dx1, double dx2, double x1_0, double x2_0) {
  if (!c || !(dx1 > 0.0) || !(dx2 > 0.0)) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->dx1 = dx1; c->dx2 = dx2; c->x1_0 = x1_0; c->x2_0 = x2_0;
  drop_graphs(c);
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  return athb_set_clock(c, h.dt_new, h.time, h.nstep);  // dt/dx factors of the new dx
}

// integrate_2d of the local interior (src/__integrate_2d__.c:100-537) into
// the other buffer, 1/dt of every updated cell folded into the context's
// running maximum; no time advance, no new dt, no ghost fill (see
// athb_finish_step).
extern "C" int athb_integrate_local(athb_ctx* c) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  return athb_launch_integrate(c, c->cur);
}

// 1/dt of the resident interior folded into the running maximum (new_dt
// before the loop, src/main.c:149).
extern "C" int athb_cfl_local(athb_ctx* c) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  return athb_launch_cfl(c, c->cur);
}

// The running maximum of 1/dt as the bits of a positive double (which order
// like the doubles): the value to reduce with a max across contexts.
extern "C" int athb_max_dti_bits(athb_ctx* c, unsigned long long* bits) {
  if (!c || !bits) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  *bits = h.max_dti_bits;
  return ATHB_OK;
}

// Impose the (global) maximum and apply the dt rule: after a step (after_step
// != 0: time += dt, nstep++, then the new dt, and the state of the other
// buffer becomes current) or before the loop (the first dt).
extern "C" int athb_finish_step(athb_ctx* c, unsigned long long max_dti_bits, int after_step) {
  if (!c) return athb_fail(ATHB_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  k_set_max_dti<<<1, 1, 0, c->stream>>>(c->st, max_dti_bits);
  k_finalize<<<1, 1, 0, c->stream>>>(c->st, c->dx1, c->dx2, after_step ? 1 : 0);
  CUDA_TRY(cudaGetLastError());
  if (after_step) c->cur ^= 1;
  return ATHB_OK;
}

// Ghost fill of the resident state: mode 1 the x1 boundaries (on the
// interior rows), 2 the x2 boundaries (whole rows), 3 both in that order;
// sides bit 0 the inner, bit 1 the outer boundary of that direction.
extern "C" int athb_ghost_fill(athb_ctx* c, int mode, int sides) {
  if (!c || mode < 1 || mode > 3 || sides < 0 || sides > 3) return athb_fail(ATHB_ERR_ARG, "bad arguments");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  if (mode == 3) {
    int rc = athb_launch_ghost_phase(c, c->cur, 1, sides);
    return rc ? rc : athb_launch_ghost_phase(c, c->cur, 2, sides);
  }
  return athb_launch_ghost_phase(c, c->cur, mode, sides);
}

// Rows [j0, j0+nrows) of all 11 planes of the resident state, ghost columns
// included, to / from a host buffer laid out [plane][row][Nx1+8].
static int rows_copy(athb_ctx* c, int j0, int nrows, double* host, bool to_host) {
  if (!c || !host || j0 < 0 || nrows < 1 || j0 + nrows > c->sy) return athb_fail(ATHB_ERR_ARG, "bad row range");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  double* dev = c->state[c->cur] + (size_t)j0 * c->pitch;
  const size_t w = sizeof(double) * c->sx;
  for (int p = 0; p < NSTATE; p++) {
    double* h = host + (size_t)p * nrows * c->sx;
    double* d = dev + (size_t)p * c->ps;
    if (to_host)
      CUDA_TRY(cudaMemcpy2DAsync(h, w, d, sizeof(double) * c->pitch, w, nrows, cudaMemcpyDeviceToHost, c->stream));
    else
      CUDA_TRY(cudaMemcpy2DAsync(d, sizeof(double) * c->pitch, h, w, w, nrows, cudaMemcpyHostToDevice, c->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return ATHB_OK;
}
extern "C" int athb_rows_get(athb_ctx* c, int j0, int nrows, double* host) {
  return rows_copy(c, j0, nrows, host, true);
}
extern "C" int athb_rows_put(athb_ctx* c, int j0, int nrows, const double* host) {
  return rows_copy(c, j0, nrows, const_cast<double*>(host), false);
}
