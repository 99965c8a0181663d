// athb_dropin.cu -- the reference's own entry points (integrate_2d, set_bvals,
// new_dt and their init/destruct companions) on host Grid buffers, so a program
// written against the reference CPU path links against this library unchanged.
//
// Each call moves only what it reads and writes between the host Grid (AoS
// Gas rows, src/athena.h:43-52) and the device planes:
//   integrate_2d  up: U, B1i, B2i (all cells)  down: the cells the reference
//                 step writes (src/__integrate_2d__.c:476-534)
//   new_dt        up: interior U               down: 8 bytes (max 1/dt)
//   set_bvals     up: the 4-cell interior band  down: the ghost frame
// Host arrays are page-locked (cudaHostRegister) on first use.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "athb_internal.h"
#include "step_types.cuh"

using namespace athb;

// reference globals (src/globals.h:18-20); weak so the host program's win
extern "C" {
__attribute__((weak)) double Gamma = 0.0;
__attribute__((weak)) double Gamma_1 = 0.0;
__attribute__((weak)) double Gamma_2 = 0.0;
__attribute__((weak)) double CourNo = 0.0;
// src/par.c:250 par_geti, provided by the host program when present
__attribute__((weak)) int par_geti(char* block, char* name);
}

namespace {

struct DropIn {
  athb_ctx* ctx = nullptr;
  int nx1 = 0, nx2 = 0;
  int bc[4] = {0, 0, 0, 0};
  bool bc_set = false;
  int flux = ATHB_FLUX_ROE;
  int device = -1;  // < 0: ATHB_DEVICE from the environment, else 0
  athb_VBCFun_t user_bc[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<void*> registered;
  unsigned long long h2d = 0, d2h = 0;  // bytes moved by the drop-in calls
  // Host-unchanged mode (opt-in): the caller does not modify the Grid
  // between the drop-in calls, so the device copy stays authoritative.
  int host_unchanged = -1;       // < 0: ATHB_DROPIN_HOST_UNCHANGED from the environment
  bool valid = false;            // device state c->cur equals the host Grid (ghosts: see below)
  bool ghosts_stale = false;     // ... except its ghost frame (after a step, before set_bvals)
  bool have_max = false;         // the CFL max of the last step's output is cached
  double max_dti = 0.0;
  const void* grid_key = nullptr;  // the Grid the device copy mirrors
};
DropIn g_drop;

[[noreturn]] void die(const char* where) {
  fprintf(stderr, "[%s]: %s\n", where, athb_last_error());
  exit(EXIT_FAILURE);
}
void check(int rc, const char* where) { if (rc) die(where); }
void check_cuda(cudaError_t e, const char* where) {
  if (e != cudaSuccess) { athb_fail(ATHB_ERR_CUDA, "%s", cudaGetErrorString(e)); die(where); }
}

// AoS Gas rows <-> SoA planes over the box [j0,j1] x [i0,i1] of a grid.
__global__ void k_aos_to_soa(const athb_Gas* __restrict__ aos, double* __restrict__ s, long long ps,
                             int pitch, int sx, int j0, int i0, int ni, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int j = j0 + t / ni, i = i0 + t % ni;
  const athb_Gas g = aos[(long long)j * sx + i];
  const long long o = (long long)j * pitch + i;
  s[0 * ps + o] = g.d; s[1 * ps + o] = g.M1; s[2 * ps + o] = g.M2; s[3 * ps + o] = g.M3;
  s[4 * ps + o] = g.E; s[5 * ps + o] = g.B1c; s[6 * ps + o] = g.B2c; s[7 * ps + o] = g.B3c;
}
__global__ void k_soa_to_aos(const double* __restrict__ s, athb_Gas* __restrict__ aos, long long ps,
                             int pitch, int sx, int j0, int i0, int ni, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int j = j0 + t / ni, i = i0 + t % ni;
  const long long o = (long long)j * pitch + i;
  athb_Gas g;
  g.d = s[0 * ps + o]; g.M1 = s[1 * ps + o]; g.M2 = s[2 * ps + o]; g.M3 = s[3 * ps + o];
  g.E = s[4 * ps + o]; g.B1c = s[5 * ps + o]; g.B2c = s[6 * ps + o]; g.B3c = s[7 * ps + o];
  aos[(long long)j * sx + i] = g;
}

// A box of cells [j0, j0+nj) x [i0, i0+ni).
struct Box { int j0, i0, nj, ni; };

bool host_unchanged_mode() {
  if (g_drop.host_unchanged < 0) {
    const char* env = getenv("ATHB_DROPIN_HOST_UNCHANGED");
    g_drop.host_unchanged = (env && atoi(env) != 0) ? 1 : 0;
  }
  return g_drop.host_unchanged == 1;
}

// The device copy can stand in for the host Grid only in host-unchanged mode,
// for the Grid it was made from.
bool device_current(athb_Grid* pG) {
  return host_unchanged_mode() && g_drop.valid && g_drop.grid_key == (const void*)pG->U[0];
}
void invalidate() {
  g_drop.valid = false;
  g_drop.ghosts_stale = false;
  g_drop.have_max = false;
}

bool contiguous(void** rows, size_t row_bytes, int nrows) {
  for (int j = 1; j < nrows; j++)
    if ((char*)rows[j] != (char*)rows[0] + (size_t)j * row_bytes) return false;
  return true;
}

void pin(void* p, size_t bytes) {
  for (void* q : g_drop.registered) if (q == p) return;
  if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) == cudaSuccess) g_drop.registered.push_back(p);
  else cudaGetLastError();  // pageable copies still work
}

athb_ctx* context_for(athb_Grid* pG, const char* where) {
  DropIn& d = g_drop;
  if (!d.bc_set) {
    if (!par_geti)
      die((athb_fail(ATHB_ERR_ARG, "boundary flags unknown: call set_bvals_init() with the host "
                                   "program's par.c linked, or athb_dropin_set_bc()"), where));
    d.bc[0] = par_geti((char*)"grid", (char*)"ibc_x1");
    d.bc[1] = par_geti((char*)"grid", (char*)"obc_x1");
    d.bc[2] = par_geti((char*)"grid", (char*)"ibc_x2");
    d.bc[3] = par_geti((char*)"grid", (char*)"obc_x2");
    d.bc_set = true;
  }
  if (d.ctx && (d.ctx->cfg.nx1 != pG->Nx1 || d.ctx->cfg.nx2 != pG->Nx2)) {
    athb_destroy(d.ctx);
    d.ctx = nullptr;
    invalidate();
  }
  if (!d.ctx) {
    athb_config cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.nx1 = pG->Nx1; cfg.nx2 = pG->Nx2;
    cfg.x1min = pG->x1_0; cfg.x1max = pG->x1_0 + pG->dx1 * pG->Nx1;
    cfg.x2min = pG->x2_0; cfg.x2max = pG->x2_0 + pG->dx2 * pG->Nx2;
    cfg.bc_ix1 = d.bc[0]; cfg.bc_ox1 = d.bc[1]; cfg.bc_ix2 = d.bc[2]; cfg.bc_ox2 = d.bc[3];
    // user boundary functions replace a side; give the kernel a valid flag
    for (int k = 0; k < 4; k++)
      if ((&cfg.bc_ix1)[k] == 0) (&cfg.bc_ix1)[k] = BC_PERIODIC;
    cfg.gamma = Gamma > 1.0 ? Gamma : 5.0 / 3.0;
    cfg.cour_no = CourNo; cfg.tlim = 0.0; cfg.nlim = -1;
    cfg.flux = d.flux;
    cfg.device = d.device;
    if (cfg.device < 0) {
      const char* env = getenv("ATHB_DEVICE");  // one process per GPU without a code change
      cfg.device = env ? atoi(env) : 0;
    }
    check(athb_create(&cfg, &d.ctx), where);
  }
  athb_ctx* c = d.ctx;
  // geometry and EOS follow the host Grid and globals at every call
  c->dx1 = pG->dx1; c->dx2 = pG->dx2; c->x1_0 = pG->x1_0; c->x2_0 = pG->x2_0;
  c->cfg.gamma = Gamma;
  c->cfg.cour_no = CourNo;
  if (pG->is != c->is || pG->js != c->js || pG->ie != c->ie || pG->je != c->je)
    die((athb_fail(ATHB_ERR_ARG, "Grid index range does not match nghost=4 layout"), where));
  check_cuda(cudaSetDevice(c->cfg.device), where);
  const size_t aos_bytes = sizeof(athb_Gas) * (size_t)c->sx * c->sy;
  if (c->aos_bytes < aos_bytes) {
    cudaFree(c->aos);
    c->aos = nullptr;
    check_cuda(cudaMalloc(&c->aos, aos_bytes), where);
    c->aos_bytes = aos_bytes;
  }
  pin(pG->U[0], aos_bytes);
  pin(pG->B1i[0], sizeof(double) * (size_t)c->sx * c->sy);
  pin(pG->B2i[0], sizeof(double) * (size_t)c->sx * c->sy);
  pin(pG->B3i[0], sizeof(double) * (size_t)c->sx * c->sy);
  return c;
}

// host -> device copies of a box of U (via the AoS staging buffer) and of
// the face-field planes listed in mask (bit 0 B1i, 1 B2i, 2 B3i).
void up_box(athb_ctx* c, athb_Grid* pG, int buf, Box b, bool with_u, int mask, const char* where) {
  if (b.nj <= 0 || b.ni <= 0) return;
  cudaStream_t s = c->stream;
  const size_t gas = sizeof(athb_Gas), dbl = sizeof(double);
  const bool ucont = contiguous((void**)pG->U, gas * c->sx, c->sy);
  if (with_u) {
    g_drop.h2d += gas * (size_t)b.ni * b.nj;
    athb_Gas* dst = (athb_Gas*)c->aos;
    if (ucont) {
      check_cuda(cudaMemcpy2DAsync(dst + (size_t)b.j0 * c->sx + b.i0, gas * c->sx,
                                   pG->U[0] + (size_t)b.j0 * c->sx + b.i0, gas * c->sx, gas * b.ni, b.nj,
                                   cudaMemcpyHostToDevice, s), where);
    } else {
      for (int j = b.j0; j < b.j0 + b.nj; j++)
        check_cuda(cudaMemcpyAsync(dst + (size_t)j * c->sx + b.i0, pG->U[j] + b.i0, gas * b.ni,
                                   cudaMemcpyHostToDevice, s), where);
    }
    const int n = b.nj * b.ni;
    k_aos_to_soa<<<(n + 255) / 256, 256, 0, s>>>(dst, c->state[buf], c->ps, c->pitch, c->sx, b.j0, b.i0, b.ni, n);
    check_cuda(cudaGetLastError(), where);
  }
  double** planes[3] = {pG->B1i, pG->B2i, pG->B3i};
  for (int k = 0; k < 3; k++) {
    if (!((mask >> k) & 1)) continue;
    g_drop.h2d += dbl * (size_t)b.ni * b.nj;
    double* dst = c->state[buf] + (P_B1I + k) * c->ps;
    if (contiguous((void**)planes[k], dbl * c->sx, c->sy)) {
      check_cuda(cudaMemcpy2DAsync(dst + (size_t)b.j0 * c->pitch + b.i0, dbl * c->pitch,
                                   planes[k][0] + (size_t)b.j0 * c->sx + b.i0, dbl * c->sx, dbl * b.ni,
                                   b.nj, cudaMemcpyHostToDevice, s), where);
    } else {
      for (int j = b.j0; j < b.j0 + b.nj; j++)
        check_cuda(cudaMemcpyAsync(dst + (size_t)j * c->pitch + b.i0, planes[k][j] + b.i0, dbl * b.ni,
                                   cudaMemcpyHostToDevice, s), where);
    }
  }
}

void down_box(athb_ctx* c, athb_Grid* pG, int buf, Box b, bool with_u, int mask, const char* where) {
  if (b.nj <= 0 || b.ni <= 0) return;
  cudaStream_t s = c->stream;
  const size_t gas = sizeof(athb_Gas), dbl = sizeof(double);
  if (with_u) {
    g_drop.d2h += gas * (size_t)b.ni * b.nj;
    athb_Gas* src = (athb_Gas*)c->aos;
    const int n = b.nj * b.ni;
    k_soa_to_aos<<<(n + 255) / 256, 256, 0, s>>>(c->state[buf], src, c->ps, c->pitch, c->sx, b.j0, b.i0, b.ni, n);
    check_cuda(cudaGetLastError(), where);
    if (contiguous((void**)pG->U, gas * c->sx, c->sy)) {
      check_cuda(cudaMemcpy2DAsync(pG->U[0] + (size_t)b.j0 * c->sx + b.i0, gas * c->sx,
                                   src + (size_t)b.j0 * c->sx + b.i0, gas * c->sx, gas * b.ni, b.nj,
                                   cudaMemcpyDeviceToHost, s), where);
    } else {
      for (int j = b.j0; j < b.j0 + b.nj; j++)
        check_cuda(cudaMemcpyAsync(pG->U[j] + b.i0, src + (size_t)j * c->sx + b.i0, gas * b.ni,
                                   cudaMemcpyDeviceToHost, s), where);
    }
  }
  double** planes[3] = {pG->B1i, pG->B2i, pG->B3i};
  for (int k = 0; k < 3; k++) {
    if (!((mask >> k) & 1)) continue;
    g_drop.d2h += dbl * (size_t)b.ni * b.nj;
    const double* src = c->state[buf] + (P_B1I + k) * c->ps;
    if (contiguous((void**)planes[k], dbl * c->sx, c->sy)) {
      check_cuda(cudaMemcpy2DAsync(planes[k][0] + (size_t)b.j0 * c->sx + b.i0, dbl * c->sx,
                                   src + (size_t)b.j0 * c->pitch + b.i0, dbl * c->pitch, dbl * b.ni, b.nj,
                                   cudaMemcpyDeviceToHost, s), where);
    } else {
      for (int j = b.j0; j < b.j0 + b.nj; j++)
        check_cuda(cudaMemcpyAsync(planes[k][j] + b.i0, src + (size_t)j * c->pitch + b.i0, dbl * b.ni,
                                   cudaMemcpyDeviceToHost, s), where);
    }
  }
}

}  // namespace

extern "C" void athb_dropin_set_bc(int ibc_x1, int obc_x1, int ibc_x2, int obc_x2) {
  g_drop.bc[0] = ibc_x1; g_drop.bc[1] = obc_x1; g_drop.bc[2] = ibc_x2; g_drop.bc[3] = obc_x2;
  g_drop.bc_set = true;
  if (g_drop.ctx) {
    g_drop.ctx->cfg.bc_ix1 = ibc_x1; g_drop.ctx->cfg.bc_ox1 = obc_x1;
    g_drop.ctx->cfg.bc_ix2 = ibc_x2; g_drop.ctx->cfg.bc_ox2 = obc_x2;
  }
}

// Opt-in: the caller promises not to modify the Grid between drop-in calls
// (the reference main loop, src/main.c:229-307, only calls integrate_2d,
// new_dt and set_bvals on it between outputs).  Every call still leaves the
// host Grid exactly as the reference would; what is skipped is the upload of
// data the device already holds.
extern "C" void athb_dropin_set_host_unchanged(int on) {
  g_drop.host_unchanged = on ? 1 : 0;
  invalidate();
}

extern "C" void athb_dropin_bytes(unsigned long long* h2d, unsigned long long* d2h) {
  if (h2d) *h2d = g_drop.h2d;
  if (d2h) *d2h = g_drop.d2h;
}

// The GPU the drop-in calls use (set before the first call; default: the
// ATHB_DEVICE environment variable, else device 0).
extern "C" void athb_dropin_set_device(int device) {
  if (g_drop.ctx && g_drop.ctx->cfg.device != device) {
    athb_destroy(g_drop.ctx);
    g_drop.ctx = nullptr;
    invalidate();
  }
  g_drop.device = device;
}

extern "C" void athb_dropin_set_flux(int flux) {
  g_drop.flux = flux;
  if (g_drop.ctx) g_drop.ctx->cfg.flux = flux;
}

// src/__integrate_2d__.c:573
extern "C" void integrate_init_2d(int nx1, int nx2) {
  g_drop.nx1 = nx1;
  g_drop.nx2 = nx2;
}

// src/__integrate_2d__.c:543
extern "C" void integrate_destruct_2d(void) {
  if (g_drop.ctx) { athb_destroy(g_drop.ctx); g_drop.ctx = nullptr; }
  invalidate();
  for (void* p : g_drop.registered) cudaHostUnregister(p);
  g_drop.registered.clear();
}

// src/lr_states_plm.c:253,270: the GPU path keeps no per-slice scratch.
extern "C" void lr_states_init(int nx1, int nx2) { (void)nx1; (void)nx2; }
extern "C" void lr_states_destruct(void) {}

// src/__integrate_2d__.c:100
// The ghost frame of a grid as four boxes.
void frame_boxes(const athb_ctx* c, Box f[4]) {
  f[0] = Box{0, 0, c->js, c->sx};                            // rows below js
  f[1] = Box{c->je + 1, 0, c->sy - c->je - 1, c->sx};        // rows above je
  f[2] = Box{c->js, 0, c->cfg.nx2, c->is};                   // left columns
  f[3] = Box{c->js, c->ie + 1, c->cfg.nx2, c->sx - c->ie - 1};  // right columns
}

extern "C" void integrate_2d(athb_Grid* pG) {
  const char* where = "integrate_2d";
  athb_ctx* c = context_for(pG, where);
  const int a = c->cur, b = a ^ 1;
  const int sx = c->sx, sy = c->sy, nx1 = c->cfg.nx1, nx2 = c->cfg.nx2;
  const bool mode = host_unchanged_mode();
  // The step reads U and B1i/B2i everywhere (B3i is only written).
  if (device_current(pG)) {
    if (g_drop.ghosts_stale) {   // set_bvals was not called: the host frame is the input
      Box f[4];
      frame_boxes(c, f);
      for (const Box& q : f) up_box(c, pG, a, q, true, 0x3, where);
    }
  } else {
    up_box(c, pG, a, Box{0, 0, sy, sx}, true, 0x3, where);
  }
  check(athb_launch_set_dt(c, pG->dt), where);
  if (mode) check_cuda(cudaMemsetAsync(&c->st->max_dti_bits, 0, sizeof(unsigned long long), c->stream), where);
  check(athb_launch_integrate(c, a), where);
  // the cells the reference writes
  down_box(c, pG, b, Box{c->js, c->is, nx2, nx1}, true, 0x4, where);  // U, B3i interior
  down_box(c, pG, b, Box{c->js, c->is, nx2, nx1 + 1}, false, 0x1, where);  // B1i + column ie+1
  down_box(c, pG, b, Box{c->js, c->is, nx2 + 1, nx1}, false, 0x2, where);  // B2i + row je+1
  unsigned long long bits = 0;
  if (mode) {   // the update kernel reduced the CFL max of the output: new_dt's value
    check_cuda(cudaMemcpyAsync(&bits, &c->st->max_dti_bits, sizeof bits, cudaMemcpyDeviceToHost, c->stream), where);
    g_drop.d2h += sizeof bits;
  }
  check_cuda(cudaStreamSynchronize(c->stream), where);
  if (mode) {
    // buffer b now holds the step's output: the host Grid's interior, with
    // the input's ghost frame still on the host until set_bvals
    c->cur = b;
    g_drop.valid = true;
    g_drop.ghosts_stale = true;
    g_drop.grid_key = pG->U[0];
    memcpy(&g_drop.max_dti, &bits, sizeof bits);
    g_drop.have_max = true;
  }
}

// src/new_dt.c:25-100
extern "C" void new_dt(athb_Grid* pG) {
  const char* where = "new_dt";
  athb_ctx* c = context_for(pG, where);
  const int a = c->cur;
  double max_dti;
  if (device_current(pG) && g_drop.have_max) {
    max_dti = g_drop.max_dti;   // reduced by the step that produced this state
  } else {
    if (!device_current(pG)) up_box(c, pG, a, Box{c->js, c->is, c->cfg.nx2, c->cfg.nx1}, true, 0, where);
    check_cuda(cudaMemsetAsync(&c->st->max_dti_bits, 0, sizeof(unsigned long long), c->stream), where);
    check(athb_launch_cfl(c, a), where);
    unsigned long long bits = 0;
    check_cuda(cudaMemcpyAsync(&bits, &c->st->max_dti_bits, sizeof bits, cudaMemcpyDeviceToHost, c->stream), where);
    g_drop.d2h += sizeof bits;
    check_cuda(cudaStreamSynchronize(c->stream), where);
    memcpy(&max_dti, &bits, sizeof max_dti);
  }
  // src/new_dt.c:93-97
  if (pG->nstep == 0) pG->dt = CourNo / max_dti;
  else pG->dt = rmin(2.0 * pG->dt, CourNo / max_dti);
}

// src/set_bvals.c:152
extern "C" void set_bvals_init(athb_Grid* pG) {
  (void)pG;
  if (g_drop.bc_set) return;
  if (!par_geti) {
    fprintf(stderr, "[set_bvals_init]: par_geti() is not linked; use athb_dropin_set_bc()\n");
    exit(EXIT_FAILURE);
  }
  int bc[4];
  const char* names[4] = {"ibc_x1", "obc_x1", "ibc_x2", "obc_x2"};
  for (int k = 0; k < 4; k++) {
    if (g_drop.user_bc[k]) { bc[k] = 0; continue; }
    bc[k] = par_geti((char*)"grid", (char*)names[k]);
    if (bc[k] != BC_REFLECT && bc[k] != BC_OUTFLOW && bc[k] != BC_PERIODIC) {
      fprintf(stderr, "[set_bvals_init]: %s = %d unknown\n", names[k], bc[k]);
      exit(EXIT_FAILURE);
    }
  }
  athb_dropin_set_bc(bc[0], bc[1], bc[2], bc[3]);
}

// src/set_bvals.c:269
extern "C" void set_bvals_fun(int dir, athb_VBCFun_t prob_bc) {
  if (dir < 0 || dir > 3) {
    fprintf(stderr, "[set_bvals_fun]: Unknown direction = %d\n", dir);
    exit(EXIT_FAILURE);
  }
  g_drop.user_bc[dir] = prob_bc;
}

// src/set_bvals.c:114
extern "C" void set_bvals(athb_Grid* pG, int var_flag) {
  const char* where = "set_bvals";
  if (var_flag == 1) return;  // every reference boundary function returns for var_flag 1
  const bool user = g_drop.user_bc[0] || g_drop.user_bc[1] || g_drop.user_bc[2] || g_drop.user_bc[3];
  athb_ctx* c = context_for(pG, where);
  const int a = c->cur, sx = c->sx, sy = c->sy, nx1 = c->cfg.nx1, nx2 = c->cfg.nx2;
  const int is = c->is, ie = c->ie, js = c->js, je = c->je;
  if (user) {
    invalidate();   // user functions write the host Grid
    // Reference order with host callbacks: the whole state goes up, built-in
    // sides run on the GPU one direction at a time, user functions run on the
    // host Grid in between.
    const int sides1 = (g_drop.user_bc[0] ? 0 : 1) | (g_drop.user_bc[1] ? 0 : 2);
    const int sides2 = (g_drop.user_bc[2] ? 0 : 1) | (g_drop.user_bc[3] ? 0 : 2);
    up_box(c, pG, a, Box{0, 0, sy, sx}, true, 0x7, where);
    check(athb_launch_ghost_phase(c, a, 1, sides1), where);
    down_box(c, pG, a, Box{0, 0, sy, sx}, true, 0x7, where);
    check_cuda(cudaStreamSynchronize(c->stream), where);
    if (g_drop.user_bc[0]) g_drop.user_bc[0](pG, var_flag);
    if (g_drop.user_bc[1]) g_drop.user_bc[1](pG, var_flag);
    up_box(c, pG, a, Box{0, 0, sy, sx}, true, 0x7, where);
    check(athb_launch_ghost_phase(c, a, 2, sides2), where);
    down_box(c, pG, a, Box{0, 0, sy, sx}, true, 0x7, where);
    check_cuda(cudaStreamSynchronize(c->stream), where);
    if (g_drop.user_bc[2]) g_drop.user_bc[2](pG, var_flag);
    if (g_drop.user_bc[3]) g_drop.user_bc[3](pG, var_flag);
    return;
  }
  if (device_current(pG)) {
    // the device state is the host Grid's interior: fill its frame there and
    // bring the frame down
    if (g_drop.ghosts_stale) check(athb_launch_ghost(c, a), where);
    g_drop.ghosts_stale = false;
    Box f[4];
    frame_boxes(c, f);
    for (const Box& q : f) down_box(c, pG, a, q, true, 0x7, where);
    check_cuda(cudaStreamSynchronize(c->stream), where);
    return;
  }
  // Sources of every ghost value: the interior band within 4 cells of a
  // boundary, plus the interior faces B1i(ie+1) and B2i(je+1).
  const Box band[4] = {
      Box{js, is, 4, nx1 + 1},          // bottom interior rows
      Box{je - 3, is, 5, nx1 + 1},      // top interior rows (+ row je+1 of B2i)
      Box{js, is, nx2 + 1, 4},          // left interior columns
      Box{js, ie - 3, nx2 + 1, 5},      // right interior columns (+ column ie+1 of B1i)
  };
  for (const Box& b : band) up_box(c, pG, a, b, true, 0x7, where);
  check(athb_launch_ghost(c, a), where);
  const Box frame[4] = {
      Box{0, 0, js, sx},                  // rows below js
      Box{je + 1, 0, sy - je - 1, sx},    // rows above je
      Box{js, 0, nx2, is},                // left columns
      Box{js, ie + 1, nx2, sx - ie - 1},  // right columns
  };
  for (const Box& b : frame) down_box(c, pG, a, b, true, 0x7, where);
  check_cuda(cudaStreamSynchronize(c->stream), where);
}
