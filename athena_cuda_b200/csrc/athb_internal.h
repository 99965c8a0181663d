// athb_internal.h -- shared between the translation units of libathena_b200.so.
#pragma once

#include <cuda_runtime.h>

#include "../../include/athena_b200.h"

namespace athb {
struct StepState;
constexpr int kNghost = 4;  // nghost, src/defs.h:82
}  // namespace athb

struct athb_ctx {
  athb_config cfg;
  int sx = 0, sy = 0, pitch = 0;  // padded host extents and device row pitch
  long long ps = 0;               // device plane stride (doubles)
  int is = 0, ie = 0, js = 0, je = 0;
  int ly = 4;                     // y-sweep march segment length
  double dx1 = 0, dx2 = 0, x1_0 = 0, x2_0 = 0;
  double* state[2] = {nullptr, nullptr};  // double-buffered state planes
  int cur = 0;                            // buffer holding the current state
  double* scr = nullptr;                  // scratch planes
  athb::StepState* st = nullptr;          // device time-stepping state
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // two-step loop, per parity
  // drop-in staging: AoS copy of the host Gas array
  void* aos = nullptr;
  size_t aos_bytes = 0;
  // cpaw2d reference solution: planes d .. B3c of the initial state, kept on
  // the device in the state layout (stride ps, row pitch)
  double* cpaw_soln = nullptr;
  // device blocks of the last adjoint / tangent-linear call, kept for the
  // next call when athb_adjoint_keep_workspace is on (athb_adjoint.cu)
  struct athb_adj_cache* adj_cache = nullptr;
  int adj_keep = 0;
};
void athb_adjoint_cache_free(athb_ctx* c);

// internal helpers (athb_core.cu)
int athb_fail(int code, const char* fmt, ...);
int athb_ctx_validate(const athb_config* cfg);
int athb_set_clock(athb_ctx* c, double dt, double time, int nstep);
int athb_launch_integrate(athb_ctx* c, int from);
int athb_launch_integrate_split(athb_ctx* c, int from, cudaEvent_t* ev);
int athb_launch_ghost(athb_ctx* c, int buf);
int athb_launch_ghost_phase(athb_ctx* c, int buf, int mode, int sides);
int athb_launch_cfl(athb_ctx* c, int buf);
int athb_launch_set_dt(athb_ctx* c, double dt);
int athb_read_clock(athb_ctx* c, athb::StepState* h);

// problem generators (problems.cpp, athb_problems_dev.cu)
enum { kProblemNone = 0, kProblemBlast, kProblemFieldLoop, kProblemCpaw2d };
int athb_builtin_problem(const char* name);  // kind of the registered generator, if built in
int athb_generate_host(athb_ctx* c, const char* name, const athb_params* p);
int athb_generate_device_into(int kind, const athb_params* p, double* state, double* az, long long ps, int pitch,
                              const athb_config& cfg, cudaStream_t stream);
// the wave of the cpaw2d problem (src/cpaw2d.c:56-120), host libm
struct athb_cpaw_wave {
  double sin_a, cos_a, k_par, b_par, b_perp, v_par, v_perp, pres, den;
};
int athb_cpaw2d_wave(const athb_params* p, int nx1, int nx2, double dx1, double dx2, athb_cpaw_wave* w);
// copy the current state's planes d .. B3c into c->cpaw_soln (allocated once)
int athb_keep_cpaw_soln(athb_ctx* c);
