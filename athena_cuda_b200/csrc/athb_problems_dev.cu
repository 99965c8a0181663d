// athb_problems_dev.cu -- the blast and field-loop initial conditions formed
// on the GPU, directly in a grid's state buffer.
//
// Per cell these generators need only + - * / and sqrt (the sin/cos of the
// blast field angle are taken once, on the host, with libm), all correctly
// rounded on both sides with --fmad=false, so the device state is bit-identical
// to the host generators of problems.cpp and to the reference's
// (src/blast.c:25-72, src/field_loop.c:40-137).  The cpaw2d generator needs
// sin/cos per cell: its device form (k_gen_cpaw_*) takes CUDA's sin/cos
// (within 2 ulp) where the host takes libm's, so it agrees with the host
// generator to a few ulp of each term, not bit for bit; athb_generate keeps
// the host generator for cpaw2d and athb_generate_device takes this one.
//
// Also the cpaw2d L1 error (src/cpaw2d.c:222-302) against the initial state
// kept on the device, summed in the reference's order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "athb_internal.h"
#include "step_kernels.cuh"

using namespace athb;

namespace {

constexpr double kPi = 3.14159265358979323846;  // PI, src/defs.h:97

// Target: the state planes of one grid, a scratch plane for A_z, geometry.
struct GenTarget {
  double* s;   // state planes (plane stride ps, row pitch)
  double* az;  // one scratch plane of the same layout
  long long ps;
  int pitch, is, ie, js, je, nx1, nx2;
  double dx1, dx2, x1_0, x2_0, gamma_1;
};

__device__ __forceinline__ double& at(const GenTarget& t, int p, int j, int i) {
  return t.s[p * t.ps + (long long)j * t.pitch + i];
}
// cell-centre position (src/cc_pos.c:25-31, idisp = -is, jdisp = -js)
__device__ __forceinline__ double cc1(const GenTarget& t, int i) { return t.x1_0 + ((i - t.is) + 0.5) * t.dx1; }
__device__ __forceinline__ double cc2(const GenTarget& t, int j) { return t.x2_0 + ((j - t.js) + 0.5) * t.dx2; }

struct BlastPars {
  double rin, pa, prat, bxa, bya, bza;
};

// src/blast.c:39-70 (da = 1, ua = va = wa = 0), one thread per interior cell.
__global__ void __launch_bounds__(kThreads) k_gen_blast(GenTarget t, BlastPars q) {
  const int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= t.nx1 * t.nx2) return;
  const int j = t.js + c / t.nx1, i = t.is + c % t.nx1;
  const double da = 1.0, ua = 0.0, va = 0.0, wa = 0.0;
  at(t, P_D, j, i) = da;
  at(t, P_M1, j, i) = da * ua;
  at(t, P_M2, j, i) = da * va;
  at(t, P_M3, j, i) = da * wa;
  at(t, P_B1I, j, i) = q.bxa;
  at(t, P_B2I, j, i) = q.bya;
  at(t, P_B3I, j, i) = q.bza;
  at(t, P_B1C, j, i) = q.bxa;
  at(t, P_B2C, j, i) = q.bya;
  at(t, P_B3C, j, i) = q.bza;
  if (i == t.ie && t.ie > t.is) at(t, P_B1I, j, i + 1) = q.bxa;
  if (j == t.je && t.je > t.js) at(t, P_B2I, j + 1, i) = q.bya;
  const double x1 = cc1(t, i), x2 = cc2(t, j);
  const double rad = sqrt(x1 * x1 + x2 * x2);
  double pressure = q.pa;
  if (rad < q.rin) pressure = q.prat * q.pa;
  at(t, P_E, j, i) = pressure / t.gamma_1 + 0.5 * (q.bxa * q.bxa + q.bya * q.bya + q.bza * q.bza) +
                     0.5 * da * (ua * ua + va * va + wa * wa);
}

struct LoopPars {
  double rad, amp, vflow, x1size, x2size, diag;
  int iprob;
};

// src/field_loop.c:62-78: A_z at the corners [is, ie+1] x [js, je+1].
__global__ void __launch_bounds__(kThreads) k_gen_loop_az(GenTarget t, LoopPars q) {
  const int w = t.nx1 + 1;
  const int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= w * (t.nx2 + 1)) return;
  const int j = t.js + c / w, i = t.is + c % w;
  const double x1f = cc1(t, i) - 0.5 * t.dx1;
  const double x2f = cc2(t, j) - 0.5 * t.dx2;
  double a = 0.0;
  if (q.iprob == 1 && (x1f * x1f + x2f * x2f) < q.rad * q.rad) a = q.amp * (q.rad - sqrt(x1f * x1f + x2f * x2f));
  t.az[(long long)j * t.pitch + i] = a;
}

// src/field_loop.c:80-110: density, momentum and the face fields from curl A_z.
__global__ void __launch_bounds__(kThreads) k_gen_loop_faces(GenTarget t, LoopPars q) {
  const int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= t.nx1 * t.nx2) return;
  const int j = t.js + c / t.nx1, i = t.is + c % t.nx1;
  auto AZ = [&](int jj, int ii) { return t.az[(long long)jj * t.pitch + ii]; };
  const double d = 1.0;
  at(t, P_D, j, i) = d;
  at(t, P_M1, j, i) = d * q.vflow * q.x1size / q.diag;
  at(t, P_M2, j, i) = d * q.vflow * q.x2size / q.diag;
  at(t, P_M3, j, i) = 0.0;
  at(t, P_B1I, j, i) = (AZ(j + 1, i) - AZ(j, i)) / t.dx2;
  at(t, P_B2I, j, i) = -(AZ(j, i + 1) - AZ(j, i)) / t.dx1;
  at(t, P_B3I, j, i) = 0.0;
  if (i == t.ie) at(t, P_B1I, j, i + 1) = (AZ(j + 1, i + 1) - AZ(j, i + 1)) / t.dx2;
  if (j == t.je) at(t, P_B2I, j + 1, i) = -(AZ(j + 1, i + 1) - AZ(j + 1, i)) / t.dx1;
}

// src/field_loop.c:112-130: cell-centred fields and total energy.
__global__ void __launch_bounds__(kThreads) k_gen_loop_centres(GenTarget t) {
  const int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= t.nx1 * t.nx2) return;
  const int j = t.js + c / t.nx1, i = t.is + c % t.nx1;
  const double b1 = 0.5 * (at(t, P_B1I, j, i) + at(t, P_B1I, j, i + 1));
  const double b2 = 0.5 * (at(t, P_B2I, j, i) + at(t, P_B2I, j + 1, i));
  const double b3 = at(t, P_B3I, j, i);
  at(t, P_B1C, j, i) = b1;
  at(t, P_B2C, j, i) = b2;
  at(t, P_B3C, j, i) = b3;
  const double m1 = at(t, P_M1, j, i), m2 = at(t, P_M2, j, i), m3 = at(t, P_M3, j, i);
  at(t, P_E, j, i) = 1.0 / t.gamma_1 + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) +
                     0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / at(t, P_D, j, i);
}

// src/cpaw2d.c:123-158: face fields from the vector potential A3
// (src/cpaw2d.c:310-314) at the faces [is, ie+1] x [js, je+1].
__device__ __forceinline__ double cpaw_A3(const athb_cpaw_wave& w, double x1, double x2) {
  return w.b_par * (x1 * w.sin_a - x2 * w.cos_a) - (w.b_perp / w.k_par) * cos(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
}

__global__ void __launch_bounds__(kThreads) k_gen_cpaw_faces(GenTarget t, athb_cpaw_wave w) {
  const int nw = t.nx1 + 1;
  const int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= nw * (t.nx2 + 1)) return;
  const int j = t.js + c / nw, i = t.is + c % nw;
  double x1 = cc1(t, i), x2 = cc2(t, j);
  const double cs = cos(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
  x1 -= 0.5 * t.dx1;
  x2 -= 0.5 * t.dx2;
  at(t, P_B1I, j, i) = -(cpaw_A3(w, x1, x2 + t.dx2) - cpaw_A3(w, x1, x2)) / t.dx2;
  at(t, P_B2I, j, i) = (cpaw_A3(w, x1 + t.dx1, x2) - cpaw_A3(w, x1, x2)) / t.dx1;
  at(t, P_B3I, j, i) = w.b_perp * cs;
}

// src/cpaw2d.c:160-180: the cell-centred state.
__global__ void __launch_bounds__(kThreads) k_gen_cpaw_centres(GenTarget t, athb_cpaw_wave w) {
  const int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= t.nx1 * t.nx2) return;
  const int j = t.js + c / t.nx1, i = t.is + c % t.nx1;
  const double x1 = cc1(t, i), x2 = cc2(t, j);
  const double sn = sin(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
  const double cs = cos(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
  const double den = w.den;
  const double m1 = den * (w.v_par * w.cos_a - w.v_perp * sn * w.sin_a);
  const double m2 = den * (w.v_par * w.sin_a + w.v_perp * sn * w.cos_a);
  const double m3 = den * w.v_perp * cs;
  at(t, P_D, j, i) = den;
  at(t, P_M1, j, i) = m1;
  at(t, P_M2, j, i) = m2;
  at(t, P_M3, j, i) = m3;
  const double b1 = 0.5 * (at(t, P_B1I, j, i) + at(t, P_B1I, j, i + 1));
  const double b2 = 0.5 * (at(t, P_B2I, j, i) + at(t, P_B2I, j + 1, i));
  const double b3 = w.b_perp * cs;
  at(t, P_B1C, j, i) = b1;
  at(t, P_B2C, j, i) = b2;
  at(t, P_B3C, j, i) = b3;
  at(t, P_E, j, i) = w.pres / t.gamma_1 + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) + 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / den;
}

// The L1 sums of src/cpaw2d.c:244-255, one warp per variable: each sum runs
// over the interior in row-major order, one addition after the other as the
// reference's loop adds (a chain of nx1*nx2 dependent additions per warp).
// The lanes form |U - Soln| of 32 consecutive cells at once and every lane
// adds them in lane order, so all lanes hold the same running sum.
__global__ void __launch_bounds__(256) k_cpaw_l1(const double* __restrict__ s, const double* __restrict__ soln,
                                                 long long ps, int pitch, int is, int js, int nx1, int nx2,
                                                 double* out) {
  const int plane = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (plane >= 8) return;
  const double* u = s + plane * ps;
  const double* v = soln + plane * ps;
  double acc = 0.0;
  for (int j = 0; j < nx2; j++) {
    const long long row = (long long)(js + j) * pitch + is;
    for (int i0 = 0; i0 < nx1; i0 += 32) {
      const int i = i0 + lane;
      const double d = i < nx1 ? fabs(u[row + i] - v[row + i]) : 0.0;
      const int n = min(32, nx1 - i0);
      for (int k = 0; k < n; k++) acc += __shfl_sync(0xffffffffu, d, k);
    }
  }
  if (lane == 0) out[plane] = acc;
}

int blocks_of(long long n) { return (int)((n + kThreads - 1) / kThreads); }

}  // namespace

// Fill the state planes at `state` (zeroed first, as a fresh host array is)
// with problem `kind`'s initial condition on `stream`.  ATHB_ERR_NOTFOUND when
// the problem has no device form.
int athb_generate_device_into(int kind, const athb_params* p, double* state, double* az, long long ps, int pitch,
                              const athb_config& cfg, cudaStream_t stream) {
  if (kind != kProblemBlast && kind != kProblemFieldLoop && kind != kProblemCpaw2d)
    return athb_fail(ATHB_ERR_NOTFOUND, "problem has no device generator");
  GenTarget t;
  t.s = state;
  t.az = az;
  t.ps = ps;
  t.pitch = pitch;
  t.nx1 = cfg.nx1;
  t.nx2 = cfg.nx2;
  t.is = kNghost; t.ie = cfg.nx1 + kNghost - 1;
  t.js = kNghost; t.je = cfg.nx2 + kNghost - 1;
  t.dx1 = (cfg.x1max - cfg.x1min) / (double)cfg.nx1;
  t.dx2 = (cfg.x2max - cfg.x2min) / (double)cfg.nx2;
  t.x1_0 = cfg.x1min;
  t.x2_0 = cfg.x2min;
  t.gamma_1 = cfg.gamma - 1.0;
  cudaError_t e = cudaMemsetAsync(state, 0, sizeof(double) * (size_t)ps * NSTATE, stream);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "generate: %s", cudaGetErrorString(e));
  const int cells = blocks_of((long long)cfg.nx1 * cfg.nx2);
  if (kind == kProblemBlast) {
    double angle = 0.0, b0 = 0.0;
    BlastPars q;
    if (athb_params_getd(p, "problem", "radius", &q.rin) || athb_params_getd(p, "problem", "pamb", &q.pa) ||
        athb_params_getd(p, "problem", "prat", &q.prat) || athb_params_getd(p, "problem", "b0", &b0) ||
        athb_params_getd(p, "problem", "angle", &angle))
      return athb_fail(ATHB_ERR_PARSE, "problem \"blast\": missing <problem> parameter");
    const double theta = (kPi / 180.0) * angle;  // host libm, as src/blast.c:44-46
    q.bxa = b0 * cos(theta);
    q.bya = b0 * sin(theta);
    q.bza = 0.0;
    k_gen_blast<<<cells, kThreads, 0, stream>>>(t, q);
  } else if (kind == kProblemCpaw2d) {
    athb_cpaw_wave w;
    if (athb_cpaw2d_wave(p, cfg.nx1, cfg.nx2, t.dx1, t.dx2, &w))
      return athb_fail(ATHB_ERR_PARSE, "problem \"cpaw2d\": missing <problem> parameter");
    k_gen_cpaw_faces<<<blocks_of((long long)(cfg.nx1 + 1) * (cfg.nx2 + 1)), kThreads, 0, stream>>>(t, w);
    k_gen_cpaw_centres<<<cells, kThreads, 0, stream>>>(t, w);
  } else {
    LoopPars q;
    double iprob = 0.0;
    if (athb_params_getd(p, "problem", "rad", &q.rad) || athb_params_getd(p, "problem", "amp", &q.amp) ||
        athb_params_getd(p, "problem", "vflow", &q.vflow) || athb_params_getd(p, "problem", "iprob", &iprob))
      return athb_fail(ATHB_ERR_PARSE, "problem \"field_loop\": missing <problem> parameter");
    q.iprob = (int)iprob;
    q.x1size = t.dx1 * (double)cfg.nx1;
    q.x2size = t.dx2 * (double)cfg.nx2;
    q.diag = sqrt(q.x1size * q.x1size + q.x2size * q.x2size);
    k_gen_loop_az<<<blocks_of((long long)(cfg.nx1 + 1) * (cfg.nx2 + 1)), kThreads, 0, stream>>>(t, q);
    k_gen_loop_faces<<<cells, kThreads, 0, stream>>>(t, q);
    k_gen_loop_centres<<<cells, kThreads, 0, stream>>>(t);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "generate: %s", cudaGetErrorString(e));
  return ATHB_OK;
}

int athb_keep_cpaw_soln(athb_ctx* c) {
  cudaError_t e = cudaSuccess;
  if (!c->cpaw_soln) e = cudaMalloc(&c->cpaw_soln, sizeof(double) * 8 * (size_t)c->ps);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->cpaw_soln, c->state[c->cur], sizeof(double) * 8 * (size_t)c->ps, cudaMemcpyDeviceToDevice,
                        c->stream);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "cpaw2d solution: %s", cudaGetErrorString(e));
  return ATHB_OK;
}

extern "C" int athb_generate_device(athb_ctx* c, const char* name, const athb_params* p) {
  if (!c || !name || !p) return athb_fail(ATHB_ERR_ARG, "null argument");
  cudaError_t e = cudaSetDevice(c->cfg.device);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "athb_generate_device: %s", cudaGetErrorString(e));
  const int kind = athb_builtin_problem(name);
  if (kind == kProblemNone)
    return athb_fail(ATHB_ERR_NOTFOUND, "problem \"%s\" has no device generator (use athb_generate)", name);
  int rc = athb_generate_device_into(kind, p, c->state[c->cur], c->scr + (size_t)S_EMF * c->ps, c->ps, c->pitch,
                                     c->cfg, c->stream);
  if (rc == ATHB_OK && kind == kProblemCpaw2d) rc = athb_keep_cpaw_soln(c);
  if (rc) return rc;
  return athb_set_clock(c, 0.0, 0.0, 0);
}

// src/cpaw2d.c:222-302 (Userwork_after_loop): the eight sums on the device in
// the reference's order (bit-identical to its host loop), then the RMS and the
// means as the reference forms them.
extern "C" int athb_cpaw2d_errors(athb_ctx* c, double err[9]) {
  if (!c || !err) return athb_fail(ATHB_ERR_ARG, "null argument");
  if (!c->cpaw_soln) return athb_fail(ATHB_ERR_ARG, "context was not created by the cpaw2d problem");
  cudaError_t e = cudaSetDevice(c->cfg.device);
  double* dsum = c->scr;   // 8 doubles of scratch (free between steps)
  if (e == cudaSuccess) {
    k_cpaw_l1<<<1, 256, 0, c->stream>>>(c->state[c->cur], c->cpaw_soln, c->ps, c->pitch, c->is, c->js, c->cfg.nx1,
                                       c->cfg.nx2, dsum);
    e = cudaGetLastError();
  }
  double s[8];
  if (e == cudaSuccess) e = cudaMemcpyAsync(s, dsum, sizeof s, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "athb_cpaw2d_errors: %s", cudaGetErrorString(e));
  // s: d M1 M2 M3 E B1c B2c B3c (state plane order)
  double rms = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + s[3] * s[3];
  rms += s[5] * s[5] + s[6] * s[6] + s[7] * s[7];
  rms += s[4] * s[4];
  const double n = (double)(c->cfg.nx1 * c->cfg.nx2);
  err[0] = sqrt(rms) / n;
  for (int k = 0; k < 8; k++) err[1 + k] = s[k] / n;
  return ATHB_OK;
}

extern "C" int athb_generate(athb_ctx* c, const char* name, const athb_params* p) {
  if (!c || !name || !p) return athb_fail(ATHB_ERR_ARG, "null argument");
  cudaError_t e = cudaSetDevice(c->cfg.device);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "athb_generate: %s", cudaGetErrorString(e));
  const int kind = athb_builtin_problem(name);
  if (kind == kProblemBlast || kind == kProblemFieldLoop) {
    int rc = athb_generate_device_into(kind, p, c->state[c->cur], c->scr + (size_t)S_EMF * c->ps, c->ps, c->pitch,
                                       c->cfg, c->stream);
    if (rc) return rc;
    return athb_set_clock(c, 0.0, 0.0, 0);
  }
  return athb_generate_host(c, name, p);
}
