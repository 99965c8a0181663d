// adjoint_host.cpp -- TEST INFRASTRUCTURE: the generic step, the
// tangent-linear model and the adjoint of the main loop
// (athena_cuda_b200/csrc/adjoint_driver.cuh) run on the host CPU through a
// loop executor, so the tests can check them without a GPU:
//   * the generic step against the oracle (bit for bit),
//   * the tangent-linear model against the adjoint (dot-product test),
//   * checkpoint schedules against storing every state (bit for bit).
// Built by tests/hostcheck/build.py into tests/_build/libathb_hostcheck.so.
#include <cstdlib>
#include <cstring>

#include "../../athena_cuda_b200/csrc/adjoint_driver.cuh"
#include "../../include/athena_b200.h"

using namespace athb;

namespace {

struct HostExec {
  template <class F> void items(const GenRange& r, const F& f) {
    for (int j = r.j0; j <= r.j1; j++)
      for (int i = r.i0; i <= r.i1; i++) f(j, i);
  }
  template <class F> void single(const F& f) { f(); }
  void argmax(const double* p, const GenRange& r, int pitch, MaxLoc* out) {
    double m = -1.0;
    long long arg = -1;
    for (int j = r.j0; j <= r.j1; j++)
      for (int i = r.i0; i <= r.i1; i++) {
        const long long o = (long long)j * pitch + i;
        if (arg < 0 || p[o] > m) { m = p[o]; arg = o; }
      }
    out->m = m;
    out->arg = arg;
  }
  void sum(const double* p, const GenRange& r, int pitch, double* out) {
    double s = 0.0;
    for (int j = r.j0; j <= r.j1; j++)
      for (int i = r.i0; i <= r.i1; i++) s += p[(long long)j * pitch + i];
    *out = s;
  }
  template <int FLUX, class D> void forward_step(D& d, int cur, bool) { d.template generic_step_double<FLUX>(cur); }
  double* alloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
  void* alloc_bytes(size_t b) { return calloc(b ? b : 1, 1); }
  void release(double* p) { free(p); }
  void release_bytes(void* p) { free(p); }
  void zero(double* p, size_t n) { memset(p, 0, n * sizeof(double)); }
  void zero_bytes(void* p, size_t b) { memset(p, 0, b); }
  void copy(double* d, const double* s, size_t n) { memcpy(d, s, n * sizeof(double)); }
  void to_host(void* d, const void* s, size_t b) { memcpy(d, s, b); }
  bool ok() const { return true; }
};

LoopGeom geom_of(const athb_config* c) {
  LoopGeom G;
  G.nx1 = c->nx1; G.nx2 = c->nx2;
  G.sx = c->nx1 + 8; G.sy = c->nx2 + 8;
  G.pitch = G.sx;   // the host arrays are unpadded
  G.ly = 4;
  G.ps = (long long)G.sx * G.sy;
  G.is = 4; G.ie = c->nx1 + 3; G.js = 4; G.je = c->nx2 + 3;
  G.dx1 = (c->x1max - c->x1min) / (double)c->nx1;
  G.dx2 = (c->x2max - c->x2min) / (double)c->nx2;
  G.cour = c->cour_no;
  G.tlim = c->tlim;
  G.eos = Eos{c->gamma, c->gamma - 1.0, c->gamma - 2.0};
  G.flux = c->flux;
  G.bc[0] = c->bc_ix1; G.bc[1] = c->bc_ox1; G.bc[2] = c->bc_ix2; G.bc[3] = c->bc_ox2;
  return G;
}

}  // namespace

extern "C" {

// The loop run through the generic double step: S0 (interior used; ghosts
// and dt^0 formed as at loop entry), N steps; writes S^N (ghosts included),
// the last dt (new_dt's value) and the time.  Returns the steps taken.
int hc_forward(const athb_config* cfg, const double* S0, int N, double* SN, double* dt_out, double* time_out) {
  HostExec x;
  AdjointDriver<HostExec> d(x, geom_of(cfg));
  d.setup(N, false);
  x.copy(d.S[0], S0, d.state_doubles());
  int cur = 0;
  d.entry();
  int n = 0;
  for (; n < N; n++) {
    if (!(*d.timev < cfg->tlim)) break;
    if (cfg->flux == ATHB_FLUX_HLLE) d.fwd_step_double<kFluxHlle>(cur); else d.fwd_step_double<kFluxRoe>(cur);
    cur ^= 1;
    x.argmax(d.tape + (long long)G_DTI * d.G.ps, d.interior(), d.G.pitch, d.ml);
    x.single(DtNextFn<double>{d.cf, d.timev, d.ml, nullptr, d.rec, n + 1, d.G.cour, d.G.tlim, d.G.dx1, d.G.dx2});
  }
  x.copy(SN, d.S[cur], d.state_doubles());
  *dt_out = d.rec[n].rule;
  *time_out = *d.timev;
  d.release();
  return n;
}

// Tangent-linear model: J and dJ (objective (B1c^2+B2c^2)/2 summed over the
// interior) after N steps from S0 along dS0; S^N and dS^N.
int hc_tlm(const athb_config* cfg, const double* S0, const double* dS0, int N, double* J, double* dJ, double* SN,
           double* dSN) {
  HostExec x;
  AdjointDriver<HostExec> d(x, geom_of(cfg));
  d.setup(N, true);
  x.copy(d.S[0], S0, d.state_doubles());
  x.copy(d.dS[0], dS0, d.state_doubles());
  int cur = 0;
  if (cfg->flux == ATHB_FLUX_HLLE) d.tlm<kFluxHlle>(N, cur); else d.tlm<kFluxRoe>(N, cur);
  *J = d.sc->J;
  *dJ = d.sc->dJ;
  if (SN) x.copy(SN, d.S[cur], d.state_doubles());
  if (dSN) x.copy(dSN, d.dS[cur], d.state_doubles());
  d.release();
  return 0;
}

// Adjoint: J and dJ/dS0 (interior entries; ghosts zero) after N steps, with
// nslot state snapshots (slot 0 holds S^0).  Returns the steps reversed.
int hc_adjoint(const athb_config* cfg, const double* S0, int N, int nslot, double* J, double* grad,
               long long* advances) {
  HostExec x;
  AdjointDriver<HostExec> d(x, geom_of(cfg));
  d.setup(N, false);
  d.nslot = nslot < 1 ? 1 : nslot;
  if (nslot < 0) {   // tape mode: every state and every step's tape kept
    d.nslot = N + 1;
    d.tapes = x.alloc((size_t)N * d.tape_doubles());
  }
  d.slots = x.alloc((size_t)d.nslot * d.state_doubles());
  x.copy(d.S[0], S0, d.state_doubles());
  int lc = 0, steps = 0;
  if (cfg->flux == ATHB_FLUX_HLLE) d.adjoint<kFluxHlle>(N, lc, steps); else d.adjoint<kFluxRoe>(N, lc, steps);
  *J = d.sc->J;
  x.copy(grad, d.lam[lc], d.state_doubles());
  if (advances) *advances = d.advances;
  d.release();
  return steps;
}

// The adjoint seeded with a cotangent of the final state (state layout,
// entries a step writes): J = <seed, S^N>, grad = (dS^N/dS^0)^T seed.
int hc_adjoint_seed(const athb_config* cfg, const double* S0, const double* seed, int N, int nslot, double* J,
                    double* grad) {
  HostExec x;
  AdjointDriver<HostExec> d(x, geom_of(cfg));
  d.setup(N, false);
  d.nslot = nslot < 1 ? 1 : nslot;
  d.slots = x.alloc((size_t)d.nslot * d.state_doubles());
  double* sd = x.alloc(d.state_doubles());
  x.copy(sd, seed, d.state_doubles());
  d.seed = sd;
  x.copy(d.S[0], S0, d.state_doubles());
  int lc = 0, steps = 0;
  if (cfg->flux == ATHB_FLUX_HLLE) d.adjoint<kFluxHlle>(N, lc, steps); else d.adjoint<kFluxRoe>(N, lc, steps);
  *J = d.sc->J;
  x.copy(grad, d.lam[lc], d.state_doubles());
  d.release();
  x.release(sd);
  return steps;
}

}  // extern "C"
