// adjoint_driver.cuh -- the tangent-linear model and the adjoint of the
// reference main loop (src/main.c:229-307: tlim clamp, integrate_2d,
// time += dt, new_dt, set_bvals) over N iterations, with binomial
// ("revolve") checkpointing of states in device memory.
//
// Written once against an executor Exec that supplies
//   items(range, f)        f(j, i) for every item of a GenRange
//   single(f)              f() once
//   argmax(plane, range, pitch, out)   max of plane over range, lowest linear
//                          index among equal maxima -> out->m, out->arg
//   sum(plane, range, pitch, out)      deterministic sum -> *out
//   alloc / release / zero / copy / to_host / from_host
// The sm_100a executor (athb_adjoint.cu) launches kernels on one stream; the
// host executor (tests/hostcheck) runs the same functors in loops, so the CPU
// tests exercise this very code.
//
// Loop differentiated, with dt as a function of the state:
//   dt_rule^0 = CourNo / m(S^0)                          (new_dt, nstep == 0)
//   dt^n      = tlim - time^n if that is smaller, else dt_rule^n   (clamp)
//   S^{n+1}   = set_bvals(integrate_2d(S^n, dt^n))
//   time^{n+1} = time^n + dt^n
//   dt_rule^{n+1} = MIN(2 dt^n, CourNo / m(S^{n+1}))      (src/new_dt.c:93-97)
// with m(S) = max over interior cells of the CFL rate (src/new_dt.c:37-85),
// differentiated through the cell that attains it (lowest index on ties).
#pragma once

#include <cstdio>
#include <vector>

#include "step_adjoint.cuh"

namespace athb {

constexpr int G_DTI = NGEN;        // tape plane: CFL rate of each interior cell of the step's output
constexpr int NTAPE = NGEN + 1;

struct MaxLoc { double m; long long arg; };

// Per-iteration record of the forward sweep.
struct StepRec {
  double dt;      // dt^n used by the step (after the clamp)
  double rule;    // dt_rule^n
  double time;    // time^n
  int clamped;    // dt^n = tlim - time^n
  int cap;        // dt_rule^n = 2 dt^{n-1} (n >= 1)
};

// Scalars of the reverse sweep.
struct AdjScal {
  double lrule;   // adjoint of dt_rule of the step after the one being reversed
  double ltime;   // adjoint of time^{n+1}
  double dtsum;   // sum of A_DT of the step being reversed
  double J;       // objective
  double dJ;      // tangent of the objective
  int nonfinite;  // a non-finite adjoint or state was seen
};

// ---------------------------------------------------------------------------
// functors
// ---------------------------------------------------------------------------
enum FwdStage { F_PLMX, F_PLMY, F_RIEX, F_RIEY, F_ECC0, F_EMF0, F_CORX, F_CORY, F_CORE, F_EMF1, F_UPD };

template <int STAGE, int FLUX, class T> struct FwdFn {
  GenArgs<T> a;
  Planes<T> dti;   // G_DTI plane for F_UPD
  ATHB_MEM void operator()(int j, int i) const {
    if (STAGE == F_PLMX) gen_plm(a, 0, j, i);
    else if (STAGE == F_PLMY) gen_plm(a, 1, j, i);
    else if (STAGE == F_RIEX) gen_riemann<FLUX>(a, 0, j, i);
    else if (STAGE == F_RIEY) gen_riemann<FLUX>(a, 1, j, i);
    else if (STAGE == F_ECC0) gen_ecc0(a, j, i);
    else if (STAGE == F_EMF0) gen_emf(a, 0, j, i);
    else if (STAGE == F_CORX) gen_correct_x<FLUX>(a, j, i);
    else if (STAGE == F_CORY) gen_correct_y<FLUX>(a, j, i);
    else if (STAGE == F_CORE) gen_correct_e(a, j, i);
    else if (STAGE == F_EMF1) gen_emf(a, 1, j, i);
    else dti.set(a.o(j, i), gen_update(a, j, i));
  }
};

// CFL rate of the cells of a state (new_dt on S^0)
template <class T> struct CflFn {
  Planes<T> s, dti;
  long long ps;
  int pitch;
  double dx1, dx2;
  Eos eos;
  ATHB_MEM void operator()(int j, int i) const {
    const long long o = (long long)j * pitch + i;
    dti.set(o, gen_cell_dti(s.get(P_D * ps + o), s.get(P_M1 * ps + o), s.get(P_M2 * ps + o),
                            s.get(P_M3 * ps + o), s.get(P_E * ps + o), eos, dx1, dx2));
  }
};

template <class T> struct GhostFn {
  Planes<T> s;
  long long ps;
  int pitch;
  GhostGeom g;
  ATHB_MEM void operator()(int j, int i) const {
    if (j >= g.js && j <= g.je && i >= g.is && i <= g.ie) return;
    gen_ghost(s, ps, pitch, g, j, i);
  }
};

enum AdjStage { R_UPD, R_EMF1, R_FLUX2, R_CORX, R_CORY, R_CORE, R_HALF, R_EMF0, R_FLUX1, R_SRC, R_RIEX, R_RIEY,
                R_PLMX, R_PLMY, R_PRIMX, R_PRIMY };

template <int STAGE, int FLUX> struct AdjFn {
  AdjArgs a;
  ATHB_MEM void operator()(int j, int i) const {
    if (STAGE == R_UPD) adj_update(a, j, i);
    else if (STAGE == R_EMF1) adj_emf1(a, j, i);
    else if (STAGE == R_FLUX2) adj_flux2(a, j, i);
    else if (STAGE == R_CORX) adj_correct_x<FLUX>(a, j, i);
    else if (STAGE == R_CORY) adj_correct_y<FLUX>(a, j, i);
    else if (STAGE == R_CORE) adj_correct_e(a, j, i);
    else if (STAGE == R_HALF) adj_half_faces(a, j, i);
    else if (STAGE == R_EMF0) adj_emf0(a, j, i);
    else if (STAGE == R_FLUX1) adj_flux1(a, j, i);
    else if (STAGE == R_SRC) adj_sources(a, j, i);
    else if (STAGE == R_RIEX) adj_riemann<FLUX>(a, 0, j, i);
    else if (STAGE == R_RIEY) adj_riemann<FLUX>(a, 1, j, i);
    else if (STAGE == R_PLMX) adj_plm(a, 0, j, i);
    else if (STAGE == R_PLMY) adj_plm(a, 1, j, i);
    else if (STAGE == R_PRIMX) adj_prim_gather(a, 0, j, i);
    else adj_prim_gather(a, 1, j, i);
  }
};

struct FoldFn {
  double* l;
  long long ps;
  int pitch;
  GhostGeom g;
  int pass;   // 2: x2 rows, 1: x1 columns, 0: clear the frame
  ATHB_MEM void operator()(int j, int i) const {
    if (pass == 2) fold_x2(l, ps, pitch, g, j, i);
    else if (pass == 1) fold_x1(l, ps, pitch, g, j, i);
    else clear_frame(l, ps, pitch, g, j, i);
  }
};

// Objective J = sum over interior cells of (B1c^2 + B2c^2)/2: per-cell value,
// its tangent, or its adjoint seed.
struct ObjFn {
  const double* s;       // state
  const double* ds;      // tangent state (mode 1)
  double* out;           // per-cell value (A_TMP-like plane) or the seed planes (mode 2)
  long long ps;
  int pitch, mode;       // 0 value, 1 tangent, 2 seed
  ATHB_MEM void operator()(int j, int i) const {
    const long long o = (long long)j * pitch + i;
    const double b1 = s[P_B1C * ps + o], b2 = s[P_B2C * ps + o];
    if (mode == 0) out[o] = 0.5 * (b1 * b1 + b2 * b2);
    else if (mode == 1) out[o] = b1 * ds[P_B1C * ps + o] + b2 * ds[P_B2C * ps + o];
    else { out[P_B1C * ps + o] = b1; out[P_B2C * ps + o] = b2; }
  }
};

// <seed, S> per cell: the 11 planes of an interior cell in plane order, then
// the outer faces B1i(ie+1) and B2i(je+1) on the last column and row (the
// entries a step writes; the seed is zero elsewhere).
struct SeedDotFn {
  const double* s;
  const double* seed;
  double* out;
  long long ps;
  int pitch, ie, je;
  ATHB_MEM void operator()(int j, int i) const {
    const long long o = (long long)j * pitch + i;
    double v = 0.0;
    for (int p = 0; p < NSTATE; p++) v += seed[p * ps + o] * s[p * ps + o];
    if (i == ie) v += seed[P_B1I * ps + o + 1] * s[P_B1I * ps + o + 1];
    if (j == je) v += seed[P_B2I * ps + o + pitch] * s[P_B2I * ps + o + pitch];
    out[o] = v;
  }
};

// dt after a forward step (value form for the records; T = Dual carries the
// tangent): time, the rule, the clamp.  cf holds the next step's factors.
template <class T> struct DtNextFn {
  StepCoef<T>* cf;
  T* time;               // running time (Exec memory)
  const MaxLoc* ml;      // max CFL rate of S^{n+1} and its cell
  const double* dti_t;   // tangent plane of the CFL rates (T = Dual), or null
  StepRec* rec;          // records (value part), index n+1
  int n1;                // n+1
  double cour, tlim, dx1, dx2;
  ATHB_MEM void operator()() const {
    const T dt = cf->dt;
    *time = *time + dt;
    T m = T(ml->m);
    set_tangent(m);
    const T cfl = cour / m;
    const T two = 2.0 * dt;
    T rule;
    int cap = 0;
    if (two < cfl) { rule = two; cap = 1; } else rule = cfl;   // rmin(2 dt, CourNo / max_dti)
    T next = rule;
    int clamped = 0;
    if ((tlim - *time) < rule) { next = tlim - *time; clamped = 1; }
    *cf = make_coef(next, dx1, dx2);
    if (rec) {
      StepRec r;
      r.dt = value_of(next); r.rule = value_of(rule); r.time = value_of(*time); r.clamped = clamped; r.cap = cap;
      rec[n1] = r;
    }
  }
  ATHB_MEM void set_tangent(double&) const {}
  ATHB_MEM void set_tangent(Dual& m) const { m.t = dti_t ? dti_t[ml->arg] : 0.0; }
};

// dt^0 at loop entry: CourNo / m(S^0), then the clamp
template <class T> struct Dt0Fn {
  StepCoef<T>* cf;
  T* time;
  const MaxLoc* ml;
  const double* dti_t;
  StepRec* rec;
  double cour, tlim, dx1, dx2;
  ATHB_MEM void operator()() const {
    *time = T(0.0);
    T m = T(ml->m);
    set_tangent(m);
    const T rule = cour / m;
    T dt = rule;
    int clamped = 0;
    if ((tlim - *time) < rule) { dt = tlim - *time; clamped = 1; }
    *cf = make_coef(dt, dx1, dx2);
    if (rec) {
      StepRec r;
      r.dt = value_of(dt); r.rule = value_of(rule); r.time = 0.0; r.clamped = clamped; r.cap = 0;
      rec[0] = r;
    }
  }
  ATHB_MEM void set_tangent(double&) const {}
  ATHB_MEM void set_tangent(Dual& m) const { m.t = dti_t ? dti_t[ml->arg] : 0.0; }
};

// coefficients of step n from the records (advances and taped steps)
struct CoefFromRecFn {
  StepCoef<double>* cf;
  const StepRec* rec;
  int n;
  double dx1, dx2;
  ATHB_MEM void operator()() const { *cf = make_coef(rec[n].dt, dx1, dx2); }
};

// Adjoint of dt_rule^{k} = CourNo / m(S^k) at the cell attaining m, added
// into the adjoint of S^k (when that branch produced dt_rule^k).
struct DtRuleAdjFn {
  const double* s;       // S^k
  double* l;             // adjoint of S^k
  const MaxLoc* ml;
  AdjScal* sc;
  const StepRec* rec;
  int k;                 // which dt_rule
  long long ps;
  double cour, dx1, dx2;
  Eos eos;
  ATHB_MEM void operator()() const {
    const double lr = sc->lrule;
    if (lr == 0.0) return;
    if (k >= 1 && rec[k].cap) return;  // the 2 dt branch: carried by the caller
    const double m = ml->m;
    const double lm = -cour / (m * m) * lr;
    const long long o = ml->arg;
    double g[5];
    cell_dti_adj(s[P_D * ps + o], s[P_M1 * ps + o], s[P_M2 * ps + o], s[P_M3 * ps + o], s[P_E * ps + o], eos, dx1,
                 dx2, lm, g);
    l[P_D * ps + o] += g[0];
    l[P_M1 * ps + o] += g[1];
    l[P_M2 * ps + o] += g[2];
    l[P_M3 * ps + o] += g[3];
    l[P_E * ps + o] += g[4];
  }
};

// After the adjoint of step n: the adjoint of dt^n, of time^n and of dt_rule^n.
struct DtStepAdjFn {
  AdjScal* sc;
  const StepRec* rec;
  int n;      // step reversed
  int last;   // n == N-1 (dt_rule^{n+1} is not used)
  ATHB_MEM void operator()() const {
    double ldt = sc->dtsum + sc->ltime;   // time^{n+1} = time^n + dt^n
    if (!last && rec[n + 1].cap) ldt += 2.0 * sc->lrule;
    double ltime = sc->ltime;
    double lrule = ldt;
    if (rec[n].clamped) {                 // dt^n = tlim - time^n
      ltime -= ldt;
      lrule = 0.0;
    }
    sc->ltime = ltime;
    sc->lrule = lrule;
    if (!(ldt == ldt) || !(ltime == ltime)) sc->nonfinite = 1;
  }
};

// ---------------------------------------------------------------------------
// the driver
// ---------------------------------------------------------------------------
struct LoopGeom {
  int nx1, nx2, sx, sy, pitch;
  int ly;          // column-march length of the fast predictor
  long long ps;
  int is, ie, js, je;
  double dx1, dx2, cour, tlim;
  Eos eos;
  int flux;
  int bc[4];
};

// binomial checkpointing: cost(l, c) = minimal number of forward steps to
// reverse l steps with c checkpoints (the start state counting as one);
// p(l, c) = t l - beta(c+1, t-1), t the least with beta(c, t) >= l,
// beta(c, t) = (c+t)! / (c! t!) (Griewank, "Achieving logarithmic growth of
// temporal and spatial complexity in reverse automatic differentiation", 1992)
inline double revolve_beta(int c, int t, double cap) {
  double b = 1.0;
  for (int k = 1; k <= t; k++) {
    b = b * (double)(c + k) / (double)k;
    if (b > cap) return cap;
  }
  return b;
}
inline long long revolve_cost(long long l, int c) {
  if (l <= 1) return 0;
  if (c <= 1) return l * (l - 1) / 2;
  int t = 0;
  while (revolve_beta(c, t, 4e18) < (double)l) t++;
  return (long long)t * l - (long long)revolve_beta(c + 1, t - 1, 4e18);
}
// best first checkpoint position in [a+1, b-1] for reversing [a, b) with s
// free slots (the start state held in its own)
inline int revolve_split(int a, int b, int s) {
  const long long l = b - a;
  long long best = -1;
  int bm = a + 1;
  for (int m = 1; m < l; m++) {
    const long long c = m + revolve_cost(l - m, s) + revolve_cost(m, s + 1);
    if (best < 0 || c < best) { best = c; bm = a + m; }
  }
  return bm;
}

template <class Exec> struct AdjointDriver {
  Exec& x;
  LoopGeom G;
  // buffers in Exec memory
  double* S[2] = {nullptr, nullptr};      // working states
  double* dS[2] = {nullptr, nullptr};     // tangent states (TLM)
  double* tape = nullptr;                 // NTAPE planes (value)
  double* dtape = nullptr;                // NTAPE planes (tangent, TLM)
  double* adj = nullptr;                  // NADJ planes
  double* lam[2] = {nullptr, nullptr};    // adjoint states
  double* slots = nullptr;                // snapshots
  int nslot = 0;
  double* tapes = nullptr;                // tape mode: the tape of every step, recorded in the first sweep
  double* tape0 = nullptr;                // the working tape
  StepRec* rec = nullptr;
  AdjScal* sc = nullptr;
  MaxLoc* ml = nullptr;
  StepCoef<double>* cf = nullptr;
  StepCoef<Dual>* cfd = nullptr;
  double* timev = nullptr;
  Dual* timed = nullptr;
  int nrec = 0;
  long long advances = 0, taped = 0;

  explicit AdjointDriver(Exec& e, const LoopGeom& g) : x(e), G(g) {}

  size_t plane() const { return (size_t)G.ps; }
  size_t state_doubles() const { return (size_t)NSTATE * G.ps; }
  GenRange full() const { return GenRange{0, G.sx - 1, 0, G.sy - 1}; }
  GenRange interior() const { return range_interior(G.is, G.ie, G.js, G.je); }
  GhostGeom ghost_geom() const {
    GhostGeom g;
    g.is = G.is; g.ie = G.ie; g.js = G.js; g.je = G.je; g.sx = G.sx; g.sy = G.sy;
    for (int k = 0; k < 4; k++) g.bc[k] = G.bc[k];
    return g;
  }

  // Allocate everything but the snapshots; nsteps bounds the records.
  int setup(int nsteps, bool tlm) {
    nrec = nsteps + 1;
    S[0] = x.alloc(state_doubles());
    S[1] = x.alloc(state_doubles());
    tape = x.alloc((size_t)NTAPE * G.ps);
    tape0 = tape;
    sc = (AdjScal*)x.alloc_bytes(sizeof(AdjScal));
    ml = (MaxLoc*)x.alloc_bytes(sizeof(MaxLoc));
    cf = (StepCoef<double>*)x.alloc_bytes(sizeof(StepCoef<double>));
    timev = x.alloc(1);
    rec = (StepRec*)x.alloc_bytes(sizeof(StepRec) * (size_t)nrec);
    if (tlm) {
      dS[0] = x.alloc(state_doubles());
      dS[1] = x.alloc(state_doubles());
      dtape = x.alloc((size_t)NTAPE * G.ps);
      cfd = (StepCoef<Dual>*)x.alloc_bytes(sizeof(StepCoef<Dual>));
      timed = (Dual*)x.alloc_bytes(sizeof(Dual));
    } else {
      adj = x.alloc((size_t)NADJ * G.ps);
      lam[0] = x.alloc(state_doubles());
      lam[1] = x.alloc(state_doubles());
    }
    if (!x.ok()) return -1;
    x.zero(S[0], state_doubles());
    x.zero(S[1], state_doubles());
    x.zero(tape, (size_t)NTAPE * G.ps);
    if (tlm) {
      x.zero(dS[0], state_doubles());
      x.zero(dS[1], state_doubles());
      x.zero(dtape, (size_t)NTAPE * G.ps);
    } else {
      x.zero(adj, (size_t)NADJ * G.ps);
      x.zero(lam[0], state_doubles());
      x.zero(lam[1], state_doubles());
    }
    x.zero_bytes(sc, sizeof(AdjScal));
    return 0;
  }
  size_t tape_doubles() const { return (size_t)NTAPE * G.ps; }
  double* tape_of(int n) const { return tapes + (size_t)n * tape_doubles(); }

  void release() {
    if (tape0) tape = tape0;
    for (double* p : {S[0], S[1], dS[0], dS[1], tape, dtape, adj, lam[0], lam[1], slots, tapes, timev}) x.release(p);
    x.release_bytes(sc); x.release_bytes(ml); x.release_bytes(cf); x.release_bytes(cfd); x.release_bytes(timed);
    x.release_bytes(rec);
  }

  template <class T> GenArgs<T> gen_args(Planes<T> in, Planes<T> out, Planes<T> scr, const StepCoef<T>* c) const {
    GenArgs<T> a;
    a.in = in; a.out = out; a.scr = scr; a.coef = c;
    a.ps = G.ps; a.pitch = G.pitch;
    a.is = G.is; a.ie = G.ie; a.js = G.js; a.je = G.je;
    a.dx1 = G.dx1; a.dx2 = G.dx2; a.eos = G.eos;
    return a;
  }

  // One generic step in -> out (interior), every intermediate into scr, the
  // CFL rates of the output into scr's G_DTI plane; then the ghost fill.
  template <int FLUX, class T>
  void step(Planes<T> in, Planes<T> out, Planes<T> scr, const StepCoef<T>* c) {
    const GenArgs<T> a = gen_args(in, out, scr, c);
    Planes<T> dti = scr;
    dti.v += (long long)G_DTI * G.ps;
    offset_tangent(dti);
    const int is = G.is, ie = G.ie, js = G.js, je = G.je;
    x.items(range_plm(is, ie, js, je), FwdFn<F_PLMX, FLUX, T>{a, dti});
    x.items(range_plm(is, ie, js, je), FwdFn<F_PLMY, FLUX, T>{a, dti});
    x.items(range_riemann_x(is, ie, js, je), FwdFn<F_RIEX, FLUX, T>{a, dti});
    x.items(range_riemann_y(is, ie, js, je), FwdFn<F_RIEY, FLUX, T>{a, dti});
    x.items(range_plm(is, ie, js, je), FwdFn<F_ECC0, FLUX, T>{a, dti});
    x.items(range_emf0(is, ie, js, je), FwdFn<F_EMF0, FLUX, T>{a, dti});
    x.items(range_correct_x(is, ie, js, je), FwdFn<F_CORX, FLUX, T>{a, dti});
    x.items(range_correct_y(is, ie, js, je), FwdFn<F_CORY, FLUX, T>{a, dti});
    x.items(range_correct_e(is, ie, js, je), FwdFn<F_CORE, FLUX, T>{a, dti});
    x.items(range_emf1(is, ie, js, je), FwdFn<F_EMF1, FLUX, T>{a, dti});
    x.items(interior(), FwdFn<F_UPD, FLUX, T>{a, dti});
    x.items(full(), GhostFn<T>{out, G.ps, G.pitch, ghost_geom()});
  }
  static void offset_tangent(Planes<double>&) {}
  void offset_tangent(Planes<Dual>& p) const { p.t += (long long)G_DTI * G.ps; }

  Planes<double> pd(double* v) const { Planes<double> p; p.v = v; return p; }
  Planes<Dual> pdual(double* v, double* t) const { Planes<Dual> p; p.v = v; p.t = t; return p; }

  template <class T> void cfl(Planes<T> s, Planes<T> dti) {
    x.items(interior(), CflFn<T>{s, dti, G.ps, G.pitch, G.dx1, G.dx2, G.eos});
  }

  // One plain step S[cur] -> S[cur^1] with the factors in cf, ghosts filled,
  // the CFL rates of the result in the G_DTI tape plane; taped: every
  // intermediate the adjoint reads is kept in the tape.  The executor runs it
  // (the GPU with the fast kernels, the host with the generic step).
  template <int FLUX> void fwd_step_double(int cur, bool taped = false) {
    x.template forward_step<FLUX>(*this, cur, taped);
  }
  template <int FLUX> void generic_step_double(int cur) {
    step<FLUX, double>(pd(S[cur]), pd(S[cur ^ 1]), pd(tape), cf);
  }

  // ---------------- tangent-linear model ----------------
  // S[0]/dS[0] hold S^0 / dS^0 (interior; ghosts are filled here).  Runs N
  // steps; J and dJ land in sc->J / sc->dJ; S[cur] / dS[cur] hold S^N / dS^N.
  template <int FLUX> int tlm(int N, int& cur) {
    cur = 0;
    Planes<Dual> s0 = pdual(S[0], dS[0]);
    x.items(full(), GhostFn<Dual>{s0, G.ps, G.pitch, ghost_geom()});
    cfl(s0, pdual(tape + (long long)G_DTI * G.ps, dtape + (long long)G_DTI * G.ps));
    x.argmax(tape + (long long)G_DTI * G.ps, interior(), G.pitch, ml);
    x.single(Dt0Fn<Dual>{cfd, timed, ml, dtape + (long long)G_DTI * G.ps, nullptr, G.cour, G.tlim, G.dx1, G.dx2});
    for (int n = 0; n < N; n++) {
      step<FLUX, Dual>(pdual(S[cur], dS[cur]), pdual(S[cur ^ 1], dS[cur ^ 1]), pdual(tape, dtape), cfd);
      cur ^= 1;
      x.argmax(tape + (long long)G_DTI * G.ps, interior(), G.pitch, ml);
      x.single(DtNextFn<Dual>{cfd, timed, ml, dtape + (long long)G_DTI * G.ps, nullptr, n + 1, G.cour, G.tlim,
                              G.dx1, G.dx2});
    }
    objective(S[cur], dS[cur]);
    return x.ok() ? 0 : -1;
  }

  // a given cotangent of the final state (Exec memory, state layout, zero
  // outside the entries a step writes), or null for the magnetic energy
  const double* seed = nullptr;

  void objective(const double* s, const double* ds) {
    double* tmp = tape;   // any plane-sized scratch: the tape's first plane is free after the step
    x.items(interior(), ObjFn{s, nullptr, tmp, G.ps, G.pitch, 0});
    x.sum(tmp, interior(), G.pitch, &sc->J);
    if (ds) {
      x.items(interior(), ObjFn{s, ds, tmp, G.ps, G.pitch, 1});
      x.sum(tmp, interior(), G.pitch, &sc->dJ);
    }
  }

  // ---------------- adjoint ----------------
  // The state the slots index: slot k -> slots + k * state_doubles.
  double* slot_ptr(int k) const { return slots + (size_t)k * state_doubles(); }

  // Advance S[cur] from step a to step b (records known), generic step.
  template <int FLUX> void advance(int& cur, int a, int b) {
    for (int n = a; n < b; n++) {
      x.single(CoefFromRecFn{cf, rec, n, G.dx1, G.dx2});
      fwd_step_double<FLUX>(cur);
      cur ^= 1;
      advances++;
    }
  }

  AdjArgs adj_args(const double* in, const double* lout, double* lin) const {
    AdjArgs a;
    a.in = in; a.tape = tape; a.lout = lout; a.lin = lin; a.adj = adj;
    a.c = StepCoef<double>{};   // filled per step from the records (host copy)
    a.ps = G.ps; a.pitch = G.pitch;
    a.is = G.is; a.ie = G.ie; a.js = G.js; a.je = G.je;
    a.dx1 = G.dx1; a.dx2 = G.dx2; a.eos = G.eos;
    return a;
  }

  // The ghost fill of a state, reversed on its adjoint l: the ghost rows'
  // adjoints added onto the rows they copy (x2), then the ghost columns'
  // onto the columns they copy (x1), then the frame cleared.  Only rows and
  // columns within kBand of an edge are copied by a ghost (periodic wraps
  // reach 4 cells in, reflection 4, outflow 1), so the passes visit those
  // bands alone; every target cell adds the same terms in the same order.
  void fold_ghosts(double* l) {
    const GhostGeom gg = ghost_geom();
    constexpr int kBand = kNghostA + 2;
    const int is = G.is, ie = G.ie, js = G.js, je = G.je;
    if (2 * kBand >= je + 2 - js) {
      x.items(GenRange{0, G.sx - 1, js, je + 1}, FoldFn{l, G.ps, G.pitch, gg, 2});
    } else {
      x.items(GenRange{0, G.sx - 1, js, js + kBand - 1}, FoldFn{l, G.ps, G.pitch, gg, 2});
      x.items(GenRange{0, G.sx - 1, je + 2 - kBand, je + 1}, FoldFn{l, G.ps, G.pitch, gg, 2});
    }
    if (2 * kBand >= ie + 2 - is) {
      x.items(GenRange{is, ie + 1, js, je + 1}, FoldFn{l, G.ps, G.pitch, gg, 1});
    } else {
      x.items(GenRange{is, is + kBand - 1, js, je + 1}, FoldFn{l, G.ps, G.pitch, gg, 1});
      x.items(GenRange{ie + 2 - kBand, ie + 1, js, je + 1}, FoldFn{l, G.ps, G.pitch, gg, 1});
    }
    // the frame: rows below js and above je (B2i's row je+1 is kept by the
    // functor), the columns left of is and right of ie on the rows between
    x.items(GenRange{0, G.sx - 1, 0, js - 1}, FoldFn{l, G.ps, G.pitch, gg, 0});
    x.items(GenRange{0, G.sx - 1, je + 1, G.sy - 1}, FoldFn{l, G.ps, G.pitch, gg, 0});
    x.items(GenRange{0, is - 1, js, je}, FoldFn{l, G.ps, G.pitch, gg, 0});
    x.items(GenRange{ie + 1, G.sx - 1, js, je}, FoldFn{l, G.ps, G.pitch, gg, 0});
  }

  // Reverse step n: S^n in S[cur].  lam[lc] holds the adjoint of S^{n+1}
  // (folded); on return lam[lc^1] holds that of S^n (folded), lc flipped.
  template <int FLUX> void reverse_step(int cur, int n, int N, int& lc, const std::vector<StepRec>& hrec) {
    const double* Sn;
    const double* Sn1;
    if (tapes) {   // tape mode: S^n, S^{n+1} in the slots, the tape of step n recorded by the first sweep
      tape = tape_of(n);
      Sn = slot_ptr(n);
      Sn1 = n + 1 < N ? slot_ptr(n + 1) : nullptr;
    } else {       // recorded forward step n: S^n -> S^{n+1}, tape, CFL rates of S^{n+1}
      x.single(CoefFromRecFn{cf, rec, n, G.dx1, G.dx2});
      fwd_step_double<FLUX>(cur, true);
      taped++;
      Sn = S[cur];
      Sn1 = S[cur ^ 1];
    }
    // dt_rule^{n+1} = CourNo / m(S^{n+1}): its adjoint into lam[lc]
    if (n + 1 < N) {
      x.argmax(tape + (long long)G_DTI * G.ps, interior(), G.pitch, ml);
      x.single(DtRuleAdjFn{Sn1, lam[lc], ml, sc, rec, n + 1, G.ps, G.cour, G.dx1, G.dx2, G.eos});
    }
    double* lin = lam[lc ^ 1];
    x.zero(lin, state_doubles());
    x.zero(adj + (long long)A_DT * G.ps, plane());
    AdjArgs a = adj_args(Sn, lam[lc], lin);
    a.c = make_coef(hrec[n].dt, G.dx1, G.dx2);
    const int is = G.is, ie = G.ie, js = G.js, je = G.je;
    x.items(GenRange{is, ie + 1, js, je + 1}, AdjFn<R_UPD, FLUX>{a});
    x.items(range_emf1(is, ie, js, je), AdjFn<R_EMF1, FLUX>{a});
    x.items(GenRange{is - 1, ie + 1, js - 1, je + 1}, AdjFn<R_FLUX2, FLUX>{a});
    x.items(range_correct_x(is, ie, js, je), AdjFn<R_CORX, FLUX>{a});
    x.items(range_correct_y(is, ie, js, je), AdjFn<R_CORY, FLUX>{a});
    x.items(range_correct_e(is, ie, js, je), AdjFn<R_CORE, FLUX>{a});
    x.items(GenRange{is - 1, ie + 2, js - 1, je + 2}, AdjFn<R_HALF, FLUX>{a});
    x.items(range_emf0(is, ie, js, je), AdjFn<R_EMF0, FLUX>{a});
    x.items(GenRange{is - 2, ie + 2, js - 2, je + 2}, AdjFn<R_FLUX1, FLUX>{a});
    x.items(GenRange{is - 1, ie + 2, js - 1, je + 2}, AdjFn<R_SRC, FLUX>{a});
    x.items(range_riemann_x(is, ie, js, je), AdjFn<R_RIEX, FLUX>{a});
    x.items(range_riemann_y(is, ie, js, je), AdjFn<R_RIEY, FLUX>{a});
    x.items(range_plm(is, ie, js, je), AdjFn<R_PLMX, FLUX>{a});
    x.items(range_plm(is, ie, js, je), AdjFn<R_PLMY, FLUX>{a});
    x.items(GenRange{is - 3, ie + 3, js - 2, je + 2}, AdjFn<R_PRIMX, FLUX>{a});
    x.items(GenRange{is - 2, ie + 2, js - 3, je + 3}, AdjFn<R_PRIMY, FLUX>{a});
    // the ghost fill of S^n, reversed: x2 rows, then x1 columns, then clear
    fold_ghosts(lin);
    // dt^n
    x.sum(adj + (long long)A_DT * G.ps, GenRange{is - 3, ie + 3, js - 3, je + 3}, G.pitch, &sc->dtsum);
    x.single(DtStepAdjFn{sc, rec, n, n + 1 == N ? 1 : 0});
    lc ^= 1;
  }

  // Reverse steps [a, b): S^a is in slot sa; free slots in `fr`.
  template <int FLUX>
  void reverse(int a, int b, int sa, std::vector<int>& fr, int N, int& lc, const std::vector<StepRec>& hrec,
               const std::vector<int>& spine_slot) {
    int cur = 0;
    if (b - a == 1) {
      x.copy(S[cur], slot_ptr(sa), state_doubles());
      reverse_step<FLUX>(cur, a, N, lc, hrec);
      return;
    }
    if (fr.empty()) {   // no free slot: recompute from S^a for every step
      for (int k = b - 1; k >= a; k--) {
        cur = 0;
        x.copy(S[cur], slot_ptr(sa), state_doubles());
        advance<FLUX>(cur, a, k);
        reverse_step<FLUX>(cur, k, N, lc, hrec);
      }
      return;
    }
    const int m = revolve_split(a, b, (int)fr.size());
    int sm;
    if (spine_slot[m] >= 0) {          // stored by the first sweep (the same slot order)
      sm = fr.back();
      fr.pop_back();
    } else {
      x.copy(S[cur], slot_ptr(sa), state_doubles());
      advance<FLUX>(cur, a, m);
      sm = fr.back();
      fr.pop_back();
      x.copy(slot_ptr(sm), S[cur], state_doubles());
    }
    std::vector<int> none(spine_slot.size(), -1);
    const std::vector<int>& sp = spine_slot[m] >= 0 ? spine_slot : none;
    reverse<FLUX>(m, b, sm, fr, N, lc, hrec, sp);
    fr.push_back(sm);
    reverse<FLUX>(a, m, sa, fr, N, lc, hrec, none);
  }

  // Full adjoint: S[0] holds S^0 (interior).  nslot snapshot slots of which
  // slot 0 is S^0.  The gradient (folded, interior) lands in lam[lc]; J in sc.
  // Loop entry on S[0] (src/main.c:139-149): set_bvals, then dt^0 from new_dt.
  void entry() {
    x.items(full(), GhostFn<double>{pd(S[0]), G.ps, G.pitch, ghost_geom()});
    cfl(pd(S[0]), pd(tape + (long long)G_DTI * G.ps));
    x.argmax(tape + (long long)G_DTI * G.ps, interior(), G.pitch, ml);
    x.single(Dt0Fn<double>{cf, timev, ml, nullptr, rec, G.cour, G.tlim, G.dx1, G.dx2});
  }

  template <int FLUX> int adjoint(int N, int& lc, int& steps_done) {
    int cur = 0;
    entry();
    x.copy(slot_ptr(0), S[0], state_doubles());
    // right spine of the checkpoint schedule, stored during the first sweep
    std::vector<int> spine(N + 1, -1);
    std::vector<int> fr;
    for (int k = nslot - 1; k >= 1; k--) fr.push_back(k);
    {
      int a = 0, s = (int)fr.size();
      std::vector<int> fr2 = fr;
      while (N - a > 1 && s > 0) {
        const int m = revolve_split(a, N, s);
        spine[m] = fr2.back();
        fr2.pop_back();
        a = m;
        s--;
      }
    }
    // first sweep: S^0 .. S^N, records, J (tape mode: every state in slot n
    // and every step's tape)
    for (int n = 0; n < N; n++) {
      if (tapes) tape = tape_of(n);
      fwd_step_double<FLUX>(cur, tapes != nullptr);
      cur ^= 1;
      if (tapes) taped++; else advances++;
      x.argmax(tape + (long long)G_DTI * G.ps, interior(), G.pitch, ml);
      x.single(DtNextFn<double>{cf, timev, ml, nullptr, rec, n + 1, G.cour, G.tlim, G.dx1, G.dx2});
      if (tapes) {
        if (n + 1 < N) x.copy(slot_ptr(n + 1), S[cur], state_doubles());
      } else if (n + 1 < N && spine[n + 1] >= 0) {
        x.copy(slot_ptr(spine[n + 1]), S[cur], state_doubles());
      }
    }
    tape = tape0;
    objective(S[cur], nullptr);
    std::vector<StepRec> hrec(N + 1);
    x.to_host(hrec.data(), rec, sizeof(StepRec) * (size_t)(N + 1));
    // stop at tlim as the main loop does
    steps_done = N;
    for (int n = 0; n < N; n++)
      if (!(hrec[n].time < G.tlim)) { steps_done = n; break; }
    const int M = steps_done;
    if (M < N) {   // the spine was built for N steps: rebuild for M
      for (int k = 0; k <= N; k++) spine[k] = -1;
      if (M > 0) {   // S^M is needed for the objective's seed: recompute from S^0
        int c2 = 0;
        x.copy(S[c2], slot_ptr(0), state_doubles());
        advance<FLUX>(c2, 0, M);
        objective(S[c2], nullptr);
        cur = c2;
      }
    }
    // seed: dJ/dS^M (the magnetic energy's, or a given cotangent of S^M,
    // whose objective is then J = <seed, S^M>)
    lc = 0;
    x.zero(lam[0], state_doubles());
    if (seed) {
      x.copy(lam[0], seed, state_doubles());
      double* tmp = tape;
      x.items(interior(), SeedDotFn{S[cur], seed, tmp, G.ps, G.pitch, G.ie, G.je});
      x.sum(tmp, interior(), G.pitch, &sc->J);
    } else {
      x.items(interior(), ObjFn{S[cur], nullptr, lam[0], G.ps, G.pitch, 2});
    }
    x.zero_bytes(&sc->lrule, sizeof(double));
    x.zero_bytes(&sc->ltime, sizeof(double));
    if (tapes && M > 0) {
      for (int n = M - 1; n >= 0; n--) reverse_step<FLUX>(0, n, M, lc, hrec);
      tape = tape0;
    } else if (M > 0) {
      reverse<FLUX>(0, M, 0, fr, M, lc, hrec, spine);
    }
    // dt_rule^0 = CourNo / m(S^0)
    x.copy(S[0], slot_ptr(0), state_doubles());
    cfl(pd(S[0]), pd(tape + (long long)G_DTI * G.ps));
    x.argmax(tape + (long long)G_DTI * G.ps, interior(), G.pitch, ml);
    x.single(DtRuleAdjFn{S[0], lam[lc], ml, sc, rec, 0, G.ps, G.cour, G.dx1, G.dx2, G.eos});
    return x.ok() ? 0 : -1;
  }
};

}  // namespace athb
