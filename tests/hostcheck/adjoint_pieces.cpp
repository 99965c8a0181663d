// adjoint_pieces.cpp -- TEST INFRASTRUCTURE: dot-product checks of the
// hand-written adjoints of the per-cell physics (athena_cuda_b200/csrc/
// mhd_adjoint.cuh) against the tangent-linear model (the same physics
// instantiated with the Dual scalar), compiled for the host CPU.
//
// For each function y = f(x) and random x, xdot, ybar:
//     <ybar, J xdot>  (one Dual evaluation)   ==   <J^T ybar, xdot>  (adjoint)
// to round-off.  Prints one line per function: trials, the largest relative
// mismatch, and how often each branch of interest was taken.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../../athena_cuda_b200/csrc/mhd_adjoint.cuh"
#include "../../athena_cuda_b200/csrc/step_generic.cuh"

using namespace athb;
using D = Dual;

static std::mt19937_64 rng(12345);
static double U(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }
static double N() { return std::normal_distribution<double>(0.0, 1.0)(rng); }

static const Eos EOS{5.0 / 3.0, 2.0 / 3.0, 5.0 / 3.0 - 2.0};

struct Stat {
  const char* name;
  int n = 0;
  double worst = 0.0;
  double worst_scaled = 0.0;
  void add(double a, double b, double scale = 0.0) {
    n++;
    const double s = std::fmax(std::fabs(a), std::fabs(b));
    const double e = s > 0 ? std::fabs(a - b) / s : 0.0;
    if (e > worst) worst = e;
    const double sc = std::fmax(scale, s);
    const double e2 = sc > 0 ? std::fabs(a - b) / sc : 0.0;
    if (e2 > worst_scaled) worst_scaled = e2;
  }
  void print(const char* extra = "") const {
    printf("%-16s trials=%d worst_rel=%.3e worst_vs_terms=%.3e %s\n", name, n, worst, worst_scaled, extra);
  }
};

static Prim1 rand_prim(double vscale = 1.0, double bscale = 1.0) {
  Prim1 w;
  w.d = U(0.2, 3.0); w.vx = vscale * U(-1.5, 1.5); w.vy = vscale * U(-1, 1); w.vz = vscale * U(-0.5, 0.5);
  w.p = U(0.05, 2.0); w.by = bscale * U(-1.5, 1.5); w.bz = bscale * U(-1.5, 1.5);
  return w;
}
static Prim1 perturb(const Prim1& w, double s) {
  Prim1 q = w;
  q.d *= std::exp(s * N()); q.p *= std::exp(s * N());
  q.vx += s * N(); q.vy += s * N(); q.vz += s * N(); q.by += s * N(); q.bz += s * N();
  return q;
}
static double* as_arr(Prim1& w) { return &w.d; }
static double* as_arr(Cons1& u) { return &u.d; }
static Prim1T<D> dual_prim(const Prim1& w, const double t[7]) {
  Prim1T<D> r;
  const double* v = &w.d;
  D* o = &r.d;
  for (int k = 0; k < 7; k++) o[k] = D(v[k], t[k]);
  return r;
}
static Cons1T<D> dual_cons(const Cons1& u, const double t[7]) {
  Cons1T<D> r;
  const double* v = &u.d;
  D* o = &r.d;
  for (int k = 0; k < 7; k++) o[k] = D(v[k], t[k]);
  return r;
}
static void rand_vec(double* v, int n) { for (int k = 0; k < n; k++) v[k] = N(); }

static void check_cons_prim(int trials) {
  Stat s1{"cons_to_prim"}, s2{"prim_to_cons"};
  for (int t = 0; t < trials; t++) {
    Prim1 w = rand_prim();
    if (t % 10 == 0) w.p = 1e-22;   // clamped pressure branch
    const double bx = U(-1.5, 1.5);
    Cons1 u = prim_to_cons(w, bx, EOS);
    double ut[7], bxt = N(), yb[7];
    rand_vec(ut, 7); rand_vec(yb, 7);
    // cons_to_prim
    {
      Prim1T<D> y = cons_to_prim(dual_cons(u, ut), D(bx, bxt), EOS);
      double lhs = 0, sc = 0; const D* yy = &y.d; for (int k = 0; k < 7; k++) { lhs += yb[k] * yy[k].t; sc += std::fabs(yb[k] * yy[k].t); }
      Prim1 wb; double* wbp = &wb.d; for (int k = 0; k < 7; k++) wbp[k] = yb[k];
      Cons1 ub; zero(ub); double bxb = 0;
      cons_to_prim_adj(u, bx, EOS, wb, ub, bxb);
      double rhs = bxb * bxt; const double* ubp = &ub.d; for (int k = 0; k < 7; k++) rhs += ubp[k] * ut[k];
      s1.add(lhs, rhs, sc);
    }
    // prim_to_cons
    {
      double wt[7]; rand_vec(wt, 7);
      Cons1T<D> y = prim_to_cons(dual_prim(w, wt), D(bx, bxt), EOS);
      double lhs = 0; const D* yy = &y.d; for (int k = 0; k < 7; k++) lhs += yb[k] * yy[k].t;
      Cons1 ub; double* ubp = &ub.d; for (int k = 0; k < 7; k++) ubp[k] = yb[k];
      Prim1 wb; zero(wb); double bxb = 0;
      prim_to_cons_adj(w, bx, EOS, ub, wb, bxb);
      double rhs = bxb * bxt; const double* wbp = &wb.d; for (int k = 0; k < 7; k++) rhs += wbp[k] * wt[k];
      s2.add(lhs, rhs);
    }
  }
  s1.print(); s2.print();
}

static constexpr int kEigN = 42;
static void eig_flat(const PrimEigT<D>& E, double* t) {
  int k = 0;
  for (int n = 0; n < 7; n++) t[k++] = E.ev[n].t;
  const D* r = &E.R00;
  for (int m = 0; m < 35; m++) t[k++] = r[m].t;
}
static void eig_unflat(PrimEig& E, const double* b) {
  int k = 0;
  for (int n = 0; n < 7; n++) E.ev[n] = b[k++];
  double* r = &E.R00;
  for (int m = 0; m < 35; m++) r[m] = b[k++];
}

static void check_esys(int trials) {
  Stat st{"esys_prim"}, sd{"esys_prim_degen"};
  int cases[4] = {0, 0, 0, 0};
  for (int t = 0; t < trials; t++) {
    double x[6] = {U(0.2, 3), U(-1, 1), U(0.05, 2), U(-1.5, 1.5), U(-1.5, 1.5), U(-1.5, 1.5)};
    if (t % 7 == 1) { x[4] = 0.0; x[5] = 0.0; }        // bt == 0
    if (t % 11 == 2) x[3] = 0.0;                       // b1 == 0
    double xt[6]; rand_vec(xt, 6);
    if (x[4] == 0.0) { xt[4] = 0.0; xt[5] = 0.0; }
    if (x[3] == 0.0) xt[3] = 0.0;
    PrimEigT<D> E;
    esys_prim(D(x[0], xt[0]), D(x[1], xt[1]), D(x[2], xt[2]), D(x[3], xt[3]), D(x[4], xt[4]), D(x[5], xt[5]), EOS, E);
    double yt[kEigN], yb[kEigN];
    eig_flat(E, yt);
    rand_vec(yb, kEigN);
    double lhs = 0, sc = 0; for (int k = 0; k < kEigN; k++) { lhs += yb[k] * yt[k]; sc += std::fabs(yb[k] * yt[k]); }
    PrimEig Eb; eig_unflat(Eb, yb);
    double xb[6] = {0, 0, 0, 0, 0, 0};
    esys_prim_adj(x[0], x[1], x[2], x[3], x[4], x[5], EOS, Eb, xb[0], xb[1], xb[2], xb[3], xb[4], xb[5]);
    double rhs = 0; for (int k = 0; k < 6; k++) { rhs += xb[k] * xt[k]; sc = std::fmax(sc, std::fabs(xb[k] * xt[k])); }
    // b2 = b3 = 0 with b1 != 0: alpha_s is the square root of a rounding
    // residue, so both linearisations are ill-conditioned there
    if (x[4] == 0.0 && x[5] == 0.0 && x[3] != 0.0) sd.add(lhs, rhs, sc); else st.add(lhs, rhs, sc);
    if (getenv("ESYS_DEBUG") && std::fabs(lhs - rhs) > 1e-10 * sc)
      printf("esys t=%d x=[%.6g %.6g %.6g %.6g %.6g %.6g] lhs=%.10g rhs=%.10g sc=%.3g\n", t, x[0], x[1], x[2], x[3], x[4], x[5], lhs, rhs, sc);
    cases[(x[4] == 0.0 ? 1 : 0) + (x[3] == 0.0 ? 2 : 0)]++;
  }
  char buf[128];
  snprintf(buf, sizeof buf, "(generic %d, bt=0 %d, b1=0 %d, both %d)", cases[0], cases[1], cases[2], cases[3]);
  st.print(buf);
  sd.print("(b2 = b3 = 0, b1 != 0)");
}

static void check_plm(int trials) {
  Stat st{"plm_cell"};
  for (int t = 0; t < trials; t++) {
    const double vs = (t % 3 == 0) ? 4.0 : 1.0;  // fast flows: all eigenvalues of one sign
    Prim1 w0 = rand_prim(vs);
    const double psc = (t % 4 == 0) ? 0.02 : 0.3;
    Prim1 wm = perturb(w0, psc), wp = perturb(w0, psc);
    if (t % 5 == 0) { wm = w0; }                         // flat left: limiter zero branch
    const double bxc = (t % 9 == 0) ? 0.0 : U(-1.5, 1.5);
    const double dtodx = U(0.05, 0.6);
    double tm[7], t0[7], tp[7], bxt = (bxc == 0.0 ? 0.0 : N()), dtt = N();
    rand_vec(tm, 7); rand_vec(t0, 7); rand_vec(tp, 7);
    Prim1T<D> yl, yr;
    plm_cell(dual_prim(wm, tm), dual_prim(w0, t0), dual_prim(wp, tp), D(bxc, bxt), D(dtodx, dtt), EOS, yl, yr);
    double ylb[7], yrb[7];
    rand_vec(ylb, 7); rand_vec(yrb, 7);
    double lhs = 0, sc = 0;
    const D* a = &yl.d; const D* b = &yr.d;
    for (int k = 0; k < 7; k++) { lhs += ylb[k] * a[k].t + yrb[k] * b[k].t; sc += std::fabs(ylb[k] * a[k].t) + std::fabs(yrb[k] * b[k].t); }
    Prim1 wlb, wrb; for (int k = 0; k < 7; k++) { (&wlb.d)[k] = ylb[k]; (&wrb.d)[k] = yrb[k]; }
    Prim1 wmb, w0b, wpb; zero(wmb); zero(w0b); zero(wpb);
    double bxcb = 0, dtb = 0;
    plm_cell_adj(wm, w0, wp, bxc, dtodx, EOS, wlb, wrb, wmb, w0b, wpb, bxcb, dtb);
    double rhs = bxcb * bxt + dtb * dtt;
    for (int k = 0; k < 7; k++) rhs += (&wmb.d)[k] * tm[k] + (&w0b.d)[k] * t0[k] + (&wpb.d)[k] * tp[k];
    st.add(lhs, rhs, sc);
    if (std::fabs(lhs - rhs) > 1e-9 * std::fmax(sc, 1e-300) && getenv("PLM_DEBUG")) {
      printf("plm mismatch t=%d lhs=%.17g rhs=%.17g\n", t, lhs, rhs);
    }
  }
  st.print();
}

// classify the Roe solver's path for the reported coverage
static int roe_path(const Cons1& Ul, const Cons1& Ur, const Prim1& Wl, const Prim1& Wr, double Bxi) {
  const RoeAvg r = roe_average(Ul, Ur, Wl, Wr, Bxi);
  const RoeSpeeds s = roe_speeds(r, Bxi, EOS);
  double ev[7] = {r.v1 - s.cf, r.v1 - s.vax, r.v1 - s.cs, r.v1, r.v1 + s.cs, r.v1 + s.vax, r.v1 + s.cf};
  if (ev[0] >= 0.0) return 1;
  if (ev[6] <= 0.0) return 2;
  RoeScal S; roe_scalars(r, s, Bxi, EOS, S);
  double dU[7]; for (int k = 0; k < 7; k++) dU[k] = (&Ur.d)[k] - (&Ul.d)[k];
  double a[7]; roe_project(S, dU, a);
  double u[7]; for (int k = 0; k < 7; k++) u[k] = (&Ul.d)[k];
  for (int n = 0; n < 6; n++) {
    double c[7]; roe_right_col(S, ev, n, c);
    for (int m = 0; m < 7; m++) if ((roe_right_mask(n) >> m) & 1) u[m] += a[n] * c[m];
    if (ev[n + 1] > ev[n]) {
      bool bad = u[0] <= 0.0;
      if (!bad) { double p = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]; p -= 0.5 * (u[5] * u[5] + u[6] * u[6] + Bxi * Bxi); bad = p < 0.0; }
      if (bad) return 3;
    }
  }
  return 0;
}

template <int FLUX>
static void check_flux(int trials, const char* name) {
  Stat st{name};
  char dname[64];
  snprintf(dname, sizeof dname, "%s_degen", name);
  Stat sd{dname};
  int paths[4] = {0, 0, 0, 0};
  for (int t = 0; t < trials; t++) {
    const int kind = t % 6;
    Prim1 wl, wr;
    double bx = U(-1.5, 1.5);
    if (kind == 0) { wl = rand_prim(); wr = perturb(wl, 0.2); }
    else if (kind == 1) { wl = rand_prim(); wr = rand_prim(); }
    else if (kind == 2) { wl = rand_prim(0.2); wl.vx = U(4, 8); wr = perturb(wl, 0.2); }       // supersonic right-moving
    else if (kind == 3) { wl = rand_prim(0.2); wl.vx = -U(4, 8); wr = perturb(wl, 0.2); }      // supersonic left-moving
    else if (kind == 4) {  // strong rarefaction: intermediate states may go negative -> HLLE
      wl = rand_prim(); wr = rand_prim(); wl.vx = -U(2, 6); wr.vx = U(2, 6); wl.d = U(0.01, 0.1); wr.d = U(0.01, 0.1);
      wl.p = U(1e-4, 1e-2); wr.p = U(1e-4, 1e-2);
    } else { wl = rand_prim(1.0, 0.0); wr = perturb(wl, 0.3); wl.by = wl.bz = wr.by = wr.bz = 0.0; }  // bt = 0
    if (kind == 5 && t % 12 == 5) bx = 0.0;
    const Cons1 ul = prim_to_cons(wl, bx, EOS), ur = prim_to_cons(wr, bx, EOS);
    paths[roe_path(ul, ur, wl, wr, bx)]++;
    double tul[7], tur[7], twl[7], twr[7], bxt = (bx == 0.0 ? 0.0 : N()), fb[7];
    rand_vec(tul, 7); rand_vec(tur, 7); rand_vec(twl, 7); rand_vec(twr, 7); rand_vec(fb, 7);
    if (kind == 5) { tul[5] = tul[6] = tur[5] = tur[6] = twl[5] = twl[6] = twr[5] = twr[6] = 0.0; }
    const Cons1T<D> F = riemann<FLUX>(dual_cons(ul, tul), dual_cons(ur, tur), dual_prim(wl, twl), dual_prim(wr, twr),
                                      D(bx, bxt), EOS);
    double lhs = 0, sc = 0; const D* f = &F.d; for (int k = 0; k < 7; k++) { lhs += fb[k] * f[k].t; sc += std::fabs(fb[k] * f[k].t); }
    Cons1 Fb; for (int k = 0; k < 7; k++) (&Fb.d)[k] = fb[k];
    Cons1 ulb, urb; Prim1 wlb, wrb; zero(ulb); zero(urb); zero(wlb); zero(wrb);
    double bxb = 0;
    riemann_adj<FLUX>(ul, ur, wl, wr, bx, EOS, Fb, ulb, urb, wlb, wrb, bxb);
    double rhs = bxb * bxt;
    for (int k = 0; k < 7; k++)
      rhs += (&ulb.d)[k] * tul[k] + (&urb.d)[k] * tur[k] + (&wlb.d)[k] * twl[k] + (&wrb.d)[k] * twr[k];
    if (kind == 5 && bx != 0.0) sd.add(lhs, rhs, sc); else st.add(lhs, rhs, sc);
    if (getenv("FLUX_DEBUG") && std::fabs(lhs - rhs) > 1e-12 * sc)
      printf("%s t=%d kind=%d path=%d bx=%g rel=%.3e\n", name, t, kind, roe_path(ul, ur, wl, wr, bx),
             bx, std::fabs(lhs - rhs) / sc);
  }
  char buf[160];
  snprintf(buf, sizeof buf, "(roe paths: subsonic %d, supersonic-left %d, supersonic-right %d, hlle-fallback %d)",
           paths[0], paths[1], paths[2], paths[3]);
  st.print(buf);
  sd.print("(transverse field zero on both sides, normal field non-zero)");
}

static void check_emf(int trials) {
  Stat st{"corner_emf"};
  for (int t = 0; t < trials; t++) {
    double f[4] = {U(-1, 1), U(-1, 1), U(-1, 1), U(-1, 1)};
    for (int k = 0; k < 4; k++) if (rng() % 5 == 0) f[k] = 0.0;
    double x[8], xt[8]; rand_vec(x, 8); rand_vec(xt, 8);
    const D r = corner_emf_gen(D(f[0]), D(x[0], xt[0]), D(f[1]), D(x[1], xt[1]), D(f[2]), D(x[2], xt[2]), D(f[3]),
                               D(x[3], xt[3]), D(x[4], xt[4]), D(x[5], xt[5]), D(x[6], xt[6]), D(x[7], xt[7]));
    double k[8]; corner_emf_coeffs(f[0], f[1], f[2], f[3], k);
    double rhs = 0, sc = 0; for (int m = 0; m < 8; m++) { rhs += k[m] * xt[m]; sc += std::fabs(k[m] * xt[m]); }
    st.add(r.t, rhs, sc);
  }
  st.print();
}

static void check_dti(int trials) {
  Stat st{"cell_dti"};
  for (int t = 0; t < trials; t++) {
    Prim1 w = rand_prim(t % 2 ? 3.0 : 0.5);
    const Cons1 u = prim_to_cons(w, U(-1, 1), EOS);
    const double e = u.e - 0.5 * (U(0, 1));   // E without the field part is what new_dt sees
    double xt[5]; rand_vec(xt, 5);
    const double dx1 = U(0.005, 0.02), dx2 = U(0.005, 0.02);
    const D m = gen_cell_dti(D(u.d, xt[0]), D(u.mx, xt[1]), D(u.my, xt[2]), D(u.mz, xt[3]), D(e, xt[4]), EOS, dx1, dx2);
    const double mb = N();
    double out[5];
    cell_dti_adj(u.d, u.mx, u.my, u.mz, e, EOS, dx1, dx2, mb, out);
    double rhs = 0, sc = 0; for (int k = 0; k < 5; k++) { rhs += out[k] * xt[k]; sc += std::fabs(out[k] * xt[k]); }
    st.add(mb * m.t, rhs, sc);
  }
  st.print();
}

int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 20000;
  check_cons_prim(trials);
  check_esys(trials);
  check_plm(trials);
  check_flux<kFluxRoe>(trials, "flux_roe");
  check_flux<kFluxHlle>(trials, "flux_hlle");
  check_emf(trials);
  check_dti(trials);
  return 0;
}
