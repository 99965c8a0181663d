// step_adjoint.cuh -- the discrete adjoint of one CTU+CT step, the adjoint
// of the ghost-zone fill and of the dt rule, and the generic ghost fill the
// tangent-linear model uses.
//
// Every stage of the step (step_generic.cuh) is reversed by one or two
// per-item functors.  Inputs of the reverse step: the step's input state S^n
// (ghosts filled), its dt, the tape of the recorded forward step (the
// GenPlane planes), and the adjoint of the step's output, lout (the cells the
// step writes: the interior, B1i column ie+1 and B2i row je+1).  Output: lin,
// the adjoint of every plane entry of S^n the step reads (ghosts included),
// and per-item contributions to the adjoint of dt in the plane A_DT.
//
// Adjoints are GATHERED, never scattered: each stage first stores the adjoint
// of its own outputs per cell or face, and the stage before it collects, for
// each of its outputs, the contributions of every consumer in a fixed order.
// No atomics are involved, so the adjoint is deterministic and a kernel never
// has two threads writing one location.
//
// Reference steps reversed (src/__integrate_2d__.c): 13, 11b, 11a, 9 (update
// and CT), 9 (corner EMF, :632-702), 8c, 8b, 7, 6b, 6a, 5b, 5a, 4 (corrector),
// 3-4 (half-step EMF), 2e, 1e (predictor Riemann), 2b-2d, 1b-1d (PLM and
// source terms), 2a, 1a (cons -> prim); set_bvals (src/set_bvals.c:114-145)
// and new_dt (src/new_dt.c:25-100).
#pragma once

#include "mhd_adjoint.cuh"
#include "step_generic.cuh"

namespace athb {

// Adjoint workspace planes.
enum AdjPlane {
  A_LB1 = 0,     // full-step face field b1 at x faces (update)
  A_LB2 = 1,     // ... b2 at y faces
  A_EMF1 = 2,    // corner emf of the full step
  A_FX2 = 3,     // corrector x flux (7)
  A_FY2 = 10,    // corrector y flux (7)
  A_ECC1 = 17,   // cell emf3 at t^{n+1/2}
  A_ULX = 18, A_URX = 25,   // corrector L/R states at x faces (7 each)
  A_ULY = 32, A_URY = 39,
  A_B1F = 46,    // half-step b1 at x faces, from the corrector flux
  A_B2F = 47,
  A_HALF = 48,   // half-step d, M1, M2, B1c, B2c of a cell (correct_e)
  A_LB1F = 53,   // half-step b1: every consumer
  A_LB2F = 54,
  A_EMF0 = 55,   // corner emf of the half step
  A_FX = 56, A_FY = 63,     // predictor fluxes (7 each)
  A_WLNX = 70, A_WRTX = 77, A_WLNY = 84, A_WRTY = 91,  // PLM outputs (7 each)
  A_BNX = 98, A_BNY = 99,   // normal face field at predictor faces
  A_SRCX = 100, A_SRCY = 101,  // the PLM source term of a cell
  A_WXM = 102, A_WX0 = 109, A_WXP = 116,  // PLM inputs: cell c-1, c, c+1 (x)
  A_WYM = 123, A_WY0 = 130, A_WYP = 137,
  A_DT = 144,    // per-item contributions to the adjoint of dt
  A_TMP = 145,   // scratch (objective per cell)
  NADJ = 146
};

struct AdjArgs {
  const double* in;     // S^n, ghosts filled
  const double* tape;   // GenPlane planes of the recorded step
  const double* lout;   // adjoint of S^{n+1} (cells the step writes)
  double* lin;          // adjoint of S^n (accumulated; zeroed before the step)
  double* adj;          // AdjPlane planes
  StepCoef<double> c;   // dt^n and its factors, exactly as the forward formed them
  long long ps;
  int pitch;
  int is, ie, js, je;
  double dx1, dx2;
  Eos eos;
  ATHB_MEM long long o(int j, int i) const { return (long long)j * pitch + i; }
  ATHB_MEM double s(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return in[p * ps + off]; }
  ATHB_MEM double t(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return tape[p * ps + off]; }
  ATHB_MEM double lo(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return lout[p * ps + off]; }
  ATHB_MEM double& li(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return lin[p * ps + off]; }
  ATHB_MEM double& a(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return adj[p * ps + off]; }
  ATHB_MEM double av(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return adj[p * ps + off]; }
};

ATHB_HD bool in_range(const GenRange& r, int j, int i) { return j >= r.j0 && j <= r.j1 && i >= r.i0 && i <= r.i1; }

// λ of the conserved vector of a sweep (as loaded by gen_cons) added to lin
ATHB_HD void lin_add_cons(const AdjArgs& a, long long o, int dir, const Cons1& ub) {
  a.li(P_D, o) += ub.d;
  a.li(P_E, o) += ub.e;
  if (dir == 0) {
    a.li(P_M1, o) += ub.mx; a.li(P_M2, o) += ub.my; a.li(P_M3, o) += ub.mz;
    a.li(P_B2C, o) += ub.by; a.li(P_B3C, o) += ub.bz;
  } else {
    a.li(P_M2, o) += ub.mx; a.li(P_M3, o) += ub.my; a.li(P_M1, o) += ub.mz;
    a.li(P_B3C, o) += ub.by; a.li(P_B1C, o) += ub.bz;
  }
}
ATHB_HD Cons1 adj_cons(const AdjArgs& a, int base, long long o) {
  Cons1 u;
  u.d = a.av(base + 0, o); u.mx = a.av(base + 1, o); u.my = a.av(base + 2, o); u.mz = a.av(base + 3, o);
  u.e = a.av(base + 4, o); u.by = a.av(base + 5, o); u.bz = a.av(base + 6, o);
  return u;
}
ATHB_HD void adj_put_cons(const AdjArgs& a, int base, long long o, const Cons1& u) {
  a.a(base + 0, o) = u.d; a.a(base + 1, o) = u.mx; a.a(base + 2, o) = u.my; a.a(base + 3, o) = u.mz;
  a.a(base + 4, o) = u.e; a.a(base + 5, o) = u.by; a.a(base + 6, o) = u.bz;
}
ATHB_HD Prim1 adj_prim(const AdjArgs& a, int base, long long o) {
  Prim1 w;
  w.d = a.av(base + 0, o); w.vx = a.av(base + 1, o); w.vy = a.av(base + 2, o); w.vz = a.av(base + 3, o);
  w.p = a.av(base + 4, o); w.by = a.av(base + 5, o); w.bz = a.av(base + 6, o);
  return w;
}
ATHB_HD void adj_put_prim(const AdjArgs& a, int base, long long o, const Prim1& w) {
  a.a(base + 0, o) = w.d; a.a(base + 1, o) = w.vx; a.a(base + 2, o) = w.vy; a.a(base + 3, o) = w.vz;
  a.a(base + 4, o) = w.p; a.a(base + 5, o) = w.by; a.a(base + 6, o) = w.bz;
}
ATHB_HD Cons1 tape_cons(const AdjArgs& a, int base, long long o) {
  Cons1 u;
  u.d = a.t(base + 0, o); u.mx = a.t(base + 1, o); u.my = a.t(base + 2, o); u.mz = a.t(base + 3, o);
  u.e = a.t(base + 4, o); u.by = a.t(base + 5, o); u.bz = a.t(base + 6, o);
  return u;
}
ATHB_HD Prim1 tape_prim(const AdjArgs& a, int base, long long o) {
  Prim1 w;
  w.d = a.t(base + 0, o); w.vx = a.t(base + 1, o); w.vy = a.t(base + 2, o); w.vz = a.t(base + 3, o);
  w.p = a.t(base + 4, o); w.by = a.t(base + 5, o); w.bz = a.t(base + 6, o);
  return w;
}
ATHB_HD Cons1 state_cons(const AdjArgs& a, long long o, int dir) {
  Cons1 u;
  u.d = a.s(P_D, o);
  u.e = a.s(P_E, o);
  if (dir == 0) {
    u.mx = a.s(P_M1, o); u.my = a.s(P_M2, o); u.mz = a.s(P_M3, o); u.by = a.s(P_B2C, o); u.bz = a.s(P_B3C, o);
  } else {
    u.mx = a.s(P_M2, o); u.my = a.s(P_M3, o); u.mz = a.s(P_M1, o); u.by = a.s(P_B3C, o); u.bz = a.s(P_B1C, o);
  }
  return u;
}

// Corner-EMF coefficients of corner (j,i) from the fluxes on the tape
// (full = 0: predictor fluxes G_FX/G_FY; 1: corrector fluxes G_FX2/G_FY2).
ATHB_HD void corner_k(const AdjArgs& a, int full, int j, int i, double k[8]) {
  const int fx = full ? G_FX2 : G_FX, fy = full ? G_FY2 : G_FY;
  const long long o = a.o(j, i);
  corner_emf_coeffs(a.t(fx, o - a.pitch), a.t(fx, o), a.t(fy, o - 1), a.t(fy, o), k);
}

// ===========================================================================
// Reverse of step 9/11/13 (update): face fields b1, b2 and the cell planes.
// Items over [is, ie+1] x [js, je+1].
// ===========================================================================
ATHB_HD void adj_update(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i), P = a.pitch;
  double dtb = 0.0;
  // b1 at x face (j,i), i in [is, ie+1], j in [js, je]
  if (j <= a.je) {
    double lb = a.lo(P_B1I, o);
    if (i <= a.ie) lb += 0.5 * a.lo(P_B1C, o);
    if (i - 1 >= a.is) lb += 0.5 * a.lo(P_B1C, o - 1);
    a.a(A_LB1, o) = lb;
    a.li(P_B1I, o) += lb;
    dtb += -lb * (a.t(G_EMF1, o + P) - a.t(G_EMF1, o)) / a.dx2;
  }
  // b2 at y face (j,i), j in [js, je+1], i in [is, ie]
  if (i <= a.ie) {
    double lb = a.lo(P_B2I, o);
    if (j <= a.je) lb += 0.5 * a.lo(P_B2C, o);
    if (j - 1 >= a.js) lb += 0.5 * a.lo(P_B2C, o - P);
    a.a(A_LB2, o) = lb;
    a.li(P_B2I, o) += lb;
    dtb += lb * (a.t(G_EMF1, o + 1) - a.t(G_EMF1, o)) / a.dx1;
  }
  // cell planes
  if (i <= a.ie && j <= a.je) {
    const double ld = a.lo(P_D, o), l1 = a.lo(P_M1, o), l2 = a.lo(P_M2, o), l3 = a.lo(P_M3, o), le = a.lo(P_E, o);
    const double lb3 = a.lo(P_B3C, o) + a.lo(P_B3I, o);
    a.li(P_D, o) += ld; a.li(P_M1, o) += l1; a.li(P_M2, o) += l2; a.li(P_M3, o) += l3; a.li(P_E, o) += le;
    a.li(P_B3C, o) += lb3;
    // d -= dtodx1 (fx(o+1) - fx(o)) ... ; d -= dtodx2 (fy(o+P) - fy(o)) ...
    double g1 = 0.0, g2 = 0.0;
    g1 += ld * (a.t(G_FX2 + 0, o + 1) - a.t(G_FX2 + 0, o));
    g1 += l1 * (a.t(G_FX2 + 1, o + 1) - a.t(G_FX2 + 1, o));
    g1 += l2 * (a.t(G_FX2 + 2, o + 1) - a.t(G_FX2 + 2, o));
    g1 += l3 * (a.t(G_FX2 + 3, o + 1) - a.t(G_FX2 + 3, o));
    g1 += le * (a.t(G_FX2 + 4, o + 1) - a.t(G_FX2 + 4, o));
    g1 += lb3 * (a.t(G_FX2 + 6, o + 1) - a.t(G_FX2 + 6, o));
    g2 += ld * (a.t(G_FY2 + 0, o + P) - a.t(G_FY2 + 0, o));
    g2 += l2 * (a.t(G_FY2 + 1, o + P) - a.t(G_FY2 + 1, o));
    g2 += l3 * (a.t(G_FY2 + 2, o + P) - a.t(G_FY2 + 2, o));
    g2 += l1 * (a.t(G_FY2 + 3, o + P) - a.t(G_FY2 + 3, o));
    g2 += le * (a.t(G_FY2 + 4, o + P) - a.t(G_FY2 + 4, o));
    g2 += lb3 * (a.t(G_FY2 + 5, o + P) - a.t(G_FY2 + 5, o));
    dtb += -g1 / a.dx1 - g2 / a.dx2;
  }
  a.a(A_DT, o) += dtb;
}

// Corner emf of the full step: corners [is, ie+1] x [js, je+1].
ATHB_HD void adj_emf1(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i), P = a.pitch;
  auto lb1 = [&](int jj, int ii) { return (jj >= a.js && jj <= a.je && ii >= a.is && ii <= a.ie + 1) ? a.av(A_LB1, a.o(jj, ii)) : 0.0; };
  auto lb2 = [&](int jj, int ii) { return (jj >= a.js && jj <= a.je + 1 && ii >= a.is && ii <= a.ie) ? a.av(A_LB2, a.o(jj, ii)) : 0.0; };
  (void)P;
  a.a(A_EMF1, o) = a.c.dtodx2 * (lb1(j, i) - lb1(j - 1, i)) + a.c.dtodx1 * (lb2(j, i - 1) - lb2(j, i));
}

// Corrector fluxes and the half-step cell emf: gathers over
// [is-1, ie+1] x [js-1, je+1].
ATHB_HD void adj_flux2(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i), P = a.pitch;
  const GenRange corners = range_emf1(a.is, a.ie, a.js, a.je);
  const GenRange interior = range_interior(a.is, a.ie, a.js, a.je);
  auto le = [&](int jj, int ii) { return in_range(corners, jj, ii) ? a.av(A_EMF1, a.o(jj, ii)) : 0.0; };
  auto lcell = [&](int p, int jj, int ii) {
    if (!in_range(interior, jj, ii)) return 0.0;
    const long long q = a.o(jj, ii);
    return p == P_B3C ? a.lo(P_B3C, q) + a.lo(P_B3I, q) : a.lo(p, q);
  };
  double k[8];
  // x face (j,i) in the corrector range
  if (in_range(range_correct_x(a.is, a.ie, a.js, a.je), j, i)) {
    static const int map[7] = {P_D, P_M1, P_M2, P_M3, P_E, -1, P_B3C};
    for (int c = 0; c < 7; c++) {
      double v = 0.0;
      if (map[c] >= 0) v = a.c.dtodx1 * (lcell(map[c], j, i) - lcell(map[c], j, i - 1));
      a.a(A_FX2 + c, o) = v;
    }
    double by = 0.0;
    if (in_range(corners, j, i)) { corner_k(a, 1, j, i, k); by += k[1] * le(j, i); }
    if (in_range(corners, j + 1, i)) { corner_k(a, 1, j + 1, i, k); by += k[0] * le(j + 1, i); }
    a.a(A_FX2 + 5, o) = by;
  }
  // y face (j,i)
  if (in_range(range_correct_y(a.is, a.ie, a.js, a.je), j, i)) {
    static const int map[7] = {P_D, P_M2, P_M3, P_M1, P_E, P_B3C, -1};
    for (int c = 0; c < 7; c++) {
      double v = 0.0;
      if (map[c] >= 0) v = a.c.dtodx2 * (lcell(map[c], j, i) - lcell(map[c], j - 1, i));
      a.a(A_FY2 + c, o) = v;
    }
    double bz = 0.0;
    if (in_range(corners, j, i)) { corner_k(a, 1, j, i, k); bz += k[3] * le(j, i); }
    if (in_range(corners, j, i + 1)) { corner_k(a, 1, j, i + 1, k); bz += k[2] * le(j, i + 1); }
    a.a(A_FY2 + 6, o) = bz;
  }
  // cell (j,i): e_c of corner (j,i), e_w of (j,i+1), e_s of (j+1,i), e_sw of (j+1,i+1)
  {
    double v = 0.0;
    if (in_range(corners, j, i)) { corner_k(a, 1, j, i, k); v += k[7] * le(j, i); }
    if (in_range(corners, j, i + 1)) { corner_k(a, 1, j, i + 1, k); v += k[6] * le(j, i + 1); }
    if (in_range(corners, j + 1, i)) { corner_k(a, 1, j + 1, i, k); v += k[5] * le(j + 1, i); }
    if (in_range(corners, j + 1, i + 1)) { corner_k(a, 1, j + 1, i + 1, k); v += k[4] * le(j + 1, i + 1); }
    a.a(A_ECC1, o) = v;
  }
  (void)P;
}

// ===========================================================================
// Reverse of the corrector (steps 4-8).
// ===========================================================================
// Corrector L/R states of x face (j,i), rebuilt exactly as gen_correct_x.
ATHB_HD void correct_x_states(const AdjArgs& a, int j, int i, Cons1& ul, Cons1& ur, double& b1f) {
  const long long o = a.o(j, i), P = a.pitch;
  const StepCoef<double>& c = a.c;
  b1f = a.s(P_B1I, o) - c.hdtodx2 * (a.t(G_EMF0, o + P) - a.t(G_EMF0, o));
  ul = tape_cons(a, G_ULX, o);
  ur = tape_cons(a, G_URX, o);
  {
    const long long on = o + P - 1, oc = o - 1;
    ul.d -= c.hdtodx2 * (a.t(G_FY + 0, on) - a.t(G_FY + 0, oc));
    ul.mx -= c.hdtodx2 * (a.t(G_FY + 3, on) - a.t(G_FY + 3, oc));
    ul.my -= c.hdtodx2 * (a.t(G_FY + 1, on) - a.t(G_FY + 1, oc));
    ul.mz -= c.hdtodx2 * (a.t(G_FY + 2, on) - a.t(G_FY + 2, oc));
    ul.e -= c.hdtodx2 * (a.t(G_FY + 4, on) - a.t(G_FY + 4, oc));
    ul.bz -= c.hdtodx2 * (a.t(G_FY + 5, on) - a.t(G_FY + 5, oc));
  }
  {
    const long long on = o + P, oc = o;
    ur.d -= c.hdtodx2 * (a.t(G_FY + 0, on) - a.t(G_FY + 0, oc));
    ur.mx -= c.hdtodx2 * (a.t(G_FY + 3, on) - a.t(G_FY + 3, oc));
    ur.my -= c.hdtodx2 * (a.t(G_FY + 1, on) - a.t(G_FY + 1, oc));
    ur.mz -= c.hdtodx2 * (a.t(G_FY + 2, on) - a.t(G_FY + 2, oc));
    ur.e -= c.hdtodx2 * (a.t(G_FY + 4, on) - a.t(G_FY + 4, oc));
    ur.bz -= c.hdtodx2 * (a.t(G_FY + 5, on) - a.t(G_FY + 5, oc));
  }
  {
    const long long ow = o - 1;
    const double dbx = a.s(P_B1I, o) - a.s(P_B1I, ow);
    const double B1 = a.s(P_B1C, ow), B2 = a.s(P_B2C, ow), B3 = a.s(P_B3C, ow);
    const double V3 = a.s(P_M3, ow) / a.s(P_D, ow);
    ul.mx += c.hdtodx1 * B1 * dbx;
    ul.my += c.hdtodx1 * B2 * dbx;
    ul.mz += c.hdtodx1 * B3 * dbx;
    ul.bz += c.hdtodx1 * V3 * dbx;
    ul.e += c.hdtodx1 * B3 * V3 * dbx;
  }
  {
    const double dbx = a.s(P_B1I, o + 1) - a.s(P_B1I, o);
    const double B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o), B3 = a.s(P_B3C, o);
    const double V3 = a.s(P_M3, o) / a.s(P_D, o);
    ur.mx += c.hdtodx1 * B1 * dbx;
    ur.my += c.hdtodx1 * B2 * dbx;
    ur.mz += c.hdtodx1 * B3 * dbx;
    ur.bz += c.hdtodx1 * V3 * dbx;
    ur.e += c.hdtodx1 * B3 * V3 * dbx;
  }
}

ATHB_HD void correct_y_states(const AdjArgs& a, int j, int i, Cons1& ul, Cons1& ur, double& b2f) {
  const long long o = a.o(j, i), P = a.pitch;
  const StepCoef<double>& c = a.c;
  b2f = a.s(P_B2I, o) + c.hdtodx1 * (a.t(G_EMF0, o + 1) - a.t(G_EMF0, o));
  ul = tape_cons(a, G_ULY, o);
  ur = tape_cons(a, G_URY, o);
  {
    const long long oe = o - P + 1, oc = o - P;
    ul.d -= c.hdtodx1 * (a.t(G_FX + 0, oe) - a.t(G_FX + 0, oc));
    ul.mx -= c.hdtodx1 * (a.t(G_FX + 2, oe) - a.t(G_FX + 2, oc));
    ul.my -= c.hdtodx1 * (a.t(G_FX + 3, oe) - a.t(G_FX + 3, oc));
    ul.mz -= c.hdtodx1 * (a.t(G_FX + 1, oe) - a.t(G_FX + 1, oc));
    ul.e -= c.hdtodx1 * (a.t(G_FX + 4, oe) - a.t(G_FX + 4, oc));
    ul.by -= c.hdtodx1 * (a.t(G_FX + 6, oe) - a.t(G_FX + 6, oc));
  }
  {
    const long long oe = o + 1, oc = o;
    ur.d -= c.hdtodx1 * (a.t(G_FX + 0, oe) - a.t(G_FX + 0, oc));
    ur.mx -= c.hdtodx1 * (a.t(G_FX + 2, oe) - a.t(G_FX + 2, oc));
    ur.my -= c.hdtodx1 * (a.t(G_FX + 3, oe) - a.t(G_FX + 3, oc));
    ur.mz -= c.hdtodx1 * (a.t(G_FX + 1, oe) - a.t(G_FX + 1, oc));
    ur.e -= c.hdtodx1 * (a.t(G_FX + 4, oe) - a.t(G_FX + 4, oc));
    ur.by -= c.hdtodx1 * (a.t(G_FX + 6, oe) - a.t(G_FX + 6, oc));
  }
  {
    const long long osn = o - P;
    const double dby = a.s(P_B2I, o) - a.s(P_B2I, osn);
    const double B1 = a.s(P_B1C, osn), B2 = a.s(P_B2C, osn), B3 = a.s(P_B3C, osn);
    const double V3 = a.s(P_M3, osn) / a.s(P_D, osn);
    ul.mz += c.hdtodx2 * B1 * dby;
    ul.mx += c.hdtodx2 * B2 * dby;
    ul.my += c.hdtodx2 * B3 * dby;
    ul.by += c.hdtodx2 * V3 * dby;
    ul.e += c.hdtodx2 * B3 * V3 * dby;
  }
  {
    const double dby = a.s(P_B2I, o + P) - a.s(P_B2I, o);
    const double B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o), B3 = a.s(P_B3C, o);
    const double V3 = a.s(P_M3, o) / a.s(P_D, o);
    ur.mz += c.hdtodx2 * B1 * dby;
    ur.mx += c.hdtodx2 * B2 * dby;
    ur.my += c.hdtodx2 * B3 * dby;
    ur.by += c.hdtodx2 * V3 * dby;
    ur.e += c.hdtodx2 * B3 * V3 * dby;
  }
}

// dt adjoint of the transverse and source terms of one corrector state
// (x face: transverse terms are x2-flux differences (hdtodx2), sources use
// hdtodx1; y face: the other way round).
ATHB_HD double correct_x_dtb(const AdjArgs& a, int j, int i, const Cons1& lul, const Cons1& lur) {
  const long long o = a.o(j, i), P = a.pitch;
  double g2 = 0.0, g1 = 0.0;
  {
    const long long on = o + P - 1, oc = o - 1;
    g2 -= lul.d * (a.t(G_FY + 0, on) - a.t(G_FY + 0, oc)) + lul.mx * (a.t(G_FY + 3, on) - a.t(G_FY + 3, oc)) +
          lul.my * (a.t(G_FY + 1, on) - a.t(G_FY + 1, oc)) + lul.mz * (a.t(G_FY + 2, on) - a.t(G_FY + 2, oc)) +
          lul.e * (a.t(G_FY + 4, on) - a.t(G_FY + 4, oc)) + lul.bz * (a.t(G_FY + 5, on) - a.t(G_FY + 5, oc));
  }
  {
    const long long on = o + P, oc = o;
    g2 -= lur.d * (a.t(G_FY + 0, on) - a.t(G_FY + 0, oc)) + lur.mx * (a.t(G_FY + 3, on) - a.t(G_FY + 3, oc)) +
          lur.my * (a.t(G_FY + 1, on) - a.t(G_FY + 1, oc)) + lur.mz * (a.t(G_FY + 2, on) - a.t(G_FY + 2, oc)) +
          lur.e * (a.t(G_FY + 4, on) - a.t(G_FY + 4, oc)) + lur.bz * (a.t(G_FY + 5, on) - a.t(G_FY + 5, oc));
  }
  {
    const long long ow = o - 1;
    const double dbx = a.s(P_B1I, o) - a.s(P_B1I, ow);
    const double B1 = a.s(P_B1C, ow), B2 = a.s(P_B2C, ow), B3 = a.s(P_B3C, ow);
    const double V3 = a.s(P_M3, ow) / a.s(P_D, ow);
    g1 += dbx * (B1 * lul.mx + B2 * lul.my + B3 * lul.mz + V3 * lul.bz + B3 * V3 * lul.e);
  }
  {
    const double dbx = a.s(P_B1I, o + 1) - a.s(P_B1I, o);
    const double B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o), B3 = a.s(P_B3C, o);
    const double V3 = a.s(P_M3, o) / a.s(P_D, o);
    g1 += dbx * (B1 * lur.mx + B2 * lur.my + B3 * lur.mz + V3 * lur.bz + B3 * V3 * lur.e);
  }
  return 0.5 * g1 / a.dx1 + 0.5 * g2 / a.dx2;
}
ATHB_HD double correct_y_dtb(const AdjArgs& a, int j, int i, const Cons1& lul, const Cons1& lur) {
  const long long o = a.o(j, i), P = a.pitch;
  double g1 = 0.0, g2 = 0.0;
  {
    const long long oe = o - P + 1, oc = o - P;
    g1 -= lul.d * (a.t(G_FX + 0, oe) - a.t(G_FX + 0, oc)) + lul.mx * (a.t(G_FX + 2, oe) - a.t(G_FX + 2, oc)) +
          lul.my * (a.t(G_FX + 3, oe) - a.t(G_FX + 3, oc)) + lul.mz * (a.t(G_FX + 1, oe) - a.t(G_FX + 1, oc)) +
          lul.e * (a.t(G_FX + 4, oe) - a.t(G_FX + 4, oc)) + lul.by * (a.t(G_FX + 6, oe) - a.t(G_FX + 6, oc));
  }
  {
    const long long oe = o + 1, oc = o;
    g1 -= lur.d * (a.t(G_FX + 0, oe) - a.t(G_FX + 0, oc)) + lur.mx * (a.t(G_FX + 2, oe) - a.t(G_FX + 2, oc)) +
          lur.my * (a.t(G_FX + 3, oe) - a.t(G_FX + 3, oc)) + lur.mz * (a.t(G_FX + 1, oe) - a.t(G_FX + 1, oc)) +
          lur.e * (a.t(G_FX + 4, oe) - a.t(G_FX + 4, oc)) + lur.by * (a.t(G_FX + 6, oe) - a.t(G_FX + 6, oc));
  }
  {
    const long long osn = o - P;
    const double dby = a.s(P_B2I, o) - a.s(P_B2I, osn);
    const double B1 = a.s(P_B1C, osn), B2 = a.s(P_B2C, osn), B3 = a.s(P_B3C, osn);
    const double V3 = a.s(P_M3, osn) / a.s(P_D, osn);
    g2 += dby * (B1 * lul.mz + B2 * lul.mx + B3 * lul.my + V3 * lul.by + B3 * V3 * lul.e);
  }
  {
    const double dby = a.s(P_B2I, o + P) - a.s(P_B2I, o);
    const double B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o), B3 = a.s(P_B3C, o);
    const double V3 = a.s(P_M3, o) / a.s(P_D, o);
    g2 += dby * (B1 * lur.mz + B2 * lur.mx + B3 * lur.my + V3 * lur.by + B3 * V3 * lur.e);
  }
  return 0.5 * g1 / a.dx1 + 0.5 * g2 / a.dx2;
}

template <int FLUX>
ATHB_HD void adj_correct_x(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i);
  Cons1 ul, ur;
  double b1f;
  correct_x_states(a, j, i, ul, ur, b1f);
  const Prim1 wl = cons_to_prim(ul, b1f, a.eos);
  const Prim1 wr = cons_to_prim(ur, b1f, a.eos);
  Cons1 ulb, urb;
  Prim1 wlb, wrb;
  zero(ulb); zero(urb); zero(wlb); zero(wrb);
  double b1fb = 0.0;
  riemann_adj<FLUX>(ul, ur, wl, wr, b1f, a.eos, adj_cons(a, A_FX2, o), ulb, urb, wlb, wrb, b1fb);
  cons_to_prim_adj(ul, b1f, a.eos, wlb, ulb, b1fb);
  cons_to_prim_adj(ur, b1f, a.eos, wrb, urb, b1fb);
  adj_put_cons(a, A_ULX, o, ulb);
  adj_put_cons(a, A_URX, o, urb);
  a.a(A_B1F, o) = b1fb;
  a.a(A_DT, o) += correct_x_dtb(a, j, i, ulb, urb);
}

template <int FLUX>
ATHB_HD void adj_correct_y(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i);
  Cons1 ul, ur;
  double b2f;
  correct_y_states(a, j, i, ul, ur, b2f);
  const Prim1 wl = cons_to_prim(ul, b2f, a.eos);
  const Prim1 wr = cons_to_prim(ur, b2f, a.eos);
  Cons1 ulb, urb;
  Prim1 wlb, wrb;
  zero(ulb); zero(urb); zero(wlb); zero(wrb);
  double b2fb = 0.0;
  riemann_adj<FLUX>(ul, ur, wl, wr, b2f, a.eos, adj_cons(a, A_FY2, o), ulb, urb, wlb, wrb, b2fb);
  cons_to_prim_adj(ul, b2f, a.eos, wlb, ulb, b2fb);
  cons_to_prim_adj(ur, b2f, a.eos, wrb, urb, b2fb);
  adj_put_cons(a, A_ULY, o, ulb);
  adj_put_cons(a, A_URY, o, urb);
  a.a(A_B2F, o) = b2fb;
  a.a(A_DT, o) += correct_y_dtb(a, j, i, ulb, urb);
}

// step 7 reversed: cells [is-1, ie+1] x [js-1, je+1]
ATHB_HD void adj_correct_e(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i), P = a.pitch;
  const StepCoef<double>& c = a.c;
  const double dfx0 = a.t(G_FX + 0, o + 1) - a.t(G_FX + 0, o), dfy0 = a.t(G_FY + 0, o + P) - a.t(G_FY + 0, o);
  const double dfx1 = a.t(G_FX + 1, o + 1) - a.t(G_FX + 1, o), dfy3 = a.t(G_FY + 3, o + P) - a.t(G_FY + 3, o);
  const double dfx2 = a.t(G_FX + 2, o + 1) - a.t(G_FX + 2, o), dfy1 = a.t(G_FY + 1, o + P) - a.t(G_FY + 1, o);
  const double d = a.s(P_D, o) - c.hdtodx1 * dfx0 - c.hdtodx2 * dfy0;
  const double M1 = a.s(P_M1, o) - c.hdtodx1 * dfx1 - c.hdtodx2 * dfy3;
  const double M2 = a.s(P_M2, o) - c.hdtodx1 * dfx2 - c.hdtodx2 * dfy1;
  const double b1f_c = a.s(P_B1I, o) - c.hdtodx2 * (a.t(G_EMF0, o + P) - a.t(G_EMF0, o));
  const double b1f_e = a.s(P_B1I, o + 1) - c.hdtodx2 * (a.t(G_EMF0, o + P + 1) - a.t(G_EMF0, o + 1));
  const double b2f_c = a.s(P_B2I, o) + c.hdtodx1 * (a.t(G_EMF0, o + 1) - a.t(G_EMF0, o));
  const double b2f_n = a.s(P_B2I, o + P) + c.hdtodx1 * (a.t(G_EMF0, o + P + 1) - a.t(G_EMF0, o + P));
  const double B1c = 0.5 * (b1f_c + b1f_e);
  const double B2c = 0.5 * (b2f_c + b2f_n);
  const double e = (B1c * M2 - B2c * M1) / d;
  const double lam = a.av(A_ECC1, o);
  const double ld = -lam * e / d, lM1 = -lam * B2c / d, lM2 = lam * B1c / d;
  a.a(A_HALF + 0, o) = ld;
  a.a(A_HALF + 1, o) = lM1;
  a.a(A_HALF + 2, o) = lM2;
  a.a(A_HALF + 3, o) = lam * M2 / d;
  a.a(A_HALF + 4, o) = -lam * M1 / d;
  a.li(P_D, o) += ld;
  a.li(P_M1, o) += lM1;
  a.li(P_M2, o) += lM2;
  a.a(A_DT, o) += 0.5 * (-(ld * dfx0 + lM1 * dfx1 + lM2 * dfx2)) / a.dx1 +
                  0.5 * (-(ld * dfy0 + lM1 * dfy3 + lM2 * dfy1)) / a.dx2;
}

// Every consumer of the half-step face fields: x faces [is-1, ie+2] x
// [js-1, je+1] and y faces [is-1, ie+1] x [js-1, je+2]; items over
// [is-1, ie+2] x [js-1, je+2].
ATHB_HD void adj_half_faces(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i), P = a.pitch;
  const GenRange E = range_correct_e(a.is, a.ie, a.js, a.je);
  double dtb = 0.0;
  if (j <= a.je + 1) {  // x face
    double lb = 0.0;
    if (in_range(range_correct_x(a.is, a.ie, a.js, a.je), j, i)) lb += a.av(A_B1F, o);
    if (in_range(E, j, i)) lb += 0.5 * a.av(A_HALF + 3, o);
    if (in_range(E, j, i - 1)) lb += 0.5 * a.av(A_HALF + 3, o - 1);
    a.a(A_LB1F, o) = lb;
    a.li(P_B1I, o) += lb;
    dtb += -lb * (a.t(G_EMF0, o + P) - a.t(G_EMF0, o)) * 0.5 / a.dx2;
  }
  if (i <= a.ie + 1) {  // y face
    double lb = 0.0;
    if (in_range(range_correct_y(a.is, a.ie, a.js, a.je), j, i)) lb += a.av(A_B2F, o);
    if (in_range(E, j, i)) lb += 0.5 * a.av(A_HALF + 4, o);
    if (in_range(E, j - 1, i)) lb += 0.5 * a.av(A_HALF + 4, o - P);
    a.a(A_LB2F, o) = lb;
    a.li(P_B2I, o) += lb;
    dtb += lb * (a.t(G_EMF0, o + 1) - a.t(G_EMF0, o)) * 0.5 / a.dx1;
  }
  a.a(A_DT, o) += dtb;
}

// Half-step corner emf: corners [is-1, ie+2] x [js-1, je+2].
ATHB_HD void adj_emf0(const AdjArgs& a, int j, int i) {
  const GenRange fx(range_correct_x(a.is, a.ie, a.js, a.je));
  auto lb1 = [&](int jj, int ii) { return (jj >= a.js - 1 && jj <= a.je + 1 && ii >= a.is - 1 && ii <= a.ie + 2) ? a.av(A_LB1F, a.o(jj, ii)) : 0.0; };
  auto lb2 = [&](int jj, int ii) { return (jj >= a.js - 1 && jj <= a.je + 2 && ii >= a.is - 1 && ii <= a.ie + 1) ? a.av(A_LB2F, a.o(jj, ii)) : 0.0; };
  (void)fx;
  a.a(A_EMF0, a.o(j, i)) = a.c.hdtodx2 * (lb1(j, i) - lb1(j - 1, i)) + a.c.hdtodx1 * (lb2(j, i - 1) - lb2(j, i));
}

// The predictor fluxes and the t^n cell emf, gathered from the corrector
// (transverse terms), correct_e and the half-step corner emf; items over
// [is-2, ie+2] x [js-2, je+2].
ATHB_HD void adj_flux1(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i);
  const StepCoef<double>& c = a.c;
  const GenRange CX = range_correct_x(a.is, a.ie, a.js, a.je), CY = range_correct_y(a.is, a.ie, a.js, a.je);
  const GenRange E = range_correct_e(a.is, a.ie, a.js, a.je), K = range_emf0(a.is, a.ie, a.js, a.je);
  auto le = [&](int jj, int ii) { return in_range(K, jj, ii) ? a.av(A_EMF0, a.o(jj, ii)) : 0.0; };
  auto half = [&](int q, int jj, int ii) { return in_range(E, jj, ii) ? a.av(A_HALF + q, a.o(jj, ii)) : 0.0; };
  double k[8];
  // x face (j,i) of the predictor
  if (in_range(range_riemann_x(a.is, a.ie, a.js, a.je), j, i)) {
    double f[7] = {0, 0, 0, 0, 0, 0, 0};
    // correct_y transverse terms: (u.d, u.mx, u.my, u.mz, u.e, u.by) <- fx (0, 2, 3, 1, 4, 6)
    auto addy = [&](int base, int jj, int ii, double w) {
      if (!in_range(CY, jj, ii)) return;
      const long long q = a.o(jj, ii);
      f[0] += w * a.av(base + 0, q); f[2] += w * a.av(base + 1, q); f[3] += w * a.av(base + 2, q);
      f[1] += w * a.av(base + 3, q); f[4] += w * a.av(base + 4, q); f[6] += w * a.av(base + 5, q);
    };
    addy(A_ULY, j + 1, i - 1, -c.hdtodx1);
    addy(A_ULY, j + 1, i, c.hdtodx1);
    addy(A_URY, j, i - 1, -c.hdtodx1);
    addy(A_URY, j, i, c.hdtodx1);
    // correct_e: d, M1, M2 of cells (j,i) and (j,i-1)
    f[0] += c.hdtodx1 * (half(0, j, i) - half(0, j, i - 1));
    f[1] += c.hdtodx1 * (half(1, j, i) - half(1, j, i - 1));
    f[2] += c.hdtodx1 * (half(2, j, i) - half(2, j, i - 1));
    // half-step corner emf: fx_by of corner (j,i), fx_by_s of corner (j+1,i)
    if (in_range(K, j, i)) { corner_k(a, 0, j, i, k); f[5] += k[1] * le(j, i); }
    if (in_range(K, j + 1, i)) { corner_k(a, 0, j + 1, i, k); f[5] += k[0] * le(j + 1, i); }
    for (int q = 0; q < 7; q++) a.a(A_FX + q, o) = f[q];
  }
  // y face (j,i)
  if (in_range(range_riemann_y(a.is, a.ie, a.js, a.je), j, i)) {
    double f[7] = {0, 0, 0, 0, 0, 0, 0};
    // correct_x transverse terms: (u.d, u.mx, u.my, u.mz, u.e, u.bz) <- fy (0, 3, 1, 2, 4, 5)
    auto addx = [&](int base, int jj, int ii, double w) {
      if (!in_range(CX, jj, ii)) return;
      const long long q = a.o(jj, ii);
      f[0] += w * a.av(base + 0, q); f[3] += w * a.av(base + 1, q); f[1] += w * a.av(base + 2, q);
      f[2] += w * a.av(base + 3, q); f[4] += w * a.av(base + 4, q); f[5] += w * a.av(base + 6, q);
    };
    addx(A_ULX, j - 1, i + 1, -c.hdtodx2);
    addx(A_ULX, j, i + 1, c.hdtodx2);
    addx(A_URX, j - 1, i, -c.hdtodx2);
    addx(A_URX, j, i, c.hdtodx2);
    // correct_e: d <- fy0, M1 <- fy3, M2 <- fy1
    f[0] += c.hdtodx2 * (half(0, j, i) - half(0, j - 1, i));
    f[3] += c.hdtodx2 * (half(1, j, i) - half(1, j - 1, i));
    f[1] += c.hdtodx2 * (half(2, j, i) - half(2, j - 1, i));
    // corner emf: fy_bz of corner (j,i), fy_bz_w of corner (j,i+1)
    if (in_range(K, j, i)) { corner_k(a, 0, j, i, k); f[6] += k[3] * le(j, i); }
    if (in_range(K, j, i + 1)) { corner_k(a, 0, j, i + 1, k); f[6] += k[2] * le(j, i + 1); }
    for (int q = 0; q < 7; q++) a.a(A_FY + q, o) = f[q];
  }
  // t^n cell emf of cell (j,i) -> the state
  {
    double v = 0.0;
    if (in_range(K, j, i)) { corner_k(a, 0, j, i, k); v += k[7] * le(j, i); }
    if (in_range(K, j, i + 1)) { corner_k(a, 0, j, i + 1, k); v += k[6] * le(j, i + 1); }
    if (in_range(K, j + 1, i)) { corner_k(a, 0, j + 1, i, k); v += k[5] * le(j + 1, i); }
    if (in_range(K, j + 1, i + 1)) { corner_k(a, 0, j + 1, i + 1, k); v += k[4] * le(j + 1, i + 1); }
    if (v != 0.0) {
      const double d = a.s(P_D, o), M1 = a.s(P_M1, o), M2 = a.s(P_M2, o), B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o);
      const double e = (B1 * M2 - B2 * M1) / d;
      a.li(P_B1C, o) += v * M2 / d;
      a.li(P_M2, o) += v * B1 / d;
      a.li(P_B2C, o) -= v * M1 / d;
      a.li(P_M1, o) -= v * B2 / d;
      a.li(P_D, o) -= v * e / d;
    }
  }
}

// The corrector's MHD source terms (steps 5b, 6b) back to the state: cells
// [is-1, ie+1] x [js-1, je+1] and the face fields of x faces [is-1, ie+2] x
// [js-1, je+1], y faces [is-1, ie+1] x [js-1, je+2]; items over
// [is-1, ie+2] x [js-1, je+2].
ATHB_HD void adj_sources(const AdjArgs& a, int j, int i) {
  const long long o = a.o(j, i), P = a.pitch;
  const double h1 = a.c.hdtodx1, h2 = a.c.hdtodx2;
  const GenRange CX = range_correct_x(a.is, a.ie, a.js, a.je), CY = range_correct_y(a.is, a.ie, a.js, a.je);
  // λ of dbx of face (jj,ii)'s left (ul) or right (ur) state, with its cell
  auto dbx_l = [&](int jj, int ii) {   // ul of x face (jj,ii): cell (jj, ii-1)
    if (!in_range(CX, jj, ii)) return 0.0;
    const long long q = a.o(jj, ii), w = q - 1;
    const double B1 = a.s(P_B1C, w), B2 = a.s(P_B2C, w), B3 = a.s(P_B3C, w), V3 = a.s(P_M3, w) / a.s(P_D, w);
    return h1 * (B1 * a.av(A_ULX + 1, q) + B2 * a.av(A_ULX + 2, q) + B3 * a.av(A_ULX + 3, q) +
                 V3 * a.av(A_ULX + 6, q) + B3 * V3 * a.av(A_ULX + 4, q));
  };
  auto dbx_r = [&](int jj, int ii) {   // ur of x face (jj,ii): cell (jj, ii)
    if (!in_range(CX, jj, ii)) return 0.0;
    const long long q = a.o(jj, ii);
    const double B1 = a.s(P_B1C, q), B2 = a.s(P_B2C, q), B3 = a.s(P_B3C, q), V3 = a.s(P_M3, q) / a.s(P_D, q);
    return h1 * (B1 * a.av(A_URX + 1, q) + B2 * a.av(A_URX + 2, q) + B3 * a.av(A_URX + 3, q) +
                 V3 * a.av(A_URX + 6, q) + B3 * V3 * a.av(A_URX + 4, q));
  };
  auto dby_l = [&](int jj, int ii) {   // ul of y face (jj,ii): cell (jj-1, ii)
    if (!in_range(CY, jj, ii)) return 0.0;
    const long long q = a.o(jj, ii), s = q - P;
    const double B1 = a.s(P_B1C, s), B2 = a.s(P_B2C, s), B3 = a.s(P_B3C, s), V3 = a.s(P_M3, s) / a.s(P_D, s);
    return h2 * (B1 * a.av(A_ULY + 3, q) + B2 * a.av(A_ULY + 1, q) + B3 * a.av(A_ULY + 2, q) +
                 V3 * a.av(A_ULY + 5, q) + B3 * V3 * a.av(A_ULY + 4, q));
  };
  auto dby_r = [&](int jj, int ii) {   // ur of y face (jj,ii): cell (jj, ii)
    if (!in_range(CY, jj, ii)) return 0.0;
    const long long q = a.o(jj, ii);
    const double B1 = a.s(P_B1C, q), B2 = a.s(P_B2C, q), B3 = a.s(P_B3C, q), V3 = a.s(P_M3, q) / a.s(P_D, q);
    return h2 * (B1 * a.av(A_URY + 3, q) + B2 * a.av(A_URY + 1, q) + B3 * a.av(A_URY + 2, q) +
                 V3 * a.av(A_URY + 5, q) + B3 * V3 * a.av(A_URY + 4, q));
  };
  // cell (j,i)
  if (in_range(range_correct_e(a.is, a.ie, a.js, a.je), j, i)) {
    const double B3 = a.s(P_B3C, o);
    const double d = a.s(P_D, o), V3 = a.s(P_M3, o) / d;
    double lB1 = 0, lB2 = 0, lB3 = 0, lV3 = 0;
    if (in_range(CX, j, i + 1)) {  // ul of x face (j,i+1)
      const long long q = o + 1;
      const double dbx = a.s(P_B1I, q) - a.s(P_B1I, o);
      lB1 += h1 * dbx * a.av(A_ULX + 1, q); lB2 += h1 * dbx * a.av(A_ULX + 2, q);
      lB3 += h1 * dbx * (a.av(A_ULX + 3, q) + V3 * a.av(A_ULX + 4, q));
      lV3 += h1 * dbx * (a.av(A_ULX + 6, q) + B3 * a.av(A_ULX + 4, q));
    }
    if (in_range(CX, j, i)) {      // ur of x face (j,i)
      const double dbx = a.s(P_B1I, o + 1) - a.s(P_B1I, o);
      lB1 += h1 * dbx * a.av(A_URX + 1, o); lB2 += h1 * dbx * a.av(A_URX + 2, o);
      lB3 += h1 * dbx * (a.av(A_URX + 3, o) + V3 * a.av(A_URX + 4, o));
      lV3 += h1 * dbx * (a.av(A_URX + 6, o) + B3 * a.av(A_URX + 4, o));
    }
    if (in_range(CY, j + 1, i)) {  // ul of y face (j+1,i): mz<-B1, mx<-B2, my<-B3, by<-V3
      const long long q = o + P;
      const double dby = a.s(P_B2I, q) - a.s(P_B2I, o);
      lB1 += h2 * dby * a.av(A_ULY + 3, q); lB2 += h2 * dby * a.av(A_ULY + 1, q);
      lB3 += h2 * dby * (a.av(A_ULY + 2, q) + V3 * a.av(A_ULY + 4, q));
      lV3 += h2 * dby * (a.av(A_ULY + 5, q) + B3 * a.av(A_ULY + 4, q));
    }
    if (in_range(CY, j, i)) {      // ur of y face (j,i)
      const double dby = a.s(P_B2I, o + P) - a.s(P_B2I, o);
      lB1 += h2 * dby * a.av(A_URY + 3, o); lB2 += h2 * dby * a.av(A_URY + 1, o);
      lB3 += h2 * dby * (a.av(A_URY + 2, o) + V3 * a.av(A_URY + 4, o));
      lV3 += h2 * dby * (a.av(A_URY + 5, o) + B3 * a.av(A_URY + 4, o));
    }
    a.li(P_B1C, o) += lB1;
    a.li(P_B2C, o) += lB2;
    a.li(P_B3C, o) += lB3;
    a.li(P_M3, o) += lV3 / d;
    a.li(P_D, o) -= lV3 * V3 / d;
  }
  // x face (j,i): B1i through dbx of ul/ur of x faces i, i+1, i-1
  if (j <= a.je + 1 && j >= a.js - 1 && i >= a.is - 1 && i <= a.ie + 2)
    a.li(P_B1I, o) += dbx_l(j, i) - dbx_l(j, i + 1) - dbx_r(j, i) + dbx_r(j, i - 1);
  // y face (j,i)
  if (i <= a.ie + 1 && i >= a.is - 1 && j >= a.js - 1 && j <= a.je + 2)
    a.li(P_B2I, o) += dby_l(j, i) - dby_l(j + 1, i) - dby_r(j, i) + dby_r(j - 1, i);
}

// ===========================================================================
// Reverse of the predictor.
// ===========================================================================
// Predictor face (j,i) of sweep dir: faces of range_riemann_x / _y.
template <int FLUX>
ATHB_HD void adj_riemann(const AdjArgs& a, int dir, int j, int i) {
  const long long o = a.o(j, i);
  const long long step = dir == 0 ? 1 : a.pitch;
  const Prim1 wl = tape_prim(a, dir == 0 ? G_WLNX : G_WLNY, o - step);
  const Prim1 wr = tape_prim(a, dir == 0 ? G_WRTX : G_WRTY, o);
  const double bn = a.s(dir == 0 ? P_B1I : P_B2I, o);
  const Cons1 ul = prim_to_cons(wl, bn, a.eos);
  const Cons1 ur = prim_to_cons(wr, bn, a.eos);
  Cons1 ulb, urb;
  Prim1 wlb, wrb;
  zero(ulb); zero(urb); zero(wlb); zero(wrb);
  double bnb = 0.0;
  riemann_adj<FLUX>(ul, ur, wl, wr, bn, a.eos, adj_cons(a, dir == 0 ? A_FX : A_FY, o), ulb, urb, wlb, wrb, bnb);
  const GenRange C = dir == 0 ? range_correct_x(a.is, a.ie, a.js, a.je) : range_correct_y(a.is, a.ie, a.js, a.je);
  if (in_range(C, j, i)) {
    addto(ulb, adj_cons(a, dir == 0 ? A_ULX : A_ULY, o));
    addto(urb, adj_cons(a, dir == 0 ? A_URX : A_URY, o));
  }
  prim_to_cons_adj(wl, bn, a.eos, ulb, wlb, bnb);
  prim_to_cons_adj(wr, bn, a.eos, urb, wrb, bnb);
  adj_put_prim(a, dir == 0 ? A_WLNX : A_WLNY, o - step, wlb);
  adj_put_prim(a, dir == 0 ? A_WRTX : A_WRTY, o, wrb);
  a.a(dir == 0 ? A_BNX : A_BNY, o) = bnb;
}

// PLM + source term of cell (j,i) of sweep dir: cells of range_plm.
ATHB_HD void adj_plm(const AdjArgs& a, int dir, int j, int i) {
  const long long o = a.o(j, i);
  const long long step = dir == 0 ? 1 : a.pitch;
  // faces fed by this cell: wln -> face c+1, wrt -> face c
  const GenRange F = dir == 0 ? range_riemann_x(a.is, a.ie, a.js, a.je) : range_riemann_y(a.is, a.ie, a.js, a.je);
  const int jn = dir == 0 ? j : j + 1, in_ = dir == 0 ? i + 1 : i;
  Prim1 lwl, lwr;
  if (in_range(F, jn, in_)) lwl = adj_prim(a, dir == 0 ? A_WLNX : A_WLNY, o); else zero(lwl);
  if (in_range(F, j, i)) lwr = adj_prim(a, dir == 0 ? A_WRTX : A_WRTY, o); else zero(lwr);
  // source term: wln.(by|bz) += hdt*src, wrt.(by|bz) += hdt*src
  const double lsum = dir == 0 ? (lwl.by + lwr.by) : (lwl.bz + lwr.bz);
  const double d = a.s(P_D, o), mt = a.s(dir == 0 ? P_M2 : P_M1, o);
  const int bnp = dir == 0 ? P_B1I : P_B2I;
  const double db = a.s(bnp, o + step) - a.s(bnp, o);
  const double dxs = dir == 0 ? a.dx1 : a.dx2;
  const double src = (mt / d) * db / dxs;
  const double lsrc = a.c.hdt * lsum;
  double dtb = 0.5 * src * lsum;
  a.a(dir == 0 ? A_SRCX : A_SRCY, o) = lsrc;
  a.li(dir == 0 ? P_M2 : P_M1, o) += lsrc * db / dxs / d;
  a.li(P_D, o) -= lsrc * (mt / d / d) * db / dxs;
  // PLM
  const Cons1 um = state_cons(a, o - step, dir), u0 = state_cons(a, o, dir), up = state_cons(a, o + step, dir);
  const int bxp = dir == 0 ? P_B1C : P_B2C;
  const Prim1 wm = cons_to_prim(um, a.s(bxp, o - step), a.eos);
  const Prim1 w0 = cons_to_prim(u0, a.s(bxp, o), a.eos);
  const Prim1 wp = cons_to_prim(up, a.s(bxp, o + step), a.eos);
  Prim1 wmb, w0b, wpb;
  zero(wmb); zero(w0b); zero(wpb);
  double bxcb = 0.0, dtodxb = 0.0;
  plm_cell_adj(wm, w0, wp, a.s(bxp, o), dir == 0 ? a.c.dtodx1 : a.c.dtodx2, a.eos, lwl, lwr, wmb, w0b, wpb, bxcb,
               dtodxb);
  adj_put_prim(a, dir == 0 ? A_WXM : A_WYM, o, wmb);
  adj_put_prim(a, dir == 0 ? A_WX0 : A_WY0, o, w0b);
  adj_put_prim(a, dir == 0 ? A_WXP : A_WYP, o, wpb);
  a.li(bxp, o) += bxcb;
  dtb += dtodxb / dxs;
  a.a(A_DT, o) += dtb;
}

// Primitive-variable adjoints of cell (j,i) gathered from the PLM of cells
// c-1, c, c+1, back through cons -> prim; and the normal face field of face
// (j,i) (Riemann states, source terms).  Items over the PLM range widened by
// one cell along the sweep.
ATHB_HD void adj_prim_gather(const AdjArgs& a, int dir, int j, int i) {
  const long long o = a.o(j, i);
  const long long step = dir == 0 ? 1 : a.pitch;
  const GenRange L = range_plm(a.is, a.ie, a.js, a.je);
  const int jm = dir == 0 ? j : j - 1, im = dir == 0 ? i - 1 : i;   // previous cell along the sweep
  const int jp = dir == 0 ? j : j + 1, ip = dir == 0 ? i + 1 : i;   // next cell
  Prim1 lw;
  zero(lw);
  bool any = false;
  if (in_range(L, j, i)) { addto(lw, adj_prim(a, dir == 0 ? A_WX0 : A_WY0, o)); any = true; }
  if (in_range(L, jm, im)) { addto(lw, adj_prim(a, dir == 0 ? A_WXP : A_WYP, o - step)); any = true; }
  if (in_range(L, jp, ip)) { addto(lw, adj_prim(a, dir == 0 ? A_WXM : A_WYM, o + step)); any = true; }
  if (any) {
    const int bxp = dir == 0 ? P_B1C : P_B2C;
    Cons1 ub;
    zero(ub);
    double bxb = 0.0;
    cons_to_prim_adj(state_cons(a, o, dir), a.s(bxp, o), a.eos, lw, ub, bxb);
    lin_add_cons(a, o, dir, ub);
    a.li(bxp, o) += bxb;
  }
  // normal face field at face (j,i)
  const GenRange F = dir == 0 ? range_riemann_x(a.is, a.ie, a.js, a.je) : range_riemann_y(a.is, a.ie, a.js, a.je);
  const int bnp = dir == 0 ? P_B1I : P_B2I;
  const int mtp = dir == 0 ? P_M2 : P_M1;
  const double dxs = dir == 0 ? a.dx1 : a.dx2;
  double lb = 0.0;
  if (in_range(F, j, i)) lb += a.av(dir == 0 ? A_BNX : A_BNY, o);
  // src(c) = (Mt/d)(c) (B(c+1) - B(c)) / dx: face (j,i) is B(c) of cell (j,i) and B(c+1) of the previous cell
  if (in_range(L, j, i)) lb -= a.av(dir == 0 ? A_SRCX : A_SRCY, o) * (a.s(mtp, o) / a.s(P_D, o)) / dxs;
  if (in_range(L, jm, im))
    lb += a.av(dir == 0 ? A_SRCX : A_SRCY, o - step) * (a.s(mtp, o - step) / a.s(P_D, o - step)) / dxs;
  a.li(bnp, o) += lb;
}

// ===========================================================================
// Ghost zones (src/set_bvals.c:114-145): the generic fill and its adjoint.
// ===========================================================================
constexpr int kNghostA = 4;   // ghost layers (nghost, src/defs.h:82)

struct GhostGeom {
  int is, ie, js, je, sx, sy;
  int bc[4];
};

// Source index of ghost position k along one direction (lo..hi interior, the
// normal-field kind keeps hi+1 interior), flip for a reflecting wall; the
// reference's index sets (src/set_bvals.c: reflect / outflow / periodic).
ATHB_HD int ghost_map1(int k, int lo, int hi, bool bnorm, int bc_in, int bc_out, bool& flip) {
  flip = false;
  if (k < lo) {
    const int m = lo - k;
    if (bc_in == BC_REFLECT) { flip = true; return lo + (m - 1); }
    if (bc_in == BC_OUTFLOW) return lo;
    return hi - (m - 1);
  }
  if (k > hi + (bnorm ? 1 : 0)) {
    const int m = k - hi;
    if (bc_out == BC_REFLECT) { flip = true; return bnorm ? hi - (m - 2) : hi - (m - 1); }
    if (bc_out == BC_OUTFLOW) return hi;
    return lo + (m - 1);
  }
  return k;
}

// Generic fill of frame cell (j,i) of every plane: x2 map then x1 map.
template <class T>
ATHB_HD void gen_ghost(const Planes<T>& s, long long ps, int pitch, const GhostGeom& g, int j, int i) {
  const bool gxa = i < g.is || i > g.ie, gya = j < g.js || j > g.je;
  for (int kind = 0; kind < 3; kind++) {
    const int ie_int = g.ie + (kind == 1 ? 1 : 0), je_int = g.je + (kind == 2 ? 1 : 0);
    const bool gx = i < g.is || i > ie_int, gy = j < g.js || j > je_int;
    if (!gx && !gy) continue;
    bool f1 = false, f2 = false;
    const int sj = gy ? ghost_map1(j, g.js, g.je, kind == 2, g.bc[2], g.bc[3], f2) : j;
    const int si = gx ? ghost_map1(i, g.is, g.ie, kind == 1, g.bc[0], g.bc[1], f1) : i;
    const long long so = (long long)sj * pitch + si, o = (long long)j * pitch + i;
    if (kind == 0) {
      for (int p = 0; p < 8; p++) {
        T v = s.get(p * ps + so);
        if ((p == P_M1 && f1) || (p == P_M2 && f2)) v = -v;
        s.set(p * ps + o, v);
      }
      s.set(P_B3I * ps + o, s.get(P_B3I * ps + so));
    } else {
      const int p = kind == 1 ? P_B1I : P_B2I;
      s.set(p * ps + o, s.get(p * ps + so));
    }
  }
  (void)gxa; (void)gya;
}

// Adjoint, pass 1 (x2): rows [js, je(+1 for B2i)], every column: add the
// adjoints of the ghost rows that copy this row.
ATHB_HD void fold_x2(double* l, long long ps, int pitch, const GhostGeom& g, int j, int i) {
  for (int kind = 0; kind < 3; kind++) {
    const int je_int = g.je + (kind == 2 ? 1 : 0);
    if (j < g.js || j > je_int) continue;
    const long long o = (long long)j * pitch + i;
    for (int gq = 0; gq < 2 * kNghostA; gq++) {   // the ghost rows: js-4..js-1, je_int+1..je_int+4
      const int jj = gq < kNghostA ? g.js - kNghostA + gq : je_int + 1 + (gq - kNghostA);
      if (jj < 0 || jj >= g.sy) continue;
      bool f = false;
      if (ghost_map1(jj, g.js, g.je, kind == 2, g.bc[2], g.bc[3], f) != j) continue;
      const long long q = (long long)jj * pitch + i;
      if (kind == 0) {
        for (int p = 0; p < 8; p++) l[p * ps + o] += (p == P_M2 && f) ? -l[p * ps + q] : l[p * ps + q];
        l[P_B3I * ps + o] += l[P_B3I * ps + q];
      } else {
        const int p = kind == 1 ? P_B1I : P_B2I;
        l[p * ps + o] += l[p * ps + q];
      }
    }
  }
}
// Adjoint, pass 2 (x1): interior cells add the adjoints of the ghost
// columns of their row that copy them.
ATHB_HD void fold_x1(double* l, long long ps, int pitch, const GhostGeom& g, int j, int i) {
  for (int kind = 0; kind < 3; kind++) {
    const int ie_int = g.ie + (kind == 1 ? 1 : 0), je_int = g.je + (kind == 2 ? 1 : 0);
    if (j < g.js || j > je_int || i < g.is || i > ie_int) continue;
    const long long o = (long long)j * pitch + i;
    for (int gq = 0; gq < 2 * kNghostA; gq++) {   // the ghost columns: is-4..is-1, ie_int+1..ie_int+4
      const int ii = gq < kNghostA ? g.is - kNghostA + gq : ie_int + 1 + (gq - kNghostA);
      if (ii < 0 || ii >= g.sx) continue;
      bool f = false;
      if (ghost_map1(ii, g.is, g.ie, kind == 1, g.bc[0], g.bc[1], f) != i) continue;
      const long long q = (long long)j * pitch + ii;
      if (kind == 0) {
        for (int p = 0; p < 8; p++) l[p * ps + o] += (p == P_M1 && f) ? -l[p * ps + q] : l[p * ps + q];
        l[P_B3I * ps + o] += l[P_B3I * ps + q];
      } else {
        const int p = kind == 1 ? P_B1I : P_B2I;
        l[p * ps + o] += l[p * ps + q];
      }
    }
  }
}
// Zero every entry that is not a cell the step writes (ghosts after the
// fold), so the folded adjoint is exactly the interior one.
ATHB_HD void clear_frame(double* l, long long ps, int pitch, const GhostGeom& g, int j, int i) {
  const long long o = (long long)j * pitch + i;
  const bool cell_int = j >= g.js && j <= g.je && i >= g.is && i <= g.ie;
  for (int p = 0; p < NSTATE; p++) {
    bool keep = cell_int;
    if (p == P_B1I) keep = j >= g.js && j <= g.je && i >= g.is && i <= g.ie + 1;
    if (p == P_B2I) keep = j >= g.js && j <= g.je + 1 && i >= g.is && i <= g.ie;
    if (!keep) l[p * ps + o] = 0.0;
  }
}

}  // namespace athb
