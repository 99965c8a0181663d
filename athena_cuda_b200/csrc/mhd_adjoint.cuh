// mhd_adjoint.cuh -- hand-written reverse (adjoint) of the per-cell and
// per-face physics of mhd_physics.cuh.
//
// Every *_adj function takes the forward inputs, recomputes the forward pass
// it needs, and ACCUMULATES (+=) the transpose of its Jacobian applied to the
// output adjoints into the input adjoints.  Branches are the forward pass's
// (limiter cases, upwind / supersonic selections, the HLLE fallback, MAX /
// MIN operands, the alpha_f / alpha_s cases), which is what the tangent-linear
// model (the physics instantiated with Dual, dual.cuh) differentiates, so the
// pair passes the dot-product test <ybar, J xdot> == <J^T ybar, xdot>.
// A square root whose argument is exactly zero passes no adjoint (the Dual
// convention for a zero tangent there).
//
// Reference functions reversed (paths within the reference project):
//   src/convert_var.c:37-95      Cons1D_to_Prim1D / Prim1D_to_Cons1D
//   src/esystem_prim.c:36-235    esys_prim_adb_mhd
//   src/lr_states_plm.c:64-248   lr_states (one cell)
//   src/flux_roe.c:91-114        Roe averages
//   src/esystem_roe.c:56-293     esys_roe_adb_mhd
//   src/flux_roe.c:54-259        flux_roe (HLLE fallback frozen)
//   src/flux_hlle.c:60-199       flux_hlle
#pragma once

#include "mhd_physics.cuh"

namespace athb {

// adjoint of y = sqrt(x) at y (zero at y == 0)
ATHB_HD double sqrt_adj(double y, double ybar) { return y > 0.0 ? ybar / (2.0 * y) : 0.0; }
// derivative of fabs(x) as the Dual convention (fabs(0) = +x)
ATHB_HD double fabs_d(double x) { return x < 0.0 ? -1.0 : 1.0; }

ATHB_HD void zero(Cons1& u) { u.d = u.mx = u.my = u.mz = u.e = u.by = u.bz = 0.0; }
ATHB_HD void zero(Prim1& w) { w.d = w.vx = w.vy = w.vz = w.p = w.by = w.bz = 0.0; }
ATHB_HD void addto(Cons1& a, const Cons1& b) {
  a.d += b.d; a.mx += b.mx; a.my += b.my; a.mz += b.mz; a.e += b.e; a.by += b.by; a.bz += b.bz;
}
ATHB_HD void addto(Prim1& a, const Prim1& b) {
  a.d += b.d; a.vx += b.vx; a.vy += b.vy; a.vz += b.vz; a.p += b.p; a.by += b.by; a.bz += b.bz;
}

// --- src/convert_var.c:37-55 -------------------------------------------------
ATHB_HD void cons_to_prim_adj(const Cons1& u, double bx, const Eos& eos, const Prim1& wb, Cons1& ub, double& bxb) {
  const double di = 1.0 / u.d;
  const double K = u.mx * u.mx + u.my * u.my + u.mz * u.mz;
  const double p2 = (u.e - 0.5 * K * di - 0.5 * (bx * bx + u.by * u.by + u.bz * u.bz)) * eos.gamma_1;
  double dib = 0.0;
  ub.d += wb.d;
  ub.by += wb.by;
  ub.bz += wb.bz;
  if (p2 > kTiny) {
    const double p1b = wb.p * eos.gamma_1;  // p0 - 0.5 |B|^2, times gamma_1
    ub.e += p1b;
    const double Kb = -0.5 * di * p1b;
    dib += -0.5 * K * p1b;
    ub.mx += 2.0 * u.mx * Kb;
    ub.my += 2.0 * u.my * Kb;
    ub.mz += 2.0 * u.mz * Kb;
    bxb += -bx * p1b;
    ub.by += -u.by * p1b;
    ub.bz += -u.bz * p1b;
  }
  ub.mx += wb.vx * di;
  ub.my += wb.vy * di;
  ub.mz += wb.vz * di;
  dib += wb.vx * u.mx + wb.vy * u.my + wb.vz * u.mz;
  ub.d += -di * di * dib;
}

// --- src/convert_var.c:64-92 -------------------------------------------------
ATHB_HD void prim_to_cons_adj(const Prim1& w, double bx, const Eos& eos, const Cons1& ub, Prim1& wb, double& bxb) {
  const double V2 = w.vx * w.vx + w.vy * w.vy + w.vz * w.vz;
  wb.d += ub.d + ub.mx * w.vx + ub.my * w.vy + ub.mz * w.vz + ub.e * 0.5 * V2;
  wb.vx += ub.mx * w.d + ub.e * w.d * w.vx;
  wb.vy += ub.my * w.d + ub.e * w.d * w.vy;
  wb.vz += ub.mz * w.d + ub.e * w.d * w.vz;
  wb.p += ub.e / eos.gamma_1;
  bxb += ub.e * bx;
  wb.by += ub.by + ub.e * w.by;
  wb.bz += ub.bz + ub.e * w.bz;
}

// --- src/esystem_prim.c:36-235 -------------------------------------------------
// Eb holds the adjoints of every PrimEig entry (ev, R.., L..).
ATHB_HD void esys_prim_adj(double d, double v1, double p, double b1, double b2, double b3, const Eos& eos,
                           const PrimEig& Eb, double& db, double& v1b, double& pb, double& b1b, double& b2b,
                           double& b3b) {
  // forward
  const double di = 1.0 / d;
  const double btsq = b2 * b2 + b3 * b3;
  const double vaxsq = b1 * b1 * di;
  const double asq = eos.gamma * p * di;
  const double ct2 = btsq * di;
  const double tsum = vaxsq + ct2 + asq;
  const double tdif = vaxsq + ct2 - asq;
  const double cf2_cs2 = sqrt(tdif * tdif + 4.0 * asq * ct2);
  const double cfsq = 0.5 * (tsum + cf2_cs2);
  const double cf = sqrt(cfsq);
  const double cssq = asq * vaxsq / cfsq;
  const double cs = sqrt(cssq);
  const double bt = sqrt(btsq);
  double bet2, bet3;
  if (bt == 0.0) { bet2 = 1.0; bet3 = 0.0; } else { bet2 = b2 / bt; bet3 = b3 / bt; }
  int acase;
  double af, as;
  if (cf2_cs2 == 0.0) { af = 1.0; as = 0.0; acase = 0; }
  else if ((asq - cssq) <= 0.0) { af = 0.0; as = 1.0; acase = 0; }
  else if ((cfsq - asq) <= 0.0) { af = 1.0; as = 0.0; acase = 0; }
  else { af = sqrt((asq - cssq) / cf2_cs2); as = sqrt((cfsq - asq) / cf2_cs2); acase = 1; }
  const double sqrtd = sqrt(d);
  const double s = rsign(b1);
  const double a = sqrt(asq);
  const double qf = cf * af * s;
  const double qs = cs * as * s;
  const double afb = a * af * sqrtd;
  const double asb = a * as * sqrtd;
  const double vax = sqrt(vaxsq);
  const double na = 0.5 / asq;
  const double qf2 = na * qf, qs2 = na * qs;
  const double afp = na * afb * di;
  const double asp = na * asb * di;

  // reverse
  double dib = 0.0, asqb = 0.0, nab = 0.0, afpb = 0.0, aspb = 0.0, qf2b = 0.0, qs2b = 0.0;
  double bet2b = 0.0, bet3b = 0.0, afb_ = 0.0, asb_ = 0.0, sqrtdb = 0.0, cfb = 0.0, csb = 0.0;
  double afbb = 0.0, asbb = 0.0, qfb = 0.0, qsb = 0.0, vaxb = 0.0, ab = 0.0;
  // L entries
  asqb += Eb.L34 / (asq * asq);
  afpb -= Eb.L26 * bet3; bet3b -= Eb.L26 * afp;
  afpb -= Eb.L25 * bet2; bet2b -= Eb.L25 * afp;
  nab += Eb.L24 * as * di; asb_ += Eb.L24 * na * di; dib += Eb.L24 * na * as;
  qf2b -= Eb.L23 * bet3; bet3b -= Eb.L23 * qf2;
  qf2b -= Eb.L22 * bet2; bet2b -= Eb.L22 * qf2;
  nab -= Eb.L21 * cs * as; csb -= Eb.L21 * na * as; asb_ -= Eb.L21 * na * cs;
  bet2b += Eb.L16 * 0.5 * s / sqrtd; sqrtdb -= Eb.L16 * (0.5 * bet2 * s / sqrtd) / sqrtd;
  bet3b -= Eb.L15 * 0.5 * s / sqrtd; sqrtdb -= Eb.L15 * (-0.5 * bet3 * s / sqrtd) / sqrtd;
  bet2b += 0.5 * Eb.L13;
  bet3b -= 0.5 * Eb.L12;
  aspb += Eb.L06 * bet3; bet3b += Eb.L06 * asp;
  aspb += Eb.L05 * bet2; bet2b += Eb.L05 * asp;
  nab += Eb.L04 * af * di; afb_ += Eb.L04 * na * di; dib += Eb.L04 * na * af;
  qs2b += Eb.L03 * bet3; bet3b += Eb.L03 * qs2;
  qs2b += Eb.L02 * bet2; bet2b += Eb.L02 * qs2;
  nab -= Eb.L01 * cf * af; cfb -= Eb.L01 * na * af; afb_ -= Eb.L01 * na * cf;
  nab += aspb * asb * di; asbb += aspb * na * di; dib += aspb * na * asb;
  nab += afpb * afb * di; afbb += afpb * na * di; dib += afpb * na * afb;
  nab += qs2b * qs; qsb += qs2b * na;
  nab += qf2b * qf; qfb += qf2b * na;
  asqb -= nab * na / asq;
  // R entries
  afbb -= Eb.R62 * bet3; bet3b -= Eb.R62 * afb;
  bet2b += Eb.R61 * s * sqrtd; sqrtdb += Eb.R61 * bet2 * s;
  asbb += Eb.R60 * bet3; bet3b += Eb.R60 * asb;
  afbb -= Eb.R52 * bet2; bet2b -= Eb.R52 * afb;
  bet3b -= Eb.R51 * s * sqrtd; sqrtdb -= Eb.R51 * bet3 * s;
  asbb += Eb.R50 * bet2; bet2b += Eb.R50 * asb;
  db += Eb.R42 * asq * as; asqb += Eb.R42 * d * as; asb_ += Eb.R42 * d * asq;
  db += Eb.R40 * asq * af; asqb += Eb.R40 * d * af; afb_ += Eb.R40 * d * asq;
  qfb -= Eb.R32 * bet3; bet3b -= Eb.R32 * qf;
  bet2b += Eb.R31;
  qsb += Eb.R30 * bet3; bet3b += Eb.R30 * qs;
  qfb -= Eb.R22 * bet2; bet2b -= Eb.R22 * qf;
  bet3b -= Eb.R21;
  qsb += Eb.R20 * bet2; bet2b += Eb.R20 * qs;
  csb -= Eb.R12 * as; asb_ -= Eb.R12 * cs;
  cfb -= Eb.R10 * af; afb_ -= Eb.R10 * cf;
  db += Eb.R02 * as; asb_ += Eb.R02 * d;
  db += Eb.R00 * af; afb_ += Eb.R00 * d;
  // eigenvalues
  v1b += Eb.ev[0] + Eb.ev[1] + Eb.ev[2] + Eb.ev[3] + Eb.ev[4] + Eb.ev[5] + Eb.ev[6];
  cfb += Eb.ev[6] - Eb.ev[0];
  vaxb += Eb.ev[5] - Eb.ev[1];
  csb += Eb.ev[4] - Eb.ev[2];
  double vaxsqb = sqrt_adj(vax, vaxb);
  ab += asbb * as * sqrtd; asb_ += asbb * a * sqrtd; sqrtdb += asbb * a * as;
  ab += afbb * af * sqrtd; afb_ += afbb * a * sqrtd; sqrtdb += afbb * a * af;
  csb += qsb * as * s; asb_ += qsb * cs * s;
  cfb += qfb * af * s; afb_ += qfb * cf * s;
  asqb += sqrt_adj(a, ab);
  db += sqrt_adj(sqrtd, sqrtdb);
  double cssqb = 0.0, cfsqb = 0.0, c2b = 0.0;
  if (acase) {
    const double Af = (asq - cssq) / cf2_cs2, As = (cfsq - asq) / cf2_cs2;
    const double Afb = afb_ / (2.0 * af), Asb = asb_ / (2.0 * as);
    asqb += Afb / cf2_cs2; cssqb -= Afb / cf2_cs2; c2b -= Afb * Af / cf2_cs2;
    cfsqb += Asb / cf2_cs2; asqb -= Asb / cf2_cs2; c2b -= Asb * As / cf2_cs2;
  }
  double btsqb = 0.0;
  if (bt != 0.0 && !(btsq < kBetaFreeze * (b1 * b1 + d * asq))) {   // freeze_beta
    const double btb = -bet2b * bet2 / bt - bet3b * bet3 / bt;
    b2b += bet2b / bt;
    b3b += bet3b / bt;
    btsqb += sqrt_adj(bt, btb);
  }
  cssqb += sqrt_adj(cs, csb);
  asqb += cssqb * vaxsq / cfsq; vaxsqb += cssqb * asq / cfsq; cfsqb -= cssqb * cssq / cfsq;
  cfsqb += sqrt_adj(cf, cfb);
  const double tsumb = 0.5 * cfsqb;
  c2b += 0.5 * cfsqb;
  const double Xb = sqrt_adj(cf2_cs2, c2b);
  const double tdifb = 2.0 * tdif * Xb;
  asqb += 4.0 * ct2 * Xb;
  double ct2b = 4.0 * asq * Xb;
  vaxsqb += tdifb + tsumb;
  ct2b += tdifb + tsumb;
  asqb += -tdifb + tsumb;
  btsqb += ct2b * di; dib += ct2b * btsq;
  pb += asqb * eos.gamma * di; dib += asqb * eos.gamma * p;
  b1b += vaxsqb * 2.0 * b1 * di; dib += vaxsqb * b1 * b1;
  b2b += 2.0 * b2 * btsqb;
  b3b += 2.0 * b3 * btsqb;
  db += -di * di * dib;
}

// Adjoint of prim_project: a = L v.  Accumulates vb (from ab) and the L part
// of Eb.
ATHB_HD void prim_project_adj(const PrimEig& E, const double v[7], const double ab[7], double vb[7], PrimEig& Eb) {
  const double s06 = ab[0] - ab[6], t06 = ab[0] + ab[6];
  const double s15 = ab[1] - ab[5], t15 = ab[1] + ab[5];
  const double s24 = ab[2] - ab[4], t24 = ab[2] + ab[4];
  vb[0] += ab[3];
  vb[1] += E.L01 * s06 + E.L21 * s24;
  vb[2] += E.L02 * s06 + E.L12 * s15 + E.L22 * s24;
  vb[3] += E.L03 * s06 + E.L13 * s15 + E.L23 * s24;
  vb[4] += E.L04 * t06 + E.L24 * t24 + E.L34 * ab[3];
  vb[5] += E.L05 * t06 + E.L15 * t15 + E.L25 * t24;
  vb[6] += E.L06 * t06 + E.L16 * t15 + E.L26 * t24;
  Eb.L01 += v[1] * s06; Eb.L02 += v[2] * s06; Eb.L03 += v[3] * s06;
  Eb.L04 += v[4] * t06; Eb.L05 += v[5] * t06; Eb.L06 += v[6] * t06;
  Eb.L12 += v[2] * s15; Eb.L13 += v[3] * s15; Eb.L15 += v[5] * t15; Eb.L16 += v[6] * t15;
  Eb.L21 += v[1] * s24; Eb.L22 += v[2] * s24; Eb.L23 += v[3] * s24;
  Eb.L24 += v[4] * t24; Eb.L25 += v[5] * t24; Eb.L26 += v[6] * t24;
  Eb.L34 += v[4] * ab[3];
}

// Accumulate the adjoint of a left-eigenvector row n (lb, 7 coefficients in
// the layout prim_left_row gives) into Eb.
ATHB_HD void prim_left_row_adj(int n, const double lb[7], PrimEig& Eb) {
  switch (n) {
  case 0: Eb.L01 += lb[1]; Eb.L02 += lb[2]; Eb.L03 += lb[3]; Eb.L04 += lb[4]; Eb.L05 += lb[5]; Eb.L06 += lb[6]; break;
  case 1: Eb.L12 += lb[2]; Eb.L13 += lb[3]; Eb.L15 += lb[5]; Eb.L16 += lb[6]; break;
  case 2: Eb.L21 += lb[1]; Eb.L22 += lb[2]; Eb.L23 += lb[3]; Eb.L24 += lb[4]; Eb.L25 += lb[5]; Eb.L26 += lb[6]; break;
  case 3: Eb.L34 += lb[4]; break;
  case 4: Eb.L21 -= lb[1]; Eb.L22 -= lb[2]; Eb.L23 -= lb[3]; Eb.L24 += lb[4]; Eb.L25 += lb[5]; Eb.L26 += lb[6]; break;
  case 5: Eb.L12 -= lb[2]; Eb.L13 -= lb[3]; Eb.L15 += lb[5]; Eb.L16 += lb[6]; break;
  default: Eb.L01 -= lb[1]; Eb.L02 -= lb[2]; Eb.L03 -= lb[3]; Eb.L04 += lb[4]; Eb.L05 += lb[5]; Eb.L06 += lb[6]; break;
  }
}
// ... and of a right-eigenvector column n.
ATHB_HD void prim_right_col_adj(int n, const double rb[7], PrimEig& Eb) {
  switch (n) {
  case 0: Eb.R00 += rb[0]; Eb.R10 += rb[1]; Eb.R20 += rb[2]; Eb.R30 += rb[3]; Eb.R40 += rb[4]; Eb.R50 += rb[5]; Eb.R60 += rb[6]; break;
  case 1: Eb.R21 += rb[2]; Eb.R31 += rb[3]; Eb.R51 += rb[5]; Eb.R61 += rb[6]; break;
  case 2: Eb.R02 += rb[0]; Eb.R12 += rb[1]; Eb.R22 += rb[2]; Eb.R32 += rb[3]; Eb.R42 += rb[4]; Eb.R52 += rb[5]; Eb.R62 += rb[6]; break;
  case 3: break;
  case 4: Eb.R02 += rb[0]; Eb.R12 -= rb[1]; Eb.R22 -= rb[2]; Eb.R32 -= rb[3]; Eb.R42 += rb[4]; Eb.R52 += rb[5]; Eb.R62 += rb[6]; break;
  case 5: Eb.R21 -= rb[2]; Eb.R31 -= rb[3]; Eb.R51 += rb[5]; Eb.R61 += rb[6]; break;
  default: Eb.R00 += rb[0]; Eb.R10 -= rb[1]; Eb.R20 -= rb[2]; Eb.R30 -= rb[3]; Eb.R40 += rb[4]; Eb.R50 += rb[5]; Eb.R60 += rb[6]; break;
  }
}

ATHB_HD void zero(PrimEig& E) {
  #pragma unroll
  for (int n = 0; n < 7; n++) E.ev[n] = 0.0;
  E.R00 = E.R02 = E.R10 = E.R12 = E.R20 = E.R21 = E.R22 = E.R30 = E.R31 = E.R32 = 0.0;
  E.R40 = E.R42 = E.R50 = E.R51 = E.R52 = E.R60 = E.R61 = E.R62 = 0.0;
  E.L01 = E.L02 = E.L03 = E.L04 = E.L05 = E.L06 = E.L12 = E.L13 = E.L15 = E.L16 = 0.0;
  E.L21 = E.L22 = E.L23 = E.L24 = E.L25 = E.L26 = E.L34 = 0.0;
}

ATHB_HD void prim_arr(const Prim1& w, double a[7]) {
  a[0] = w.d; a[1] = w.vx; a[2] = w.vy; a[3] = w.vz; a[4] = w.p; a[5] = w.by; a[6] = w.bz;
}
ATHB_HD void prim_add_arr(Prim1& w, const double a[7]) {
  w.d += a[0]; w.vx += a[1]; w.vy += a[2]; w.vz += a[3]; w.p += a[4]; w.by += a[5]; w.bz += a[6];
}

// --- src/lr_states_plm.c:95-233, one cell -------------------------------------
// Forward: plm_cell(wm, w0, wp, bxc, dtodx) -> (wl_next, wr_this).
// Adjoint: wlb, wrb (adjoints of wl_next, wr_this) -> wmb, w0b, wpb, bxcb, dtodxb.
ATHB_HD void plm_cell_adj(const Prim1& wm, const Prim1& w0, const Prim1& wp, double bxc, double dtodx,
                          const Eos& eos, const Prim1& wlb, const Prim1& wrb, Prim1& wmb, Prim1& w0b, Prim1& wpb,
                          double& bxcb, double& dtodxb) {
  // ---- forward, keeping what the reverse needs ----
  PrimEig E;
  esys_prim(w0.d, w0.vx, w0.p, bxc, w0.by, w0.bz, eos, E);
  double Wm[7], W0[7], Wp[7];
  prim_arr(wm, Wm); prim_arr(w0, W0); prim_arr(wp, Wp);
  double dWc[7], dWl[7], dWr[7], dWg[7];
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    dWc[n] = Wp[n] - Wm[n];
    dWl[n] = W0[n] - Wm[n];
    dWr[n] = Wp[n] - W0[n];
    if (dWl[n] * dWr[n] > 0.0) dWg[n] = 2.0 * dWl[n] * dWr[n] / (dWl[n] + dWr[n]);
    else dWg[n] = 0.0;
  }
  double dac[7], dal[7], dar[7], dag[7];
  prim_project(E, dWc, dac);
  prim_project(E, dWl, dal);
  prim_project(E, dWr, dar);
  prim_project(E, dWg, dag);
  double da[7];
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    da[n] = 0.0;
    if (dal[n] * dar[n] > 0.0) {
      const double lim_slope1 = rmin(fabs(dal[n]), fabs(dar[n]));
      const double lim_slope2 = rmin(0.5 * fabs(dac[n]), fabs(dag[n]));
      da[n] = rsign(dac[n]) * rmin(2.0 * lim_slope1, lim_slope2);
    }
  }
  double dWm[7];
  dWm[0] = da[0] * E.R00 + da[2] * E.R02 + da[3] + da[4] * E.R02 + da[6] * E.R00;
  dWm[1] = da[0] * E.R10 + da[2] * E.R12 + da[4] * -E.R12 + da[6] * -E.R10;
  dWm[2] = da[0] * E.R20 + da[1] * E.R21 + da[2] * E.R22 + da[4] * -E.R22 + da[5] * -E.R21 + da[6] * -E.R20;
  dWm[3] = da[0] * E.R30 + da[1] * E.R31 + da[2] * E.R32 + da[4] * -E.R32 + da[5] * -E.R31 + da[6] * -E.R30;
  dWm[4] = da[0] * E.R40 + da[2] * E.R42 + da[4] * E.R42 + da[6] * E.R40;
  dWm[5] = da[0] * E.R50 + da[1] * E.R51 + da[2] * E.R52 + da[4] * E.R52 + da[5] * E.R51 + da[6] * E.R50;
  dWm[6] = da[0] * E.R60 + da[1] * E.R61 + da[2] * E.R62 + da[4] * E.R62 + da[5] * E.R61 + da[6] * E.R60;
  double dW[7];
  unsigned lsel = 0, rsel = 0;  // 2 bits per component: 0 = own value, 1 = first clip operand, 2 = second
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    const double l0 = W0[n] - 0.5 * dWm[n];
    const double r0 = W0[n] + 0.5 * dWm[n];
    // l = min(max(W0,Wm), max(min(W0,Wm), l0))
    const double lo = rmin(W0[n], Wm[n]), hi = rmax(W0[n], Wm[n]);
    double l = l0;
    unsigned sl = 0;
    if (lo > l) { l = lo; sl = 1; }      // rmax(lo, l) picks lo only when lo > l
    if (hi < l) { l = hi; sl = 2; }      // rmin(hi, l) picks hi only when hi < l
    const double lor = rmin(W0[n], Wp[n]), hir = rmax(W0[n], Wp[n]);
    double r = r0;
    unsigned sr = 0;
    if (lor > r) { r = lor; sr = 1; }
    if (hir < r) { r = hir; sr = 2; }
    lsel |= sl << (2 * n);
    rsel |= sr << (2 * n);
    dW[n] = r - l;
  }
  const double qx = 0.5 * rmax(E.ev[6], 0.0) * dtodx;
  const double qy = -0.5 * rmin(E.ev[0], 0.0) * dtodx;

  // ---- reverse ----
  double pWlb[7], pWrb[7];
  prim_arr(wlb, pWlb);
  prim_arr(wrb, pWrb);
  PrimEig Eb;
  zero(Eb);
  double dWb[7] = {0, 0, 0, 0, 0, 0, 0};
  // step 9, second loop (waves moving left)
  #pragma unroll
  for (int n = 6; n >= 0; n--) {
    if (!(E.ev[n] < 0.)) continue;
    double l[7], r[7], h[7], lb[7] = {0, 0, 0, 0, 0, 0, 0}, rb[7] = {0, 0, 0, 0, 0, 0, 0};
    prim_left_row(E, n, l);
    prim_right_col(E, n, r);
    #pragma unroll
    for (int m = 0; m < 7; m++) h[m] = l[m] * 0.5 * dtodx;
    double hb[7] = {0, 0, 0, 0, 0, 0, 0};
    const int lm = prim_left_mask(n), rm = prim_right_mask(n);
    {  // pWl[m] -= qa2 * r[m], qa2 = sum h[m] dev2 dW[m], dev2 = ev[n] - ev[6]
      const double dev2 = E.ev[n] - E.ev[6];
      double qa2 = 0.0, hdw = 0.0;
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((lm >> m) & 1) { qa2 += h[m] * dev2 * dW[m]; hdw += h[m] * dW[m]; }
      double qa2b = 0.0;
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((rm >> m) & 1) { qa2b -= pWlb[m] * r[m]; rb[m] -= qa2 * pWlb[m]; }
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((lm >> m) & 1) { hb[m] += qa2b * dev2 * dW[m]; dWb[m] += qa2b * h[m] * dev2; }
      const double dev2b = qa2b * hdw;
      Eb.ev[n] += dev2b;
      Eb.ev[6] -= dev2b;
    }
    if (n != 0) {  // pWr[m] += qa * r[m], qa = sum h[m] dev dW[m], dev = ev[0] - ev[n]
      const double dev = E.ev[0] - E.ev[n];
      double qa = 0.0, hdw = 0.0;
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((lm >> m) & 1) { qa += h[m] * dev * dW[m]; hdw += h[m] * dW[m]; }
      double qab = 0.0;
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((rm >> m) & 1) { qab += pWrb[m] * r[m]; rb[m] += qa * pWrb[m]; }
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((lm >> m) & 1) { hb[m] += qab * dev * dW[m]; dWb[m] += qab * h[m] * dev; }
      const double devb = qab * hdw;
      Eb.ev[0] += devb;
      Eb.ev[n] -= devb;
    }
    #pragma unroll
    for (int m = 0; m < 7; m++) {
      lb[m] += hb[m] * 0.5 * dtodx;
      dtodxb += hb[m] * l[m] * 0.5;
    }
    prim_left_row_adj(n, lb, Eb);
    prim_right_col_adj(n, rb, Eb);
  }
  // step 9, first loop (waves moving right)
  #pragma unroll
  for (int n = 5; n >= 0; n--) {
    if (!(E.ev[n] > 0.)) continue;
    double l[7], r[7], lb[7] = {0, 0, 0, 0, 0, 0, 0}, rb[7] = {0, 0, 0, 0, 0, 0, 0};
    prim_left_row(E, n, l);
    prim_right_col(E, n, r);
    const int lm = prim_left_mask(n), rm = prim_right_mask(n);
    const double dev = E.ev[6] - E.ev[n];
    double qa = 0.0, ldw = 0.0;
    #pragma unroll
    for (int m = 0; m < 7; m++)
      if ((lm >> m) & 1) { qa += l[m] * 0.5 * dtodx * dev * dW[m]; ldw += l[m] * dW[m]; }
    double qab = 0.0;
    #pragma unroll
    for (int m = 0; m < 7; m++)
      if ((rm >> m) & 1) { qab += pWlb[m] * r[m]; rb[m] += qa * pWlb[m]; }
    #pragma unroll
    for (int m = 0; m < 7; m++)
      if ((lm >> m) & 1) {
        lb[m] += qab * 0.5 * dtodx * dev * dW[m];
        dWb[m] += qab * l[m] * 0.5 * dtodx * dev;
      }
    const double devb = qab * 0.5 * dtodx * ldw;
    dtodxb += qab * 0.5 * dev * ldw;
    Eb.ev[6] += devb;
    Eb.ev[n] -= devb;
    prim_left_row_adj(n, lb, Eb);
    prim_right_col_adj(n, rb, Eb);
  }
  // step 8: pWl = Wrv - qx dW, pWr = Wlv + qy dW
  double Wlvb[7], Wrvb[7];
  double qxb = 0.0, qyb = 0.0;
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    Wrvb[n] = pWlb[n];
    qxb -= pWlb[n] * dW[n];
    dWb[n] -= qx * pWlb[n];
    Wlvb[n] = pWrb[n];
    qyb += pWrb[n] * dW[n];
    dWb[n] += qy * pWrb[n];
  }
  if (E.ev[6] > 0.0) Eb.ev[6] += qxb * 0.5 * dtodx;
  dtodxb += qxb * 0.5 * rmax(E.ev[6], 0.0);
  if (E.ev[0] < 0.0) Eb.ev[0] += -0.5 * dtodx * qyb;
  dtodxb += qyb * (-0.5 * rmin(E.ev[0], 0.0));
  // step 7: dW = r - l, and the clips
  double Wmb[7] = {0, 0, 0, 0, 0, 0, 0}, W0b[7] = {0, 0, 0, 0, 0, 0, 0}, Wpb[7] = {0, 0, 0, 0, 0, 0, 0};
  double dWmb[7];
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    Wrvb[n] += dWb[n];
    Wlvb[n] -= dWb[n];
    dWmb[n] = 0.0;
    const unsigned sl = (lsel >> (2 * n)) & 3u, sr = (rsel >> (2 * n)) & 3u;
    // left value
    if (sl == 0) { W0b[n] += Wlvb[n]; dWmb[n] -= 0.5 * Wlvb[n]; }
    else if (sl == 1) { if (W0[n] < Wm[n]) W0b[n] += Wlvb[n]; else Wmb[n] += Wlvb[n]; }   // lo = min(W0, Wm)
    else { if (W0[n] > Wm[n]) W0b[n] += Wlvb[n]; else Wmb[n] += Wlvb[n]; }                // hi = max(W0, Wm)
    // right value
    if (sr == 0) { W0b[n] += Wrvb[n]; dWmb[n] += 0.5 * Wrvb[n]; }
    else if (sr == 1) { if (W0[n] < Wp[n]) W0b[n] += Wrvb[n]; else Wpb[n] += Wrvb[n]; }
    else { if (W0[n] > Wp[n]) W0b[n] += Wrvb[n]; else Wpb[n] += Wrvb[n]; }
  }
  // step 5: dWm = R da
  double dab[7];
  dab[0] = dWmb[0] * E.R00 + dWmb[1] * E.R10 + dWmb[2] * E.R20 + dWmb[3] * E.R30 + dWmb[4] * E.R40 +
           dWmb[5] * E.R50 + dWmb[6] * E.R60;
  dab[1] = dWmb[2] * E.R21 + dWmb[3] * E.R31 + dWmb[5] * E.R51 + dWmb[6] * E.R61;
  dab[2] = dWmb[0] * E.R02 + dWmb[1] * E.R12 + dWmb[2] * E.R22 + dWmb[3] * E.R32 + dWmb[4] * E.R42 +
           dWmb[5] * E.R52 + dWmb[6] * E.R62;
  dab[3] = dWmb[0];
  dab[4] = dWmb[0] * E.R02 - dWmb[1] * E.R12 - dWmb[2] * E.R22 - dWmb[3] * E.R32 + dWmb[4] * E.R42 +
           dWmb[5] * E.R52 + dWmb[6] * E.R62;
  dab[5] = -dWmb[2] * E.R21 - dWmb[3] * E.R31 + dWmb[5] * E.R51 + dWmb[6] * E.R61;
  dab[6] = dWmb[0] * E.R00 - dWmb[1] * E.R10 - dWmb[2] * E.R20 - dWmb[3] * E.R30 + dWmb[4] * E.R40 +
           dWmb[5] * E.R50 + dWmb[6] * E.R60;
  Eb.R00 += dWmb[0] * (da[0] + da[6]); Eb.R02 += dWmb[0] * (da[2] + da[4]);
  Eb.R10 += dWmb[1] * (da[0] - da[6]); Eb.R12 += dWmb[1] * (da[2] - da[4]);
  Eb.R20 += dWmb[2] * (da[0] - da[6]); Eb.R21 += dWmb[2] * (da[1] - da[5]); Eb.R22 += dWmb[2] * (da[2] - da[4]);
  Eb.R30 += dWmb[3] * (da[0] - da[6]); Eb.R31 += dWmb[3] * (da[1] - da[5]); Eb.R32 += dWmb[3] * (da[2] - da[4]);
  Eb.R40 += dWmb[4] * (da[0] + da[6]); Eb.R42 += dWmb[4] * (da[2] + da[4]);
  Eb.R50 += dWmb[5] * (da[0] + da[6]); Eb.R51 += dWmb[5] * (da[1] + da[5]); Eb.R52 += dWmb[5] * (da[2] + da[4]);
  Eb.R60 += dWmb[6] * (da[0] + da[6]); Eb.R61 += dWmb[6] * (da[1] + da[5]); Eb.R62 += dWmb[6] * (da[2] + da[4]);
  // step 4: limiter, branch frozen
  double dacb[7] = {0, 0, 0, 0, 0, 0, 0}, dalb[7] = {0, 0, 0, 0, 0, 0, 0};
  double darb[7] = {0, 0, 0, 0, 0, 0, 0}, dagb[7] = {0, 0, 0, 0, 0, 0, 0};
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    if (!(dal[n] * dar[n] > 0.0)) continue;
    const double sg = rsign(dac[n]);
    const double al = fabs(dal[n]), ar = fabs(dar[n]);
    const double lim1 = rmin(al, ar);
    const double ac = 0.5 * fabs(dac[n]), ag = fabs(dag[n]);
    const double lim2 = rmin(ac, ag);
    const double mb = sg * dab[n];
    if (2.0 * lim1 < lim2) {   // rmin(2 lim1, lim2) picks 2 lim1
      const double l1b = 2.0 * mb;
      if (al < ar) dalb[n] += l1b * fabs_d(dal[n]); else darb[n] += l1b * fabs_d(dar[n]);
    } else {
      if (ac < ag) dacb[n] += mb * 0.5 * fabs_d(dac[n]); else dagb[n] += mb * fabs_d(dag[n]);
    }
  }
  // step 3: projections
  double dWcb[7] = {0, 0, 0, 0, 0, 0, 0}, dWlb[7] = {0, 0, 0, 0, 0, 0, 0};
  double dWrb[7] = {0, 0, 0, 0, 0, 0, 0}, dWgb[7] = {0, 0, 0, 0, 0, 0, 0};
  prim_project_adj(E, dWc, dacb, dWcb, Eb);
  prim_project_adj(E, dWl, dalb, dWlb, Eb);
  prim_project_adj(E, dWr, darb, dWrb, Eb);
  prim_project_adj(E, dWg, dagb, dWgb, Eb);
  // step 2: differences and the van Leer mean
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    if (dWl[n] * dWr[n] > 0.0) {
      const double s = dWl[n] + dWr[n];
      dWlb[n] += dWgb[n] * 2.0 * dWr[n] * dWr[n] / (s * s);
      dWrb[n] += dWgb[n] * 2.0 * dWl[n] * dWl[n] / (s * s);
    }
    Wpb[n] += dWcb[n] + dWrb[n];
    Wmb[n] -= dWcb[n] + dWlb[n];
    W0b[n] += dWlb[n] - dWrb[n];
  }
  // eigensystem of the centre cell
  double db = 0.0, v1b = 0.0, pb = 0.0, b2b = 0.0, b3b = 0.0;
  esys_prim_adj(w0.d, w0.vx, w0.p, bxc, w0.by, w0.bz, eos, Eb, db, v1b, pb, bxcb, b2b, b3b);
  W0b[0] += db; W0b[1] += v1b; W0b[4] += pb; W0b[5] += b2b; W0b[6] += b3b;
  prim_add_arr(wmb, Wmb);
  prim_add_arr(w0b, W0b);
  prim_add_arr(wpb, Wpb);
}

// ---------------------------------------------------------------------------
// Roe solver pieces
// ---------------------------------------------------------------------------
ATHB_HD void zero(RoeAvg& r) {
  r.sqrtdl = r.sqrtdr = r.isdlpdr = r.droe = r.v1 = r.v2 = r.v3 = r.b2 = r.b3 = r.x = r.y = r.pbl = r.pbr = r.h = 0.0;
}
ATHB_HD void zero(RoeSpeeds& s) {
  s.di = s.vsq = s.btsq = s.bt_starsq = s.vaxsq = s.hp = s.twid_asq = s.cfsq = s.cf = s.cssq = s.cs = s.vax = s.gfac = 0.0;
}
ATHB_HD void zero(RoeScal& S) {
  S.v1 = S.v2 = S.v3 = S.b2 = S.b3 = S.vsq = S.hp = S.cf = S.cs = 0.0;
  S.af = S.as = S.qf = S.qs = 0.0;
  S.bet2 = S.bet3 = S.bet2s = S.bet3s = S.vbet = S.aspbb = S.afpbb = S.sgn = S.isqrtd = S.sqrtd = 0.0;
  S.asp = S.afp = S.gx = 0.0;
  S.afn = S.asn = S.cff = S.css = S.qfn = S.qsn = S.Afn = S.Asn = S.afpb = S.aspb = S.q2s = S.q3s = 0.0;
  S.vqstr = S.norm2 = 0.0;
}

// src/flux_roe.c:91-114
ATHB_HD void roe_average_adj(const Cons1& Ul, const Cons1& Ur, const Prim1& Wl, const Prim1& Wr, double Bxi,
                             const RoeAvg& rb_in, Cons1& Ulb, Cons1& Urb, Prim1& Wlb, Prim1& Wrb, double& Bxib) {
  const RoeAvg r = roe_average(Ul, Ur, Wl, Wr, Bxi);
  RoeAvg rb = rb_in;
  // h = Q * isd, Q = A / sl + B / sr
  const double A = Ul.e + Wl.p + r.pbl, B = Ur.e + Wr.p + r.pbr;
  const double Q = A / r.sqrtdl + B / r.sqrtdr;
  const double Qb = rb.h * r.isdlpdr;
  rb.isdlpdr += rb.h * Q;
  const double Ab = Qb / r.sqrtdl, Bb = Qb / r.sqrtdr;
  rb.sqrtdl -= Qb * A / (r.sqrtdl * r.sqrtdl);
  rb.sqrtdr -= Qb * B / (r.sqrtdr * r.sqrtdr);
  Ulb.e += Ab; Wlb.p += Ab; rb.pbl += Ab;
  Urb.e += Bb; Wrb.p += Bb; rb.pbr += Bb;
  Bxib += (rb.pbl + rb.pbr) * Bxi;
  Wlb.by += rb.pbl * Wl.by; Wlb.bz += rb.pbl * Wl.bz;
  Wrb.by += rb.pbr * Wr.by; Wrb.bz += rb.pbr * Wr.bz;
  // y = 0.5 (dl + dr) / droe
  Wlb.d += 0.5 * rb.y / r.droe;
  Wrb.d += 0.5 * rb.y / r.droe;
  rb.droe -= rb.y * r.y / r.droe;
  // x = 0.5 (dby^2 + dbz^2) / ss^2
  {
    const double dby = Wl.by - Wr.by, dbz = Wl.bz - Wr.bz, ss = r.sqrtdl + r.sqrtdr;
    const double ss2 = ss * ss;
    const double Nb = 0.5 * rb.x / ss2;
    const double ss2b = -rb.x * r.x / ss2;
    const double ssb = 2.0 * ss * ss2b;
    Wlb.by += 2.0 * dby * Nb; Wrb.by -= 2.0 * dby * Nb;
    Wlb.bz += 2.0 * dbz * Nb; Wrb.bz -= 2.0 * dbz * Nb;
    rb.sqrtdl += ssb;
    rb.sqrtdr += ssb;
  }
  // transverse field averages (note the crossed weights)
  {
    const double n2 = r.sqrtdr * Wl.by + r.sqrtdl * Wr.by, n3 = r.sqrtdr * Wl.bz + r.sqrtdl * Wr.bz;
    const double n2b = rb.b2 * r.isdlpdr, n3b = rb.b3 * r.isdlpdr;
    rb.isdlpdr += rb.b2 * n2 + rb.b3 * n3;
    rb.sqrtdr += n2b * Wl.by + n3b * Wl.bz;
    rb.sqrtdl += n2b * Wr.by + n3b * Wr.bz;
    Wlb.by += n2b * r.sqrtdr; Wrb.by += n2b * r.sqrtdl;
    Wlb.bz += n3b * r.sqrtdr; Wrb.bz += n3b * r.sqrtdl;
  }
  // velocity averages
  {
    const double n1 = r.sqrtdl * Wl.vx + r.sqrtdr * Wr.vx;
    const double n2 = r.sqrtdl * Wl.vy + r.sqrtdr * Wr.vy;
    const double n3 = r.sqrtdl * Wl.vz + r.sqrtdr * Wr.vz;
    const double n1b = rb.v1 * r.isdlpdr, n2b = rb.v2 * r.isdlpdr, n3b = rb.v3 * r.isdlpdr;
    rb.isdlpdr += rb.v1 * n1 + rb.v2 * n2 + rb.v3 * n3;
    rb.sqrtdl += n1b * Wl.vx + n2b * Wl.vy + n3b * Wl.vz;
    rb.sqrtdr += n1b * Wr.vx + n2b * Wr.vy + n3b * Wr.vz;
    Wlb.vx += n1b * r.sqrtdl; Wlb.vy += n2b * r.sqrtdl; Wlb.vz += n3b * r.sqrtdl;
    Wrb.vx += n1b * r.sqrtdr; Wrb.vy += n2b * r.sqrtdr; Wrb.vz += n3b * r.sqrtdr;
  }
  rb.sqrtdl += rb.droe * r.sqrtdr;
  rb.sqrtdr += rb.droe * r.sqrtdl;
  rb.sqrtdl -= rb.isdlpdr * r.isdlpdr * r.isdlpdr;
  rb.sqrtdr -= rb.isdlpdr * r.isdlpdr * r.isdlpdr;
  Wlb.d += sqrt_adj(r.sqrtdl, rb.sqrtdl);
  Wrb.d += sqrt_adj(r.sqrtdr, rb.sqrtdr);
}

// src/esystem_roe.c:68-87,136-144
ATHB_HD void roe_speeds_adj(const RoeAvg& r, double b1, const Eos& eos, const RoeSpeeds& s, const RoeSpeeds& sb_in,
                            RoeAvg& rb, double& b1b) {
  RoeSpeeds sb = sb_in;
  const double T0 = eos.gamma_1 * (s.hp - 0.5 * s.vsq) - eos.gamma_2 * r.x;
  const double ct2 = s.bt_starsq * s.di;
  const double tdif = s.vaxsq + ct2 - s.twid_asq;
  const double cf2_cs2 = sqrt(tdif * tdif + 4.0 * s.twid_asq * ct2);
  sb.vaxsq += sqrt_adj(s.vax, sb.vax);
  sb.cssq += sqrt_adj(s.cs, sb.cs);
  sb.twid_asq += sb.cssq * s.vaxsq / s.cfsq;
  sb.vaxsq += sb.cssq * s.twid_asq / s.cfsq;
  sb.cfsq -= sb.cssq * s.cssq / s.cfsq;
  sb.cfsq += sqrt_adj(s.cf, sb.cf);
  const double tsumb = 0.5 * sb.cfsq;
  const double c2b = 0.5 * sb.cfsq;
  const double Xb = sqrt_adj(cf2_cs2, c2b);
  const double tdifb = 2.0 * tdif * Xb;
  sb.twid_asq += 4.0 * ct2 * Xb;
  double ct2b = 4.0 * s.twid_asq * Xb;
  sb.vaxsq += tdifb + tsumb;
  ct2b += tdifb + tsumb;
  sb.twid_asq += -tdifb + tsumb;
  sb.bt_starsq += ct2b * s.di;
  sb.di += ct2b * s.bt_starsq;
  if (T0 > kTiny) {
    sb.hp += eos.gamma_1 * sb.twid_asq;
    sb.vsq -= 0.5 * eos.gamma_1 * sb.twid_asq;
    rb.x -= eos.gamma_2 * sb.twid_asq;
  }
  rb.h += sb.hp;
  sb.vaxsq -= sb.hp;
  sb.btsq -= sb.hp * s.di;
  sb.di -= sb.hp * s.btsq;
  b1b += sb.vaxsq * 2.0 * b1 * s.di;
  sb.di += sb.vaxsq * b1 * b1;
  sb.gfac += sb.bt_starsq * s.btsq;
  sb.btsq += sb.bt_starsq * s.gfac;
  rb.y -= eos.gamma_2 * sb.gfac;
  rb.b2 += 2.0 * r.b2 * sb.btsq;
  rb.b3 += 2.0 * r.b3 * sb.btsq;
  rb.v1 += 2.0 * r.v1 * sb.vsq;
  rb.v2 += 2.0 * r.v2 * sb.vsq;
  rb.v3 += 2.0 * r.v3 * sb.vsq;
  rb.droe -= sb.di * s.di * s.di;
}

// src/esystem_roe.c:91-291 (the scalars of the eigenvectors)
ATHB_HD void roe_scalars_adj(const RoeAvg& r, const RoeSpeeds& s, double b1, const Eos& eos, const RoeScal& Sb,
                             RoeAvg& rb, RoeSpeeds& sb) {
  // forward
  const double v2 = r.v2, v3 = r.v3, b2 = r.b2, b3 = r.b3, d = r.droe;
  const double bt = sqrt(s.btsq);
  const double bt_star = sqrt(s.bt_starsq);
  double bet2, bet3;
  if (bt == 0.0) { bet2 = 1.0; bet3 = 0.0; } else { bet2 = b2 / bt; bet3 = b3 / bt; }
  const double sg = sqrt(s.gfac);
  const double bet2s = bet2 / sg, bet3s = bet3 / sg;
  const double bsq = bet2s * bet2s + bet3s * bet3s;
  int acase;
  double af, as;
  if ((s.cfsq - s.cssq) == 0.0) { af = 1.0; as = 0.0; acase = 0; }
  else if ((s.twid_asq - s.cssq) <= 0.0) { af = 0.0; as = 1.0; acase = 0; }
  else if ((s.cfsq - s.twid_asq) <= 0.0) { af = 1.0; as = 0.0; acase = 0; }
  else {
    af = sqrt((s.twid_asq - s.cssq) / (s.cfsq - s.cssq));
    as = sqrt((s.cfsq - s.twid_asq) / (s.cfsq - s.cssq));
    acase = 1;
  }
  const double sqrtd = sqrt(d);
  const double isqrtd = 1.0 / sqrtd;
  const double sgn = rsign(b1);
  const double twid_a = sqrt(s.twid_asq);
  const double qf = s.cf * af * sgn;
  const double qs = s.cs * as * sgn;
  const double afp = twid_a * af * isqrtd;
  const double asp = twid_a * as * isqrtd;
  const double norm = 0.5 / s.twid_asq;
  const double norm1 = norm * eos.gamma_1;
  const double q2s = bet2s / bsq, q3s = bet3s / bsq;

  // reverse
  double norm1b = 2.0 * Sb.norm2;
  double v2b = Sb.vqstr * q2s + Sb.v2, v3b = Sb.vqstr * q3s + Sb.v3;
  double q2sb = Sb.vqstr * v2 + Sb.q2s, q3sb = Sb.vqstr * v3 + Sb.q3s;
  double bet2sb = Sb.bet2s, bet3sb = Sb.bet3s, bsqb = 0.0;
  bet3sb += q3sb / bsq; bsqb -= q3sb * q3s / bsq;
  bet2sb += q2sb / bsq; bsqb -= q2sb * q2s / bsq;
  double asb_ = Sb.as + Sb.asn * norm1, afb_ = Sb.af + Sb.afn * norm1;
  norm1b += Sb.asn * as + Sb.afn * af;
  double normb = norm1b * eos.gamma_1;
  double aspb = Sb.asp, afpb = Sb.afp, btsb = 0.0;
  normb += Sb.aspb * asp * bt_star; aspb += Sb.aspb * norm * bt_star; btsb += Sb.aspb * norm * asp;
  normb += Sb.afpb * afp * bt_star; afpb += Sb.afpb * norm * bt_star; btsb += Sb.afpb * norm * afp;
  double db = 0.0;
  normb += Sb.Asn * asp * d; aspb += Sb.Asn * norm * d; db += Sb.Asn * norm * asp;
  normb += Sb.Afn * afp * d; afpb += Sb.Afn * norm * d; db += Sb.Afn * norm * afp;
  double qsb = Sb.qs + Sb.qsn * norm, qfb = Sb.qf + Sb.qfn * norm;
  normb += Sb.qsn * qs + Sb.qfn * qf;
  double csb = Sb.cs, cfb = Sb.cf;
  normb += Sb.css * as * s.cs; asb_ += Sb.css * norm * s.cs; csb += Sb.css * norm * as;
  normb += Sb.cff * af * s.cf; afb_ += Sb.cff * norm * s.cf; cfb += Sb.cff * norm * af;
  double twb = -normb * norm / s.twid_asq;
  rb.x += Sb.gx * eos.gamma_2 / eos.gamma_1;
  double sqrtdb = Sb.sqrtd, isqrtdb = Sb.isqrtd;
  aspb += Sb.aspbb * bt_star * bsq; btsb += Sb.aspbb * asp * bsq; bsqb += Sb.aspbb * asp * bt_star;
  afpb += Sb.afpbb * bt_star * bsq; btsb += Sb.afpbb * afp * bsq; bsqb += Sb.afpbb * afp * bt_star;
  double twab = aspb * as * isqrtd + afpb * af * isqrtd;
  asb_ += aspb * twid_a * isqrtd; afb_ += afpb * twid_a * isqrtd;
  isqrtdb += aspb * twid_a * as + afpb * twid_a * af;
  csb += qsb * as * sgn; asb_ += qsb * s.cs * sgn;
  cfb += qfb * af * sgn; afb_ += qfb * s.cf * sgn;
  twb += sqrt_adj(twid_a, twab);
  sqrtdb -= isqrtdb * isqrtd * isqrtd;
  db += sqrt_adj(sqrtd, sqrtdb);
  double cfsqb = 0.0, cssqb = 0.0;
  if (acase) {
    const double Den = s.cfsq - s.cssq;
    const double Af = (s.twid_asq - s.cssq) / Den, As = (s.cfsq - s.twid_asq) / Den;
    const double Afb = afb_ / (2.0 * af), Asb = asb_ / (2.0 * as);
    twb += Afb / Den; cssqb -= Afb / Den;
    cfsqb += Asb / Den; twb -= Asb / Den;
    const double Denb = -Afb * Af / Den - Asb * As / Den;
    cfsqb += Denb; cssqb -= Denb;
  }
  v2b += Sb.vbet * bet2s; bet2sb += Sb.vbet * v2;
  v3b += Sb.vbet * bet3s; bet3sb += Sb.vbet * v3;
  bet2sb += 2.0 * bet2s * bsqb;
  bet3sb += 2.0 * bet3s * bsqb;
  double bet2b = Sb.bet2 + bet2sb / sg, bet3b = Sb.bet3 + bet3sb / sg;
  const double sgb = -bet2sb * bet2s / sg - bet3sb * bet3s / sg;
  sb.gfac += sqrt_adj(sg, sgb);
  double b2b = Sb.b2, b3b = Sb.b3;
  if (bt != 0.0 && !(s.btsq < kBetaFreeze * (b1 * b1 + d * s.twid_asq))) {   // freeze_beta
    const double btb = -bet2b * bet2 / bt - bet3b * bet3 / bt;
    b2b += bet2b / bt;
    b3b += bet3b / bt;
    sb.btsq += sqrt_adj(bt, btb);
  }
  sb.bt_starsq += sqrt_adj(bt_star, btsb);
  rb.v1 += Sb.v1;
  rb.v2 += v2b;
  rb.v3 += v3b;
  rb.b2 += b2b;
  rb.b3 += b3b;
  rb.droe += db;
  sb.vsq += Sb.vsq;
  sb.hp += Sb.hp;
  sb.cf += cfb;
  sb.cs += csb;
  sb.twid_asq += twb;
  sb.cfsq += cfsqb;
  sb.cssq += cssqb;
}

// adjoint of column n of the Roe right-eigenmatrix
ATHB_HD void roe_right_col_adj(const RoeScal& S, const double ev[7], int n, const double cb[7], RoeScal& Sb,
                               double evb[7]) {
  switch (n) {
  case 0:
  case 6: {
    const double sg = n == 0 ? 1.0 : -1.0;   // c(6) = c(0) with qs, v1*cf terms negated
    // c0 = af; c1 = af*ev; c2 = af*v2 + sg*qs*bet2s; c3 = af*v3 + sg*qs*bet3s;
    // c4 = af*(hp - sg*v1*cf) + sg*qs*vbet + aspbb; c5 = asp*bet2s; c6 = asp*bet3s
    Sb.af += cb[0] + cb[1] * ev[n] + cb[2] * S.v2 + cb[3] * S.v3 + cb[4] * (S.hp - sg * S.v1 * S.cf);
    evb[n] += cb[1] * S.af;
    Sb.v2 += cb[2] * S.af;
    Sb.v3 += cb[3] * S.af;
    Sb.qs += sg * (cb[2] * S.bet2s + cb[3] * S.bet3s + cb[4] * S.vbet);
    Sb.bet2s += sg * cb[2] * S.qs + cb[5] * S.asp;
    Sb.bet3s += sg * cb[3] * S.qs + cb[6] * S.asp;
    Sb.hp += cb[4] * S.af;
    Sb.v1 -= sg * cb[4] * S.af * S.cf;
    Sb.cf -= sg * cb[4] * S.af * S.v1;
    Sb.vbet += sg * cb[4] * S.qs;
    Sb.aspbb += cb[4];
    Sb.asp += cb[5] * S.bet2s + cb[6] * S.bet3s;
    break;
  }
  case 1:
  case 5: {
    const double sg = n == 1 ? 1.0 : -1.0;
    // c2 = -sg*bet3; c3 = sg*bet2; c4 = -sg*(v2*bet3 - v3*bet2); c5 = -bet3*sgn*isqrtd; c6 = bet2*sgn*isqrtd
    Sb.bet3 += -sg * cb[2] - sg * cb[4] * S.v2 - cb[5] * S.sgn * S.isqrtd;
    Sb.bet2 += sg * cb[3] + sg * cb[4] * S.v3 + cb[6] * S.sgn * S.isqrtd;
    Sb.v2 += -sg * cb[4] * S.bet3;
    Sb.v3 += sg * cb[4] * S.bet2;
    Sb.isqrtd += (-cb[5] * S.bet3 + cb[6] * S.bet2) * S.sgn;
    break;
  }
  case 2:
  case 4: {
    const double sg = n == 2 ? -1.0 : 1.0;  // c(2): -qf terms, -v1*cs; c(4): +qf, +v1*cs
    // c0 = as; c1 = as*ev; c2 = as*v2 + sg*qf*bet2s; c3 = as*v3 + sg*qf*bet3s;
    // c4 = as*(hp + sg*v1*cs) + sg*qf*vbet - afpbb; c5 = -afp*bet2s; c6 = -afp*bet3s
    Sb.as += cb[0] + cb[1] * ev[n] + cb[2] * S.v2 + cb[3] * S.v3 + cb[4] * (S.hp + sg * S.v1 * S.cs);
    evb[n] += cb[1] * S.as;
    Sb.v2 += cb[2] * S.as;
    Sb.v3 += cb[3] * S.as;
    Sb.qf += sg * (cb[2] * S.bet2s + cb[3] * S.bet3s + cb[4] * S.vbet);
    Sb.bet2s += sg * cb[2] * S.qf - cb[5] * S.afp;
    Sb.bet3s += sg * cb[3] * S.qf - cb[6] * S.afp;
    Sb.hp += cb[4] * S.as;
    Sb.v1 += sg * cb[4] * S.as * S.cs;
    Sb.cs += sg * cb[4] * S.as * S.v1;
    Sb.vbet += sg * cb[4] * S.qf;
    Sb.afpbb -= cb[4];
    Sb.afp -= cb[5] * S.bet2s + cb[6] * S.bet3s;
    break;
  }
  default: {  // n == 3: (1, v1, v2, v3, 0.5 vsq + gx, 0, 0)
    Sb.v1 += cb[1];
    Sb.v2 += cb[2];
    Sb.v3 += cb[3];
    Sb.vsq += 0.5 * cb[4];
    Sb.gx += cb[4];
    break;
  }
  }
}

// adjoint of a = L u (roe_project)
ATHB_HD void roe_project_adj(const RoeScal& S, const double u[7], const double ab[7], double ub[7], RoeScal& Sb) {
  const double vh = S.vsq - S.hp;
  double vhb = 0.0;
  {  // rows 0 and 6
    const double a0 = ab[0], a6 = ab[6], t = a0 + a6, d = a0 - a6;
    // M00 = afn vh + cff (cf + v1) - qsn vqstr - aspb ; M60 = afn vh + cff (cf - v1) + qsn vqstr - aspb
    ub[0] += (S.afn * vh + S.cff * (S.cf + S.v1) - S.qsn * S.vqstr - S.aspb) * a0 +
             (S.afn * vh + S.cff * (S.cf - S.v1) + S.qsn * S.vqstr - S.aspb) * a6;
    ub[1] += (-S.afn * S.v1 - S.cff) * a0 + (-S.afn * S.v1 + S.cff) * a6;
    ub[2] += (-S.afn * S.v2 + S.qsn * S.q2s) * a0 + (-S.afn * S.v2 - S.qsn * S.q2s) * a6;
    ub[3] += (-S.afn * S.v3 + S.qsn * S.q3s) * a0 + (-S.afn * S.v3 - S.qsn * S.q3s) * a6;
    ub[4] += S.afn * t;
    ub[5] += (S.Asn * S.q2s - S.afn * S.b2) * t;
    ub[6] += (S.Asn * S.q3s - S.afn * S.b3) * t;
    const double u0 = u[0];
    Sb.afn += vh * u0 * t - S.v1 * u[1] * t - S.v2 * u[2] * t - S.v3 * u[3] * t + u[4] * t - S.b2 * u[5] * t -
              S.b3 * u[6] * t;
    vhb += S.afn * u0 * t;
    Sb.cff += (S.cf + S.v1) * u0 * a0 + (S.cf - S.v1) * u0 * a6 - u[1] * d;
    Sb.cf += S.cff * u0 * t;
    Sb.v1 += S.cff * u0 * d - S.afn * u[1] * t;
    Sb.qsn += -S.vqstr * u0 * d + S.q2s * u[2] * d + S.q3s * u[3] * d;
    Sb.vqstr += -S.qsn * u0 * d;
    Sb.aspb += -u0 * t;
    Sb.v2 += -S.afn * u[2] * t;
    Sb.v3 += -S.afn * u[3] * t;
    Sb.q2s += S.qsn * u[2] * d + S.Asn * u[5] * t;
    Sb.q3s += S.qsn * u[3] * d + S.Asn * u[6] * t;
    Sb.Asn += S.q2s * u[5] * t + S.q3s * u[6] * t;
    Sb.b2 += -S.afn * u[5] * t;
    Sb.b3 += -S.afn * u[6] * t;
  }
  {  // rows 1 and 5: a1 = p0+p2+p3+p5+p6, a5 = -p0-p2-p3+p5+p6
    const double d = ab[1] - ab[5], t = ab[1] + ab[5];
    ub[0] += (0.5 * (S.v2 * S.bet3 - S.v3 * S.bet2)) * d;
    ub[2] += (-0.5 * S.bet3) * d;
    ub[3] += (0.5 * S.bet2) * d;
    ub[5] += (-0.5 * S.sqrtd * S.bet3 * S.sgn) * t;
    ub[6] += (0.5 * S.sqrtd * S.bet2 * S.sgn) * t;
    Sb.v2 += 0.5 * S.bet3 * u[0] * d;
    Sb.v3 += -0.5 * S.bet2 * u[0] * d;
    Sb.bet3 += 0.5 * S.v2 * u[0] * d - 0.5 * u[2] * d - 0.5 * S.sqrtd * S.sgn * u[5] * t;
    Sb.bet2 += -0.5 * S.v3 * u[0] * d + 0.5 * u[3] * d + 0.5 * S.sqrtd * S.sgn * u[6] * t;
    Sb.sqrtd += (-0.5 * S.bet3 * u[5] + 0.5 * S.bet2 * u[6]) * S.sgn * t;
  }
  {  // rows 2 and 4
    const double a2 = ab[2], a4 = ab[4], t = a2 + a4, d = a2 - a4;
    // M20 = asn vh + css (cs + v1) + qfn vqstr + afpb ; M40 = asn vh + css (cs - v1) - qfn vqstr + afpb
    ub[0] += (S.asn * vh + S.css * (S.cs + S.v1) + S.qfn * S.vqstr + S.afpb) * a2 +
             (S.asn * vh + S.css * (S.cs - S.v1) - S.qfn * S.vqstr + S.afpb) * a4;
    ub[1] += (-S.asn * S.v1 - S.css) * a2 + (-S.asn * S.v1 + S.css) * a4;
    ub[2] += (-S.asn * S.v2 - S.qfn * S.q2s) * a2 + (-S.asn * S.v2 + S.qfn * S.q2s) * a4;
    ub[3] += (-S.asn * S.v3 - S.qfn * S.q3s) * a2 + (-S.asn * S.v3 + S.qfn * S.q3s) * a4;
    ub[4] += S.asn * t;
    ub[5] += (-S.Afn * S.q2s - S.asn * S.b2) * t;
    ub[6] += (-S.Afn * S.q3s - S.asn * S.b3) * t;
    const double u0 = u[0];
    Sb.asn += vh * u0 * t - S.v1 * u[1] * t - S.v2 * u[2] * t - S.v3 * u[3] * t + u[4] * t - S.b2 * u[5] * t -
              S.b3 * u[6] * t;
    vhb += S.asn * u0 * t;
    Sb.css += (S.cs + S.v1) * u0 * a2 + (S.cs - S.v1) * u0 * a4 - u[1] * d;
    Sb.cs += S.css * u0 * t;
    Sb.v1 += S.css * u0 * d - S.asn * u[1] * t;
    Sb.qfn += S.vqstr * u0 * d - S.q2s * u[2] * d - S.q3s * u[3] * d;
    Sb.vqstr += S.qfn * u0 * d;
    Sb.afpb += u0 * t;
    Sb.v2 += -S.asn * u[2] * t;
    Sb.v3 += -S.asn * u[3] * t;
    Sb.q2s += -S.qfn * u[2] * d - S.Afn * u[5] * t;
    Sb.q3s += -S.qfn * u[3] * d - S.Afn * u[6] * t;
    Sb.Afn += -S.q2s * u[5] * t - S.q3s * u[6] * t;
    Sb.b2 += -S.asn * u[5] * t;
    Sb.b3 += -S.asn * u[6] * t;
  }
  {  // row 3
    const double a3 = ab[3];
    ub[0] += (1.0 - S.norm2 * (0.5 * S.vsq - S.gx)) * a3;
    ub[1] += (S.norm2 * S.v1) * a3;
    ub[2] += (S.norm2 * S.v2) * a3;
    ub[3] += (S.norm2 * S.v3) * a3;
    ub[4] += (-S.norm2) * a3;
    ub[5] += (S.norm2 * S.b2) * a3;
    ub[6] += (S.norm2 * S.b3) * a3;
    Sb.norm2 += (-(0.5 * S.vsq - S.gx) * u[0] + S.v1 * u[1] + S.v2 * u[2] + S.v3 * u[3] - u[4] + S.b2 * u[5] +
                 S.b3 * u[6]) * a3;
    Sb.vsq += -0.5 * S.norm2 * u[0] * a3;
    Sb.gx += S.norm2 * u[0] * a3;
    Sb.v1 += S.norm2 * u[1] * a3;
    Sb.v2 += S.norm2 * u[2] * a3;
    Sb.v3 += S.norm2 * u[3] * a3;
    Sb.b2 += S.norm2 * u[5] * a3;
    Sb.b3 += S.norm2 * u[6] * a3;
  }
  Sb.vsq += vhb;
  Sb.hp -= vhb;
}

// src/flux_roe.c:136-172 (one side's physical flux)
ATHB_HD void side_flux_adj(const Cons1& U, const Prim1& W, double Bxi, double pb, const Cons1& Fb, Cons1& Ub,
                           Prim1& Wb, double& Bxib, double& pbb) {
  Ub.mx += Fb.d + Fb.mx * W.vx + Fb.my * W.vy + Fb.mz * W.vz;
  Ub.e += Fb.e * W.vx;
  Wb.vx += Fb.mx * U.mx + Fb.e * (U.e + W.p) + Fb.e * (pb - Bxi * Bxi) + Fb.by * W.by + Fb.bz * W.bz;
  Wb.vy += Fb.my * U.mx - Fb.e * Bxi * W.by - Fb.by * Bxi;
  Wb.vz += Fb.mz * U.mx - Fb.e * Bxi * W.bz - Fb.bz * Bxi;
  Wb.p += Fb.mx + Fb.e * W.vx;
  Wb.by += Fb.mx * W.by - Fb.my * Bxi - Fb.e * Bxi * W.vy + Fb.by * W.vx;
  Wb.bz += Fb.mx * W.bz - Fb.mz * Bxi - Fb.e * Bxi * W.vz + Fb.bz * W.vx;
  Bxib += -Fb.mx * Bxi - Fb.my * W.by - Fb.mz * W.bz -
          Fb.e * (2.0 * Bxi * W.vx + W.by * W.vy + W.bz * W.vz) - Fb.by * W.vy - Fb.bz * W.vz;
  pbb += Fb.e * W.vx;
}

// --- src/flux_hlle.c:60-199 ----------------------------------------------------
ATHB_HD void flux_hlle_adj(const Cons1& Ul, const Cons1& Ur, const Prim1& Wl, const Prim1& Wr, double Bxi,
                           const Eos& eos, const Cons1& Fb, Cons1& Ulb, Cons1& Urb, Prim1& Wlb, Prim1& Wrb,
                           double& Bxib) {
  const RoeAvg r = roe_average(Ul, Ur, Wl, Wr, Bxi);
  const RoeSpeeds s = roe_speeds(r, Bxi, eos);
  const double ev0 = r.v1 - s.cf, ev6 = r.v1 + s.cf;
  // fast speeds of the two sides
  const double asql = eos.gamma * Wl.p / Wl.d, vaxl = Bxi * Bxi / Wl.d;
  const double ct2l = (Ul.by * Ul.by + Ul.bz * Ul.bz) / Wl.d;
  const double tmpl = vaxl + ct2l - asql;
  const double sql = sqrt(tmpl * tmpl + 4.0 * asql * ct2l);
  const double cfl = sqrt(0.5 * (vaxl + ct2l + asql + sql));
  const double asqr = eos.gamma * Wr.p / Wr.d, vaxr = Bxi * Bxi / Wr.d;
  const double ct2r = (Ur.by * Ur.by + Ur.bz * Ur.bz) / Wr.d;
  const double tmpr = vaxr + ct2r - asqr;
  const double sqr = sqrt(tmpr * tmpr + 4.0 * asqr * ct2r);
  const double cfr = sqrt(0.5 * (vaxr + ct2r + asqr + sqr));
  const double ar = rmax(ev6, (Wr.vx + cfr));
  const double al = rmin(ev0, (Wl.vx - cfl));
  const double bp = rmax(ar, 0.0);
  const double bm = rmin(al, 0.0);
  Cons1 Fl, Fr;
  Fl.d = Ul.mx - bm * Ul.d;
  Fr.d = Ur.mx - bp * Ur.d;
  Fl.mx = Ul.mx * (Wl.vx - bm) + Wl.p - 0.5 * (Bxi * Bxi - Wl.by * Wl.by - Wl.bz * Wl.bz);
  Fr.mx = Ur.mx * (Wr.vx - bp) + Wr.p - 0.5 * (Bxi * Bxi - Wr.by * Wr.by - Wr.bz * Wr.bz);
  Fl.my = Ul.my * (Wl.vx - bm) - Bxi * Wl.by;
  Fr.my = Ur.my * (Wr.vx - bp) - Bxi * Wr.by;
  Fl.mz = Ul.mz * (Wl.vx - bm) - Bxi * Wl.bz;
  Fr.mz = Ur.mz * (Wr.vx - bp) - Bxi * Wr.bz;
  Fl.e = Ul.e * (Wl.vx - bm) + Wl.p * Wl.vx + (r.pbl * Wl.vx - Bxi * (Bxi * Wl.vx + Wl.by * Wl.vy + Wl.bz * Wl.vz));
  Fr.e = Ur.e * (Wr.vx - bp) + Wr.p * Wr.vx + (r.pbr * Wr.vx - Bxi * (Bxi * Wr.vx + Wr.by * Wr.vy + Wr.bz * Wr.vz));
  Fl.by = Wl.by * (Wl.vx - bm) - Bxi * Wl.vy;
  Fr.by = Wr.by * (Wr.vx - bp) - Bxi * Wr.vy;
  Fl.bz = Wl.bz * (Wl.vx - bm) - Bxi * Wl.vz;
  Fr.bz = Wr.bz * (Wr.vx - bp) - Bxi * Wr.vz;
  const double t = 0.5 * (bp + bm) / (bp - bm);

  // F = 0.5 (Fl + Fr) + (Fl - Fr) t
  const double fb[7] = {Fb.d, Fb.mx, Fb.my, Fb.mz, Fb.e, Fb.by, Fb.bz};
  const double fl[7] = {Fl.d, Fl.mx, Fl.my, Fl.mz, Fl.e, Fl.by, Fl.bz};
  const double fr[7] = {Fr.d, Fr.mx, Fr.my, Fr.mz, Fr.e, Fr.by, Fr.bz};
  double tb = 0.0;
  Cons1 Flb, Frb;
  double* flb = &Flb.d;
  double* frb = &Frb.d;
  #pragma unroll
  for (int k = 0; k < 7; k++) {
    flb[k] = (0.5 + t) * fb[k];
    frb[k] = (0.5 - t) * fb[k];
    tb += (fl[k] - fr[k]) * fb[k];
  }
  // t = 0.5 (bp + bm) / (bp - bm)
  double bpb = 0.5 * tb / (bp - bm) - tb * t / (bp - bm);
  double bmb = 0.5 * tb / (bp - bm) + tb * t / (bp - bm);
  double pblb = 0.0, pbrb = 0.0;
  // left flux
  {
    const double vm = Wl.vx - bm;
    Ulb.mx += Flb.d + Flb.mx * vm;
    Ulb.d -= Flb.d * bm;
    bmb -= Flb.d * Ul.d + Flb.mx * Ul.mx + Flb.my * Ul.my + Flb.mz * Ul.mz + Flb.e * Ul.e + Flb.by * Wl.by +
           Flb.bz * Wl.bz;
    Ulb.my += Flb.my * vm;
    Ulb.mz += Flb.mz * vm;
    Ulb.e += Flb.e * vm;
    Wlb.vx += Flb.mx * Ul.mx + Flb.my * Ul.my + Flb.mz * Ul.mz + Flb.e * Ul.e + Flb.e * Wl.p +
              Flb.e * (r.pbl - Bxi * Bxi) + Flb.by * Wl.by + Flb.bz * Wl.bz;
    Wlb.p += Flb.mx + Flb.e * Wl.vx;
    Wlb.by += Flb.mx * Wl.by - Flb.my * Bxi - Flb.e * Bxi * Wl.vy + Flb.by * vm;
    Wlb.bz += Flb.mx * Wl.bz - Flb.mz * Bxi - Flb.e * Bxi * Wl.vz + Flb.bz * vm;
    Wlb.vy += -Flb.e * Bxi * Wl.by - Flb.by * Bxi;
    Wlb.vz += -Flb.e * Bxi * Wl.bz - Flb.bz * Bxi;
    Bxib += -Flb.mx * Bxi - Flb.my * Wl.by - Flb.mz * Wl.bz -
            Flb.e * (2.0 * Bxi * Wl.vx + Wl.by * Wl.vy + Wl.bz * Wl.vz) - Flb.by * Wl.vy - Flb.bz * Wl.vz;
    pblb += Flb.e * Wl.vx;
  }
  {
    const double vp = Wr.vx - bp;
    Urb.mx += Frb.d + Frb.mx * vp;
    Urb.d -= Frb.d * bp;
    bpb -= Frb.d * Ur.d + Frb.mx * Ur.mx + Frb.my * Ur.my + Frb.mz * Ur.mz + Frb.e * Ur.e + Frb.by * Wr.by +
           Frb.bz * Wr.bz;
    Urb.my += Frb.my * vp;
    Urb.mz += Frb.mz * vp;
    Urb.e += Frb.e * vp;
    Wrb.vx += Frb.mx * Ur.mx + Frb.my * Ur.my + Frb.mz * Ur.mz + Frb.e * Ur.e + Frb.e * Wr.p +
              Frb.e * (r.pbr - Bxi * Bxi) + Frb.by * Wr.by + Frb.bz * Wr.bz;
    Wrb.p += Frb.mx + Frb.e * Wr.vx;
    Wrb.by += Frb.mx * Wr.by - Frb.my * Bxi - Frb.e * Bxi * Wr.vy + Frb.by * vp;
    Wrb.bz += Frb.mx * Wr.bz - Frb.mz * Bxi - Frb.e * Bxi * Wr.vz + Frb.bz * vp;
    Wrb.vy += -Frb.e * Bxi * Wr.by - Frb.by * Bxi;
    Wrb.vz += -Frb.e * Bxi * Wr.bz - Frb.bz * Bxi;
    Bxib += -Frb.mx * Bxi - Frb.my * Wr.by - Frb.mz * Wr.bz -
            Frb.e * (2.0 * Bxi * Wr.vx + Wr.by * Wr.vy + Wr.bz * Wr.vz) - Frb.by * Wr.vy - Frb.bz * Wr.vz;
    pbrb += Frb.e * Wr.vx;
  }
  // bp = max(max(ev6, Wr.vx + cfr), 0), bm = min(min(ev0, Wl.vx - cfl), 0)
  double ev6b = 0.0, ev0b = 0.0, cfrb = 0.0, cflb = 0.0;
  if (ar > 0.0) {
    if (ev6 > Wr.vx + cfr) ev6b += bpb; else { Wrb.vx += bpb; cfrb += bpb; }
  }
  if (al < 0.0) {
    if (ev0 < Wl.vx - cfl) ev0b += bmb; else { Wlb.vx += bmb; cflb -= bmb; }
  }
  // cf of each side
  {
    const double cfsqb = sqrt_adj(cfl, cflb);
    const double sqb = sqrt_adj(sql, 0.5 * cfsqb);
    const double tmpb = 2.0 * tmpl * sqb;
    const double asqb = 0.5 * cfsqb - tmpb + 4.0 * ct2l * sqb;
    const double vaxb = 0.5 * cfsqb + tmpb;
    const double ct2b = 0.5 * cfsqb + tmpb + 4.0 * asql * sqb;
    Wlb.p += asqb * eos.gamma / Wl.d;
    Wlb.d -= asqb * asql / Wl.d + vaxb * vaxl / Wl.d + ct2b * ct2l / Wl.d;
    Bxib += vaxb * 2.0 * Bxi / Wl.d;
    Ulb.by += ct2b * 2.0 * Ul.by / Wl.d;
    Ulb.bz += ct2b * 2.0 * Ul.bz / Wl.d;
  }
  {
    const double cfsqb = sqrt_adj(cfr, cfrb);
    const double sqb = sqrt_adj(sqr, 0.5 * cfsqb);
    const double tmpb = 2.0 * tmpr * sqb;
    const double asqb = 0.5 * cfsqb - tmpb + 4.0 * ct2r * sqb;
    const double vaxb = 0.5 * cfsqb + tmpb;
    const double ct2b = 0.5 * cfsqb + tmpb + 4.0 * asqr * sqb;
    Wrb.p += asqb * eos.gamma / Wr.d;
    Wrb.d -= asqb * asqr / Wr.d + vaxb * vaxr / Wr.d + ct2b * ct2r / Wr.d;
    Bxib += vaxb * 2.0 * Bxi / Wr.d;
    Urb.by += ct2b * 2.0 * Ur.by / Wr.d;
    Urb.bz += ct2b * 2.0 * Ur.bz / Wr.d;
  }
  // Roe average and speeds
  RoeAvg rb;
  zero(rb);
  RoeSpeeds sb;
  zero(sb);
  rb.v1 += ev0b + ev6b;
  sb.cf += ev6b - ev0b;
  rb.pbl += pblb;
  rb.pbr += pbrb;
  roe_speeds_adj(r, Bxi, eos, s, sb, rb, Bxib);
  roe_average_adj(Ul, Ur, Wl, Wr, Bxi, rb, Ulb, Urb, Wlb, Wrb, Bxib);
}

// --- src/flux_roe.c:54-259 -----------------------------------------------------
ATHB_HD void flux_roe_adj(const Cons1& Ul, const Cons1& Ur, const Prim1& Wl, const Prim1& Wr, double Bxi,
                          const Eos& eos, const Cons1& Fb, Cons1& Ulb, Cons1& Urb, Prim1& Wlb, Prim1& Wrb,
                          double& Bxib) {
  const RoeAvg r = roe_average(Ul, Ur, Wl, Wr, Bxi);
  const RoeSpeeds s = roe_speeds(r, Bxi, eos);
  double ev[7];
  ev[0] = r.v1 - s.cf; ev[1] = r.v1 - s.vax; ev[2] = r.v1 - s.cs; ev[3] = r.v1;
  ev[4] = r.v1 + s.cs; ev[5] = r.v1 + s.vax; ev[6] = r.v1 + s.cf;
  RoeAvg rb;
  zero(rb);
  if (ev[0] >= 0.0 || ev[6] <= 0.0) {  // supersonic: the upwind side's flux
    const bool left = ev[0] >= 0.0;
    double pbb = 0.0;
    side_flux_adj(left ? Ul : Ur, left ? Wl : Wr, Bxi, left ? r.pbl : r.pbr, Fb, left ? Ulb : Urb,
                  left ? Wlb : Wrb, Bxib, pbb);
    if (left) rb.pbl += pbb; else rb.pbr += pbb;
    roe_average_adj(Ul, Ur, Wl, Wr, Bxi, rb, Ulb, Urb, Wlb, Wrb, Bxib);
    return;
  }
  RoeScal S;
  roe_scalars(r, s, Bxi, eos, S);
  const double dU[7] = {Ur.d - Ul.d, Ur.mx - Ul.mx, Ur.my - Ul.my, Ur.mz - Ul.mz,
                        Ur.e - Ul.e, Ur.by - Ul.by, Ur.bz - Ul.bz};
  double a[7];
  roe_project(S, dU, a);
  // the forward's intermediate-state test (the HLLE fallback, frozen)
  {
    double u[7] = {Ul.d, Ul.mx, Ul.my, Ul.mz, Ul.e, Ul.by, Ul.bz};
    #pragma unroll
    for (int n = 0; n < 6; n++) {
      double c[7];
      roe_right_col(S, ev, n, c);
      #pragma unroll
      for (int m = 0; m < 7; m++)
        if ((roe_right_mask(n) >> m) & 1) u[m] += a[n] * c[m];
      if (ev[n + 1] > ev[n]) {
        bool bad = (u[0] <= 0.0);
        if (!bad) {
          double p_inter = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
          p_inter -= 0.5 * (u[5] * u[5] + u[6] * u[6] + Bxi * Bxi);
          bad = (p_inter < 0.0);
        }
        if (bad) {
          flux_hlle_adj(Ul, Ur, Wl, Wr, Bxi, eos, Fb, Ulb, Urb, Wlb, Wrb, Bxib);
          return;
        }
      }
    }
  }
  // F = 0.5 (Fl + Fr) - sum_n 0.5 |ev_n| a_n c_n
  const double fb[7] = {Fb.d, Fb.mx, Fb.my, Fb.mz, Fb.e, Fb.by, Fb.bz};
  RoeScal Sb;
  zero(Sb);
  double evb[7] = {0, 0, 0, 0, 0, 0, 0}, abar[7];
  #pragma unroll
  for (int n = 0; n < 7; n++) {
    double c[7], cb[7];
    roe_right_col(S, ev, n, c);
    const double coeff = 0.5 * rmax(fabs(ev[n]), 0.0) * a[n];
    double coeffb = 0.0;
    #pragma unroll
    for (int k = 0; k < 7; k++) {
      if ((roe_right_mask(n) >> k) & 1) { coeffb -= fb[k] * c[k]; cb[k] = -coeff * fb[k]; }
      else cb[k] = 0.0;
    }
    abar[n] = 0.5 * fabs(ev[n]) * coeffb;
    // MAX(fabs(ev), 0) takes the constant 0 when ev == 0
    if (fabs(ev[n]) > 0.0) evb[n] += 0.5 * fabs_d(ev[n]) * a[n] * coeffb;
    roe_right_col_adj(S, ev, n, cb, Sb, evb);
  }
  double dUb[7] = {0, 0, 0, 0, 0, 0, 0};
  roe_project_adj(S, dU, abar, dUb, Sb);
  Urb.d += dUb[0]; Urb.mx += dUb[1]; Urb.my += dUb[2]; Urb.mz += dUb[3]; Urb.e += dUb[4]; Urb.by += dUb[5]; Urb.bz += dUb[6];
  Ulb.d -= dUb[0]; Ulb.mx -= dUb[1]; Ulb.my -= dUb[2]; Ulb.mz -= dUb[3]; Ulb.e -= dUb[4]; Ulb.by -= dUb[5]; Ulb.bz -= dUb[6];
  {
    Cons1 Fhb;
    Fhb.d = 0.5 * Fb.d; Fhb.mx = 0.5 * Fb.mx; Fhb.my = 0.5 * Fb.my; Fhb.mz = 0.5 * Fb.mz;
    Fhb.e = 0.5 * Fb.e; Fhb.by = 0.5 * Fb.by; Fhb.bz = 0.5 * Fb.bz;
    side_flux_adj(Ul, Wl, Bxi, r.pbl, Fhb, Ulb, Wlb, Bxib, rb.pbl);
    side_flux_adj(Ur, Wr, Bxi, r.pbr, Fhb, Urb, Wrb, Bxib, rb.pbr);
  }
  RoeSpeeds sb;
  zero(sb);
  roe_scalars_adj(r, s, Bxi, eos, Sb, rb, sb);
  rb.v1 += evb[0] + evb[1] + evb[2] + evb[3] + evb[4] + evb[5] + evb[6];
  sb.cf += evb[6] - evb[0];
  sb.vax += evb[5] - evb[1];
  sb.cs += evb[4] - evb[2];
  roe_speeds_adj(r, Bxi, eos, s, sb, rb, Bxib);
  roe_average_adj(Ul, Ur, Wl, Wr, Bxi, rb, Ulb, Urb, Wlb, Wrb, Bxib);
}

template <int FLUX>
ATHB_HD void riemann_adj(const Cons1& Ul, const Cons1& Ur, const Prim1& Wl, const Prim1& Wr, double Bxi,
                         const Eos& eos, const Cons1& Fb, Cons1& Ulb, Cons1& Urb, Prim1& Wlb, Prim1& Wrb,
                         double& Bxib) {
  if (FLUX == kFluxHlle) flux_hlle_adj(Ul, Ur, Wl, Wr, Bxi, eos, Fb, Ulb, Urb, Wlb, Wrb, Bxib);
  else flux_roe_adj(Ul, Ur, Wl, Wr, Bxi, eos, Fb, Ulb, Urb, Wlb, Wrb, Bxib);
}

// ---------------------------------------------------------------------------
// Corner EMF: partial derivatives (linear once the upwind branches are fixed)
// with respect to its 8 varying inputs, in the order
// fx_by_s, fx_by, fy_bz_w, fy_bz, e_sw, e_s, e_w, e_c.
// ---------------------------------------------------------------------------
ATHB_HD void corner_emf_coeffs(double fx_d_s, double fx_d, double fy_d_w, double fy_d, double k[8]) {
  for (int m = 0; m < 8; m++) k[m] = 0.0;
  // l2 (fx_d_s): -fx_by_s + ...
  k[0] -= 1.0;
  if (fx_d_s > 0.0) { k[2] += 1.0; k[4] -= 1.0; }
  else if (fx_d_s < 0.0) { k[3] += 1.0; k[5] -= 1.0; }
  else { k[2] += 0.5; k[4] -= 0.5; k[3] += 0.5; k[5] -= 0.5; }
  // r2 (fx_d): -fx_by + ...
  k[1] -= 1.0;
  if (fx_d > 0.0) { k[2] += 1.0; k[6] -= 1.0; }
  else if (fx_d < 0.0) { k[3] += 1.0; k[7] -= 1.0; }
  else { k[2] += 0.5; k[6] -= 0.5; k[3] += 0.5; k[7] -= 0.5; }
  // l1 (fy_d_w): fy_bz_w + ...
  k[2] += 1.0;
  if (fy_d_w > 0.0) { k[0] -= 1.0; k[4] -= 1.0; }
  else if (fy_d_w < 0.0) { k[1] -= 1.0; k[6] -= 1.0; }
  else { k[0] -= 0.5; k[4] -= 0.5; k[1] -= 0.5; k[6] -= 0.5; }
  // r1 (fy_d): fy_bz + ...
  k[3] += 1.0;
  if (fy_d > 0.0) { k[0] -= 1.0; k[5] -= 1.0; }
  else if (fy_d < 0.0) { k[1] -= 1.0; k[7] -= 1.0; }
  else { k[0] -= 0.5; k[5] -= 0.5; k[1] -= 0.5; k[7] -= 0.5; }
  for (int m = 0; m < 8; m++) k[m] *= 0.25;
}

// new_dt per cell (src/new_dt.c:37-85): adjoint with respect to (d, M1, M2,
// M3, E) of the winning term, given the adjoint mb of the cell's rate.
ATHB_HD void cell_dti_adj(double d, double m1, double m2, double m3, double e, const Eos& eos, double dx1,
                          double dx2, double mb, double out[5]) {
  const double di = 1.0 / d;
  const double v1 = m1 * di, v2 = m2 * di, v3 = m3 * di;
  const double qsq = v1 * v1 + v2 * v2 + v3 * v3;
  const double p0 = eos.gamma_1 * (e - 0.5 * d * qsq);
  const double p = rmax(p0, kTiny);
  const double asq = eos.gamma * p * di;
  const double ca = sqrt(asq);
  const double t1 = (fabs(v1) + ca) / dx1, t2 = (fabs(v2) + ca) / dx2;
  // m = MAX(MAX(0, t1), t2): MAX(a, b) = (a > b) ? a : b takes b on a tie
  const double m = rmax(0.0, t1);
  double v1b = 0.0, v2b = 0.0, cab = 0.0;
  if (!(m > t2)) { v2b += fabs_d(v2) * mb / dx2; cab += mb / dx2; }
  else if (!(0.0 > t1)) { v1b += fabs_d(v1) * mb / dx1; cab += mb / dx1; }
  const double asqb = sqrt_adj(ca, cab);
  const double pb = asqb * eos.gamma * di;
  double dib = asqb * eos.gamma * p;
  double db = 0.0, qsqb = 0.0, eb = 0.0;
  if (p0 > kTiny) {
    eb += eos.gamma_1 * pb;
    db += -0.5 * eos.gamma_1 * qsq * pb;
    qsqb += -0.5 * eos.gamma_1 * d * pb;
  }
  v1b += 2.0 * v1 * qsqb; v2b += 2.0 * v2 * qsqb;
  const double v3b = 2.0 * v3 * qsqb;
  out[1] = v1b * di; out[2] = v2b * di; out[3] = v3b * di;
  dib += v1b * m1 + v2b * m2 + v3b * m3;
  out[0] = db - di * di * dib;
  out[4] = eb;
}

}  // namespace athb
