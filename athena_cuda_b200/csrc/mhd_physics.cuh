// mhd_physics.cuh -- per-cell / per-face physics of the 2D adiabatic ideal-MHD
// CTU step, written for FP64 SIMT on sm_100a.
//
// Every function here reproduces, operation for operation, the IEEE-754
// binary64 arithmetic of the reference CPU path (same operands, same
// association, same branch tests) so that a kernel built with --fmad=false is
// bit-identical to it.  What differs is the shape of the work:
//   * eigenmatrices are never materialised as dense 7x7 arrays: only the
//     structurally non-zero entries are formed, and products whose factor is an
//     exact 0.0 in the reference are skipped (x + (+-0) == x for every finite x,
//     so sums over the remaining terms, kept in the reference order, are
//     unchanged; only the sign of an exact zero result can differ);
//   * entries that the reference defines as exact negations / copies of other
//     entries reuse one product (-(a*b) == (-a)*b exactly in IEEE-754);
//   * eigenvalues are formed first and the Roe solver returns the upwind flux
//     before any eigenvector work when the face is supersonic.
//
// The functions are __host__ __device__ so the very same source can be checked
// on a CPU against the reference routines; on the device they are inlined into
// the step kernels.
//
// Reference sources restated (paths within the reference project):
//   src/convert_var.c:37-95      Cons1D_to_Prim1D / Prim1D_to_Cons1D
//   src/esystem_prim.c:36-235    esys_prim_adb_mhd   (eigensystem in primitives)
//   src/lr_states_plm.c:64-248   lr_states           (characteristic PLM)
//   src/esystem_roe.c:56-293     esys_roe_adb_mhd    (Roe-matrix eigensystem)
//   src/flux_roe.c:54-259        flux_roe            (with HLLE fallback)
//   src/flux_hlle.c:60-199       flux_hlle
#pragma once

#include <math.h>

#include <type_traits>

#include "dual.cuh"

#if defined(__CUDACC__)
#define ATHB_HD __host__ __device__ __forceinline__
#else
#define ATHB_HD static inline
#endif

namespace athb {

constexpr double kTiny = 1.0e-20;   // TINY_NUMBER, src/defs.h:100

// Derivatives only (the tangent-linear model and the adjoint; the plain step
// is untouched): the unit vector of the transverse field, (b2, b3)/|b_t|,
// turns at a rate ~1/|b_t|, and near |b_t| = 0 the wave terms that carry it
// cancel in exact arithmetic but not in floating point, whereas their exact
// contribution to the derivative is O(|b_t|).  Where the transverse magnetic
// pressure is below kBetaFreeze times the pressure scale (b_n^2 + d a^2) the
// unit vector is therefore differentiated as a constant.
constexpr double kBetaFreeze = 1.0e-12;
template <class T>
ATHB_HD void freeze_beta(T& bet2, T& bet3, double btsq, double scale) {
  if constexpr (!std::is_same<T, double>::value) {
    if (btsq < kBetaFreeze * scale) {
      bet2 = no_tangent(bet2);
      bet3 = no_tangent(bet3);
    }
  }
}

// Conserved / primitive variables of one 1D slice, in the slice frame
// (x = sweep direction).  Field order is that of Cons1D / Prim1D
// (src/athena.h:75-98).
template <class T> struct Cons1T { T d, mx, my, mz, e, by, bz; };
template <class T> struct Prim1T { T d, vx, vy, vz, p, by, bz; };
using Cons1 = Cons1T<double>;
using Prim1 = Prim1T<double>;

// Equation-of-state constants (the reference globals Gamma, Gamma_1, Gamma_2).
struct Eos { double gamma, gamma_1, gamma_2; };

// MAX / MIN / SIGN exactly as the reference macros (src/defs.h:87-94).
template <class T> ATHB_HD T rmax(T a, T b) { return (a > b) ? a : b; }
template <class T> ATHB_HD T rmin(T a, T b) { return (a < b) ? a : b; }
template <class T> ATHB_HD T rsign(T a) { return (a < 0.) ? T(-1.) : T(1.); }

template <class T>
ATHB_HD T cget(const Cons1T<T>& u, int n) {
  return n == 0 ? u.d : n == 1 ? u.mx : n == 2 ? u.my : n == 3 ? u.mz : n == 4 ? u.e : n == 5 ? u.by : u.bz;
}

// --- src/convert_var.c:37-55 -------------------------------------------------
template <class T>
ATHB_HD Prim1T<T> cons_to_prim(const Cons1T<T>& u, T bx, const Eos& eos) {
  Prim1T<T> w;
  const T di = 1.0 / u.d;
  w.d = u.d;
  w.vx = u.mx * di;
  w.vy = u.my * di;
  w.vz = u.mz * di;
  T p = u.e - 0.5 * (u.mx * u.mx + u.my * u.my + u.mz * u.mz) * di;
  p -= 0.5 * (bx * bx + u.by * u.by + u.bz * u.bz);
  p *= eos.gamma_1;
  w.p = rmax(p, T(kTiny));
  w.by = u.by;
  w.bz = u.bz;
  return w;
}

// --- src/convert_var.c:64-92 -------------------------------------------------
template <class T>
ATHB_HD Cons1T<T> prim_to_cons(const Prim1T<T>& w, T bx, const Eos& eos) {
  Cons1T<T> u;
  u.d = w.d;
  u.mx = w.d * w.vx;
  u.my = w.d * w.vy;
  u.mz = w.d * w.vz;
  u.e = w.p / eos.gamma_1 + 0.5 * w.d * (w.vx * w.vx + w.vy * w.vy + w.vz * w.vz);
  u.e += 0.5 * (bx * bx + w.by * w.by + w.bz * w.bz);
  u.by = w.by;
  u.bz = w.bz;
  return u;
}

// ---------------------------------------------------------------------------
// Primitive-variable eigensystem (src/esystem_prim.c:36-235), kept as the few
// distinct scalars the 7x7 matrices are built from.
//   Right eigenvectors (columns) R[row][col]:
//     row0: R00=d*af  R02=d*as  R03=1  R04=R02  R06=R00
//     row1: R10=-cf*af R12=-cs*as R14=-R12 R16=-R10
//     row2: R20=qs*b2 R21=-b3 R22=-qf*b2 R24=-R22 R25=b3 R26=-R20
//     row3: R30=qs*b3 R31=b2  R32=-qf*b3 R34=-R32 R35=-b2 R36=-R30
//     row4: R40=d*asq*af R42=d*asq*as R44=R42 R46=R40
//     row5: R50=as*b2 R51=-b3*s*sqrtd R52=-af*b2 R54=R52 R55=R51 R56=R50
//     row6: R60=as*b3 R61=b2*s*sqrtd  R62=-af*b3 R64=R62 R65=R61 R66=R60
//   Left eigenvectors (rows) L[row][col]:
//     row0: L01..L06 ; row1: L12 L13 L15 L16 ; row2: L21..L26 ;
//     row3: L30=1 L34=-1/asq ; row4 = (-L21,-L22,-L23, L24,L25,L26) ;
//     row5 = (-L12,-L13, L15,L16) ; row6 = (-L01,-L02,-L03, L04,L05,L06)
// ---------------------------------------------------------------------------
template <class T> struct PrimEigT {
  T ev[7];
  T R00, R02, R10, R12, R20, R21, R22, R30, R31, R32, R40, R42, R50, R51, R52, R60, R61, R62;
  T L01, L02, L03, L04, L05, L06, L12, L13, L15, L16, L21, L22, L23, L24, L25, L26, L34;
};
using PrimEig = PrimEigT<double>;

template <class T>
ATHB_HD void esys_prim(T d, T v1, T p, T b1, T b2, T b3,
                       const Eos& eos, PrimEigT<T>& E) {
  const T di = 1.0 / d;
  const T btsq = b2 * b2 + b3 * b3;
  const T vaxsq = b1 * b1 * di;
  const T asq = eos.gamma * p * di;

  const T ct2 = btsq * di;
  const T tsum = vaxsq + ct2 + asq;
  const T tdif = vaxsq + ct2 - asq;
  const T cf2_cs2 = sqrt(tdif * tdif + 4.0 * asq * ct2);
  const T cfsq = 0.5 * (tsum + cf2_cs2);
  const T cf = sqrt(cfsq);
  const T cssq = asq * vaxsq / cfsq;
  const T cs = sqrt(cssq);

  const T bt = sqrt(btsq);
  T bet2, bet3;
  if (bt == 0.0) { bet2 = 1.0; bet3 = 0.0; } else { bet2 = b2 / bt; bet3 = b3 / bt; }
  freeze_beta(bet2, bet3, value_of(btsq), value_of(b1) * value_of(b1) + value_of(d) * value_of(asq));

  T alpha_f, alpha_s;
  if (cf2_cs2 == 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
  else if ((asq - cssq) <= 0.0) { alpha_f = 0.0; alpha_s = 1.0; }
  else if ((cfsq - asq) <= 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
  else { alpha_f = sqrt((asq - cssq) / cf2_cs2); alpha_s = sqrt((cfsq - asq) / cf2_cs2); }

  const T sqrtd = sqrt(d);
  const T s = rsign(b1);
  const T a = sqrt(asq);
  T qf = cf * alpha_f * s;
  T qs = cs * alpha_s * s;
  const T af = a * alpha_f * sqrtd;
  const T as = a * alpha_s * sqrtd;

  const T vax = sqrt(vaxsq);
  E.ev[0] = v1 - cf; E.ev[1] = v1 - vax; E.ev[2] = v1 - cs; E.ev[3] = v1;
  E.ev[4] = v1 + cs; E.ev[5] = v1 + vax; E.ev[6] = v1 + cf;

  E.R00 = d * alpha_f;        E.R02 = d * alpha_s;
  E.R10 = -cf * alpha_f;      E.R12 = -cs * alpha_s;
  E.R20 = qs * bet2;          E.R21 = -bet3;      E.R22 = -qf * bet2;
  E.R30 = qs * bet3;          E.R31 = bet2;       E.R32 = -qf * bet3;
  E.R40 = d * asq * alpha_f;  E.R42 = d * asq * alpha_s;
  E.R50 = as * bet2;          E.R51 = -bet3 * s * sqrtd;  E.R52 = -af * bet2;
  E.R60 = as * bet3;          E.R61 = bet2 * s * sqrtd;   E.R62 = -af * bet3;

  const T na = 0.5 / asq;
  qf = na * qf;
  qs = na * qs;
  const T af_prime = na * af * di;
  const T as_prime = na * as * di;

  E.L01 = -na * cf * alpha_f; E.L02 = qs * bet2; E.L03 = qs * bet3;
  E.L04 = na * alpha_f * di;  E.L05 = as_prime * bet2; E.L06 = as_prime * bet3;
  E.L12 = -0.5 * bet3; E.L13 = 0.5 * bet2;
  E.L15 = -0.5 * bet3 * s / sqrtd; E.L16 = 0.5 * bet2 * s / sqrtd;
  E.L21 = -na * cs * alpha_s; E.L22 = -qf * bet2; E.L23 = -qf * bet3;
  E.L24 = na * alpha_s * di;  E.L25 = -af_prime * bet2; E.L26 = -af_prime * bet3;
  E.L34 = -1.0 / asq;
}

// a = L * v for the primitive eigensystem, terms in the reference's column
// order (src/lr_states_plm.c:122-133), exact zeros skipped.
template <class T>
ATHB_HD void prim_project(const PrimEigT<T>& E, const T v[7], T a[7]) {
  const T p01 = E.L01 * v[1], p02 = E.L02 * v[2], p03 = E.L03 * v[3];
  const T p04 = E.L04 * v[4], p05 = E.L05 * v[5], p06 = E.L06 * v[6];
  a[0] = p01 + p02 + p03 + p04 + p05 + p06;
  a[6] = -p01 - p02 - p03 + p04 + p05 + p06;
  const T p12 = E.L12 * v[2], p13 = E.L13 * v[3], p15 = E.L15 * v[5], p16 = E.L16 * v[6];
  a[1] = p12 + p13 + p15 + p16;
  a[5] = -p12 - p13 + p15 + p16;
  const T p21 = E.L21 * v[1], p22 = E.L22 * v[2], p23 = E.L23 * v[3];
  const T p24 = E.L24 * v[4], p25 = E.L25 * v[5], p26 = E.L26 * v[6];
  a[2] = p21 + p22 + p23 + p24 + p25 + p26;
  a[4] = -p21 - p22 - p23 + p24 + p25 + p26;
  a[3] = v[0] + E.L34 * v[4];
}

// One left eigenvector of the primitive system, as 7 coefficients (for the
// characteristic tracing loop, src/lr_states_plm.c:201-224).
template <class T>
ATHB_HD void prim_left_row(const PrimEigT<T>& E, int n, T l[7]) {
  for (int m = 0; m < 7; m++) l[m] = 0.0;
  switch (n) {
  case 0: l[1] = E.L01; l[2] = E.L02; l[3] = E.L03; l[4] = E.L04; l[5] = E.L05; l[6] = E.L06; break;
  case 1: l[2] = E.L12; l[3] = E.L13; l[5] = E.L15; l[6] = E.L16; break;
  case 2: l[1] = E.L21; l[2] = E.L22; l[3] = E.L23; l[4] = E.L24; l[5] = E.L25; l[6] = E.L26; break;
  case 3: l[0] = 1.0; l[4] = E.L34; break;
  case 4: l[1] = -E.L21; l[2] = -E.L22; l[3] = -E.L23; l[4] = E.L24; l[5] = E.L25; l[6] = E.L26; break;
  case 5: l[2] = -E.L12; l[3] = -E.L13; l[5] = E.L15; l[6] = E.L16; break;
  default: l[1] = -E.L01; l[2] = -E.L02; l[3] = -E.L03; l[4] = E.L04; l[5] = E.L05; l[6] = E.L06; break;
  }
}

// One right eigenvector (column n) of the primitive system.
template <class T>
ATHB_HD void prim_right_col(const PrimEigT<T>& E, int n, T r[7]) {
  switch (n) {
  case 0: r[0] = E.R00; r[1] = E.R10;  r[2] = E.R20;  r[3] = E.R30;  r[4] = E.R40; r[5] = E.R50; r[6] = E.R60; break;
  case 1: r[0] = 0.0;   r[1] = 0.0;    r[2] = E.R21;  r[3] = E.R31;  r[4] = 0.0;   r[5] = E.R51; r[6] = E.R61; break;
  case 2: r[0] = E.R02; r[1] = E.R12;  r[2] = E.R22;  r[3] = E.R32;  r[4] = E.R42; r[5] = E.R52; r[6] = E.R62; break;
  case 3: r[0] = 1.0;   r[1] = 0.0;    r[2] = 0.0;    r[3] = 0.0;    r[4] = 0.0;   r[5] = 0.0;   r[6] = 0.0;   break;
  case 4: r[0] = E.R02; r[1] = -E.R12; r[2] = -E.R22; r[3] = -E.R32; r[4] = E.R42; r[5] = E.R52; r[6] = E.R62; break;
  case 5: r[0] = 0.0;   r[1] = 0.0;    r[2] = -E.R21; r[3] = -E.R31; r[4] = 0.0;   r[5] = E.R51; r[6] = E.R61; break;
  default: r[0] = E.R00; r[1] = -E.R10; r[2] = -E.R20; r[3] = -E.R30; r[4] = E.R40; r[5] = E.R50; r[6] = E.R60; break;
  }
}

// Structural non-zero masks of the primitive eigenmatrices (bit m of row n).
// Used to skip exact-zero products; constant-folded after unrolling.
ATHB_HD int prim_left_mask(int n) {
  return n == 3 ? 0x11 : (n == 1 || n == 5) ? 0x6C : 0x7E;
}
ATHB_HD int prim_right_mask(int n) {  // column n
  return n == 3 ? 0x01 : (n == 1 || n == 5) ? 0x6C : 0x7F;
}

// ---------------------------------------------------------------------------
// Characteristic PLM for one cell (src/lr_states_plm.c:95-233).
//   wm, w0, wp : primitive states of cells i-1, i, i+1
//   bxc        : cell-centred normal field of cell i
// Returns wl_next = W_L at face i+1/2 (reference Wl[i+1]) and
//         wr_this = W_R at face i-1/2 (reference Wr[i]).
// ---------------------------------------------------------------------------
template <class T>
ATHB_HD void plm_cell(const Prim1T<T>& wm, const Prim1T<T>& w0, const Prim1T<T>& wp, T bxc,
                      T dtodx, const Eos& eos, Prim1T<T>& wl_next, Prim1T<T>& wr_this) {
  PrimEigT<T> E;
  esys_prim(w0.d, w0.vx, w0.p, bxc, w0.by, w0.bz, eos, E);

  const T Wm[7] = {wm.d, wm.vx, wm.vy, wm.vz, wm.p, wm.by, wm.bz};
  const T W0[7] = {w0.d, w0.vx, w0.vy, w0.vz, w0.p, w0.by, w0.bz};
  const T Wp[7] = {wp.d, wp.vx, wp.vy, wp.vz, wp.p, wp.by, wp.bz};

  // Step 2: centred, left, right and van Leer differences.
  T dWc[7], dWl[7], dWr[7], dWg[7];
#pragma unroll
  for (int n = 0; n < 7; n++) {
    dWc[n] = Wp[n] - Wm[n];
    dWl[n] = W0[n] - Wm[n];
    dWr[n] = Wp[n] - W0[n];
    if (dWl[n] * dWr[n] > 0.0) dWg[n] = 2.0 * dWl[n] * dWr[n] / (dWl[n] + dWr[n]);
    else dWg[n] = 0.0;
  }

  // Step 3: characteristic projections.
  T dac[7], dal[7], dar[7], dag[7];
  prim_project(E, dWc, dac);
  prim_project(E, dWl, dal);
  prim_project(E, dWr, dar);
  prim_project(E, dWg, dag);

  // Step 4: monotonicity constraints.
  T da[7];
#pragma unroll
  for (int n = 0; n < 7; n++) {
    da[n] = 0.0;
    if (dal[n] * dar[n] > 0.0) {
      const T lim_slope1 = rmin(fabs(dal[n]), fabs(dar[n]));
      const T lim_slope2 = rmin(0.5 * fabs(dac[n]), fabs(dag[n]));
      da[n] = rsign(dac[n]) * rmin(2.0 * lim_slope1, lim_slope2);
    }
  }

  // Step 5: back to primitive slopes, dWm[n] = sum_m da[m]*R[n][m].
  T dWm[7];
  dWm[0] = da[0] * E.R00 + da[2] * E.R02 + da[3] + da[4] * E.R02 + da[6] * E.R00;
  dWm[1] = da[0] * E.R10 + da[2] * E.R12 + da[4] * -E.R12 + da[6] * -E.R10;
  dWm[2] = da[0] * E.R20 + da[1] * E.R21 + da[2] * E.R22 + da[4] * -E.R22 + da[5] * -E.R21 + da[6] * -E.R20;
  dWm[3] = da[0] * E.R30 + da[1] * E.R31 + da[2] * E.R32 + da[4] * -E.R32 + da[5] * -E.R31 + da[6] * -E.R30;
  dWm[4] = da[0] * E.R40 + da[2] * E.R42 + da[4] * E.R42 + da[6] * E.R40;
  dWm[5] = da[0] * E.R50 + da[1] * E.R51 + da[2] * E.R52 + da[4] * E.R52 + da[5] * E.R51 + da[6] * E.R50;
  dWm[6] = da[0] * E.R60 + da[1] * E.R61 + da[2] * E.R62 + da[4] * E.R62 + da[5] * E.R61 + da[6] * E.R60;

  // Step 7: L/R values, bounded by the neighbouring cell centres.
  T Wlv[7], Wrv[7], dW[7];
#pragma unroll
  for (int n = 0; n < 7; n++) {
    T l = W0[n] - 0.5 * dWm[n];
    T r = W0[n] + 0.5 * dWm[n];
    l = rmax(rmin(W0[n], Wm[n]), l);
    l = rmin(rmax(W0[n], Wm[n]), l);
    r = rmax(rmin(W0[n], Wp[n]), r);
    r = rmin(rmax(W0[n], Wp[n]), r);
    Wlv[n] = l;
    Wrv[n] = r;
    dW[n] = r - l;
  }

  // Step 8: integrate over the domain of dependence of the extreme waves.
  T pWl[7], pWr[7];
  {
    const T qx = 0.5 * rmax(E.ev[6], T(0.0)) * dtodx;
#pragma unroll
    for (int n = 0; n < 7; n++) pWl[n] = Wrv[n] - qx * dW[n];
    const T qy = -0.5 * rmin(E.ev[0], T(0.0)) * dtodx;
#pragma unroll
    for (int n = 0; n < 7; n++) pWr[n] = Wlv[n] + qy * dW[n];
  }

  // Step 9: subtract the waves that do not reach the interface.  Wave 6 in the
  // first loop and wave 0's first part in the second contribute (ev-ev)=0
  // multiples of exact-zero size and are skipped.
#pragma unroll
  for (int n = 0; n < 6; n++) {
    if (E.ev[n] > 0.) {
      T l[7], r[7];
      prim_left_row(E, n, l);
      const T dev = E.ev[6] - E.ev[n];
      T qa = T(0.0);
      bool first = true;
#pragma unroll
      for (int m = 0; m < 7; m++) {
        if (!((prim_left_mask(n) >> m) & 1)) continue;
        const T t = l[m] * 0.5 * dtodx * dev * dW[m];
        qa = first ? t : qa + t;
        first = false;
      }
      prim_right_col(E, n, r);
#pragma unroll
      for (int m = 0; m < 7; m++)
        if ((prim_right_mask(n) >> m) & 1) pWl[m] += qa * r[m];
    }
  }
#pragma unroll
  for (int n = 0; n < 7; n++) {
    if (E.ev[n] < 0.) {
      T l[7], r[7], h[7];
      prim_left_row(E, n, l);
      prim_right_col(E, n, r);
#pragma unroll
      for (int m = 0; m < 7; m++) h[m] = l[m] * 0.5 * dtodx;
      if (n != 0) {
        const T dev = E.ev[0] - E.ev[n];
        T qa = T(0.0);
        bool first = true;
#pragma unroll
        for (int m = 0; m < 7; m++) {
          if (!((prim_left_mask(n) >> m) & 1)) continue;
          const T t = h[m] * dev * dW[m];
          qa = first ? t : qa + t;
          first = false;
        }
#pragma unroll
        for (int m = 0; m < 7; m++)
          if ((prim_right_mask(n) >> m) & 1) pWr[m] += qa * r[m];
      }
      {
        const T dev = E.ev[n] - E.ev[6];
        T qa = T(0.0);
        bool first = true;
#pragma unroll
        for (int m = 0; m < 7; m++) {
          if (!((prim_left_mask(n) >> m) & 1)) continue;
          const T t = h[m] * dev * dW[m];
          qa = first ? t : qa + t;
          first = false;
        }
#pragma unroll
        for (int m = 0; m < 7; m++)
          if ((prim_right_mask(n) >> m) & 1) pWl[m] -= qa * r[m];
      }
    }
  }

  wl_next.d = pWl[0]; wl_next.vx = pWl[1]; wl_next.vy = pWl[2]; wl_next.vz = pWl[3];
  wl_next.p = pWl[4]; wl_next.by = pWl[5]; wl_next.bz = pWl[6];
  wr_this.d = pWr[0]; wr_this.vx = pWr[1]; wr_this.vy = pWr[2]; wr_this.vz = pWr[3];
  wr_this.p = pWr[4]; wr_this.by = pWr[5]; wr_this.bz = pWr[6];
}

// ---------------------------------------------------------------------------
// Roe-averaged state shared by the Roe and HLLE solvers
// (src/flux_roe.c:91-114, src/flux_hlle.c:87-110).
// ---------------------------------------------------------------------------
template <class T> struct RoeAvgT {
  T sqrtdl, sqrtdr, isdlpdr, droe, v1, v2, v3, b2, b3, x, y, pbl, pbr, h;
};
using RoeAvg = RoeAvgT<double>;

template <class T>
ATHB_HD RoeAvgT<T> roe_average(const Cons1T<T>& Ul, const Cons1T<T>& Ur, const Prim1T<T>& Wl, const Prim1T<T>& Wr,
                           T Bxi) {
  RoeAvgT<T> r;
  r.sqrtdl = sqrt(Wl.d);
  r.sqrtdr = sqrt(Wr.d);
  r.isdlpdr = 1.0 / (r.sqrtdl + r.sqrtdr);
  r.droe = r.sqrtdl * r.sqrtdr;
  r.v1 = (r.sqrtdl * Wl.vx + r.sqrtdr * Wr.vx) * r.isdlpdr;
  r.v2 = (r.sqrtdl * Wl.vy + r.sqrtdr * Wr.vy) * r.isdlpdr;
  r.v3 = (r.sqrtdl * Wl.vz + r.sqrtdr * Wr.vz) * r.isdlpdr;
  r.b2 = (r.sqrtdr * Wl.by + r.sqrtdl * Wr.by) * r.isdlpdr;
  r.b3 = (r.sqrtdr * Wl.bz + r.sqrtdl * Wr.bz) * r.isdlpdr;
  const T dby = Wl.by - Wr.by, dbz = Wl.bz - Wr.bz, ss = r.sqrtdl + r.sqrtdr;
  r.x = 0.5 * (dby * dby + dbz * dbz) / (ss * ss);
  r.y = 0.5 * (Wl.d + Wr.d) / r.droe;
  r.pbl = 0.5 * (Bxi * Bxi + Wl.by * Wl.by + Wl.bz * Wl.bz);
  r.pbr = 0.5 * (Bxi * Bxi + Wr.by * Wr.by + Wr.bz * Wr.bz);
  r.h = ((Ul.e + Wl.p + r.pbl) / r.sqrtdl + (Ur.e + Wr.p + r.pbr) / r.sqrtdr) * r.isdlpdr;
  return r;
}

// Roe-matrix wave speeds (src/esystem_roe.c:68-87,136-144).
template <class T> struct RoeSpeedsT {
  T di, vsq, btsq, bt_starsq, vaxsq, hp, twid_asq, cfsq, cf, cssq, cs, vax, gfac;
};
using RoeSpeeds = RoeSpeedsT<double>;

template <class T>
ATHB_HD RoeSpeedsT<T> roe_speeds(const RoeAvgT<T>& r, T b1, const Eos& eos) {
  RoeSpeedsT<T> s;
  s.di = 1.0 / r.droe;
  s.vsq = r.v1 * r.v1 + r.v2 * r.v2 + r.v3 * r.v3;
  s.btsq = r.b2 * r.b2 + r.b3 * r.b3;
  s.gfac = eos.gamma_1 - eos.gamma_2 * r.y;
  s.bt_starsq = s.gfac * s.btsq;
  s.vaxsq = b1 * b1 * s.di;
  s.hp = r.h - (s.vaxsq + s.btsq * s.di);
  s.twid_asq = rmax((eos.gamma_1 * (s.hp - 0.5 * s.vsq) - eos.gamma_2 * r.x), T(kTiny));
  const T ct2 = s.bt_starsq * s.di;
  const T tsum = s.vaxsq + ct2 + s.twid_asq;
  const T tdif = s.vaxsq + ct2 - s.twid_asq;
  const T cf2_cs2 = sqrt(tdif * tdif + 4.0 * s.twid_asq * ct2);
  s.cfsq = 0.5 * (tsum + cf2_cs2);
  s.cf = sqrt(s.cfsq);
  s.cssq = s.twid_asq * s.vaxsq / s.cfsq;
  s.cs = sqrt(s.cssq);
  s.vax = sqrt(s.vaxsq);
  return s;
}

// Roe eigenvectors (src/esystem_roe.c:91-291), kept as the scalars the 7x7
// matrices are built from.  Rows of L and columns of R are formed one at a
// time where they are consumed, so no matrix is ever live in registers.
//   R columns (n-th right eigenvector), rows 0..6:
//     c0 = (af, af*ev0, af*v2+qs*b2*, af*v3+qs*b3*, R40, as'*b2*, as'*b3*)
//     c1 = (0, 0, -b3, b2, R41, -b3*s*isd, b2*s*isd)
//     c2 = (as, as*ev2, as*v2-qf*b2*, as*v3-qf*b3*, R42, -af'*b2*, -af'*b3*)
//     c3 = (1, v1, v2, v3, R43, 0, 0)
//     c4 = (as, as*ev4, as*v2+qf*b2*, as*v3+qf*b3*, R44, -af'*b2*, -af'*b3*)
//     c5 = (0, 0, b3, -b2, -R41, -b3*s*isd, b2*s*isd)
//     c6 = (af, af*ev6, af*v2-qs*b2*, af*v3-qs*b3*, R46, as'*b2*, as'*b3*)
//   L rows: row 5 = (-L10, 0, -L12, -L13, 0, L15, L16) of row 1; rows 2/4 and
//   0/6 share their last three entries.
template <class T> struct RoeScalT {
  T v1, v2, v3, b2, b3, vsq, hp, cf, cs;
  T af, as, qf, qs;            // alpha_f, alpha_s, qf, qs (right vectors)
  T bet2, bet3, bet2s, bet3s, vbet, aspbb, afpbb, sgn, isqrtd, sqrtd, asp, afp, gx;
  T afn, asn, cff, css, qfn, qsn, Afn, Asn, afpb, aspb, q2s, q3s, vqstr, norm2;  // left vectors
};
using RoeScal = RoeScalT<double>;

template <class T>
ATHB_HD void roe_scalars(const RoeAvgT<T>& r, const RoeSpeedsT<T>& s, T b1, const Eos& eos, RoeScalT<T>& S) {
  const T v2 = r.v2, v3 = r.v3, b2 = r.b2, b3 = r.b3, d = r.droe;
  S.v1 = r.v1; S.v2 = v2; S.v3 = v3; S.b2 = b2; S.b3 = b3;
  S.vsq = s.vsq; S.hp = s.hp; S.cf = s.cf; S.cs = s.cs;
  const T bt = sqrt(s.btsq);
  const T bt_star = sqrt(s.bt_starsq);
  T bet2, bet3;
  if (bt == 0.0) { bet2 = 1.0; bet3 = 0.0; } else { bet2 = b2 / bt; bet3 = b3 / bt; }
  freeze_beta(bet2, bet3, value_of(s.btsq), value_of(b1) * value_of(b1) + value_of(d) * value_of(s.twid_asq));
  const T sg = sqrt(s.gfac);
  const T bet2_star = bet2 / sg;
  const T bet3_star = bet3 / sg;
  const T bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
  S.bet2 = bet2; S.bet3 = bet3; S.bet2s = bet2_star; S.bet3s = bet3_star;
  S.vbet = v2 * bet2_star + v3 * bet3_star;

  T alpha_f, alpha_s;
  if ((s.cfsq - s.cssq) == 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
  else if ((s.twid_asq - s.cssq) <= 0.0) { alpha_f = 0.0; alpha_s = 1.0; }
  else if ((s.cfsq - s.twid_asq) <= 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
  else {
    alpha_f = sqrt((s.twid_asq - s.cssq) / (s.cfsq - s.cssq));
    alpha_s = sqrt((s.cfsq - s.twid_asq) / (s.cfsq - s.cssq));
  }
  const T sqrtd = sqrt(d);
  const T isqrtd = 1.0 / sqrtd;
  const T sgn = rsign(b1);
  const T twid_a = sqrt(s.twid_asq);
  const T qf = s.cf * alpha_f * sgn;
  const T qs = s.cs * alpha_s * sgn;
  const T af_prime = twid_a * alpha_f * isqrtd;
  const T as_prime = twid_a * alpha_s * isqrtd;
  S.af = alpha_f; S.as = alpha_s; S.qf = qf; S.qs = qs;
  S.afpbb = af_prime * bt_star * bet_starsq;
  S.aspbb = as_prime * bt_star * bet_starsq;
  S.sgn = sgn; S.isqrtd = isqrtd; S.sqrtd = sqrtd; S.asp = as_prime; S.afp = af_prime;
  S.gx = eos.gamma_2 * r.x / eos.gamma_1;

  T norm = 0.5 / s.twid_asq;
  S.cff = norm * alpha_f * s.cf;
  S.css = norm * alpha_s * s.cs;
  S.qfn = qf * norm;
  S.qsn = qs * norm;
  S.Afn = norm * af_prime * d;
  S.Asn = norm * as_prime * d;
  S.afpb = norm * af_prime * bt_star;
  S.aspb = norm * as_prime * bt_star;
  norm *= eos.gamma_1;
  S.afn = alpha_f * norm;
  S.asn = alpha_s * norm;
  S.q2s = bet2_star / bet_starsq;
  S.q3s = bet3_star / bet_starsq;
  S.vqstr = (v2 * S.q2s + v3 * S.q3s);
  S.norm2 = norm * 2.0;
}

// Column n of the Roe right-eigenmatrix.
template <class T>
ATHB_HD void roe_right_col(const RoeScalT<T>& S, const T ev[7], int n, T c[7]) {
  switch (n) {
  case 0:
    c[0] = S.af; c[1] = S.af * ev[0]; c[2] = S.af * S.v2 + S.qs * S.bet2s; c[3] = S.af * S.v3 + S.qs * S.bet3s;
    c[4] = S.af * (S.hp - S.v1 * S.cf) + S.qs * S.vbet + S.aspbb;
    c[5] = S.asp * S.bet2s; c[6] = S.asp * S.bet3s; break;
  case 1:
    c[0] = 0.0; c[1] = 0.0; c[2] = -S.bet3; c[3] = S.bet2; c[4] = -(S.v2 * S.bet3 - S.v3 * S.bet2);
    c[5] = -S.bet3 * S.sgn * S.isqrtd; c[6] = S.bet2 * S.sgn * S.isqrtd; break;
  case 2:
    c[0] = S.as; c[1] = S.as * ev[2]; c[2] = S.as * S.v2 - S.qf * S.bet2s; c[3] = S.as * S.v3 - S.qf * S.bet3s;
    c[4] = S.as * (S.hp - S.v1 * S.cs) - S.qf * S.vbet - S.afpbb;
    c[5] = -S.afp * S.bet2s; c[6] = -S.afp * S.bet3s; break;
  case 3:
    c[0] = 1.0; c[1] = S.v1; c[2] = S.v2; c[3] = S.v3; c[4] = 0.5 * S.vsq + S.gx; c[5] = 0.0; c[6] = 0.0; break;
  case 4:
    c[0] = S.as; c[1] = S.as * ev[4]; c[2] = S.as * S.v2 + S.qf * S.bet2s; c[3] = S.as * S.v3 + S.qf * S.bet3s;
    c[4] = S.as * (S.hp + S.v1 * S.cs) + S.qf * S.vbet - S.afpbb;
    c[5] = -S.afp * S.bet2s; c[6] = -S.afp * S.bet3s; break;
  case 5:
    c[0] = 0.0; c[1] = 0.0; c[2] = S.bet3; c[3] = -S.bet2; c[4] = (S.v2 * S.bet3 - S.v3 * S.bet2);
    c[5] = -S.bet3 * S.sgn * S.isqrtd; c[6] = S.bet2 * S.sgn * S.isqrtd; break;
  default:
    c[0] = S.af; c[1] = S.af * ev[6]; c[2] = S.af * S.v2 - S.qs * S.bet2s; c[3] = S.af * S.v3 - S.qs * S.bet3s;
    c[4] = S.af * (S.hp + S.v1 * S.cf) - S.qs * S.vbet + S.aspbb;
    c[5] = S.asp * S.bet2s; c[6] = S.asp * S.bet3s; break;
  }
}
ATHB_HD int roe_right_mask(int n) {  // structural non-zeros of column n
  return (n == 1 || n == 5) ? 0x7C : (n == 3) ? 0x1F : 0x7F;
}

// a = L * dU (src/flux_roe.c:200-204), terms in column order, zeros skipped,
// rows formed in pairs that share entries.
template <class T>
ATHB_HD void roe_project(const RoeScalT<T>& S, const T u[7], T a[7]) {
  const T vh = S.vsq - S.hp;
  {  // rows 0 and 6
    const T p4 = S.afn * u[4];
    const T p5 = (S.Asn * S.q2s - S.afn * S.b2) * u[5];
    const T p6 = (S.Asn * S.q3s - S.afn * S.b3) * u[6];
    a[0] = (S.afn * vh + S.cff * (S.cf + S.v1) - S.qsn * S.vqstr - S.aspb) * u[0] +
           (-S.afn * S.v1 - S.cff) * u[1] + (-S.afn * S.v2 + S.qsn * S.q2s) * u[2] +
           (-S.afn * S.v3 + S.qsn * S.q3s) * u[3] + p4 + p5 + p6;
    a[6] = (S.afn * vh + S.cff * (S.cf - S.v1) + S.qsn * S.vqstr - S.aspb) * u[0] +
           (-S.afn * S.v1 + S.cff) * u[1] + (-S.afn * S.v2 - S.qsn * S.q2s) * u[2] +
           (-S.afn * S.v3 - S.qsn * S.q3s) * u[3] + p4 + p5 + p6;
  }
  {  // rows 1 and 5
    const T p0 = (0.5 * (S.v2 * S.bet3 - S.v3 * S.bet2)) * u[0];
    const T p2 = (-0.5 * S.bet3) * u[2];
    const T p3 = (0.5 * S.bet2) * u[3];
    const T p5 = (-0.5 * S.sqrtd * S.bet3 * S.sgn) * u[5];
    const T p6 = (0.5 * S.sqrtd * S.bet2 * S.sgn) * u[6];
    a[1] = p0 + p2 + p3 + p5 + p6;
    a[5] = -p0 - p2 - p3 + p5 + p6;
  }
  {  // rows 2 and 4
    const T p4 = S.asn * u[4];
    const T p5 = (-S.Afn * S.q2s - S.asn * S.b2) * u[5];
    const T p6 = (-S.Afn * S.q3s - S.asn * S.b3) * u[6];
    a[2] = (S.asn * vh + S.css * (S.cs + S.v1) + S.qfn * S.vqstr + S.afpb) * u[0] +
           (-S.asn * S.v1 - S.css) * u[1] + (-S.asn * S.v2 - S.qfn * S.q2s) * u[2] +
           (-S.asn * S.v3 - S.qfn * S.q3s) * u[3] + p4 + p5 + p6;
    a[4] = (S.asn * vh + S.css * (S.cs - S.v1) - S.qfn * S.vqstr + S.afpb) * u[0] +
           (-S.asn * S.v1 + S.css) * u[1] + (-S.asn * S.v2 + S.qfn * S.q2s) * u[2] +
           (-S.asn * S.v3 + S.qfn * S.q3s) * u[3] + p4 + p5 + p6;
  }
  {  // row 3
    a[3] = (1.0 - S.norm2 * (0.5 * S.vsq - S.gx)) * u[0] + (S.norm2 * S.v1) * u[1] + (S.norm2 * S.v2) * u[2] +
           (S.norm2 * S.v3) * u[3] + (-S.norm2) * u[4] + (S.norm2 * S.b2) * u[5] + (S.norm2 * S.b3) * u[6];
  }
}

// Physical flux of one side (src/flux_roe.c:136-172).
template <class T>
ATHB_HD Cons1T<T> side_flux(const Cons1T<T>& U, const Prim1T<T>& W, T Bxi, T pb) {
  Cons1T<T> F;
  F.d = U.mx;
  F.mx = U.mx * W.vx;
  F.my = U.mx * W.vy;
  F.mz = U.mx * W.vz;
  F.mx += W.p;
  F.e = (U.e + W.p) * W.vx;
  F.mx -= 0.5 * (Bxi * Bxi - W.by * W.by - W.bz * W.bz);
  F.my -= Bxi * W.by;
  F.mz -= Bxi * W.bz;
  F.e += (pb * W.vx - Bxi * (Bxi * W.vx + W.by * W.vy + W.bz * W.vz));
  F.by = W.by * W.vx - Bxi * W.vy;
  F.bz = W.bz * W.vx - Bxi * W.vz;
  return F;
}

// --- src/flux_hlle.c:60-199 ---------------------------------------------------
template <class T>
ATHB_HD Cons1T<T> flux_hlle(const Cons1T<T>& Ul, const Cons1T<T>& Ur, const Prim1T<T>& Wl, const Prim1T<T>& Wr,
                        T Bxi, const Eos& eos) {
  const RoeAvgT<T> r = roe_average(Ul, Ur, Wl, Wr, Bxi);
  const RoeSpeedsT<T> s = roe_speeds(r, Bxi, eos);
  const T ev0 = r.v1 - s.cf, ev6 = r.v1 + s.cf;

  T asq = eos.gamma * Wl.p / Wl.d;
  T vaxsq = Bxi * Bxi / Wl.d;
  T ct2 = (Ul.by * Ul.by + Ul.bz * Ul.bz) / Wl.d;
  T qsq = vaxsq + ct2 + asq;
  T tmp = vaxsq + ct2 - asq;
  T cfsq = 0.5 * (qsq + sqrt(tmp * tmp + 4.0 * asq * ct2));
  const T cfl = sqrt(cfsq);

  asq = eos.gamma * Wr.p / Wr.d;
  vaxsq = Bxi * Bxi / Wr.d;
  ct2 = (Ur.by * Ur.by + Ur.bz * Ur.bz) / Wr.d;
  qsq = vaxsq + ct2 + asq;
  tmp = vaxsq + ct2 - asq;
  cfsq = 0.5 * (qsq + sqrt(tmp * tmp + 4.0 * asq * ct2));
  const T cfr = sqrt(cfsq);

  const T ar = rmax(ev6, (Wr.vx + cfr));
  const T al = rmin(ev0, (Wl.vx - cfl));
  const T bp = rmax(ar, T(0.0));
  const T bm = rmin(al, T(0.0));

  Cons1T<T> Fl, Fr;
  Fl.d = Ul.mx - bm * Ul.d;
  Fr.d = Ur.mx - bp * Ur.d;
  Fl.mx = Ul.mx * (Wl.vx - bm);
  Fr.mx = Ur.mx * (Wr.vx - bp);
  Fl.my = Ul.my * (Wl.vx - bm);
  Fr.my = Ur.my * (Wr.vx - bp);
  Fl.mz = Ul.mz * (Wl.vx - bm);
  Fr.mz = Ur.mz * (Wr.vx - bp);
  Fl.mx += Wl.p;
  Fr.mx += Wr.p;
  Fl.e = Ul.e * (Wl.vx - bm) + Wl.p * Wl.vx;
  Fr.e = Ur.e * (Wr.vx - bp) + Wr.p * Wr.vx;
  Fl.mx -= 0.5 * (Bxi * Bxi - Wl.by * Wl.by - Wl.bz * Wl.bz);
  Fr.mx -= 0.5 * (Bxi * Bxi - Wr.by * Wr.by - Wr.bz * Wr.bz);
  Fl.my -= Bxi * Wl.by;
  Fr.my -= Bxi * Wr.by;
  Fl.mz -= Bxi * Wl.bz;
  Fr.mz -= Bxi * Wr.bz;
  Fl.e += (r.pbl * Wl.vx - Bxi * (Bxi * Wl.vx + Wl.by * Wl.vy + Wl.bz * Wl.vz));
  Fr.e += (r.pbr * Wr.vx - Bxi * (Bxi * Wr.vx + Wr.by * Wr.vy + Wr.bz * Wr.vz));
  Fl.by = Wl.by * (Wl.vx - bm) - Bxi * Wl.vy;
  Fr.by = Wr.by * (Wr.vx - bp) - Bxi * Wr.vy;
  Fl.bz = Wl.bz * (Wl.vx - bm) - Bxi * Wl.vz;
  Fr.bz = Wr.bz * (Wr.vx - bp) - Bxi * Wr.vz;

  const T t = 0.5 * (bp + bm) / (bp - bm);
  Cons1T<T> F;
  F.d = 0.5 * (Fl.d + Fr.d) + (Fl.d - Fr.d) * t;
  F.mx = 0.5 * (Fl.mx + Fr.mx) + (Fl.mx - Fr.mx) * t;
  F.my = 0.5 * (Fl.my + Fr.my) + (Fl.my - Fr.my) * t;
  F.mz = 0.5 * (Fl.mz + Fr.mz) + (Fl.mz - Fr.mz) * t;
  F.e = 0.5 * (Fl.e + Fr.e) + (Fl.e - Fr.e) * t;
  F.by = 0.5 * (Fl.by + Fr.by) + (Fl.by - Fr.by) * t;
  F.bz = 0.5 * (Fl.bz + Fr.bz) + (Fl.bz - Fr.bz) * t;
  return F;
}

// --- src/flux_roe.c:54-259 ----------------------------------------------------
template <class T>
ATHB_HD Cons1T<T> flux_roe(const Cons1T<T>& Ul, const Cons1T<T>& Ur, const Prim1T<T>& Wl, const Prim1T<T>& Wr,
                       T Bxi, const Eos& eos) {
  const RoeAvgT<T> r = roe_average(Ul, Ur, Wl, Wr, Bxi);
  const RoeSpeedsT<T> s = roe_speeds(r, Bxi, eos);
  T ev[7];
  ev[0] = r.v1 - s.cf; ev[1] = r.v1 - s.vax; ev[2] = r.v1 - s.cs; ev[3] = r.v1;
  ev[4] = r.v1 + s.cs; ev[5] = r.v1 + s.vax; ev[6] = r.v1 + s.cf;

  // Step 5: supersonic faces take the upwind flux.
  if (ev[0] >= 0.0) return side_flux(Ul, Wl, Bxi, r.pbl);
  if (ev[6] <= 0.0) return side_flux(Ur, Wr, Bxi, r.pbr);

  RoeScalT<T> S;
  roe_scalars(r, s, Bxi, eos, S);

  // Step 6: wave strengths.
  T a[7];
  {
    const T dU[7] = {Ur.d - Ul.d, Ur.mx - Ul.mx, Ur.my - Ul.my, Ur.mz - Ul.mz,
                          Ur.e - Ul.e, Ur.by - Ul.by, Ur.bz - Ul.bz};
    roe_project(S, dU, a);
  }
  // Step 8 starts from the mean of the side fluxes (src/flux_roe.c:252)
  T F[7];
  {
    const Cons1T<T> Fl = side_flux(Ul, Wl, Bxi, r.pbl);
    const Cons1T<T> Fr = side_flux(Ur, Wr, Bxi, r.pbr);
    F[0] = 0.5 * (Fl.d + Fr.d); F[1] = 0.5 * (Fl.mx + Fr.mx); F[2] = 0.5 * (Fl.my + Fr.my);
    F[3] = 0.5 * (Fl.mz + Fr.mz); F[4] = 0.5 * (Fl.e + Fr.e); F[5] = 0.5 * (Fl.by + Fr.by);
    F[6] = 0.5 * (Fl.bz + Fr.bz);
  }
  // Steps 7 and 8 fused over the right eigenvectors: the intermediate states
  // (positivity test, HLLE on failure) and the Roe flux subtract the same
  // column n; per component the flux terms keep the reference's order.
  T u[7] = {Ul.d, Ul.mx, Ul.my, Ul.mz, Ul.e, Ul.by, Ul.bz};
#pragma unroll
  for (int n = 0; n < 7; n++) {
    T c[7];
    roe_right_col(S, ev, n, c);
    if (n < 6) {
#pragma unroll
      for (int m = 0; m < 7; m++)
        if ((roe_right_mask(n) >> m) & 1) u[m] += a[n] * c[m];
      if (ev[n + 1] > ev[n]) {
        bool bad = (u[0] <= 0.0);
        if (!bad) {
          T p_inter = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
          p_inter -= 0.5 * (u[5] * u[5] + u[6] * u[6] + Bxi * Bxi);
          bad = (p_inter < 0.0);
        }
        if (bad) return flux_hlle(Ul, Ur, Wl, Wr, Bxi, eos);
      }
    }
    const T coeff = 0.5 * rmax(fabs(ev[n]), T(0.0)) * a[n];
#pragma unroll
    for (int k = 0; k < 7; k++)
      if ((roe_right_mask(n) >> k) & 1) F[k] -= coeff * c[k];
  }
  Cons1T<T> out;
  out.d = F[0]; out.mx = F[1]; out.my = F[2]; out.mz = F[3]; out.e = F[4]; out.by = F[5]; out.bz = F[6];
  return out;
}

// Flux selection: the reference always calls flux_roe (src/__integrate_2d__.c:178,
// 238,444,461); HLLE everywhere is the optional alternative.
enum FluxKind { kFluxRoe = 0, kFluxHlle = 1 };

template <int FLUX, class T>
ATHB_HD Cons1T<T> riemann(const Cons1T<T>& Ul, const Cons1T<T>& Ur, const Prim1T<T>& Wl, const Prim1T<T>& Wr,
                          T Bxi, const Eos& eos) {
  if (FLUX == kFluxHlle) return flux_hlle(Ul, Ur, Wl, Wr, Bxi, eos);
  return flux_roe(Ul, Ur, Wl, Wr, Bxi, eos);
}

}  // namespace athb
