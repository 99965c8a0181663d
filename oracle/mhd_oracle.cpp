// mhd_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's 2D adiabatic ideal-MHD step (the path
// integrate_2d -> new_dt -> set_bvals of awasiljew/athena-cuda), used as the
// parity oracle of the CUDA library and, instantiated with a counting scalar,
// to count the algorithmic FP64 operations of each stage.  It is written from
// the published algorithm (Stone et al. 2008, ApJS 178, 137, App. A/B;
// Gardiner & Stone 2005, JCP 205, 509) and keeps the reference's evaluation
// order in every expression so that its results are bit-identical; the
// eigenmatrices are formed densely (7x7) and every product is evaluated, as in
// the reference, so the operation counts are the reference's.
//
// Nothing here is used by the library; only tests/, smoke() and bench.py's
// CPU leg may load it.
//
// Reference functions restated (paths within the reference project):
//   src/convert_var.c:37-95          cons_to_prim / prim_to_cons
//   src/esystem_prim.c:36-235        eig_prim
//   src/lr_states_plm.c:64-248       plm_slice
//   src/esystem_roe.c:56-293         eig_roe
//   src/flux_roe.c:54-259            flux_roe
//   src/flux_hlle.c:60-199           flux_hlle
//   src/__integrate_2d__.c:100-537   Stepper::integrate
//   src/__integrate_2d__.c:632-702   Stepper::corner_emf
//   src/set_bvals.c:114-1031         Stepper::bvals
//   src/new_dt.c:25-100              Stepper::new_dt
//   src/main.c:221-318               oracle_run (main loop)
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// scalar types: plain double, or a counting wrapper
// ---------------------------------------------------------------------------
struct Counts {
  uint64_t add = 0, mul = 0, div = 0, sqrt = 0, neg = 0;
};
static Counts g_cnt;

struct Cnt {
  double v;
  Cnt() : v(0.0) {}
  Cnt(double x) : v(x) {}
  explicit operator double() const { return v; }
};
inline Cnt operator+(Cnt a, Cnt b) { g_cnt.add++; return Cnt(a.v + b.v); }
inline Cnt operator-(Cnt a, Cnt b) { g_cnt.add++; return Cnt(a.v - b.v); }
inline Cnt operator*(Cnt a, Cnt b) { g_cnt.mul++; return Cnt(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { g_cnt.div++; return Cnt(a.v / b.v); }
inline Cnt operator-(Cnt a) { g_cnt.neg++; return Cnt(-a.v); }
inline Cnt& operator+=(Cnt& a, Cnt b) { a = a + b; return a; }
inline Cnt& operator-=(Cnt& a, Cnt b) { a = a - b; return a; }
inline Cnt& operator*=(Cnt& a, Cnt b) { a = a * b; return a; }
inline bool operator<(Cnt a, Cnt b) { return a.v < b.v; }
inline bool operator>(Cnt a, Cnt b) { return a.v > b.v; }
inline bool operator<=(Cnt a, Cnt b) { return a.v <= b.v; }
inline bool operator>=(Cnt a, Cnt b) { return a.v >= b.v; }
inline bool operator==(Cnt a, Cnt b) { return a.v == b.v; }
inline Cnt sqrt(Cnt a) { g_cnt.sqrt++; return Cnt(std::sqrt(a.v)); }
inline Cnt fabs(Cnt a) { return Cnt(std::fabs(a.v)); }
inline double val(Cnt a) { return a.v; }
inline double val(double a) { return a; }
using std::fabs;
using std::sqrt;

template <class R> inline R MAXR(R a, R b) { return (a > b) ? a : b; }
template <class R> inline R MINR(R a, R b) { return (a < b) ? a : b; }
template <class R> inline R SIGNR(R a) { return (a < R(0.)) ? R(-1.) : R(1.); }
template <class R> inline R SQ(R x) { return x * x; }

constexpr int NW = 7;
constexpr int NG = 4;
constexpr double TINY = 1.0e-20;

template <class R> using Vec = std::array<R, NW>;
template <class R> using Mat = std::array<std::array<R, NW>, NW>;

// Slice vectors in the sweep frame: conserved (d, Mx, My, Mz, E, By, Bz),
// primitive (d, Vx, Vy, Vz, P, By, Bz).
enum { D = 0, VX = 1, VY = 2, VZ = 3, PE = 4, BY = 5, BZ = 6 };

template <class R> struct Eos { R gamma, g1, g2; };

// ---------------------------------------------------------------------------
// conversions (src/convert_var.c)
// ---------------------------------------------------------------------------
template <class R> Vec<R> cons_to_prim(const Vec<R>& u, R bx, const Eos<R>& e) {
  Vec<R> w;
  R di = R(1.0) / u[D];
  w[D] = u[D];
  w[VX] = u[VX] * di;
  w[VY] = u[VY] * di;
  w[VZ] = u[VZ] * di;
  w[PE] = u[PE] - R(0.5) * (SQ(u[VX]) + SQ(u[VY]) + SQ(u[VZ])) * di;
  w[PE] -= R(0.5) * (SQ(bx) + SQ(u[BY]) + SQ(u[BZ]));
  w[PE] *= e.g1;
  w[PE] = MAXR(w[PE], R(TINY));
  w[BY] = u[BY];
  w[BZ] = u[BZ];
  return w;
}

template <class R> Vec<R> prim_to_cons(const Vec<R>& w, R bx, const Eos<R>& e) {
  Vec<R> u;
  u[D] = w[D];
  u[VX] = w[D] * w[VX];
  u[VY] = w[D] * w[VY];
  u[VZ] = w[D] * w[VZ];
  u[PE] = w[PE] / e.g1 + R(0.5) * w[D] * (SQ(w[VX]) + SQ(w[VY]) + SQ(w[VZ]));
  u[PE] += R(0.5) * (SQ(bx) + SQ(w[BY]) + SQ(w[BZ]));
  u[BY] = w[BY];
  u[BZ] = w[BZ];
  return u;
}

// ---------------------------------------------------------------------------
// primitive eigensystem (src/esystem_prim.c; Athena paper eqs. A9-A18)
// ---------------------------------------------------------------------------
template <class R>
void eig_prim(R d, R v1, R p, R b1, R b2, R b3, const Eos<R>& e, Vec<R>& ev, Mat<R>& rem, Mat<R>& lem) {
  for (auto& row : rem) row.fill(R(0.0));
  for (auto& row : lem) row.fill(R(0.0));
  R di = R(1.0) / d;
  R btsq = b2 * b2 + b3 * b3;
  R vaxsq = b1 * b1 * di;
  R asq = e.gamma * p * di;
  R ct2 = btsq * di;
  R tsum = vaxsq + ct2 + asq;
  R tdif = vaxsq + ct2 - asq;
  R cf2_cs2 = sqrt(tdif * tdif + R(4.0) * asq * ct2);
  R cfsq = R(0.5) * (tsum + cf2_cs2);
  R cf = sqrt(cfsq);
  R cssq = asq * vaxsq / cfsq;
  R cs = sqrt(cssq);
  R bt = sqrt(btsq);
  R bet2, bet3;
  if (bt == R(0.0)) { bet2 = R(1.0); bet3 = R(0.0); } else { bet2 = b2 / bt; bet3 = b3 / bt; }
  R af, as;
  if (cf2_cs2 == R(0.0)) { af = R(1.0); as = R(0.0); }
  else if ((asq - cssq) <= R(0.0)) { af = R(0.0); as = R(1.0); }
  else if ((cfsq - asq) <= R(0.0)) { af = R(1.0); as = R(0.0); }
  else { af = sqrt((asq - cssq) / cf2_cs2); as = sqrt((cfsq - asq) / cf2_cs2); }
  R sqrtd = sqrt(d);
  R s = SIGNR(b1);
  R a = sqrt(asq);
  R qf = cf * af * s;
  R qs = cs * as * s;
  R Af = a * af * sqrtd;
  R As = a * as * sqrtd;
  R vax = sqrt(vaxsq);
  ev = {v1 - cf, v1 - vax, v1 - cs, v1, v1 + cs, v1 + vax, v1 + cf};

  rem[0][0] = d * af; rem[0][2] = d * as; rem[0][3] = R(1.0); rem[0][4] = rem[0][2]; rem[0][6] = rem[0][0];
  rem[1][0] = -cf * af; rem[1][2] = -cs * as; rem[1][4] = -rem[1][2]; rem[1][6] = -rem[1][0];
  rem[2][0] = qs * bet2; rem[2][1] = -bet3; rem[2][2] = -qf * bet2; rem[2][4] = -rem[2][2];
  rem[2][5] = bet3; rem[2][6] = -rem[2][0];
  rem[3][0] = qs * bet3; rem[3][1] = bet2; rem[3][2] = -qf * bet3; rem[3][4] = -rem[3][2];
  rem[3][5] = -bet2; rem[3][6] = -rem[3][0];
  rem[4][0] = d * asq * af; rem[4][2] = d * asq * as; rem[4][4] = rem[4][2]; rem[4][6] = rem[4][0];
  rem[5][0] = As * bet2; rem[5][1] = -bet3 * s * sqrtd; rem[5][2] = -Af * bet2; rem[5][4] = rem[5][2];
  rem[5][5] = rem[5][1]; rem[5][6] = rem[5][0];
  rem[6][0] = As * bet3; rem[6][1] = bet2 * s * sqrtd; rem[6][2] = -Af * bet3; rem[6][4] = rem[6][2];
  rem[6][5] = rem[6][1]; rem[6][6] = rem[6][0];

  R na = R(0.5) / asq;
  qf = na * qf;
  qs = na * qs;
  R afp = na * Af * di;
  R asp = na * As * di;
  lem[0][1] = -na * cf * af; lem[0][2] = qs * bet2; lem[0][3] = qs * bet3; lem[0][4] = na * af * di;
  lem[0][5] = asp * bet2; lem[0][6] = asp * bet3;
  lem[1][2] = R(-0.5) * bet3; lem[1][3] = R(0.5) * bet2;
  lem[1][5] = R(-0.5) * bet3 * s / sqrtd; lem[1][6] = R(0.5) * bet2 * s / sqrtd;
  lem[2][1] = -na * cs * as; lem[2][2] = -qf * bet2; lem[2][3] = -qf * bet3; lem[2][4] = na * as * di;
  lem[2][5] = -afp * bet2; lem[2][6] = -afp * bet3;
  lem[3][0] = R(1.0); lem[3][4] = R(-1.0) / asq;
  lem[4][1] = -lem[2][1]; lem[4][2] = -lem[2][2]; lem[4][3] = -lem[2][3];
  lem[4][4] = lem[2][4]; lem[4][5] = lem[2][5]; lem[4][6] = lem[2][6];
  lem[5][2] = -lem[1][2]; lem[5][3] = -lem[1][3]; lem[5][5] = lem[1][5]; lem[5][6] = lem[1][6];
  lem[6][1] = -lem[0][1]; lem[6][2] = -lem[0][2]; lem[6][3] = -lem[0][3];
  lem[6][4] = lem[0][4]; lem[6][5] = lem[0][5]; lem[6][6] = lem[0][6];
}

// ---------------------------------------------------------------------------
// characteristic PLM over one slice (src/lr_states_plm.c:64-248):
// cells i in [lo, hi]; writes wl[i+1] and wr[i].
// ---------------------------------------------------------------------------
template <class R>
void plm_slice(const std::vector<Vec<R>>& W, const std::vector<R>& Bxc, R dtodx, int lo, int hi,
               std::vector<Vec<R>>& wl, std::vector<Vec<R>>& wr, const Eos<R>& e) {
  Vec<R> ev;
  Mat<R> rem, lem;
  for (int i = lo; i <= hi; i++) {
    const Vec<R>&Wm = W[i - 1], &W0 = W[i], &Wp = W[i + 1];
    eig_prim(W0[D], W0[VX], W0[PE], Bxc[i], W0[BY], W0[BZ], e, ev, rem, lem);
    Vec<R> dWc, dWl, dWr, dWg;
    for (int n = 0; n < NW; n++) {
      dWc[n] = Wp[n] - Wm[n];
      dWl[n] = W0[n] - Wm[n];
      dWr[n] = Wp[n] - W0[n];
      if (dWl[n] * dWr[n] > R(0.0)) dWg[n] = R(2.0) * dWl[n] * dWr[n] / (dWl[n] + dWr[n]);
      else dWg[n] = R(0.0);
    }
    Vec<R> dac, dal, dar, dag;
    for (int n = 0; n < NW; n++) {
      dac[n] = lem[n][0] * dWc[0];
      dal[n] = lem[n][0] * dWl[0];
      dar[n] = lem[n][0] * dWr[0];
      dag[n] = lem[n][0] * dWg[0];
      for (int m = 1; m < NW; m++) {
        dac[n] += lem[n][m] * dWc[m];
        dal[n] += lem[n][m] * dWl[m];
        dar[n] += lem[n][m] * dWr[m];
        dag[n] += lem[n][m] * dWg[m];
      }
    }
    Vec<R> da;
    for (int n = 0; n < NW; n++) {
      da[n] = R(0.0);
      if (dal[n] * dar[n] > R(0.0)) {
        R l1 = MINR(fabs(dal[n]), fabs(dar[n]));
        R l2 = MINR(R(0.5) * fabs(dac[n]), fabs(dag[n]));
        da[n] = SIGNR(dac[n]) * MINR(R(2.0) * l1, l2);
      }
    }
    Vec<R> dWm;
    for (int n = 0; n < NW; n++) {
      dWm[n] = da[0] * rem[n][0];
      for (int m = 1; m < NW; m++) dWm[n] += da[m] * rem[n][m];
    }
    Vec<R> Wlv, Wrv, dW;
    for (int n = 0; n < NW; n++) {
      Wlv[n] = W0[n] - R(0.5) * dWm[n];
      Wrv[n] = W0[n] + R(0.5) * dWm[n];
    }
    for (int n = 0; n < NW; n++) {
      Wlv[n] = MAXR(MINR(W0[n], Wm[n]), Wlv[n]);
      Wlv[n] = MINR(MAXR(W0[n], Wm[n]), Wlv[n]);
      Wrv[n] = MAXR(MINR(W0[n], Wp[n]), Wrv[n]);
      Wrv[n] = MINR(MAXR(W0[n], Wp[n]), Wrv[n]);
    }
    for (int n = 0; n < NW; n++) dW[n] = Wrv[n] - Wlv[n];
    Vec<R>& pl = wl[i + 1];
    Vec<R>& pr = wr[i];
    R qx = R(0.5) * MAXR(ev[NW - 1], R(0.0)) * dtodx;
    for (int n = 0; n < NW; n++) pl[n] = Wrv[n] - qx * dW[n];
    qx = R(-0.5) * MINR(ev[0], R(0.0)) * dtodx;
    for (int n = 0; n < NW; n++) pr[n] = Wlv[n] + qx * dW[n];
    for (int n = 0; n < NW; n++) {
      if (ev[n] > R(0.)) {
        R qa = R(0.0);
        for (int m = 0; m < NW; m++) qa += lem[n][m] * R(0.5) * dtodx * (ev[NW - 1] - ev[n]) * dW[m];
        for (int m = 0; m < NW; m++) pl[m] += qa * rem[m][n];
      }
    }
    for (int n = 0; n < NW; n++) {
      if (ev[n] < R(0.)) {
        R qa = R(0.0);
        for (int m = 0; m < NW; m++) qa += lem[n][m] * R(0.5) * dtodx * (ev[0] - ev[n]) * dW[m];
        for (int m = 0; m < NW; m++) pr[m] += qa * rem[m][n];
        qa = R(0.0);
        for (int m = 0; m < NW; m++) qa += lem[n][m] * R(0.5) * dtodx * (ev[n] - ev[NW - 1]) * dW[m];
        for (int m = 0; m < NW; m++) pl[m] -= qa * rem[m][n];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Roe eigensystem (src/esystem_roe.c; Athena paper App. B)
// ---------------------------------------------------------------------------
template <class R>
void eig_roe(R d, R v1, R v2, R v3, R h, R b1, R b2, R b3, R x, R y, const Eos<R>& e, Vec<R>& ev,
             Mat<R>* remp, Mat<R>* lemp) {
  R di = R(1.0) / d;
  R vsq = v1 * v1 + v2 * v2 + v3 * v3;
  R btsq = b2 * b2 + b3 * b3;
  R bt_starsq = (e.g1 - e.g2 * y) * btsq;
  R vaxsq = b1 * b1 * di;
  R hp = h - (vaxsq + btsq * di);
  R twid_asq = MAXR((e.g1 * (hp - R(0.5) * vsq) - e.g2 * x), R(TINY));
  R ct2 = bt_starsq * di;
  R tsum = vaxsq + ct2 + twid_asq;
  R tdif = vaxsq + ct2 - twid_asq;
  R cf2_cs2 = sqrt(tdif * tdif + R(4.0) * twid_asq * ct2);
  R cfsq = R(0.5) * (tsum + cf2_cs2);
  R cf = sqrt(cfsq);
  R cssq = twid_asq * vaxsq / cfsq;
  R cs = sqrt(cssq);
  R bt = sqrt(btsq);
  R bt_star = sqrt(bt_starsq);
  R bet2, bet3;
  if (bt == R(0.0)) { bet2 = R(1.0); bet3 = R(0.0); } else { bet2 = b2 / bt; bet3 = b3 / bt; }
  R bet2_star = bet2 / sqrt(e.g1 - e.g2 * y);
  R bet3_star = bet3 / sqrt(e.g1 - e.g2 * y);
  R bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
  R vbet = v2 * bet2_star + v3 * bet3_star;
  R af, as;
  if ((cfsq - cssq) == R(0.0)) { af = R(1.0); as = R(0.0); }
  else if ((twid_asq - cssq) <= R(0.0)) { af = R(0.0); as = R(1.0); }
  else if ((cfsq - twid_asq) <= R(0.0)) { af = R(1.0); as = R(0.0); }
  else { af = sqrt((twid_asq - cssq) / (cfsq - cssq)); as = sqrt((cfsq - twid_asq) / (cfsq - cssq)); }
  R sqrtd = sqrt(d);
  R isqrtd = R(1.0) / sqrtd;
  R s = SIGNR(b1);
  R twid_a = sqrt(twid_asq);
  R qf = cf * af * s;
  R qs = cs * as * s;
  R afp = twid_a * af * isqrtd;
  R asp = twid_a * as * isqrtd;
  R afpbb = afp * bt_star * bet_starsq;
  R aspbb = asp * bt_star * bet_starsq;
  R vax = sqrt(vaxsq);
  ev = {v1 - cf, v1 - vax, v1 - cs, v1, v1 + cs, v1 + vax, v1 + cf};
  if (!remp || !lemp) return;
  Mat<R>& rem = *remp;
  Mat<R>& lem = *lemp;
  for (auto& row : rem) row.fill(R(0.0));
  for (auto& row : lem) row.fill(R(0.0));

  rem[0][0] = af; rem[0][2] = as; rem[0][3] = R(1.0); rem[0][4] = as; rem[0][6] = af;
  rem[1][0] = af * ev[0]; rem[1][2] = as * ev[2]; rem[1][3] = v1; rem[1][4] = as * ev[4]; rem[1][6] = af * ev[6];
  R qa = af * v2, qb = as * v2, qc = qs * bet2_star, qd = qf * bet2_star;
  rem[2][0] = qa + qc; rem[2][1] = -bet3; rem[2][2] = qb - qd; rem[2][3] = v2;
  rem[2][4] = qb + qd; rem[2][5] = bet3; rem[2][6] = qa - qc;
  qa = af * v3; qb = as * v3; qc = qs * bet3_star; qd = qf * bet3_star;
  rem[3][0] = qa + qc; rem[3][1] = bet2; rem[3][2] = qb - qd; rem[3][3] = v3;
  rem[3][4] = qb + qd; rem[3][5] = -bet2; rem[3][6] = qa - qc;
  rem[4][0] = af * (hp - v1 * cf) + qs * vbet + aspbb;
  rem[4][1] = -(v2 * bet3 - v3 * bet2);
  rem[4][2] = as * (hp - v1 * cs) - qf * vbet - afpbb;
  rem[4][3] = R(0.5) * vsq + e.g2 * x / e.g1;
  rem[4][4] = as * (hp + v1 * cs) + qf * vbet - afpbb;
  rem[4][5] = -rem[4][1];
  rem[4][6] = af * (hp + v1 * cf) - qs * vbet + aspbb;
  rem[5][0] = asp * bet2_star; rem[5][1] = -bet3 * s * isqrtd; rem[5][2] = -afp * bet2_star;
  rem[5][4] = rem[5][2]; rem[5][5] = rem[5][1]; rem[5][6] = rem[5][0];
  rem[6][0] = asp * bet3_star; rem[6][1] = bet2 * s * isqrtd; rem[6][2] = -afp * bet3_star;
  rem[6][4] = rem[6][2]; rem[6][5] = rem[6][1]; rem[6][6] = rem[6][0];

  R norm = R(0.5) / twid_asq;
  R cff = norm * af * cf;
  R css = norm * as * cs;
  qf *= norm;
  qs *= norm;
  R Af = norm * afp * d;
  R As = norm * asp * d;
  R afpb = norm * afp * bt_star;
  R aspb = norm * asp * bt_star;
  norm *= e.g1;
  af *= norm;
  as *= norm;
  R q2_star = bet2_star / bet_starsq;
  R q3_star = bet3_star / bet_starsq;
  R vqstr = (v2 * q2_star + v3 * q3_star);
  norm *= R(2.0);
  lem[0][0] = af * (vsq - hp) + cff * (cf + v1) - qs * vqstr - aspb;
  lem[0][1] = -af * v1 - cff;
  lem[0][2] = -af * v2 + qs * q2_star;
  lem[0][3] = -af * v3 + qs * q3_star;
  lem[0][4] = af;
  lem[0][5] = As * q2_star - af * b2;
  lem[0][6] = As * q3_star - af * b3;
  lem[1][0] = R(0.5) * (v2 * bet3 - v3 * bet2);
  lem[1][2] = R(-0.5) * bet3;
  lem[1][3] = R(0.5) * bet2;
  lem[1][5] = R(-0.5) * sqrtd * bet3 * s;
  lem[1][6] = R(0.5) * sqrtd * bet2 * s;
  lem[2][0] = as * (vsq - hp) + css * (cs + v1) + qf * vqstr + afpb;
  lem[2][1] = -as * v1 - css;
  lem[2][2] = -as * v2 - qf * q2_star;
  lem[2][3] = -as * v3 - qf * q3_star;
  lem[2][4] = as;
  lem[2][5] = -Af * q2_star - as * b2;
  lem[2][6] = -Af * q3_star - as * b3;
  lem[3][0] = R(1.0) - norm * (R(0.5) * vsq - e.g2 * x / e.g1);
  lem[3][1] = norm * v1;
  lem[3][2] = norm * v2;
  lem[3][3] = norm * v3;
  lem[3][4] = -norm;
  lem[3][5] = norm * b2;
  lem[3][6] = norm * b3;
  lem[4][0] = as * (vsq - hp) + css * (cs - v1) - qf * vqstr + afpb;
  lem[4][1] = -as * v1 + css;
  lem[4][2] = -as * v2 + qf * q2_star;
  lem[4][3] = -as * v3 + qf * q3_star;
  lem[4][4] = as;
  lem[4][5] = lem[2][5];
  lem[4][6] = lem[2][6];
  lem[5][0] = -lem[1][0];
  lem[5][2] = -lem[1][2];
  lem[5][3] = -lem[1][3];
  lem[5][5] = lem[1][5];
  lem[5][6] = lem[1][6];
  lem[6][0] = af * (vsq - hp) + cff * (cf - v1) + qs * vqstr - aspb;
  lem[6][1] = -af * v1 + cff;
  lem[6][2] = -af * v2 - qs * q2_star;
  lem[6][3] = -af * v3 - qs * q3_star;
  lem[6][4] = af;
  lem[6][5] = lem[0][5];
  lem[6][6] = lem[0][6];
}

// Roe-averaged quantities shared by both solvers (src/flux_roe.c:91-114).
template <class R> struct RoeIn { R sl, sr, isd, droe, v1, v2, v3, b2, b3, x, y, pbl, pbr, h; };

template <class R>
RoeIn<R> roe_in(const Vec<R>& Ul, const Vec<R>& Ur, const Vec<R>& Wl, const Vec<R>& Wr, R Bxi) {
  RoeIn<R> r;
  r.sl = sqrt(Wl[D]);
  r.sr = sqrt(Wr[D]);
  r.isd = R(1.0) / (r.sl + r.sr);
  r.droe = r.sl * r.sr;
  r.v1 = (r.sl * Wl[VX] + r.sr * Wr[VX]) * r.isd;
  r.v2 = (r.sl * Wl[VY] + r.sr * Wr[VY]) * r.isd;
  r.v3 = (r.sl * Wl[VZ] + r.sr * Wr[VZ]) * r.isd;
  r.b2 = (r.sr * Wl[BY] + r.sl * Wr[BY]) * r.isd;
  r.b3 = (r.sr * Wl[BZ] + r.sl * Wr[BZ]) * r.isd;
  r.x = R(0.5) * (SQ(Wl[BY] - Wr[BY]) + SQ(Wl[BZ] - Wr[BZ])) / (SQ(r.sl + r.sr));
  r.y = R(0.5) * (Wl[D] + Wr[D]) / r.droe;
  r.pbl = R(0.5) * (SQ(Bxi) + SQ(Wl[BY]) + SQ(Wl[BZ]));
  r.pbr = R(0.5) * (SQ(Bxi) + SQ(Wr[BY]) + SQ(Wr[BZ]));
  r.h = ((Ul[PE] + Wl[PE] + r.pbl) / r.sl + (Ur[PE] + Wr[PE] + r.pbr) / r.sr) * r.isd;
  return r;
}

// src/flux_hlle.c:60-199
template <class R>
Vec<R> flux_hlle(const Vec<R>& Ul, const Vec<R>& Ur, const Vec<R>& Wl, const Vec<R>& Wr, R Bxi, const Eos<R>& e) {
  RoeIn<R> r = roe_in(Ul, Ur, Wl, Wr, Bxi);
  Vec<R> ev;
  eig_roe<R>(r.droe, r.v1, r.v2, r.v3, r.h, Bxi, r.b2, r.b3, r.x, r.y, e, ev, nullptr, nullptr);
  R asq = e.gamma * Wl[PE] / Wl[D];
  R vaxsq = Bxi * Bxi / Wl[D];
  R ct2 = (Ul[BY] * Ul[BY] + Ul[BZ] * Ul[BZ]) / Wl[D];
  R qsq = vaxsq + ct2 + asq;
  R tmp = vaxsq + ct2 - asq;
  R cfsq = R(0.5) * (qsq + sqrt(tmp * tmp + R(4.0) * asq * ct2));
  R cfl = sqrt(cfsq);
  asq = e.gamma * Wr[PE] / Wr[D];
  vaxsq = Bxi * Bxi / Wr[D];
  ct2 = (Ur[BY] * Ur[BY] + Ur[BZ] * Ur[BZ]) / Wr[D];
  qsq = vaxsq + ct2 + asq;
  tmp = vaxsq + ct2 - asq;
  cfsq = R(0.5) * (qsq + sqrt(tmp * tmp + R(4.0) * asq * ct2));
  R cfr = sqrt(cfsq);
  R ar = MAXR(ev[NW - 1], (Wr[VX] + cfr));
  R al = MINR(ev[0], (Wl[VX] - cfl));
  R bp = MAXR(ar, R(0.0));
  R bm = MINR(al, R(0.0));
  Vec<R> Fl, Fr;
  Fl[D] = Ul[VX] - bm * Ul[D];
  Fr[D] = Ur[VX] - bp * Ur[D];
  Fl[VX] = Ul[VX] * (Wl[VX] - bm);
  Fr[VX] = Ur[VX] * (Wr[VX] - bp);
  Fl[VY] = Ul[VY] * (Wl[VX] - bm);
  Fr[VY] = Ur[VY] * (Wr[VX] - bp);
  Fl[VZ] = Ul[VZ] * (Wl[VX] - bm);
  Fr[VZ] = Ur[VZ] * (Wr[VX] - bp);
  Fl[VX] += Wl[PE];
  Fr[VX] += Wr[PE];
  Fl[PE] = Ul[PE] * (Wl[VX] - bm) + Wl[PE] * Wl[VX];
  Fr[PE] = Ur[PE] * (Wr[VX] - bp) + Wr[PE] * Wr[VX];
  Fl[VX] -= R(0.5) * (Bxi * Bxi - SQ(Wl[BY]) - SQ(Wl[BZ]));
  Fr[VX] -= R(0.5) * (Bxi * Bxi - SQ(Wr[BY]) - SQ(Wr[BZ]));
  Fl[VY] -= Bxi * Wl[BY];
  Fr[VY] -= Bxi * Wr[BY];
  Fl[VZ] -= Bxi * Wl[BZ];
  Fr[VZ] -= Bxi * Wr[BZ];
  Fl[PE] += (r.pbl * Wl[VX] - Bxi * (Bxi * Wl[VX] + Wl[BY] * Wl[VY] + Wl[BZ] * Wl[VZ]));
  Fr[PE] += (r.pbr * Wr[VX] - Bxi * (Bxi * Wr[VX] + Wr[BY] * Wr[VY] + Wr[BZ] * Wr[VZ]));
  Fl[BY] = Wl[BY] * (Wl[VX] - bm) - Bxi * Wl[VY];
  Fr[BY] = Wr[BY] * (Wr[VX] - bp) - Bxi * Wr[VY];
  Fl[BZ] = Wl[BZ] * (Wl[VX] - bm) - Bxi * Wl[VZ];
  Fr[BZ] = Wr[BZ] * (Wr[VX] - bp) - Bxi * Wr[VZ];
  R t = R(0.5) * (bp + bm) / (bp - bm);
  Vec<R> F;
  for (int n = 0; n < NW; n++) F[n] = R(0.5) * (Fl[n] + Fr[n]) + (Fl[n] - Fr[n]) * t;
  return F;
}

// src/flux_roe.c:54-259
template <class R>
Vec<R> flux_roe(const Vec<R>& Ul, const Vec<R>& Ur, const Vec<R>& Wl, const Vec<R>& Wr, R Bxi, const Eos<R>& e) {
  Mat<R> rem, lem;
  RoeIn<R> r = roe_in(Ul, Ur, Wl, Wr, Bxi);
  Vec<R> ev;
  eig_roe<R>(r.droe, r.v1, r.v2, r.v3, r.h, Bxi, r.b2, r.b3, r.x, r.y, e, ev, &rem, &lem);
  Vec<R> Fl, Fr;
  Fl[D] = Ul[VX];
  Fr[D] = Ur[VX];
  Fl[VX] = Ul[VX] * Wl[VX];
  Fr[VX] = Ur[VX] * Wr[VX];
  Fl[VY] = Ul[VX] * Wl[VY];
  Fr[VY] = Ur[VX] * Wr[VY];
  Fl[VZ] = Ul[VX] * Wl[VZ];
  Fr[VZ] = Ur[VX] * Wr[VZ];
  Fl[VX] += Wl[PE];
  Fr[VX] += Wr[PE];
  Fl[PE] = (Ul[PE] + Wl[PE]) * Wl[VX];
  Fr[PE] = (Ur[PE] + Wr[PE]) * Wr[VX];
  Fl[VX] -= R(0.5) * (Bxi * Bxi - SQ(Wl[BY]) - SQ(Wl[BZ]));
  Fr[VX] -= R(0.5) * (Bxi * Bxi - SQ(Wr[BY]) - SQ(Wr[BZ]));
  Fl[VY] -= Bxi * Wl[BY];
  Fr[VY] -= Bxi * Wr[BY];
  Fl[VZ] -= Bxi * Wl[BZ];
  Fr[VZ] -= Bxi * Wr[BZ];
  Fl[PE] += (r.pbl * Wl[VX] - Bxi * (Bxi * Wl[VX] + Wl[BY] * Wl[VY] + Wl[BZ] * Wl[VZ]));
  Fr[PE] += (r.pbr * Wr[VX] - Bxi * (Bxi * Wr[VX] + Wr[BY] * Wr[VY] + Wr[BZ] * Wr[VZ]));
  Fl[BY] = Wl[BY] * Wl[VX] - Bxi * Wl[VY];
  Fr[BY] = Wr[BY] * Wr[VX] - Bxi * Wr[VY];
  Fl[BZ] = Wl[BZ] * Wl[VX] - Bxi * Wl[VZ];
  Fr[BZ] = Wr[BZ] * Wr[VX] - Bxi * Wr[VZ];
  if (ev[0] >= R(0.0)) return Fl;
  if (ev[NW - 1] <= R(0.0)) return Fr;
  Vec<R> dU, a;
  for (int n = 0; n < NW; n++) dU[n] = Ur[n] - Ul[n];
  for (int n = 0; n < NW; n++) {
    a[n] = R(0.0);
    for (int m = 0; m < NW; m++) a[n] += lem[n][m] * dU[m];
  }
  Vec<R> u = Ul;
  for (int n = 0; n < NW - 1; n++) {
    for (int m = 0; m < NW; m++) u[m] += a[n] * rem[m][n];
    if (ev[n + 1] > ev[n]) {
      if (u[0] <= R(0.0)) return flux_hlle(Ul, Ur, Wl, Wr, Bxi, e);
      R p = u[4] - R(0.5) * (SQ(u[1]) + SQ(u[2]) + SQ(u[3])) / u[0];
      p -= R(0.5) * (SQ(u[NW - 2]) + SQ(u[NW - 1]) + SQ(Bxi));
      if (p < R(0.0)) return flux_hlle(Ul, Ur, Wl, Wr, Bxi, e);
    }
  }
  Vec<R> coeff, F;
  for (int m = 0; m < NW; m++) coeff[m] = R(0.5) * MAXR(fabs(ev[m]), R(0.0)) * a[m];
  for (int n = 0; n < NW; n++) {
    F[n] = R(0.5) * (Fl[n] + Fr[n]);
    for (int m = 0; m < NW; m++) F[n] -= coeff[m] * rem[n][m];
  }
  return F;
}

// ---------------------------------------------------------------------------
// the grid and the step
// ---------------------------------------------------------------------------
enum Plane { PD = 0, PM1, PM2, PM3, PE_, PB1C, PB2C, PB3C, PB1I, PB2I, PB3I, NPL };
enum Stage { ST_PREDICT = 0, ST_EMF_HALF, ST_CORRECT, ST_EMF_FULL, ST_UPDATE, ST_NEWDT, NSTAGE };

template <class R> struct Stepper {
  int nx1, nx2, sx, sy, is, ie, js, je, nmax;
  R dx1, dx2, x1_0 = R(0.0), x2_0 = R(0.0);
  Eos<R> eos;
  R cour_no;
  int bc[4];
  int flux;
  std::vector<R> q[NPL];
  Counts stage_counts[NSTAGE];

  // scratch, row-major [j][i] like the reference's 2D arrays
  std::vector<Vec<R>> ul1, ur1, f1, ul2, ur2, f2;
  std::vector<R> emf, ecc, b1f, b2f;

  R& at(int p, int j, int i) { return q[p][(size_t)j * sx + i]; }
  size_t ix(int j, int i) const { return (size_t)j * sx + i; }

  Stepper(int nx1_, int nx2_, double dx1_, double dx2_, double gamma, double cour, const int* bc_, int flux_)
      : nx1(nx1_), nx2(nx2_), sx(nx1_ + 2 * NG), sy(nx2_ + 2 * NG), is(NG), ie(nx1_ + NG - 1), js(NG),
        je(nx2_ + NG - 1), dx1(dx1_), dx2(dx2_), cour_no(cour), flux(flux_) {
    nmax = sx > sy ? sx : sy;
    eos.gamma = R(gamma);
    eos.g1 = R(gamma - 1.0);
    eos.g2 = R(gamma - 2.0);
    for (int k = 0; k < 4; k++) bc[k] = bc_[k];
    for (auto& p : q) p.assign((size_t)sx * sy, R(0.0));
    const size_t n = (size_t)sx * sy;
    ul1.assign(n, Vec<R>()); ur1 = ul1; f1 = ul1; ul2 = ul1; ur2 = ul1; f2 = ul1;
    emf.assign(n, R(0.0)); ecc = emf; b1f = emf; b2f = emf;
  }

  Vec<R> riemann(const Vec<R>& Ul, const Vec<R>& Ur, const Vec<R>& Wl, const Vec<R>& Wr, R bx) {
    return flux == 1 ? flux_hlle(Ul, Ur, Wl, Wr, bx, eos) : flux_roe(Ul, Ur, Wl, Wr, bx, eos);
  }

  void mark(int stage, Counts& before) {
    Counts now = g_cnt;
    Counts& s = stage_counts[stage];
    s.add += now.add - before.add; s.mul += now.mul - before.mul; s.div += now.div - before.div;
    s.sqrt += now.sqrt - before.sqrt; s.neg += now.neg - before.neg;
    before = now;
  }

  // upwind CT corner EMF (src/__integrate_2d__.c:632-702) at (j,i)
  R corner_emf(int j, int i) {
    const Vec<R>&fxs = f1[ix(j - 1, i)], &fxc = f1[ix(j, i)], &fyw = f2[ix(j, i - 1)], &fyc = f2[ix(j, i)];
    R esw = ecc[ix(j - 1, i - 1)], es = ecc[ix(j - 1, i)], ew = ecc[ix(j, i - 1)], ec = ecc[ix(j, i)];
    R l2, r2, l1, r1;
    if (fxs[D] > R(0.0)) l2 = -fxs[BY] + (fyw[BZ] - esw);
    else if (fxs[D] < R(0.0)) l2 = -fxs[BY] + (fyc[BZ] - es);
    else l2 = -fxs[BY] + R(0.5) * (fyw[BZ] - esw + fyc[BZ] - es);
    if (fxc[D] > R(0.0)) r2 = -fxc[BY] + (fyw[BZ] - ew);
    else if (fxc[D] < R(0.0)) r2 = -fxc[BY] + (fyc[BZ] - ec);
    else r2 = -fxc[BY] + R(0.5) * (fyw[BZ] - ew + fyc[BZ] - ec);
    if (fyw[D] > R(0.0)) l1 = fyw[BZ] + (-fxs[BY] - esw);
    else if (fyw[D] < R(0.0)) l1 = fyw[BZ] + (-fxc[BY] - ew);
    else l1 = fyw[BZ] + R(0.5) * (-fxs[BY] - esw - fxc[BY] - ew);
    if (fyc[D] > R(0.0)) r1 = fyc[BZ] + (-fxs[BY] - es);
    else if (fyc[D] < R(0.0)) r1 = fyc[BZ] + (-fxc[BY] - ec);
    else r1 = fyc[BZ] + R(0.5) * (-fxs[BY] - es - fxc[BY] - ec);
    return R(0.25) * (l1 + r1 + l2 + r2);
  }

  // src/__integrate_2d__.c:100-537
  void integrate(R dt) {
    Counts c0 = g_cnt;
    const R dtodx1 = dt / dx1, dtodx2 = dt / dx2, hdtodx1 = R(0.5) * dtodx1, hdtodx2 = R(0.5) * dtodx2;
    const R hdt = R(0.5) * dt;
    const int il = is - 2, iu = ie + 2, jl = js - 2, ju = je + 2;
    std::vector<Vec<R>> W(nmax), Wl(nmax + 1), Wr(nmax + 1);
    std::vector<R> Bxc(nmax);

    // steps 1a-1e: x-sweep
    for (int j = jl; j <= ju; j++) {
      for (int i = is - NG; i <= ie + NG; i++) {
        Vec<R> u = {at(PD, j, i), at(PM1, j, i), at(PM2, j, i), at(PM3, j, i), at(PE_, j, i), at(PB2C, j, i),
                    at(PB3C, j, i)};
        Bxc[i] = at(PB1C, j, i);
        W[i] = cons_to_prim(u, Bxc[i], eos);
      }
      plm_slice(W, Bxc, dtodx1, is - 2, ie + 2, Wl, Wr, eos);
      for (int i = is - 1; i <= iu; i++) {
        R src = (at(PM2, j, i - 1) / at(PD, j, i - 1)) * (at(PB1I, j, i) - at(PB1I, j, i - 1)) / dx1;
        Wl[i][BY] += hdt * src;
        src = (at(PM2, j, i) / at(PD, j, i)) * (at(PB1I, j, i + 1) - at(PB1I, j, i)) / dx1;
        Wr[i][BY] += hdt * src;
      }
      for (int i = is - 1; i <= iu; i++) {
        const R bx = at(PB1I, j, i);
        ul1[ix(j, i)] = prim_to_cons(Wl[i], bx, eos);
        ur1[ix(j, i)] = prim_to_cons(Wr[i], bx, eos);
        f1[ix(j, i)] = riemann(ul1[ix(j, i)], ur1[ix(j, i)], Wl[i], Wr[i], bx);
      }
    }
    // steps 2a-2e: y-sweep, slice frame (d, M2, M3, M1, E, B3c, B1c)
    for (int i = il; i <= iu; i++) {
      for (int j = js - NG; j <= je + NG; j++) {
        Vec<R> u = {at(PD, j, i), at(PM2, j, i), at(PM3, j, i), at(PM1, j, i), at(PE_, j, i), at(PB3C, j, i),
                    at(PB1C, j, i)};
        Bxc[j] = at(PB2C, j, i);
        W[j] = cons_to_prim(u, Bxc[j], eos);
      }
      plm_slice(W, Bxc, dtodx2, js - 2, je + 2, Wl, Wr, eos);
      for (int j = js - 1; j <= ju; j++) {
        R src = (at(PM1, j - 1, i) / at(PD, j - 1, i)) * (at(PB2I, j, i) - at(PB2I, j - 1, i)) / dx2;
        Wl[j][BZ] += hdt * src;
        src = (at(PM1, j, i) / at(PD, j, i)) * (at(PB2I, j + 1, i) - at(PB2I, j, i)) / dx2;
        Wr[j][BZ] += hdt * src;
      }
      for (int j = js - 1; j <= ju; j++) {
        const R bx = at(PB2I, j, i);
        ul2[ix(j, i)] = prim_to_cons(Wl[j], bx, eos);
        ur2[ix(j, i)] = prim_to_cons(Wr[j], bx, eos);
        f2[ix(j, i)] = riemann(ul2[ix(j, i)], ur2[ix(j, i)], Wl[j], Wr[j], bx);
      }
    }
    // step 3: cell-centred emf3 at t^n
    for (int j = jl; j <= ju; j++)
      for (int i = il; i <= iu; i++)
        ecc[ix(j, i)] = (at(PB1C, j, i) * at(PM2, j, i) - at(PB2C, j, i) * at(PM1, j, i)) / at(PD, j, i);
    mark(ST_PREDICT, c0);

    // step 4: corner EMF and half-step CT on the face copies
    for (int j = js - 1; j <= je + 2; j++)
      for (int i = is - 1; i <= ie + 2; i++) emf[ix(j, i)] = corner_emf(j, i);
    for (int j = 0; j < sy; j++)
      for (int i = 0; i < sx; i++) { b1f[ix(j, i)] = at(PB1I, j, i); b2f[ix(j, i)] = at(PB2I, j, i); }
    for (int j = js - 1; j <= je + 1; j++) {
      for (int i = is - 1; i <= ie + 1; i++) {
        b1f[ix(j, i)] -= hdtodx2 * (emf[ix(j + 1, i)] - emf[ix(j, i)]);
        b2f[ix(j, i)] += hdtodx1 * (emf[ix(j, i + 1)] - emf[ix(j, i)]);
      }
      b1f[ix(j, iu)] -= hdtodx2 * (emf[ix(j + 1, iu)] - emf[ix(j, iu)]);
    }
    for (int i = is - 1; i <= ie + 1; i++) b2f[ix(ju, i)] += hdtodx1 * (emf[ix(ju, i + 1)] - emf[ix(ju, i)]);
    mark(ST_EMF_HALF, c0);

    // step 5a/5b: x1-face states, transverse x2-flux gradients + MHD terms
    const int mx[6] = {D, VZ, VX, VY, PE, BY};  // x2-flux component feeding (d,Mx,My,Mz,E,Bz)
    const int dst1[6] = {D, VX, VY, VZ, PE, BZ};
    for (int j = js - 1; j <= je + 1; j++)
      for (int i = is - 1; i <= iu; i++)
        for (int k = 0; k < 6; k++) {
          ul1[ix(j, i)][dst1[k]] -= hdtodx2 * (f2[ix(j + 1, i - 1)][mx[k]] - f2[ix(j, i - 1)][mx[k]]);
          ur1[ix(j, i)][dst1[k]] -= hdtodx2 * (f2[ix(j + 1, i)][mx[k]] - f2[ix(j, i)][mx[k]]);
        }
    for (int j = js - 1; j <= je + 1; j++)
      for (int i = is - 1; i <= iu; i++) {
        for (int side = 0; side < 2; side++) {
          const int c = side == 0 ? i - 1 : i;
          R dbx = at(PB1I, j, c + 1) - at(PB1I, j, c);
          R B1 = at(PB1C, j, c), B2 = at(PB2C, j, c), B3 = at(PB3C, j, c);
          R V3 = at(PM3, j, c) / at(PD, j, c);
          Vec<R>& u = side == 0 ? ul1[ix(j, i)] : ur1[ix(j, i)];
          u[VX] += hdtodx1 * B1 * dbx;
          u[VY] += hdtodx1 * B2 * dbx;
          u[VZ] += hdtodx1 * B3 * dbx;
          u[BZ] += hdtodx1 * V3 * dbx;
          u[PE] += hdtodx1 * B3 * V3 * dbx;
        }
      }
    // step 6a/6b: x2-face states, transverse x1-flux gradients + MHD terms
    const int my[6] = {D, VY, VZ, VX, PE, BZ};  // x1-flux component feeding (d,Mx,My,Mz,E,By)
    const int dst2[6] = {D, VX, VY, VZ, PE, BY};
    for (int j = js - 1; j <= ju; j++)
      for (int i = is - 1; i <= ie + 1; i++)
        for (int k = 0; k < 6; k++) {
          ul2[ix(j, i)][dst2[k]] -= hdtodx1 * (f1[ix(j - 1, i + 1)][my[k]] - f1[ix(j - 1, i)][my[k]]);
          ur2[ix(j, i)][dst2[k]] -= hdtodx1 * (f1[ix(j, i + 1)][my[k]] - f1[ix(j, i)][my[k]]);
        }
    for (int j = js - 1; j <= ju; j++)
      for (int i = is - 1; i <= ie + 1; i++) {
        for (int side = 0; side < 2; side++) {
          const int c = side == 0 ? j - 1 : j;
          R dby = at(PB2I, c + 1, i) - at(PB2I, c, i);
          R B1 = at(PB1C, c, i), B2 = at(PB2C, c, i), B3 = at(PB3C, c, i);
          R V3 = at(PM3, c, i) / at(PD, c, i);
          Vec<R>& u = side == 0 ? ul2[ix(j, i)] : ur2[ix(j, i)];
          u[VZ] += hdtodx2 * B1 * dby;
          u[VX] += hdtodx2 * B2 * dby;
          u[VY] += hdtodx2 * B3 * dby;
          u[BY] += hdtodx2 * V3 * dby;
          u[PE] += hdtodx2 * B3 * V3 * dby;
        }
      }
    // step 7: cell-centred emf3 at t^{n+1/2}
    for (int j = js - 1; j <= je + 1; j++)
      for (int i = is - 1; i <= ie + 1; i++) {
        // cell position computed and unused by the reference (src/__integrate_2d__.c:414)
        R x1 = x1_0 + (R((double)(i - is)) + R(0.5)) * dx1;
        R x2 = x2_0 + (R((double)(j - js)) + R(0.5)) * dx2;
        (void)x1; (void)x2;
        R d = at(PD, j, i) - hdtodx1 * (f1[ix(j, i + 1)][D] - f1[ix(j, i)][D]) -
              hdtodx2 * (f2[ix(j + 1, i)][D] - f2[ix(j, i)][D]);
        R M1 = at(PM1, j, i) - hdtodx1 * (f1[ix(j, i + 1)][VX] - f1[ix(j, i)][VX]) -
               hdtodx2 * (f2[ix(j + 1, i)][VZ] - f2[ix(j, i)][VZ]);
        R M2 = at(PM2, j, i) - hdtodx1 * (f1[ix(j, i + 1)][VY] - f1[ix(j, i)][VY]) -
               hdtodx2 * (f2[ix(j + 1, i)][VX] - f2[ix(j, i)][VX]);
        R B1c = R(0.5) * (b1f[ix(j, i)] + b1f[ix(j, i + 1)]);
        R B2c = R(0.5) * (b2f[ix(j, i)] + b2f[ix(j + 1, i)]);
        ecc[ix(j, i)] = (B1c * M2 - B2c * M1) / d;
      }
    // steps 8b/8c: corrector fluxes
    for (int j = js - 1; j <= je + 1; j++)
      for (int i = is; i <= ie + 1; i++) {
        const R bx = b1f[ix(j, i)];
        Vec<R> wl = cons_to_prim(ul1[ix(j, i)], bx, eos), wr = cons_to_prim(ur1[ix(j, i)], bx, eos);
        f1[ix(j, i)] = riemann(ul1[ix(j, i)], ur1[ix(j, i)], wl, wr, bx);
      }
    for (int j = js; j <= je + 1; j++)
      for (int i = is - 1; i <= ie + 1; i++) {
        const R bx = b2f[ix(j, i)];
        Vec<R> wl = cons_to_prim(ul2[ix(j, i)], bx, eos), wr = cons_to_prim(ur2[ix(j, i)], bx, eos);
        f2[ix(j, i)] = riemann(ul2[ix(j, i)], ur2[ix(j, i)], wl, wr, bx);
      }
    mark(ST_CORRECT, c0);

    // step 9: corner EMF at t^{n+1/2} over the reference's full range
    // (src/__integrate_2d__.c:641-642); the CT update reads [is,ie+1]x[js,je+1]
    for (int j = js - 1; j <= je + 2; j++)
      for (int i = is - 1; i <= ie + 2; i++) emf[ix(j, i)] = corner_emf(j, i);
    mark(ST_EMF_FULL, c0);
    for (int j = js; j <= je; j++) {
      for (int i = is; i <= ie; i++) {
        at(PB1I, j, i) -= dtodx2 * (emf[ix(j + 1, i)] - emf[ix(j, i)]);
        at(PB2I, j, i) += dtodx1 * (emf[ix(j, i + 1)] - emf[ix(j, i)]);
      }
      at(PB1I, j, ie + 1) -= dtodx2 * (emf[ix(j + 1, ie + 1)] - emf[ix(j, ie + 1)]);
    }
    for (int i = is; i <= ie; i++) at(PB2I, je + 1, i) += dtodx1 * (emf[ix(je + 1, i + 1)] - emf[ix(je + 1, i)]);
    // steps 11a/11b: conservative update
    const int p1[7] = {PD, PM1, PM2, PM3, PE_, PB2C, PB3C};
    for (int j = js; j <= je; j++)
      for (int i = is; i <= ie; i++)
        for (int k = 0; k < 7; k++) at(p1[k], j, i) -= dtodx1 * (f1[ix(j, i + 1)][k] - f1[ix(j, i)][k]);
    const int p2[7] = {PD, PM2, PM3, PM1, PE_, PB3C, PB1C};
    for (int j = js; j <= je; j++)
      for (int i = is; i <= ie; i++)
        for (int k = 0; k < 7; k++) at(p2[k], j, i) -= dtodx2 * (f2[ix(j + 1, i)][k] - f2[ix(j, i)][k]);
    // step 13: cell-centred field from the faces
    for (int j = js; j <= je; j++)
      for (int i = is; i <= ie; i++) {
        at(PB1C, j, i) = R(0.5) * (at(PB1I, j, i) + at(PB1I, j, i + 1));
        at(PB2C, j, i) = R(0.5) * (at(PB2I, j, i) + at(PB2I, j + 1, i));
        at(PB3I, j, i) = at(PB3C, j, i);
      }
    mark(ST_UPDATE, c0);
  }

  // src/new_dt.c:25-100; returns max 1/dt
  R max_dti() {
    Counts c0 = g_cnt;
    R m = R(0.0);
    for (int j = js; j <= je; j++)
      for (int i = is; i <= ie; i++) {
        R di = R(1.0) / at(PD, j, i);
        R v1 = at(PM1, j, i) * di, v2 = at(PM2, j, i) * di, v3 = at(PM3, j, i) * di;
        R qsq = v1 * v1 + v2 * v2 + v3 * v3;
        // magnetic fast speeds (src/new_dt.c:46-63), overwritten by the sound
        // speed at src/new_dt.c:66-77: formed, then discarded
        {
          R b1 = at(PB1C, j, i) + fabs(at(PB1I, j, i) - at(PB1C, j, i));
          R b2 = at(PB2C, j, i) + fabs(at(PB2I, j, i) - at(PB2C, j, i));
          R b3 = at(PB3C, j, i) + fabs(at(PB3I, j, i) - at(PB3C, j, i));
          R bsq = b1 * b1 + b2 * b2 + b3 * b3;
          R pm = MAXR(eos.g1 * (at(PE_, j, i) - R(0.5) * at(PD, j, i) * qsq - R(0.5) * bsq), R(TINY));
          R asqm = eos.gamma * pm * di;
          R tsum = bsq * di + asqm;
          R tdif = bsq * di - asqm;
          R c1 = R(0.5) * (tsum + sqrt(tdif * tdif + R(4.0) * asqm * (b2 * b2 + b3 * b3) * di));
          R c2 = R(0.5) * (tsum + sqrt(tdif * tdif + R(4.0) * asqm * (b1 * b1 + b3 * b3) * di));
          R c3 = R(0.5) * (tsum + sqrt(tdif * tdif + R(4.0) * asqm * (b1 * b1 + b2 * b2) * di));
          (void)c1; (void)c2; (void)c3;
        }
        R p = MAXR(eos.g1 * (at(PE_, j, i) - R(0.5) * at(PD, j, i) * qsq), R(TINY));
        R asq = eos.gamma * p * di;
        m = MAXR(m, (fabs(v1) + sqrt(asq)) / dx1);
        m = MAXR(m, (fabs(v2) + sqrt(asq)) / dx2);
      }
    mark(ST_NEWDT, c0);
    return m;
  }

  // ghost zones (src/set_bvals.c): x1 boundaries on rows [js,je] ([js,je+1]
  // for B2i), then x2 boundaries on whole rows
  void bvals() {
    const int cc[9] = {PD, PM1, PM2, PM3, PE_, PB1C, PB2C, PB3C, PB3I};
    for (int side = 0; side < 2; side++) {  // x1
      const int kind = bc[side];
      for (int j = js; j <= je + 1; j++)
        for (int g = 1; g <= NG; g++) {
          const int dst = side == 0 ? is - g : ie + g;
          int src = 0;
          if (kind == 1) src = side == 0 ? is + (g - 1) : ie - (g - 1);
          else if (kind == 2) src = side == 0 ? is : ie;
          else src = side == 0 ? ie - (g - 1) : is + (g - 1);
          if (j <= je) {
            for (int p : cc) at(p, j, dst) = at(p, j, src);
            if (kind == 1) at(PM1, j, dst) = -at(PM1, j, dst);
            // B1i: outer side starts at ie+2; reflect/outflow use ie-(g-2) / ie
            if (side == 0) at(PB1I, j, dst) = at(PB1I, j, src);
            else if (g >= 2) {
              int s1 = kind == 1 ? ie - (g - 2) : kind == 2 ? ie : is + (g - 1);
              at(PB1I, j, dst) = at(PB1I, j, s1);
            }
          }
          at(PB2I, j, dst) = at(PB2I, j, src);
        }
    }
    for (int side = 0; side < 2; side++) {  // x2
      const int kind = bc[2 + side];
      for (int g = 1; g <= NG; g++) {
        const int dst = side == 0 ? js - g : je + g;
        int src = 0;
        if (kind == 1) src = side == 0 ? js + (g - 1) : je - (g - 1);
        else if (kind == 2) src = side == 0 ? js : je;
        else src = side == 0 ? je - (g - 1) : js + (g - 1);
        for (int i = 0; i < sx; i++) {
          for (int p : cc) at(p, dst, i) = at(p, src, i);
          if (kind == 1) at(PM2, dst, i) = -at(PM2, dst, i);
          at(PB1I, dst, i) = at(PB1I, src, i);
          if (side == 0) at(PB2I, dst, i) = at(PB2I, src, i);
          else if (g >= 2) {
            int s2 = kind == 1 ? je - (g - 2) : kind == 2 ? je : js + (g - 1);
            at(PB2I, dst, i) = at(PB2I, s2, i);
          }
        }
      }
    }
  }
};

}  // namespace orc

using namespace orc;

template <class R>
static int run_loop(Stepper<R>& S, double tlim, int nlim, int max_steps, double* dt_io, double* time_io,
                    int* nstep_io) {
  // src/main.c:139-149: boundary values and the first dt
  S.bvals();
  R dt = S.cour_no / S.max_dti();
  R time = R(*time_io);
  int nstep = 0;
  int done = 0;
  while (val(time) < tlim && (nlim < 0 || nstep < nlim) && (max_steps < 0 || done < max_steps)) {
    if ((R(tlim) - time) < dt) dt = (R(tlim) - time);
    S.integrate(dt);
    nstep++;
    time += dt;
    R m = S.max_dti();
    dt = MINR(R(2.0) * dt, S.cour_no / m);
    S.bvals();
    done++;
  }
  *dt_io = val(dt);
  *time_io = val(time);
  *nstep_io = nstep;
  return done;
}

extern "C" {

// Run the reference main loop from an initial state (11 planes of
// (nx2+8) x (nx1+8) doubles; ghosts are filled first, as src/main.c does).
// Returns the number of steps run; the final state overwrites planes.
int oracle_run(int nx1, int nx2, double dx1, double dx2, const int* bc, double gamma, double cour_no,
               double tlim, int nlim, int flux, int max_steps, double* planes, double* dt_out,
               double* time_out, int* nstep_out) {
  Stepper<double> S(nx1, nx2, dx1, dx2, gamma, cour_no, bc, flux);
  const size_t n = (size_t)S.sx * S.sy;
  for (int p = 0; p < NPL; p++) std::memcpy(S.q[p].data(), planes + p * n, n * sizeof(double));
  double dt = 0, t = 0;
  int ns = 0;
  int done = run_loop(S, tlim, nlim, max_steps, &dt, &t, &ns);
  for (int p = 0; p < NPL; p++) std::memcpy(planes + p * n, S.q[p].data(), n * sizeof(double));
  *dt_out = dt;
  *time_out = t;
  *nstep_out = ns;
  return done;
}

// Same loop with the counting scalar; counts[stage*5 + {add, mul, div, sqrt,
// neg}] for the stages predict, emf_half, correct, emf_full, update, new_dt,
// summed over the steps run (the initial new_dt is excluded).
int oracle_opcount(int nx1, int nx2, double dx1, double dx2, const int* bc, double gamma, double cour_no,
                   double tlim, int nlim, int flux, int max_steps, const double* planes, double* counts) {
  Stepper<Cnt> S(nx1, nx2, dx1, dx2, gamma, cour_no, bc, flux);
  const size_t n = (size_t)S.sx * S.sy;
  for (int p = 0; p < NPL; p++)
    for (size_t k = 0; k < n; k++) S.q[p][k] = Cnt(planes[p * n + k]);
  S.bvals();
  Cnt dt = S.cour_no / S.max_dti();
  for (auto& s : S.stage_counts) s = Counts();
  Cnt time = Cnt(0.0);
  int nstep = 0;
  while (time.v < tlim && (nlim < 0 || nstep < nlim) && (max_steps < 0 || nstep < max_steps)) {
    if ((Cnt(tlim) - time) < dt) dt = (Cnt(tlim) - time);
    S.integrate(dt);
    nstep++;
    time = Cnt(time.v + dt.v);
    Cnt m = S.max_dti();
    dt = Cnt(std::fmin(2.0 * dt.v, S.cour_no.v / m.v));
    S.bvals();
  }
  for (int s = 0; s < NSTAGE; s++) {
    counts[s * 5 + 0] = (double)S.stage_counts[s].add;
    counts[s * 5 + 1] = (double)S.stage_counts[s].mul;
    counts[s * 5 + 2] = (double)S.stage_counts[s].div;
    counts[s * 5 + 3] = (double)S.stage_counts[s].sqrt;
    counts[s * 5 + 4] = (double)S.stage_counts[s].neg;
  }
  return nstep;
}

}  // extern "C"
