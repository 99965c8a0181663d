// step_generic.cuh -- one CTU+CT step written per work item and templated on
// the scalar type, for the tangent-linear model and for the recorded
// ("taped") forward step of the adjoint.
//
// The fast forward kernels (step_kernels.cuh) fuse the predictor's PLM and
// Riemann solver per warp and march columns through shared memory; here every
// stage is a plain per-cell or per-face item that reads planes and writes
// planes, so that
//   * T = double gives the plain step with every intermediate kept in HBM
//     (the tape the adjoint kernels read); its state is bit-identical to the
//     fast kernels' (same operations in the same order);
//   * T = Dual gives the tangent-linear step: values bit-identical to the
//     plain step, tangents its derivative (dual.cuh);
//   * the items are __host__ __device__, so the same code runs on a CPU (the
//     host checks in tests/) as in the sm_100a kernels (athb_adjoint.cu).
//
// Stages (reference src/__integrate_2d__.c:100-537):
//   gen_plm      1b-1d / 2b-2d  PLM of one cell of a sweep + the half-dt MHD
//                               source (:156-164, :216-224)
//   gen_riemann  1e / 2e        predictor L/R conserved states and flux at a face
//   gen_ecc0     3              cell-centred emf3 at t^n
//   gen_emf      4 / 9          upwind corner EMF (:632-702)
//   gen_correct_x / _y          4, 5a/5b, 8b / 4, 6a/6b, 8c
//   gen_correct_e 7             cell-centred emf3 at t^{n+1/2}
//   gen_update   9, 11a/11b, 13 CT, conservative update, cell-centred B
//   gen_cell_dti                new_dt's per-cell CFL rate (src/new_dt.c:37-85)
#pragma once

#include "dual.cuh"
#include "step_types.cuh"

namespace athb {

// ---------------------------------------------------------------------------
// Plane access for either scalar kind: a double plane set, or a value plane
// set plus a tangent plane set with the same layout.
// ---------------------------------------------------------------------------
template <class T> struct Planes;
template <> struct Planes<double> {
  double* v = nullptr;
  ATHB_MEM double get(long long i) const { return v[i]; }
  ATHB_MEM void set(long long i, double x) const { v[i] = x; }
};
template <> struct Planes<Dual> {
  double* v = nullptr;
  double* t = nullptr;
  ATHB_MEM Dual get(long long i) const { return Dual(v[i], t[i]); }
  ATHB_MEM void set(long long i, Dual x) const { v[i] = x.v; t[i] = x.t; }
};

// Tape / scratch planes of the generic step (each group of 7 is one Cons1 or
// Prim1 in the sweep frame), laid out as the fast kernels' scratch planes
// (step_types.cuh) followed by the taped planes, so that a taped step of the
// fast kernels and one of the generic step leave the same tape.
enum GenPlane {
  G_ULX = S_ULX, G_URX = S_URX, G_FX = S_FX,   // predictor states and fluxes at x faces
  G_ULY = S_ULY, G_URY = S_URY, G_FY = S_FY,
  G_FX2 = S_FX2, G_FY2 = S_FY2,                // corrector fluxes
  G_ECC1 = S_ECC,   // cell emf3 at t^{n+1/2}
  G_EMF1 = S_EMF,   // corner emf of the full step
  G_WLNX = T_WLNX,  // W_L at face i+1/2 from cell i (x sweep), after the source term
  G_WRTX = T_WRTX,  // W_R at face i-1/2 from cell i
  G_WLNY = T_WLNY,
  G_WRTY = T_WRTY,
  G_ECC0 = T_ECC0,  // cell emf3 at t^n
  G_EMF0 = T_EMF0,  // corner emf at t^n (half step)
  NGEN = NTAPED
};

// dt and its derived factors (src/__integrate_2d__.c:102-110), as the scalar
// kind of the step (a Dual carries d(dt) of the tangent-linear model).
template <class T> struct StepCoef {
  T dt, dtodx1, dtodx2, hdtodx1, hdtodx2, hdt;
};

template <class T>
ATHB_HD StepCoef<T> make_coef(T dt, double dx1, double dx2) {
  StepCoef<T> c;
  c.dt = dt;
  c.dtodx1 = dt / dx1;
  c.dtodx2 = dt / dx2;
  c.hdtodx1 = 0.5 * c.dtodx1;
  c.hdtodx2 = 0.5 * c.dtodx2;
  c.hdt = 0.5 * dt;
  return c;
}

// Host test builds define ATHB_HOST_BOUNDS: every plane access is checked to
// stay inside its plane (the kernels' index ranges are verified on the CPU).
#if defined(ATHB_HOST_BOUNDS) && !defined(__CUDA_ARCH__)
#include <cstdio>
#include <cstdlib>
#define ATHB_CHECK_OFF(off, ps)                                                           \
  do {                                                                                    \
    if ((off) < 0 || (off) >= (ps)) {                                                     \
      std::fprintf(stderr, "plane offset %lld outside [0, %lld) at %s:%d\n", (long long)(off), \
                   (long long)(ps), __FILE__, __LINE__);                                  \
      std::abort();                                                                       \
    }                                                                                     \
  } while (0)
#else
#define ATHB_CHECK_OFF(off, ps) do { } while (0)
#endif

template <class T> struct GenArgs {
  Planes<T> in, out, scr;
  const StepCoef<T>* coef;
  long long ps;       // plane stride of in / out / scr
  int pitch;
  int is, ie, js, je;
  double dx1, dx2;
  Eos eos;
  ATHB_MEM long long o(int j, int i) const { return (long long)j * pitch + i; }
  ATHB_MEM T s(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return in.get(p * ps + off); }
  ATHB_MEM T g(int p, long long off) const { ATHB_CHECK_OFF(off, ps); return scr.get(p * ps + off); }
  ATHB_MEM void put(int p, long long off, T x) const { ATHB_CHECK_OFF(off, ps); scr.set(p * ps + off, x); }
};

// Ranges (inclusive) of the stages over an interior [is,ie] x [js,je].
struct GenRange { int i0, i1, j0, j1; };
ATHB_HD GenRange range_plm(int is, int ie, int js, int je) { return {is - 2, ie + 2, js - 2, je + 2}; }
ATHB_HD GenRange range_riemann_x(int is, int ie, int js, int je) { return {is - 1, ie + 2, js - 2, je + 2}; }
ATHB_HD GenRange range_riemann_y(int is, int ie, int js, int je) { return {is - 2, ie + 2, js - 1, je + 2}; }
ATHB_HD GenRange range_emf0(int is, int ie, int js, int je) { return {is - 1, ie + 2, js - 1, je + 2}; }
ATHB_HD GenRange range_correct_x(int is, int ie, int js, int je) { return {is, ie + 1, js - 1, je + 1}; }
ATHB_HD GenRange range_correct_y(int is, int ie, int js, int je) { return {is - 1, ie + 1, js, je + 1}; }
ATHB_HD GenRange range_correct_e(int is, int ie, int js, int je) { return {is - 1, ie + 1, js - 1, je + 1}; }
ATHB_HD GenRange range_emf1(int is, int ie, int js, int je) { return {is, ie + 1, js, je + 1}; }
ATHB_HD GenRange range_interior(int is, int ie, int js, int je) { return {is, ie, js, je}; }
ATHB_HD long long range_count(const GenRange& r) {
  return (long long)(r.i1 - r.i0 + 1) * (r.j1 - r.j0 + 1);
}
ATHB_HD void range_item(const GenRange& r, long long t, int& j, int& i) {
  const int w = r.i1 - r.i0 + 1;
  j = r.j0 + (int)(t / w);
  i = r.i0 + (int)(t % w);
}

// Sweep-frame conserved vector of a cell and its normal field
// (src/__integrate_2d__.c:130-139 for x, :191-201 for y).
template <class T>
ATHB_HD Cons1T<T> gen_cons(const GenArgs<T>& a, long long o, int dir) {
  Cons1T<T> u;
  u.d = a.s(P_D, o);
  u.e = a.s(P_E, o);
  if (dir == 0) {
    u.mx = a.s(P_M1, o); u.my = a.s(P_M2, o); u.mz = a.s(P_M3, o);
    u.by = a.s(P_B2C, o); u.bz = a.s(P_B3C, o);
  } else {
    u.mx = a.s(P_M2, o); u.my = a.s(P_M3, o); u.mz = a.s(P_M1, o);
    u.by = a.s(P_B3C, o); u.bz = a.s(P_B1C, o);
  }
  return u;
}
template <class T>
ATHB_HD Prim1T<T> gen_prim(const GenArgs<T>& a, long long o, int dir) {
  return cons_to_prim(gen_cons(a, o, dir), a.s(dir == 0 ? P_B1C : P_B2C, o), a.eos);
}

template <class T>
ATHB_HD void put_prim(const GenArgs<T>& a, int base, long long o, const Prim1T<T>& w) {
  a.put(base + 0, o, w.d); a.put(base + 1, o, w.vx); a.put(base + 2, o, w.vy); a.put(base + 3, o, w.vz);
  a.put(base + 4, o, w.p); a.put(base + 5, o, w.by); a.put(base + 6, o, w.bz);
}
template <class T>
ATHB_HD Prim1T<T> get_prim(const GenArgs<T>& a, int base, long long o) {
  Prim1T<T> w;
  w.d = a.g(base + 0, o); w.vx = a.g(base + 1, o); w.vy = a.g(base + 2, o); w.vz = a.g(base + 3, o);
  w.p = a.g(base + 4, o); w.by = a.g(base + 5, o); w.bz = a.g(base + 6, o);
  return w;
}
template <class T>
ATHB_HD void put_cons(const GenArgs<T>& a, int base, long long o, const Cons1T<T>& u) {
  a.put(base + 0, o, u.d); a.put(base + 1, o, u.mx); a.put(base + 2, o, u.my); a.put(base + 3, o, u.mz);
  a.put(base + 4, o, u.e); a.put(base + 5, o, u.by); a.put(base + 6, o, u.bz);
}
template <class T>
ATHB_HD Cons1T<T> get_cons(const GenArgs<T>& a, int base, long long o) {
  Cons1T<T> u;
  u.d = a.g(base + 0, o); u.mx = a.g(base + 1, o); u.my = a.g(base + 2, o); u.mz = a.g(base + 3, o);
  u.e = a.g(base + 4, o); u.by = a.g(base + 5, o); u.bz = a.g(base + 6, o);
  return u;
}

// ---- 1b-1d / 2b-2d: PLM of cell (j,i) in sweep dir, plus the MHD source ----
template <class T>
ATHB_HD void gen_plm(const GenArgs<T>& a, int dir, int j, int i) {
  const StepCoef<T>& c = *a.coef;
  const long long o = a.o(j, i);
  const long long step = dir == 0 ? 1 : a.pitch;
  const Prim1T<T> wm = gen_prim(a, o - step, dir);
  const Prim1T<T> w0 = gen_prim(a, o, dir);
  const Prim1T<T> wp = gen_prim(a, o + step, dir);
  Prim1T<T> wln, wrt;
  plm_cell(wm, w0, wp, a.s(dir == 0 ? P_B1C : P_B2C, o), dir == 0 ? c.dtodx1 : c.dtodx2, a.eos, wln, wrt);
  if (dir == 0) {
    // src/__integrate_2d__.c:156-164
    const T src = (a.s(P_M2, o) / a.s(P_D, o)) * (a.s(P_B1I, o + 1) - a.s(P_B1I, o)) / a.dx1;
    wln.by += c.hdt * src;
    wrt.by += c.hdt * src;
    put_prim(a, G_WLNX, o, wln);
    put_prim(a, G_WRTX, o, wrt);
  } else {
    // src/__integrate_2d__.c:216-224
    const T src = (a.s(P_M1, o) / a.s(P_D, o)) * (a.s(P_B2I, o + a.pitch) - a.s(P_B2I, o)) / a.dx2;
    wln.bz += c.hdt * src;
    wrt.bz += c.hdt * src;
    put_prim(a, G_WLNY, o, wln);
    put_prim(a, G_WRTY, o, wrt);
  }
}

// ---- 1e / 2e: predictor states and flux at the face (j,i) of sweep dir -----
template <int FLUX, class T>
ATHB_HD void gen_riemann(const GenArgs<T>& a, int dir, int j, int i) {
  const long long o = a.o(j, i);
  const long long step = dir == 0 ? 1 : a.pitch;
  const Prim1T<T> wl = get_prim(a, dir == 0 ? G_WLNX : G_WLNY, o - step);
  const Prim1T<T> wr = get_prim(a, dir == 0 ? G_WRTX : G_WRTY, o);
  const T bn = a.s(dir == 0 ? P_B1I : P_B2I, o);
  const Cons1T<T> ul = prim_to_cons(wl, bn, a.eos);
  const Cons1T<T> ur = prim_to_cons(wr, bn, a.eos);
  put_cons(a, dir == 0 ? G_ULX : G_ULY, o, ul);
  put_cons(a, dir == 0 ? G_URX : G_URY, o, ur);
  put_cons(a, dir == 0 ? G_FX : G_FY, o, riemann<FLUX>(ul, ur, wl, wr, bn, a.eos));
}

// ---- 3: cell-centred emf3 at t^n (src/__integrate_2d__.c:249-255) ----------
template <class T>
ATHB_HD void gen_ecc0(const GenArgs<T>& a, int j, int i) {
  const long long o = a.o(j, i);
  a.put(G_ECC0, o, (a.s(P_B1C, o) * a.s(P_M2, o) - a.s(P_B2C, o) * a.s(P_M1, o)) / a.s(P_D, o));
}

// ---- 4 / 9: upwind corner EMF (src/__integrate_2d__.c:632-702) -------------
// Inputs of corner (j,i): x-fluxes at (j-1,i) and (j,i) (mass and By = -E3),
// y-fluxes at (j,i-1) and (j,i) (mass and Bz = +E3), cell emf3 at (j-1,i-1),
// (j-1,i), (j,i-1), (j,i).
template <class T>
ATHB_HD T corner_emf_gen(T fx_d_s, T fx_by_s, T fx_d, T fx_by, T fy_d_w, T fy_bz_w, T fy_d, T fy_bz, T e_sw, T e_s,
                         T e_w, T e_c) {
  T emf_l2, emf_r2, emf_l1, emf_r1;
  if (fx_d_s > 0.0) emf_l2 = -fx_by_s + (fy_bz_w - e_sw);
  else if (fx_d_s < 0.0) emf_l2 = -fx_by_s + (fy_bz - e_s);
  else emf_l2 = -fx_by_s + 0.5 * (fy_bz_w - e_sw + fy_bz - e_s);

  if (fx_d > 0.0) emf_r2 = -fx_by + (fy_bz_w - e_w);
  else if (fx_d < 0.0) emf_r2 = -fx_by + (fy_bz - e_c);
  else emf_r2 = -fx_by + 0.5 * (fy_bz_w - e_w + fy_bz - e_c);

  if (fy_d_w > 0.0) emf_l1 = fy_bz_w + (-fx_by_s - e_sw);
  else if (fy_d_w < 0.0) emf_l1 = fy_bz_w + (-fx_by - e_w);
  else emf_l1 = fy_bz_w + 0.5 * (-fx_by_s - e_sw - fx_by - e_w);

  if (fy_d > 0.0) emf_r1 = fy_bz + (-fx_by_s - e_s);
  else if (fy_d < 0.0) emf_r1 = fy_bz + (-fx_by - e_c);
  else emf_r1 = fy_bz + 0.5 * (-fx_by_s - e_s - fx_by - e_c);

  return 0.25 * (emf_l1 + emf_r1 + emf_l2 + emf_r2);
}

template <class T>
ATHB_HD void gen_emf(const GenArgs<T>& a, int full, int j, int i) {
  const int fxp = full ? G_FX2 : G_FX, fyp = full ? G_FY2 : G_FY, ep = full ? G_ECC1 : G_ECC0;
  const long long o = a.o(j, i), os = o - a.pitch;
  a.put(full ? G_EMF1 : G_EMF0, o,
        corner_emf_gen(a.g(fxp + 0, os), a.g(fxp + 5, os), a.g(fxp + 0, o), a.g(fxp + 5, o), a.g(fyp + 0, o - 1),
                       a.g(fyp + 6, o - 1), a.g(fyp + 0, o), a.g(fyp + 6, o), a.g(ep, os - 1), a.g(ep, os),
                       a.g(ep, o - 1), a.g(ep, o)));
}

// ---- 4, 5a, 5b, 8b: corrector flux at x face (j,i) -------------------------
template <int FLUX, class T>
ATHB_HD void gen_correct_x(const GenArgs<T>& a, int j, int i) {
  const StepCoef<T>& c = *a.coef;
  const long long o = a.o(j, i), P = a.pitch;
  // step 4 (src/__integrate_2d__.c:268,271)
  const T b1f = a.s(P_B1I, o) - c.hdtodx2 * (a.g(G_EMF0, o + P) - a.g(G_EMF0, o));
  Cons1T<T> ul = get_cons(a, G_ULX, o);
  Cons1T<T> ur = get_cons(a, G_URX, o);
  // step 5a: x2-flux gradients, (x,y,z) -> (z,x,y) (src/__integrate_2d__.c:284-301)
  {
    const long long on = o + P - 1, oc = o - 1;
    ul.d -= c.hdtodx2 * (a.g(G_FY + 0, on) - a.g(G_FY + 0, oc));
    ul.mx -= c.hdtodx2 * (a.g(G_FY + 3, on) - a.g(G_FY + 3, oc));
    ul.my -= c.hdtodx2 * (a.g(G_FY + 1, on) - a.g(G_FY + 1, oc));
    ul.mz -= c.hdtodx2 * (a.g(G_FY + 2, on) - a.g(G_FY + 2, oc));
    ul.e -= c.hdtodx2 * (a.g(G_FY + 4, on) - a.g(G_FY + 4, oc));
    ul.bz -= c.hdtodx2 * (a.g(G_FY + 5, on) - a.g(G_FY + 5, oc));
  }
  {
    const long long on = o + P, oc = o;
    ur.d -= c.hdtodx2 * (a.g(G_FY + 0, on) - a.g(G_FY + 0, oc));
    ur.mx -= c.hdtodx2 * (a.g(G_FY + 3, on) - a.g(G_FY + 3, oc));
    ur.my -= c.hdtodx2 * (a.g(G_FY + 1, on) - a.g(G_FY + 1, oc));
    ur.mz -= c.hdtodx2 * (a.g(G_FY + 2, on) - a.g(G_FY + 2, oc));
    ur.e -= c.hdtodx2 * (a.g(G_FY + 4, on) - a.g(G_FY + 4, oc));
    ur.bz -= c.hdtodx2 * (a.g(G_FY + 5, on) - a.g(G_FY + 5, oc));
  }
  // step 5b: MHD source terms (src/__integrate_2d__.c:308-333)
  {
    const long long ow = o - 1;
    const T dbx = a.s(P_B1I, o) - a.s(P_B1I, ow);
    const T B1 = a.s(P_B1C, ow), B2 = a.s(P_B2C, ow), B3 = a.s(P_B3C, ow);
    const T V3 = a.s(P_M3, ow) / a.s(P_D, ow);
    ul.mx += c.hdtodx1 * B1 * dbx;
    ul.my += c.hdtodx1 * B2 * dbx;
    ul.mz += c.hdtodx1 * B3 * dbx;
    ul.bz += c.hdtodx1 * V3 * dbx;
    ul.e += c.hdtodx1 * B3 * V3 * dbx;
  }
  {
    const T dbx = a.s(P_B1I, o + 1) - a.s(P_B1I, o);
    const T B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o), B3 = a.s(P_B3C, o);
    const T V3 = a.s(P_M3, o) / a.s(P_D, o);
    ur.mx += c.hdtodx1 * B1 * dbx;
    ur.my += c.hdtodx1 * B2 * dbx;
    ur.mz += c.hdtodx1 * B3 * dbx;
    ur.bz += c.hdtodx1 * V3 * dbx;
    ur.e += c.hdtodx1 * B3 * V3 * dbx;
  }
  // step 8b (src/__integrate_2d__.c:438-447)
  const Prim1T<T> wl = cons_to_prim(ul, b1f, a.eos);
  const Prim1T<T> wr = cons_to_prim(ur, b1f, a.eos);
  put_cons(a, G_FX2, o, riemann<FLUX>(ul, ur, wl, wr, b1f, a.eos));
}

// ---- 4, 6a, 6b, 8c: corrector flux at y face (j,i) -------------------------
template <int FLUX, class T>
ATHB_HD void gen_correct_y(const GenArgs<T>& a, int j, int i) {
  const StepCoef<T>& c = *a.coef;
  const long long o = a.o(j, i), P = a.pitch;
  // step 4 (src/__integrate_2d__.c:269,274)
  const T b2f = a.s(P_B2I, o) + c.hdtodx1 * (a.g(G_EMF0, o + 1) - a.g(G_EMF0, o));
  Cons1T<T> ul = get_cons(a, G_ULY, o);
  Cons1T<T> ur = get_cons(a, G_URY, o);
  // step 6a: x1-flux gradients, (x,y,z) -> (y,z,x) (src/__integrate_2d__.c:343-360)
  {
    const long long oe = o - P + 1, oc = o - P;
    ul.d -= c.hdtodx1 * (a.g(G_FX + 0, oe) - a.g(G_FX + 0, oc));
    ul.mx -= c.hdtodx1 * (a.g(G_FX + 2, oe) - a.g(G_FX + 2, oc));
    ul.my -= c.hdtodx1 * (a.g(G_FX + 3, oe) - a.g(G_FX + 3, oc));
    ul.mz -= c.hdtodx1 * (a.g(G_FX + 1, oe) - a.g(G_FX + 1, oc));
    ul.e -= c.hdtodx1 * (a.g(G_FX + 4, oe) - a.g(G_FX + 4, oc));
    ul.by -= c.hdtodx1 * (a.g(G_FX + 6, oe) - a.g(G_FX + 6, oc));
  }
  {
    const long long oe = o + 1, oc = o;
    ur.d -= c.hdtodx1 * (a.g(G_FX + 0, oe) - a.g(G_FX + 0, oc));
    ur.mx -= c.hdtodx1 * (a.g(G_FX + 2, oe) - a.g(G_FX + 2, oc));
    ur.my -= c.hdtodx1 * (a.g(G_FX + 3, oe) - a.g(G_FX + 3, oc));
    ur.mz -= c.hdtodx1 * (a.g(G_FX + 1, oe) - a.g(G_FX + 1, oc));
    ur.e -= c.hdtodx1 * (a.g(G_FX + 4, oe) - a.g(G_FX + 4, oc));
    ur.by -= c.hdtodx1 * (a.g(G_FX + 6, oe) - a.g(G_FX + 6, oc));
  }
  // step 6b: MHD source terms (src/__integrate_2d__.c:367-392)
  {
    const long long osn = o - P;
    const T dby = a.s(P_B2I, o) - a.s(P_B2I, osn);
    const T B1 = a.s(P_B1C, osn), B2 = a.s(P_B2C, osn), B3 = a.s(P_B3C, osn);
    const T V3 = a.s(P_M3, osn) / a.s(P_D, osn);
    ul.mz += c.hdtodx2 * B1 * dby;
    ul.mx += c.hdtodx2 * B2 * dby;
    ul.my += c.hdtodx2 * B3 * dby;
    ul.by += c.hdtodx2 * V3 * dby;
    ul.e += c.hdtodx2 * B3 * V3 * dby;
  }
  {
    const T dby = a.s(P_B2I, o + P) - a.s(P_B2I, o);
    const T B1 = a.s(P_B1C, o), B2 = a.s(P_B2C, o), B3 = a.s(P_B3C, o);
    const T V3 = a.s(P_M3, o) / a.s(P_D, o);
    ur.mz += c.hdtodx2 * B1 * dby;
    ur.mx += c.hdtodx2 * B2 * dby;
    ur.my += c.hdtodx2 * B3 * dby;
    ur.by += c.hdtodx2 * V3 * dby;
    ur.e += c.hdtodx2 * B3 * V3 * dby;
  }
  // step 8c (src/__integrate_2d__.c:455-464)
  const Prim1T<T> wl = cons_to_prim(ul, b2f, a.eos);
  const Prim1T<T> wr = cons_to_prim(ur, b2f, a.eos);
  put_cons(a, G_FY2, o, riemann<FLUX>(ul, ur, wl, wr, b2f, a.eos));
}

// ---- 7: cell-centred emf3 at t^{n+1/2} (src/__integrate_2d__.c:402-431) -----
template <class T>
ATHB_HD void gen_correct_e(const GenArgs<T>& a, int j, int i) {
  const StepCoef<T>& c = *a.coef;
  const long long o = a.o(j, i), P = a.pitch;
  const T d = a.s(P_D, o) - c.hdtodx1 * (a.g(G_FX + 0, o + 1) - a.g(G_FX + 0, o)) -
              c.hdtodx2 * (a.g(G_FY + 0, o + P) - a.g(G_FY + 0, o));
  const T M1 = a.s(P_M1, o) - c.hdtodx1 * (a.g(G_FX + 1, o + 1) - a.g(G_FX + 1, o)) -
               c.hdtodx2 * (a.g(G_FY + 3, o + P) - a.g(G_FY + 3, o));
  const T M2 = a.s(P_M2, o) - c.hdtodx1 * (a.g(G_FX + 2, o + 1) - a.g(G_FX + 2, o)) -
               c.hdtodx2 * (a.g(G_FY + 1, o + P) - a.g(G_FY + 1, o));
  const T b1f_c = a.s(P_B1I, o) - c.hdtodx2 * (a.g(G_EMF0, o + P) - a.g(G_EMF0, o));
  const T b1f_e = a.s(P_B1I, o + 1) - c.hdtodx2 * (a.g(G_EMF0, o + P + 1) - a.g(G_EMF0, o + 1));
  const T b2f_c = a.s(P_B2I, o) + c.hdtodx1 * (a.g(G_EMF0, o + 1) - a.g(G_EMF0, o));
  const T b2f_n = a.s(P_B2I, o + P) + c.hdtodx1 * (a.g(G_EMF0, o + P + 1) - a.g(G_EMF0, o + P));
  const T B1c = 0.5 * (b1f_c + b1f_e);
  const T B2c = 0.5 * (b2f_c + b2f_n);
  a.put(G_ECC1, o, (B1c * M2 - B2c * M1) / d);
}

// ---- new_dt per cell (src/new_dt.c:37-85; the fast speeds it forms are
// overwritten by the sound speed and are not formed) -------------------------
template <class T>
ATHB_HD T gen_cell_dti(T d, T m1, T m2, T m3, T e, const Eos& eos, double dx1, double dx2) {
  const T di = 1.0 / d;
  const T v1 = m1 * di, v2 = m2 * di, v3 = m3 * di;
  const T qsq = v1 * v1 + v2 * v2 + v3 * v3;
  const T p = rmax(eos.gamma_1 * (e - 0.5 * d * qsq), T(kTiny));
  const T asq = eos.gamma * p * di;
  const T ca = sqrt(asq);
  T m = rmax(T(0.0), (fabs(v1) + ca) / dx1);
  m = rmax(m, (fabs(v2) + ca) / dx2);
  return m;
}

// ---- 9, 11a, 11b, 13: update of interior cell (j,i); returns its CFL rate ---
template <class T>
ATHB_HD T gen_update(const GenArgs<T>& a, int j, int i) {
  const StepCoef<T>& c = *a.coef;
  const long long ps = a.ps, o = a.o(j, i), P = a.pitch;
  const T dtodx1 = c.dtodx1, dtodx2 = c.dtodx2;
  // step 9 (src/__integrate_2d__.c:476-485)
  const T e00 = a.g(G_EMF1, o), e01 = a.g(G_EMF1, o + 1), e10 = a.g(G_EMF1, o + P), e11 = a.g(G_EMF1, o + P + 1);
  const T b1 = a.s(P_B1I, o) - dtodx2 * (e10 - e00);
  const T b1e = a.s(P_B1I, o + 1) - dtodx2 * (e11 - e01);
  const T b2 = a.s(P_B2I, o) + dtodx1 * (e01 - e00);
  const T b2n = a.s(P_B2I, o + P) + dtodx1 * (e11 - e10);
  a.out.set(P_B1I * ps + o, b1);
  if (i == a.ie) a.out.set(P_B1I * ps + o + 1, b1e);
  a.out.set(P_B2I * ps + o, b2);
  if (j == a.je) a.out.set(P_B2I * ps + o + P, b2n);
  // step 11a (src/__integrate_2d__.c:491-501)
  T d = a.s(P_D, o), m1 = a.s(P_M1, o), m2 = a.s(P_M2, o);
  T m3 = a.s(P_M3, o), e = a.s(P_E, o), b3c = a.s(P_B3C, o);
  d -= dtodx1 * (a.g(G_FX2 + 0, o + 1) - a.g(G_FX2 + 0, o));
  m1 -= dtodx1 * (a.g(G_FX2 + 1, o + 1) - a.g(G_FX2 + 1, o));
  m2 -= dtodx1 * (a.g(G_FX2 + 2, o + 1) - a.g(G_FX2 + 2, o));
  m3 -= dtodx1 * (a.g(G_FX2 + 3, o + 1) - a.g(G_FX2 + 3, o));
  e -= dtodx1 * (a.g(G_FX2 + 4, o + 1) - a.g(G_FX2 + 4, o));
  b3c -= dtodx1 * (a.g(G_FX2 + 6, o + 1) - a.g(G_FX2 + 6, o));
  // step 11b (src/__integrate_2d__.c:508-518)
  d -= dtodx2 * (a.g(G_FY2 + 0, o + P) - a.g(G_FY2 + 0, o));
  m1 -= dtodx2 * (a.g(G_FY2 + 3, o + P) - a.g(G_FY2 + 3, o));
  m2 -= dtodx2 * (a.g(G_FY2 + 1, o + P) - a.g(G_FY2 + 1, o));
  m3 -= dtodx2 * (a.g(G_FY2 + 2, o + P) - a.g(G_FY2 + 2, o));
  e -= dtodx2 * (a.g(G_FY2 + 4, o + P) - a.g(G_FY2 + 4, o));
  b3c -= dtodx2 * (a.g(G_FY2 + 5, o + P) - a.g(G_FY2 + 5, o));
  a.out.set(P_D * ps + o, d);
  a.out.set(P_M1 * ps + o, m1);
  a.out.set(P_M2 * ps + o, m2);
  a.out.set(P_M3 * ps + o, m3);
  a.out.set(P_E * ps + o, e);
  // step 13 (src/__integrate_2d__.c:526-534)
  a.out.set(P_B1C * ps + o, 0.5 * (b1 + b1e));
  a.out.set(P_B2C * ps + o, 0.5 * (b2 + b2n));
  a.out.set(P_B3C * ps + o, b3c);
  a.out.set(P_B3I * ps + o, b3c);
  return gen_cell_dti(d, m1, m2, m3, e, a.eos, a.dx1, a.dx2);
}

}  // namespace athb
