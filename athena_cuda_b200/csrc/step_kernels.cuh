// step_kernels.cuh -- sm_100a kernels for one CTU+CT step of the 2D ideal-MHD
// solver, its CFL reduction and its ghost-zone fill.
//
// Data layout in HBM (one grid): structure-of-arrays FP64 planes of
// (Nx2+8) rows x pitch doubles, pitch = Nx1+8 rounded up to 16 doubles so that
// every row starts on a 128-byte boundary.  The state (11 planes: d, M1, M2, M3,
// E, B1c, B2c, B3c, B1i, B2i, B3i) is double-buffered: a step reads buffer A
// everywhere and writes the interior of buffer B; the ghost kernel then fills
// B's ghosts from B's interior.  Face scratch planes hold the predictor L/R
// states and fluxes of both sweeps, the corrector fluxes and two EMF planes.
//
// One step (reference src/__integrate_2d__.c:100-537, src/main.c:229-307):
//   k_predict   role X: steps 1a-1e   (x-sweep: prims, PLM, MHD source, Roe)
//               role Y: steps 2a-2e   (y-sweep, marching along x2)
//   k_emf_half  steps 3-4             (upwind corner EMF at t^n)
//   k_correct   role X: 4,5a,5b,8b    (half-step face field, transverse
//                                      correction, source terms, corrector flux)
//               role Y: 4,6a,6b,8c
//               role E: 7             (cell-centred EMF at t^{n+1/2})
//   k_emf_full  step 9 corner EMF
//   k_update    steps 9 (CT), 11a, 11b, 13 + new_dt per cell (src/new_dt.c)
//               with warp-shuffle / block max and one 64-bit atomicMax
//   k_finalize  time += dt, nstep++, dt rule (src/new_dt.c:93-97), tlim clamp
//               (src/main.c:230-232)
//   k_ghost     set_bvals (src/set_bvals.c:114-1031) for both directions in
//               one pass through composed index maps
#pragma once

#include <cstdint>
#include "step_types.cuh"

namespace athb {

__device__ __forceinline__ long long off(const GridArgs& g, int j, int i) {
  return (long long)j * g.pitch + i;
}

// ---------------------------------------------------------------------------
// Slice loads
// ---------------------------------------------------------------------------
// x-sweep conserved vector (d, M1, M2, M3, E, B2c, B3c), normal field B1c
// (src/__integrate_2d__.c:130-139)
__device__ __forceinline__ Prim1 prim_x(const GridArgs& g, const double* s, long long o) {
  Cons1 u;
  u.d = s[P_D * g.ps + o]; u.mx = s[P_M1 * g.ps + o]; u.my = s[P_M2 * g.ps + o];
  u.mz = s[P_M3 * g.ps + o]; u.e = s[P_E * g.ps + o];
  u.by = s[P_B2C * g.ps + o]; u.bz = s[P_B3C * g.ps + o];
  return cons_to_prim(u, s[P_B1C * g.ps + o], g.eos);
}
// y-sweep conserved vector (d, M2, M3, M1, E, B3c, B1c), normal field B2c
// (src/__integrate_2d__.c:191-201)
__device__ __forceinline__ Prim1 prim_y(const GridArgs& g, const double* s, long long o) {
  Cons1 u;
  u.d = s[P_D * g.ps + o]; u.mx = s[P_M2 * g.ps + o]; u.my = s[P_M3 * g.ps + o];
  u.mz = s[P_M1 * g.ps + o]; u.e = s[P_E * g.ps + o];
  u.by = s[P_B3C * g.ps + o]; u.bz = s[P_B1C * g.ps + o];
  return cons_to_prim(u, s[P_B2C * g.ps + o], g.eos);
}

__device__ __forceinline__ Prim1 shfl_prim(unsigned mask, const Prim1& w, int delta, bool up) {
  Prim1 r;
  if (up) {
    r.d = __shfl_up_sync(mask, w.d, delta); r.vx = __shfl_up_sync(mask, w.vx, delta);
    r.vy = __shfl_up_sync(mask, w.vy, delta); r.vz = __shfl_up_sync(mask, w.vz, delta);
    r.p = __shfl_up_sync(mask, w.p, delta); r.by = __shfl_up_sync(mask, w.by, delta);
    r.bz = __shfl_up_sync(mask, w.bz, delta);
  } else {
    r.d = __shfl_down_sync(mask, w.d, delta); r.vx = __shfl_down_sync(mask, w.vx, delta);
    r.vy = __shfl_down_sync(mask, w.vy, delta); r.vz = __shfl_down_sync(mask, w.vz, delta);
    r.p = __shfl_down_sync(mask, w.p, delta); r.by = __shfl_down_sync(mask, w.by, delta);
    r.bz = __shfl_down_sync(mask, w.bz, delta);
  }
  return r;
}

__device__ __forceinline__ void store_cons(double* base, long long ps, long long o, const Cons1& u) {
  base[0 * ps + o] = u.d; base[1 * ps + o] = u.mx; base[2 * ps + o] = u.my; base[3 * ps + o] = u.mz;
  base[4 * ps + o] = u.e; base[5 * ps + o] = u.by; base[6 * ps + o] = u.bz;
}
__device__ __forceinline__ Cons1 load_cons(const double* base, long long ps, long long o) {
  Cons1 u;
  u.d = base[0 * ps + o]; u.mx = base[1 * ps + o]; u.my = base[2 * ps + o]; u.mz = base[3 * ps + o];
  u.e = base[4 * ps + o]; u.by = base[5 * ps + o]; u.bz = base[6 * ps + o];
  return u;
}

// Launch geometry shared by the host launcher and the kernels.
constexpr int kThreads = 128;
constexpr int kXFacesPerWarp = 31;              // 32 PLM cells -> 31 faces

// Role X: a warp per 31-face row segment, four rows per block.  Role Y: one
// thread per (column, segment of ly faces), flattened column-fastest over
// the blocks so that narrow grids leave no idle columns.
struct PredictGeom {
  int xseg, xrowblk, nx_blocks;  // role X blocks = xseg * xrowblk
  int ycols, yseg, ny_blocks;    // role Y threads = ycols * yseg, in ny_blocks blocks
};

// Faces [is-1, ie+2] x rows [js-2, je+2] (role X) and columns [is-2, ie+2]
// x faces [js-1, je+2] (role Y) of an nx1 x nx2 interior, in blocks of nt
// threads (a multiple of 32; the single-grid kernels use kThreads).
inline PredictGeom make_predict_geom(int nx1, int nx2, int ly, int nt = kThreads) {
  PredictGeom pg;
  const int rows_per_block = nt / 32;
  pg.xseg = (nx1 + 3 + kXFacesPerWarp - 1) / kXFacesPerWarp;
  pg.xrowblk = (nx2 + 4 + rows_per_block - 1) / rows_per_block;
  pg.nx_blocks = pg.xseg * pg.xrowblk;
  pg.ycols = nx1 + 4;
  pg.yseg = (nx2 + 3 + ly - 1) / ly;
  pg.ny_blocks = (int)(((long long)pg.ycols * pg.yseg + nt - 1) / nt);
  return pg;
}

// ---------------------------------------------------------------------------
// k_predict: predictor L/R states and fluxes of both sweeps.
// ---------------------------------------------------------------------------
// TAPE: also keep the face states W_L, W_R of every predictor face in the
// T_WLN* / T_WRT* planes (the recorded step of the adjoint).
__device__ __forceinline__ void store_prim(double* base, long long ps, long long o, const Prim1& w) {
  base[0 * ps + o] = w.d; base[1 * ps + o] = w.vx; base[2 * ps + o] = w.vy; base[3 * ps + o] = w.vz;
  base[4 * ps + o] = w.p; base[5 * ps + o] = w.by; base[6 * ps + o] = w.bz;
}

template <int FLUX, bool TAPE = false, int NT = kThreads>
__device__ __forceinline__ void predict_x(const GridArgs& g, int bx, int by) {
  const StepState& st = *g.st;
  const int lane = threadIdx.x & 31;
  const int j = g.js - 2 + by * (NT / 32) + (threadIdx.x >> 5);
  if (j > g.je + 2) return;                        // warp-uniform
  const int c = g.is - 2 + bx * kXFacesPerWarp + lane;
  const int ce = c < g.ie + 3 ? c : g.ie + 3;      // keep c+1 inside the array
  const double* s = g.in;
  const long long o = off(g, j, ce);

  const Prim1 w0 = prim_x(g, s, o);
  Prim1 wm = shfl_prim(0xffffffffu, w0, 1, true);
  Prim1 wp = shfl_prim(0xffffffffu, w0, 1, false);
  if (lane == 0) wm = prim_x(g, s, o - 1);
  if (lane == 31) wp = prim_x(g, s, o + 1);

  Prim1 wln, wrt;
  plm_cell(wm, w0, wp, s[P_B1C * g.ps + o], st.dtodx1, g.eos, wln, wrt);

  // "MHD source terms" for 0.5*dt (src/__integrate_2d__.c:156-164)
  const double d0 = s[P_D * g.ps + o];
  const double b1l = s[P_B1I * g.ps + o], b1r = s[P_B1I * g.ps + o + 1];
  const double src = (s[P_M2 * g.ps + o] / d0) * (b1r - b1l) / g.dx1;
  wln.by += st.hdt * src;
  wrt.by += st.hdt * src;

  const Prim1 wl = shfl_prim(0xffffffffu, wln, 1, true);  // W_L of face c
  if (lane >= 1 && c <= g.ie + 2) {
    // step 1e (src/__integrate_2d__.c:172-180)
    const Cons1 ul = prim_to_cons(wl, b1l, g.eos);
    const Cons1 ur = prim_to_cons(wrt, b1l, g.eos);
    store_cons(g.scr + S_ULX * g.ps, g.ps, o, ul);
    store_cons(g.scr + S_URX * g.ps, g.ps, o, ur);
    store_cons(g.scr + S_FX * g.ps, g.ps, o, riemann<FLUX>(ul, ur, wl, wrt, b1l, g.eos));
    if constexpr (TAPE) {
      store_prim(g.scr + T_WLNX * g.ps, g.ps, o - 1, wl);
      store_prim(g.scr + T_WRTX * g.ps, g.ps, o, wrt);
    }
  }
  // step 3: emf3_cc at t^n on [is-2,ie+2] x [js-2,je+2] (src/__integrate_2d__.c:249-255)
  if ((lane >= 1 || bx == 0) && c <= g.ie + 2) {
    g.scr[S_ECC * g.ps + o] =
        (s[P_B1C * g.ps + o] * s[P_M2 * g.ps + o] - s[P_B2C * g.ps + o] * s[P_M1 * g.ps + o]) / d0;
  }
}

// The y role carries three cell states and one face state from row to row;
// they live in a per-thread ring in shared memory rather than in registers.
template <int NT = kThreads>
__device__ __forceinline__ void sh_store(double* sh, int slot, int tid, const Prim1& w) {
  double* p = sh + slot * 7 * NT + tid;
  p[0 * NT] = w.d; p[1 * NT] = w.vx; p[2 * NT] = w.vy; p[3 * NT] = w.vz;
  p[4 * NT] = w.p; p[5 * NT] = w.by; p[6 * NT] = w.bz;
}
template <int NT = kThreads>
__device__ __forceinline__ Prim1 sh_load(const double* sh, int slot, int tid) {
  const double* p = sh + slot * 7 * NT + tid;
  Prim1 w;
  w.d = p[0 * NT]; w.vx = p[1 * NT]; w.vy = p[2 * NT]; w.vz = p[3 * NT];
  w.p = p[4 * NT]; w.by = p[5 * NT]; w.bz = p[6 * NT];
  return w;
}

template <int FLUX, bool TAPE = false, int NT = kThreads>
__device__ __forceinline__ void predict_y(const GridArgs& g, const PredictGeom& pg, int b) {
  // slots 0..2: prims of rows k-1, k, k+1 (ring); slot 3: W_L of face k.
  // Above 128 threads the ring (4 x 7 x NT doubles) exceeds the 48 KB of
  // static shared memory: the launch supplies it as dynamic shared memory.
  double* sh;
  if constexpr (NT <= 128) {
    __shared__ double sh_static[4 * 7 * NT];
    sh = sh_static;
  } else {
    extern __shared__ double sh_dynamic[];
    sh = sh_dynamic;
  }
  const StepState& st = *g.st;
  const int tid = threadIdx.x;
  const int T = b * NT + tid;
  if (T >= pg.ycols * pg.yseg) return;
  const int i = g.is - 2 + T % pg.ycols;
  const int ja = g.js - 1 + (T / pg.ycols) * g.ly;
  const int jb = min(ja + g.ly - 1, g.je + 2);
  const double* s = g.in;

  sh_store<NT>(sh, 0, tid, prim_y(g, s, off(g, ja - 2, i)));
  sh_store<NT>(sh, 1, tid, prim_y(g, s, off(g, ja - 1, i)));
  int r0 = 0;  // ring slot of row k-1
  for (int k = ja - 1; k <= jb; k++) {
    const long long o = off(g, k, i);
    const int r1 = r0 == 2 ? 0 : r0 + 1, r2 = r1 == 2 ? 0 : r1 + 1;
    sh_store<NT>(sh, r2, tid, prim_y(g, s, o + g.pitch));
    Prim1 wln, wrt;
    plm_cell(sh_load<NT>(sh, r0, tid), sh_load<NT>(sh, r1, tid), sh_load<NT>(sh, r2, tid), s[P_B2C * g.ps + o],
             st.dtodx2, g.eos, wln, wrt);
    // "MHD source terms" for 0.5*dt (src/__integrate_2d__.c:216-224)
    const double b2l = s[P_B2I * g.ps + o], b2r = s[P_B2I * g.ps + o + g.pitch];
    const double src = (s[P_M1 * g.ps + o] / s[P_D * g.ps + o]) * (b2r - b2l) / g.dx2;
    wln.bz += st.hdt * src;
    wrt.bz += st.hdt * src;
    if (k >= ja) {
      // step 2e (src/__integrate_2d__.c:233-241)
      const Prim1 wl = sh_load<NT>(sh, 3, tid);
      const Cons1 ul = prim_to_cons(wl, b2l, g.eos);
      const Cons1 ur = prim_to_cons(wrt, b2l, g.eos);
      store_cons(g.scr + S_ULY * g.ps, g.ps, o, ul);
      store_cons(g.scr + S_URY * g.ps, g.ps, o, ur);
      store_cons(g.scr + S_FY * g.ps, g.ps, o, riemann<FLUX>(ul, ur, wl, wrt, b2l, g.eos));
      if constexpr (TAPE) {
        store_prim(g.scr + T_WLNY * g.ps, g.ps, o - g.pitch, wl);
        store_prim(g.scr + T_WRTY * g.ps, g.ps, o, wrt);
      }
    }
    sh_store<NT>(sh, 3, tid, wln);
    r0 = r1;
  }
}

// Resident blocks per SM the heavy kernels are compiled for (register caps of
// 168 and 128 per thread): measured faster on B200 than the uncapped 255
// registers and 2 blocks per SM despite the spills they cause.
#ifndef ATHB_PREDICT_MIN_BLOCKS
#define ATHB_PREDICT_MIN_BLOCKS 3
#endif
#ifndef ATHB_CORRECT_MIN_BLOCKS
#define ATHB_CORRECT_MIN_BLOCKS 4
#endif
constexpr int kPredictMinBlocks = ATHB_PREDICT_MIN_BLOCKS;
constexpr int kCorrectMinBlocks = ATHB_CORRECT_MIN_BLOCKS;

// Block b of the predictor: the long role-Y column marches (ly rows each)
// come first and the short role-X row segments (31 faces) last, so the
// block scheduler ends the launch on small blocks instead of a tail of
// marches.
template <int FLUX, bool TAPE = false, int NT = kThreads>
__device__ __forceinline__ void predict_block(const GridArgs& g, const PredictGeom& pg, int b) {
  if (b < pg.ny_blocks) {
    predict_y<FLUX, TAPE, NT>(g, pg, b);
  } else {
    b -= pg.ny_blocks;
    predict_x<FLUX, TAPE, NT>(g, b % pg.xseg, b / pg.xseg);
  }
}

template <int FLUX, bool TAPE = false>
static __global__ void __launch_bounds__(kThreads, kPredictMinBlocks) k_predict(GridArgs g, PredictGeom pg) {
  if (g.st->done) return;
  predict_block<FLUX, TAPE>(g, pg, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Upwind corner EMF (src/__integrate_2d__.c:632-702) from x1-fluxes (component
// By = -E3), x2-fluxes (component Bz = +E3) and cell-centred emf3.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double corner_emf(const GridArgs& g, const double* fx, const double* fy,
                                             const double* ecc, int j, int i) {
  const long long ps = g.ps;
  const long long o = off(g, j, i), os = o - g.pitch;       // (j,i), (j-1,i)
  const double fx_d_s = fx[0 * ps + os], fx_by_s = fx[5 * ps + os];  // x1Flux[j-1][i]
  const double fx_d = fx[0 * ps + o], fx_by = fx[5 * ps + o];        // x1Flux[j][i]
  const double fy_d_w = fy[0 * ps + o - 1], fy_bz_w = fy[6 * ps + o - 1];  // x2Flux[j][i-1]
  const double fy_d = fy[0 * ps + o], fy_bz = fy[6 * ps + o];              // x2Flux[j][i]
  const double e_sw = ecc[os - 1], e_s = ecc[os], e_w = ecc[o - 1], e_c = ecc[o];

  double emf_l2, emf_r2, emf_l1, emf_r1;
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

// Corner EMF over [i0, i0+ni) x [j0, j0+nj): work item t.
__device__ __forceinline__ void emf_item(const GridArgs& g, int i0, int j0, int ni, int nj, int fx_plane,
                                         int fy_plane, int t) {
  if (t >= ni * nj) return;
  const int j = j0 + t / ni, i = i0 + t % ni;
  g.scr[S_EMF * g.ps + off(g, j, i)] =
      corner_emf(g, g.scr + fx_plane * g.ps, g.scr + fy_plane * g.ps, g.scr + S_ECC * g.ps, j, i);
}

static __global__ void __launch_bounds__(kThreads) k_emf(GridArgs g, int i0, int j0, int ni, int nj,
                                                  int fx_plane, int fy_plane) {
  if (g.st->done) return;
  emf_item(g, i0, j0, ni, nj, fx_plane, fy_plane, blockIdx.x * kThreads + threadIdx.x);
}

// ---------------------------------------------------------------------------
// k_correct: corrector fluxes of both directions and the half-step cell EMF.
// ---------------------------------------------------------------------------
struct CorrectGeom {
  int xw, xn;   // role X: faces [is, ie+1] x [js-1, je+1]
  int yw, yn;   // role Y: faces [is-1, ie+1] x [js, je+1]
  int ew, en;   // role E: cells [is-1, ie+1] x [js-1, je+1]
  int xb, yb, eb;
};

template <int FLUX>
__device__ __forceinline__ void correct_x(const GridArgs& g, int t, int w) {
  const StepState& st = *g.st;
  const int j = g.js - 1 + t / w, i = g.is + t % w;
  const long long ps = g.ps, o = off(g, j, i);
  const double* s = g.in;
  const double* emf = g.scr + S_EMF * ps;
  // step 4: half-step CT on the x1-face field (src/__integrate_2d__.c:268,271)
  const double b1f = s[P_B1I * ps + o] - st.hdtodx2 * (emf[o + g.pitch] - emf[o]);

  // step 5a: transverse x2-flux gradients, (x,y,z) -> (z,x,y)
  const double* fy = g.scr + S_FY * ps;
  Cons1 ul = load_cons(g.scr + S_ULX * ps, ps, o);
  Cons1 ur = load_cons(g.scr + S_URX * ps, ps, o);
  {
    const long long on = o + g.pitch - 1, oc = o - 1;  // x2Flux[j+1][i-1], x2Flux[j][i-1]
    ul.d -= st.hdtodx2 * (fy[0 * ps + on] - fy[0 * ps + oc]);
    ul.mx -= st.hdtodx2 * (fy[3 * ps + on] - fy[3 * ps + oc]);
    ul.my -= st.hdtodx2 * (fy[1 * ps + on] - fy[1 * ps + oc]);
    ul.mz -= st.hdtodx2 * (fy[2 * ps + on] - fy[2 * ps + oc]);
    ul.e -= st.hdtodx2 * (fy[4 * ps + on] - fy[4 * ps + oc]);
    ul.bz -= st.hdtodx2 * (fy[5 * ps + on] - fy[5 * ps + oc]);
  }
  {
    const long long on = o + g.pitch, oc = o;
    ur.d -= st.hdtodx2 * (fy[0 * ps + on] - fy[0 * ps + oc]);
    ur.mx -= st.hdtodx2 * (fy[3 * ps + on] - fy[3 * ps + oc]);
    ur.my -= st.hdtodx2 * (fy[1 * ps + on] - fy[1 * ps + oc]);
    ur.mz -= st.hdtodx2 * (fy[2 * ps + on] - fy[2 * ps + oc]);
    ur.e -= st.hdtodx2 * (fy[4 * ps + on] - fy[4 * ps + oc]);
    ur.bz -= st.hdtodx2 * (fy[5 * ps + on] - fy[5 * ps + oc]);
  }
  // step 5b: MHD source terms (src/__integrate_2d__.c:308-333)
  {
    const long long ow = o - 1;
    const double dbx = s[P_B1I * ps + o] - s[P_B1I * ps + ow];
    const double B1 = s[P_B1C * ps + ow], B2 = s[P_B2C * ps + ow], B3 = s[P_B3C * ps + ow];
    const double V3 = s[P_M3 * ps + ow] / s[P_D * ps + ow];
    ul.mx += st.hdtodx1 * B1 * dbx;
    ul.my += st.hdtodx1 * B2 * dbx;
    ul.mz += st.hdtodx1 * B3 * dbx;
    ul.bz += st.hdtodx1 * V3 * dbx;
    ul.e += st.hdtodx1 * B3 * V3 * dbx;
  }
  {
    const double dbx = s[P_B1I * ps + o + 1] - s[P_B1I * ps + o];
    const double B1 = s[P_B1C * ps + o], B2 = s[P_B2C * ps + o], B3 = s[P_B3C * ps + o];
    const double V3 = s[P_M3 * ps + o] / s[P_D * ps + o];
    ur.mx += st.hdtodx1 * B1 * dbx;
    ur.my += st.hdtodx1 * B2 * dbx;
    ur.mz += st.hdtodx1 * B3 * dbx;
    ur.bz += st.hdtodx1 * V3 * dbx;
    ur.e += st.hdtodx1 * B3 * V3 * dbx;
  }
  // step 8b (src/__integrate_2d__.c:438-447)
  const Prim1 wl = cons_to_prim(ul, b1f, g.eos);
  const Prim1 wr = cons_to_prim(ur, b1f, g.eos);
  store_cons(g.scr + S_FX2 * ps, ps, o, riemann<FLUX>(ul, ur, wl, wr, b1f, g.eos));
}

template <int FLUX>
__device__ __forceinline__ void correct_y(const GridArgs& g, int t, int w) {
  const StepState& st = *g.st;
  const int j = g.js + t / w, i = g.is - 1 + t % w;
  const long long ps = g.ps, o = off(g, j, i);
  const double* s = g.in;
  const double* emf = g.scr + S_EMF * ps;
  // step 4: half-step CT on the x2-face field (src/__integrate_2d__.c:269,274)
  const double b2f = s[P_B2I * ps + o] + st.hdtodx1 * (emf[o + 1] - emf[o]);

  // step 6a: transverse x1-flux gradients, (x,y,z) -> (y,z,x)
  const double* fx = g.scr + S_FX * ps;
  Cons1 ul = load_cons(g.scr + S_ULY * ps, ps, o);
  Cons1 ur = load_cons(g.scr + S_URY * ps, ps, o);
  {
    const long long oe = o - g.pitch + 1, oc = o - g.pitch;  // x1Flux[j-1][i+1], x1Flux[j-1][i]
    ul.d -= st.hdtodx1 * (fx[0 * ps + oe] - fx[0 * ps + oc]);
    ul.mx -= st.hdtodx1 * (fx[2 * ps + oe] - fx[2 * ps + oc]);
    ul.my -= st.hdtodx1 * (fx[3 * ps + oe] - fx[3 * ps + oc]);
    ul.mz -= st.hdtodx1 * (fx[1 * ps + oe] - fx[1 * ps + oc]);
    ul.e -= st.hdtodx1 * (fx[4 * ps + oe] - fx[4 * ps + oc]);
    ul.by -= st.hdtodx1 * (fx[6 * ps + oe] - fx[6 * ps + oc]);
  }
  {
    const long long oe = o + 1, oc = o;
    ur.d -= st.hdtodx1 * (fx[0 * ps + oe] - fx[0 * ps + oc]);
    ur.mx -= st.hdtodx1 * (fx[2 * ps + oe] - fx[2 * ps + oc]);
    ur.my -= st.hdtodx1 * (fx[3 * ps + oe] - fx[3 * ps + oc]);
    ur.mz -= st.hdtodx1 * (fx[1 * ps + oe] - fx[1 * ps + oc]);
    ur.e -= st.hdtodx1 * (fx[4 * ps + oe] - fx[4 * ps + oc]);
    ur.by -= st.hdtodx1 * (fx[6 * ps + oe] - fx[6 * ps + oc]);
  }
  // step 6b: MHD source terms (src/__integrate_2d__.c:367-392)
  {
    const long long osn = o - g.pitch;
    const double dby = s[P_B2I * ps + o] - s[P_B2I * ps + osn];
    const double B1 = s[P_B1C * ps + osn], B2 = s[P_B2C * ps + osn], B3 = s[P_B3C * ps + osn];
    const double V3 = s[P_M3 * ps + osn] / s[P_D * ps + osn];
    ul.mz += st.hdtodx2 * B1 * dby;
    ul.mx += st.hdtodx2 * B2 * dby;
    ul.my += st.hdtodx2 * B3 * dby;
    ul.by += st.hdtodx2 * V3 * dby;
    ul.e += st.hdtodx2 * B3 * V3 * dby;
  }
  {
    const double dby = s[P_B2I * ps + o + g.pitch] - s[P_B2I * ps + o];
    const double B1 = s[P_B1C * ps + o], B2 = s[P_B2C * ps + o], B3 = s[P_B3C * ps + o];
    const double V3 = s[P_M3 * ps + o] / s[P_D * ps + o];
    ur.mz += st.hdtodx2 * B1 * dby;
    ur.mx += st.hdtodx2 * B2 * dby;
    ur.my += st.hdtodx2 * B3 * dby;
    ur.by += st.hdtodx2 * V3 * dby;
    ur.e += st.hdtodx2 * B3 * V3 * dby;
  }
  // step 8c (src/__integrate_2d__.c:455-464)
  const Prim1 wl = cons_to_prim(ul, b2f, g.eos);
  const Prim1 wr = cons_to_prim(ur, b2f, g.eos);
  store_cons(g.scr + S_FY2 * ps, ps, o, riemann<FLUX>(ul, ur, wl, wr, b2f, g.eos));
}

// step 7: cell-centred emf3 at t^{n+1/2} (src/__integrate_2d__.c:402-431)
__device__ __forceinline__ void correct_e(const GridArgs& g, int t, int w) {
  const StepState& st = *g.st;
  const int j = g.js - 1 + t / w, i = g.is - 1 + t % w;
  const long long ps = g.ps, o = off(g, j, i), P = g.pitch;
  const double* s = g.in;
  const double* fx = g.scr + S_FX * ps;
  const double* fy = g.scr + S_FY * ps;
  const double* emf = g.scr + S_EMF * ps;
  const double d = s[P_D * ps + o]
      - st.hdtodx1 * (fx[0 * ps + o + 1] - fx[0 * ps + o])
      - st.hdtodx2 * (fy[0 * ps + o + P] - fy[0 * ps + o]);
  const double M1 = s[P_M1 * ps + o]
      - st.hdtodx1 * (fx[1 * ps + o + 1] - fx[1 * ps + o])
      - st.hdtodx2 * (fy[3 * ps + o + P] - fy[3 * ps + o]);
  const double M2 = s[P_M2 * ps + o]
      - st.hdtodx1 * (fx[2 * ps + o + 1] - fx[2 * ps + o])
      - st.hdtodx2 * (fy[1 * ps + o + P] - fy[1 * ps + o]);
  // half-step face fields, exactly as step 4 forms them
  const double b1f_c = s[P_B1I * ps + o] - st.hdtodx2 * (emf[o + P] - emf[o]);
  const double b1f_e = s[P_B1I * ps + o + 1] - st.hdtodx2 * (emf[o + P + 1] - emf[o + 1]);
  const double b2f_c = s[P_B2I * ps + o] + st.hdtodx1 * (emf[o + 1] - emf[o]);
  const double b2f_n = s[P_B2I * ps + o + P] + st.hdtodx1 * (emf[o + P + 1] - emf[o + P]);
  const double B1c = 0.5 * (b1f_c + b1f_e);
  const double B2c = 0.5 * (b2f_c + b2f_n);
  // written to the scratch ECC plane: the t^n values were consumed by k_emf
  g.scr[S_ECC * ps + o] = (B1c * M2 - B2c * M1) / d;
}

template <int FLUX, int NT = kThreads>
__device__ __forceinline__ void correct_block(const GridArgs& g, const CorrectGeom& cg, int b) {
  if (b < cg.xb) {
    const int t = b * NT + threadIdx.x;
    if (t < cg.xw * cg.xn) correct_x<FLUX>(g, t, cg.xw);
  } else if (b < cg.xb + cg.yb) {
    const int t = (b - cg.xb) * NT + threadIdx.x;
    if (t < cg.yw * cg.yn) correct_y<FLUX>(g, t, cg.yw);
  } else {
    const int t = (b - cg.xb - cg.yb) * NT + threadIdx.x;
    if (t < cg.ew * cg.en) correct_e(g, t, cg.ew);
  }
}

template <int FLUX>
static __global__ void __launch_bounds__(kThreads, kCorrectMinBlocks) k_correct(GridArgs g, CorrectGeom cg) {
  if (g.st->done) return;
  correct_block<FLUX>(g, cg, blockIdx.x);
}

// ---------------------------------------------------------------------------
// new_dt for one cell (src/new_dt.c:37-85).  The magnetic fast speeds the
// reference computes are overwritten by the sound speed (src/new_dt.c:66-77)
// and are therefore not formed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double cell_dti(double d, double m1, double m2, double m3, double e,
                                           const Eos& eos, double dx1, double dx2) {
  const double di = 1.0 / d;
  const double v1 = m1 * di, v2 = m2 * di, v3 = m3 * di;
  const double qsq = v1 * v1 + v2 * v2 + v3 * v3;
  const double p = rmax(eos.gamma_1 * (e - 0.5 * d * qsq), kTiny);
  const double asq = eos.gamma * p * di;
  const double ca = sqrt(asq);
  double m = rmax(0.0, (fabs(v1) + ca) / dx1);
  m = rmax(m, (fabs(v2) + ca) / dx2);
  return m;
}

// Block max of a non-negative double, then one atomicMax on its bit pattern
// (blocks of NT threads).
template <int NT = kThreads>
__device__ __forceinline__ void block_max_to(double v, unsigned long long* dst, int* flags) {
  __shared__ double red[NT / 32];
  if (!(v >= 0.0) || isinf(v)) { atomicOr(flags, kErrNonFinite); v = 0.0; }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, d));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
#pragma unroll
    for (int k = 1; k < NT / 32; k++) m = fmax(m, red[k]);
    atomicMax(dst, (unsigned long long)__double_as_longlong(m));
  }
}

__device__ __forceinline__ double update_cell(const GridArgs& g, int nx1, int ncell, int t);

// ---------------------------------------------------------------------------
// k_update: CT on the face fields, conservative update, cell-centred B and the
// per-cell CFL rate.  One thread per interior cell.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(kThreads) k_update(GridArgs g, int nx1, int ncell) {
  const StepState& st = *g.st;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (st.done) {
    // the loop has ended: carry the state over unchanged so that the buffer
    // parity of later (no-op) steps stays consistent
    if (t < ncell) {
      const int j = g.js + t / nx1, i = g.is + t % nx1;
      const long long o = off(g, j, i);
      for (int p = 0; p < NSTATE; p++) g.out[p * g.ps + o] = g.in[p * g.ps + o];
      if (i == g.ie) g.out[P_B1I * g.ps + o + 1] = g.in[P_B1I * g.ps + o + 1];
      if (j == g.je) g.out[P_B2I * g.ps + o + g.pitch] = g.in[P_B2I * g.ps + o + g.pitch];
    }
    return;
  }
  block_max_to(update_cell(g, nx1, ncell, t), &g.st->max_dti_bits, &g.st->flags);
}

// CT, conservative update and cell-centred field of interior cell t; returns
// the cell's CFL rate (0 for t >= ncell).
__device__ __forceinline__ double update_cell(const GridArgs& g, int nx1, int ncell, int t) {
  const StepState& st = *g.st;
  double dti = 0.0;
  if (t < ncell) {
    const int j = g.js + t / nx1, i = g.is + t % nx1;
    const long long ps = g.ps, o = off(g, j, i), P = g.pitch;
    const double* s = g.in;
    double* out = g.out;
    const double* emf = g.scr + S_EMF * ps;
    const double* fx = g.scr + S_FX2 * ps;
    const double* fy = g.scr + S_FY2 * ps;
    const double dtodx1 = st.dtodx1, dtodx2 = st.dtodx2;
    // step 9: CT for a full step (src/__integrate_2d__.c:476-485)
    const double e00 = emf[o], e01 = emf[o + 1], e10 = emf[o + P], e11 = emf[o + P + 1];
    const double b1 = s[P_B1I * ps + o] - dtodx2 * (e10 - e00);
    const double b1e = s[P_B1I * ps + o + 1] - dtodx2 * (e11 - e01);
    const double b2 = s[P_B2I * ps + o] + dtodx1 * (e01 - e00);
    const double b2n = s[P_B2I * ps + o + P] + dtodx1 * (e11 - e10);
    out[P_B1I * ps + o] = b1;
    if (i == g.ie) out[P_B1I * ps + o + 1] = b1e;
    out[P_B2I * ps + o] = b2;
    if (j == g.je) out[P_B2I * ps + o + P] = b2n;
    // step 11a (src/__integrate_2d__.c:491-501)
    double d = s[P_D * ps + o], m1 = s[P_M1 * ps + o], m2 = s[P_M2 * ps + o];
    double m3 = s[P_M3 * ps + o], e = s[P_E * ps + o], b3c = s[P_B3C * ps + o];
    d -= dtodx1 * (fx[0 * ps + o + 1] - fx[0 * ps + o]);
    m1 -= dtodx1 * (fx[1 * ps + o + 1] - fx[1 * ps + o]);
    m2 -= dtodx1 * (fx[2 * ps + o + 1] - fx[2 * ps + o]);
    m3 -= dtodx1 * (fx[3 * ps + o + 1] - fx[3 * ps + o]);
    e -= dtodx1 * (fx[4 * ps + o + 1] - fx[4 * ps + o]);
    b3c -= dtodx1 * (fx[6 * ps + o + 1] - fx[6 * ps + o]);
    // step 11b (src/__integrate_2d__.c:508-518); the B1c/B2c updates of 11a/11b
    // are overwritten by step 13 and are not formed
    d -= dtodx2 * (fy[0 * ps + o + P] - fy[0 * ps + o]);
    m1 -= dtodx2 * (fy[3 * ps + o + P] - fy[3 * ps + o]);
    m2 -= dtodx2 * (fy[1 * ps + o + P] - fy[1 * ps + o]);
    m3 -= dtodx2 * (fy[2 * ps + o + P] - fy[2 * ps + o]);
    e -= dtodx2 * (fy[4 * ps + o + P] - fy[4 * ps + o]);
    b3c -= dtodx2 * (fy[5 * ps + o + P] - fy[5 * ps + o]);
    out[P_D * ps + o] = d;
    out[P_M1 * ps + o] = m1;
    out[P_M2 * ps + o] = m2;
    out[P_M3 * ps + o] = m3;
    out[P_E * ps + o] = e;
    // step 13 (src/__integrate_2d__.c:526-534)
    out[P_B1C * ps + o] = 0.5 * (b1 + b1e);
    out[P_B2C * ps + o] = 0.5 * (b2 + b2n);
    out[P_B3C * ps + o] = b3c;
    out[P_B3I * ps + o] = b3c;
    dti = cell_dti(d, m1, m2, m3, e, g.eos, g.dx1, g.dx2);
  }
  return dti;
}

// Standalone CFL reduction over the interior of the step's input buffer
// (the reference new_dt(), used before the first step and by the drop-in ABI).
static __global__ void __launch_bounds__(kThreads) k_cfl(GridArgs g, int nx1, int ncell) {
  const int t = blockIdx.x * kThreads + threadIdx.x;
  double dti = 0.0;
  if (t < ncell) {
    const int j = g.js + t / nx1, i = g.is + t % nx1;
    const long long ps = g.ps, o = off(g, j, i);
    const double* s = g.in;
    dti = cell_dti(s[P_D * ps + o], s[P_M1 * ps + o], s[P_M2 * ps + o], s[P_M3 * ps + o],
                   s[P_E * ps + o], g.eos, g.dx1, g.dx2);
  }
  block_max_to(dti, &g.st->max_dti_bits, &g.st->flags);
}

__device__ __forceinline__ void set_step_coeffs(StepState& st, double dx1, double dx2) {
  st.dtodx1 = st.dt / dx1;
  st.dtodx2 = st.dt / dx2;
  st.hdtodx1 = 0.5 * st.dtodx1;
  st.hdtodx2 = 0.5 * st.dtodx2;
  st.hdt = 0.5 * st.dt;
}

// dt rule of src/new_dt.c:93-97 applied to the reduced max_dti.  mode 0: the
// initial call (nstep == 0 rule); mode 1: end of a step (time += dt, nstep++
// first, as src/main.c:268-271).  Then the tlim clamp of the next iteration
// (src/main.c:230-232) is applied if the loop continues.
__device__ __forceinline__ void finalize_state(StepState& st, double dx1, double dx2, int mode) {
  if (mode == 1) {
    if (st.done) return;
    st.nstep++;
    st.time += st.dt;
  }
  const double max_dti = __longlong_as_double((long long)st.max_dti_bits);
  st.max_dti_bits = 0ull;
  if (st.nstep == 0) st.dt = st.cour_no / max_dti;
  else st.dt = rmin(2.0 * st.dt, st.cour_no / max_dti);
  st.dt_new = st.dt;
  const bool more = (st.time < st.tlim) && (st.nlim < 0 || st.nstep < st.nlim);
  st.done = more ? 0 : 1;
  if (more && (st.tlim - st.time) < st.dt) st.dt = (st.tlim - st.time);
  if (more && st.has_pause && st.time >= st.tpause) st.done = 2;  // a host output is due first
  set_step_coeffs(st, dx1, dx2);
}

// Set (on != 0) or clear the pause time; a grid that has not ended runs or
// stays paused according to it.
static __global__ void k_set_pause(StepState* stp, double tpause, int on) {
  StepState& st = *stp;
  st.has_pause = on;
  st.tpause = tpause;
  if (st.done != 1) st.done = (on && st.time >= tpause) ? 2 : 0;
}

static __global__ void k_finalize(StepState* stp, double dx1, double dx2, int mode) {
  finalize_state(*stp, dx1, dx2, mode);
}

// Set dt from the host value without any rule (drop-in integrate_2d path).
static __global__ void k_set_dt(StepState* stp, double dt, double dx1, double dx2) {
  stp->dt = dt;
  stp->dt_new = dt;
  stp->done = 0;
  set_step_coeffs(*stp, dx1, dx2);
}

// ---------------------------------------------------------------------------
// Ghost zones (src/set_bvals.c).  x1 boundaries are applied on rows [js,je]
// (B2i: [js,je+1]) and x2 boundaries then copy whole rows including the x1
// ghosts, so every ghost value equals an interior value reached through the
// x2 map followed by the x1 map.  One thread per frame cell handles all planes.
// ---------------------------------------------------------------------------
// x1 source column for ghost column i, normal-field variant when bnorm
__device__ __forceinline__ int map_x1(const GridArgs& g, int i, bool bnorm, bool& flip) {
  flip = false;
  if (i < g.is) {
    const int k = g.is - i;  // 1..4
    switch (g.bc[0]) {
    case BC_REFLECT: flip = true; return g.is + (k - 1);
    case BC_OUTFLOW: return g.is;
    default: return g.ie - (k - 1);
    }
  }
  if (i > g.ie + (bnorm ? 1 : 0)) {   // i = ie+1 is an interior face of B1i
    const int k = i - g.ie;  // 1..4 (2..4 for B1i)
    switch (g.bc[1]) {
    case BC_REFLECT: flip = true; return bnorm ? g.ie - (k - 2) : g.ie - (k - 1);
    case BC_OUTFLOW: return g.ie;
    default: return g.is + (k - 1);
    }
  }
  return i;
}
__device__ __forceinline__ int map_x2(const GridArgs& g, int j, bool bnorm, bool& flip) {
  flip = false;
  if (j < g.js) {
    const int k = g.js - j;
    switch (g.bc[2]) {
    case BC_REFLECT: flip = true; return g.js + (k - 1);
    case BC_OUTFLOW: return g.js;
    default: return g.je - (k - 1);
    }
  }
  if (j > g.je + (bnorm ? 1 : 0)) {   // j = je+1 is an interior face of B2i
    const int k = j - g.je;  // 1..4 (2..4 for B2i)
    switch (g.bc[3]) {
    case BC_REFLECT: flip = true; return bnorm ? g.je - (k - 2) : g.je - (k - 1);
    case BC_OUTFLOW: return g.je;
    default: return g.js + (k - 1);
    }
  }
  return j;
}

// Ghost source of frame cell (j,i) for one plane kind: cell-centred planes
// and B3i (kind 0), B1i (kind 1: column ie+1 is an interior face), B2i (kind 2:
// row je+1 is an interior face).  mode 3: both directions composed (x2 map
// then x1 map); mode 1: the x1 boundaries alone on rows [js,je] (B2i
// [js,je+1]); mode 2: the x2 boundaries alone on whole rows.  sides: bit 0
// inner, bit 1 outer side of the direction(s) applied.  Returns false when
// the plane's value at (j,i) is not set by this mode.
__device__ __forceinline__ bool ghost_src(const GridArgs& g, int kind, int j, int i, int mode,
                                          int sides, int& sj, int& si, bool& f1, bool& f2) {
  const int ie_int = g.ie + (kind == 1 ? 1 : 0);
  const int je_int = g.je + (kind == 2 ? 1 : 0);
  const bool gx = (i < g.is && (sides & 1)) || (i > ie_int && (sides & 2));
  const bool gy = (j < g.js && (sides & 1)) || (j > je_int && (sides & 2));
  const bool in_rows = (j >= g.js && j <= je_int);
  sj = j; si = i; f1 = false; f2 = false;
  if (mode == 1) {
    if (!(gx && in_rows)) return false;
    si = map_x1(g, i, kind == 1, f1);
    return true;
  }
  if (mode == 2) {
    if (!gy) return false;
    sj = map_x2(g, j, kind == 2, f2);
    return true;
  }
  if (!gx && !gy) return false;
  if (gy) sj = map_x2(g, j, kind == 2, f2);
  if (gx) si = map_x1(g, i, kind == 1, f1);
  return true;
}

// Frame enumeration: rows [0,js) and (je,sy) full width, then rows [js,je]
// columns [0,is) and (ie,sx).  One thread per frame cell handles all planes.
__device__ __forceinline__ void ghost_item(const GridArgs& g, int sx, int sy, int nframe, int mode, int sides,
                                           int t) {
  if (t >= nframe) return;
  const int nbot = g.js * sx, ntop = (sy - g.je - 1) * sx;
  int j, i;
  if (t < nbot) { j = t / sx; i = t % sx; }
  else if (t < nbot + ntop) { j = g.je + 1 + (t - nbot) / sx; i = (t - nbot) % sx; }
  else {
    const int u = t - nbot - ntop, side = 2 * g.is;
    j = g.js + u / side;
    const int k = u % side;
    i = k < g.is ? k : g.ie + 1 + (k - g.is);
  }
  double* s = g.out;
  const long long ps = g.ps, o = off(g, j, i);
  int sj, si;
  bool f1, f2;
  if (ghost_src(g, 0, j, i, mode, sides, sj, si, f1, f2)) {
    const long long so = off(g, sj, si);
#pragma unroll
    for (int p = 0; p < 8; p++) {
      double v = s[p * ps + so];
      if ((p == P_M1 && f1) || (p == P_M2 && f2)) v = -v;  // reflecting walls
      s[p * ps + o] = v;
    }
    s[P_B3I * ps + o] = s[P_B3I * ps + so];
  }
  if (ghost_src(g, 1, j, i, mode, sides, sj, si, f1, f2))
    s[P_B1I * ps + o] = s[P_B1I * ps + off(g, sj, si)];
  if (ghost_src(g, 2, j, i, mode, sides, sj, si, f1, f2))
    s[P_B2I * ps + o] = s[P_B2I * ps + off(g, sj, si)];
}

static __global__ void __launch_bounds__(kThreads) k_ghost(GridArgs g, int sx, int sy, int nframe, int mode,
                                                   int sides) {
  ghost_item(g, sx, sy, nframe, mode, sides, blockIdx.x * kThreads + threadIdx.x);
}

}  // namespace athb
