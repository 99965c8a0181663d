// step_types.cuh -- data layout and time-stepping state shared by the kernels
// (step_kernels.cuh) and the host-side launchers.
#pragma once

#include "mhd_physics.cuh"

namespace athb {


enum StatePlane { P_D = 0, P_M1, P_M2, P_M3, P_E, P_B1C, P_B2C, P_B3C, P_B1I, P_B2I, P_B3I, NSTATE };

// Scratch plane offsets (each group of 7 is one Cons1 in the sweep frame).
enum ScratchPlane {
  S_ULX = 0, S_URX = 7, S_FX = 14,
  S_ULY = 21, S_URY = 28, S_FY = 35,
  S_FX2 = 42, S_FY2 = 49,
  S_ECC = 56,   // cell-centred emf3 (t^n, then t^{n+1/2})
  S_EMF = 57,   // corner emf3 (half step, then full step)
  NSCRATCH = 58
};

// Planes after the scratch planes that a recorded ("taped") step keeps for
// the adjoint: the predictor's face states in primitive form (W_L of the
// face on the right of a cell, W_R of the face on its left; each group of 7
// is one Prim1 in the sweep frame) and the half-step emfs, which the plain
// step overwrites.
enum TapePlane {
  T_WLNX = NSCRATCH, T_WRTX = NSCRATCH + 7, T_WLNY = NSCRATCH + 14, T_WRTY = NSCRATCH + 21,
  T_ECC0 = NSCRATCH + 28,   // cell emf3 at t^n
  T_EMF0 = NSCRATCH + 29,   // corner emf of the half step
  NTAPED = NSCRATCH + 30
};

enum BcKind { BC_REFLECT = 1, BC_OUTFLOW = 2, BC_PERIODIC = 4 };

// Device-resident time-stepping state of one grid.
struct StepState {
  double dt;        // dt of the next step (after the tlim clamp of src/main.c:230-232)
  double dt_new;    // dt as the reference Grid holds it between iterations:
                    // new_dt's value, before the next iteration's tlim clamp
  double time;
  double tlim;
  double cour_no;
  // derived from the dt the next step uses (src/__integrate_2d__.c:102-110)
  double dtodx1, dtodx2, hdtodx1, hdtodx2, hdt;
  double tpause;    // with has_pause: stop stepping once time >= tpause
  int nstep;
  int nlim;         // < 0: no cycle limit
  int done;         // 1 once time >= tlim or nstep >= nlim (ended), 2 paused at
                    // tpause; either way steps are no-ops
  int flags;        // error bits, see kErr*
  int has_pause;
  unsigned long long max_dti_bits;  // running max of 1/dt (positive doubles
                                    // order like their bit patterns)
};

constexpr int kErrNonFinite = 1;  // a non-finite or negative 1/dt was reduced

// Geometry and pointers of one grid, passed by value to every kernel.
struct GridArgs {
  const double* __restrict__ in;  // state planes read by the step
  double* __restrict__ out;       // state planes written by the step
  double* __restrict__ scr;       // scratch planes
  StepState* st;
  long long ps;                   // plane stride in doubles
  int pitch;
  int is, ie, js, je;
  int ly;                         // rows per y-sweep march segment
  double dx1, dx2;
  Eos eos;
  int bc[4];                      // ix1, ox1, ix2, ox2
};

}  // namespace athb
