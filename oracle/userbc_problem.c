/*
 * userbc_problem.c -- TEST INFRASTRUCTURE ONLY: a problem generator that
 * registers a user boundary condition through the reference's problem-file
 * hook, set_bvals_fun (src/set_bvals.c:269), the way a reference problem file
 * does it (problem() runs before set_bvals_init, src/main.c:139-144, and
 * set_bvals_init keeps a function that is already set).
 *
 * Linked (by oracle/build_ref.py) into two programs that run the same main
 * loop (oracle/ref_harness.c):
 *   athref_userbc_roe  -- with the reference's own src/set_bvals.c;
 *   athdrop_userbc     -- with libathena_b200.so's set_bvals / set_bvals_fun.
 * Their outputs must be identical.
 *
 * State: a uniform magnetised medium (rho = 1, P = 0.6, B = (0.5, 0.3, 0.1))
 * with a dense blob at the centre; the left x1 boundary is a fixed supersonic
 * inflow (rho = 1.2, v = (1.6, 0.1, 0), same P and B), written into the four
 * ghost columns of rows js..je (B2i rows js..je+1) like the reference's own
 * x1 boundary functions (src/set_bvals.c:553-600).  B is uniform, so the
 * ghost faces keep div B = 0.
 */
#include <math.h>
#include <stdio.h>
#include "defs.h"
#include "athena.h"
#include "globals.h"
#include "prototypes.h"

static const Real B0[3] = {0.5, 0.3, 0.1};
static const Real P0 = 0.6;

static Real total_energy(Real d, Real v1, Real v2, Real v3)
{
  return P0 / Gamma_1 + 0.5 * d * (v1 * v1 + v2 * v2 + v3 * v3) +
         0.5 * (B0[0] * B0[0] + B0[1] * B0[1] + B0[2] * B0[2]);
}

static void inflow_ix1(Grid *pG, int var_flag)
{
  int is = pG->is, js = pG->js, je = pG->je;
  const Real d = 1.2, v1 = 1.6, v2 = 0.1, v3 = 0.0;
  if (var_flag == 1) return;
  for (int j = js; j <= je; j++) {
    for (int i = 1; i <= nghost; i++) {
      Gas *u = &pG->U[j][is - i];
      u->d = d;
      u->M1 = d * v1;
      u->M2 = d * v2;
      u->M3 = d * v3;
      u->E = total_energy(d, v1, v2, v3);
      u->B1c = B0[0];
      u->B2c = B0[1];
      u->B3c = B0[2];
      pG->B1i[j][is - i] = B0[0];
      pG->B3i[j][is - i] = B0[2];
    }
  }
  for (int j = js; j <= je + 1; j++)
    for (int i = 1; i <= nghost; i++) pG->B2i[j][is - i] = B0[1];
}

void problem(Grid *pG)
{
  Real x1, x2;
  for (int j = pG->js; j <= pG->je; j++) {
    for (int i = pG->is; i <= pG->ie; i++) {
      cc_pos(pG, i, j, &x1, &x2);
      Real r2 = x1 * x1 + x2 * x2;
      Real d = (r2 < 0.04) ? 3.0 : 1.0;
      Gas *u = &pG->U[j][i];
      u->d = d;
      u->M1 = u->M2 = u->M3 = 0.0;
      u->E = total_energy(d, 0.0, 0.0, 0.0);
      u->B1c = B0[0];
      u->B2c = B0[1];
      u->B3c = B0[2];
      pG->B1i[j][i] = B0[0];
      pG->B2i[j][i] = B0[1];
      pG->B3i[j][i] = B0[2];
    }
    pG->B1i[j][pG->ie + 1] = B0[0];
  }
  for (int i = pG->is; i <= pG->ie; i++) pG->B2i[pG->je + 1][i] = B0[1];
  set_bvals_fun(left_x1, inflow_ix1);
}

void problem_write_restart(Grid *pG, FILE *fp) { (void)pG; (void)fp; }
void problem_read_restart(Grid *pG, FILE *fp) { (void)pG; (void)fp; }
Gasfun_t get_usr_expr(const char *expr) { (void)expr; return NULL; }
void Userwork_in_loop(Grid *pGrid) { (void)pGrid; }
void Userwork_after_loop(Grid *pGrid) { (void)pGrid; }
