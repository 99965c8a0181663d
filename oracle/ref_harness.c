/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * A driver that links the reference's own, unmodified CPU sources
 * (src/__integrate_2d__.c, src/set_bvals.c, src/new_dt.c, src/lr_states_plm.c,
 * src/flux_roe.c, src/flux_hlle.c, src/esystem_*.c, src/convert_var.c,
 * src/init_grid.c, src/par.c and one problem file) and reproduces the main loop
 * of src/main.c:221-318 without any output.  It replaces src/main.c only: the
 * physics is the reference's.
 *
 * It is built by oracle/build_ref.py into oracle/_ref/ and is used only by
 * tests/ (parity pins) and by bench.py's CPU-baseline leg.
 *
 * Usage:
 *   athref_<problem>_<flux> -i <athinput> [--steps N] [--dump FILE]
 *                           [--init FILE] [--l1] [--quiet]
 *
 *   --steps N   stop after N steps (default: run to time/tlim, or time/nlim)
 *   --dump F    write the final state (raw state file, format below)
 *   --init F    (problem "file" builds only) initial state read from F
 *   --l1        (cpaw2d builds) call Userwork_after_loop (cpaw2d.c:222) which
 *               appends the L1 errors to ./cpaw2d-errors.dat
 *   --bench     print one JSON line with the main-loop time (zone-cycles/s)
 *   --max-seconds T  also stop once the main loop has run for T seconds
 *   --warmup N  run N untimed iterations before the timed loop (--steps
 *               counts the timed ones); --warmup-seconds T stops the
 *               warm-up once it has run for T seconds
 *
 * Raw state file format (little endian):
 *   int32  magic 0x41544842 ("ATHB"), version 1
 *   int32  Nx1, Nx2, nghost, nstep
 *   double dt, time, dx1, dx2, x1_0, x2_0
 *   11 planes of (Nx2+2*nghost) x (Nx1+2*nghost) doubles, row-major,
 *   in the order d, M1, M2, M3, E, B1c, B2c, B3c, B1i, B2i, B3i.
 */
#define MAIN_C
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "defs.h"
#include "athena.h"
#include "globals.h"
#include "prototypes.h"

#define RAW_MAGIC 0x41544842
#define NPLANES 11

static const char *g_init_file = NULL;

static double now_s(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static double *plane_ptr(Grid *g, int p, int j, int i)
{
  Gas *u = &g->U[j][i];
  switch (p) {
  case 0: return &u->d;
  case 1: return &u->M1;
  case 2: return &u->M2;
  case 3: return &u->M3;
  case 4: return &u->E;
  case 5: return &u->B1c;
  case 6: return &u->B2c;
  case 7: return &u->B3c;
  case 8: return &g->B1i[j][i];
  case 9: return &g->B2i[j][i];
  default: return &g->B3i[j][i];
  }
}

static void dump_state(Grid *g, const char *path)
{
  int sx = g->Nx1 + 2 * nghost, sy = g->Nx2 + 2 * nghost;
  int hdr[6] = {RAW_MAGIC, 1, g->Nx1, g->Nx2, nghost, g->nstep};
  double dh[6] = {g->dt, g->time, g->dx1, g->dx2, g->x1_0, g->x2_0};
  FILE *fp = fopen(path, "wb");
  if (!fp) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
  fwrite(hdr, sizeof(int), 6, fp);
  fwrite(dh, sizeof(double), 6, fp);
  for (int p = 0; p < NPLANES; p++)
    for (int j = 0; j < sy; j++)
      for (int i = 0; i < sx; i++)
        fwrite(plane_ptr(g, p, j, i), sizeof(double), 1, fp);
  fclose(fp);
}

/* problem "file": the initial state (every cell, ghosts included) comes from a
 * raw state file.  Only linked into the athref_file_* builds. */
#ifdef HARNESS_FILE_PROBLEM
void problem(Grid *g)
{
  int sx = g->Nx1 + 2 * nghost, sy = g->Nx2 + 2 * nghost;
  int hdr[6];
  double dh[6];
  FILE *fp;
  if (!g_init_file) { fprintf(stderr, "--init FILE required\n"); exit(2); }
  fp = fopen(g_init_file, "rb");
  if (!fp) { fprintf(stderr, "cannot read %s\n", g_init_file); exit(2); }
  if (fread(hdr, sizeof(int), 6, fp) != 6 || hdr[0] != RAW_MAGIC ||
      hdr[2] != g->Nx1 || hdr[3] != g->Nx2 || hdr[4] != nghost) {
    fprintf(stderr, "bad init file %s\n", g_init_file); exit(2);
  }
  if (fread(dh, sizeof(double), 6, fp) != 6) exit(2);
  for (int p = 0; p < NPLANES; p++)
    for (int j = 0; j < sy; j++)
      for (int i = 0; i < sx; i++)
        if (fread(plane_ptr(g, p, j, i), sizeof(double), 1, fp) != 1) exit(2);
  fclose(fp);
}
void problem_write_restart(Grid *pG, FILE *fp) { (void)pG; (void)fp; }
void problem_read_restart(Grid *pG, FILE *fp) { (void)pG; (void)fp; }
Gasfun_t get_usr_expr(const char *expr) { (void)expr; return NULL; }
void Userwork_in_loop(Grid *pGrid) { (void)pGrid; }
void Userwork_after_loop(Grid *pGrid) { (void)pGrid; }
#endif

int main(int argc, char **argv)
{
  const char *athinput = NULL, *dump = NULL;
  long steps = -1;
  int want_l1 = 0, bench = 0;
  double max_seconds = -1.0;
  long warmup = 0;
  double warmup_seconds = -1.0;
  Grid G;
  memset(&G, 0, sizeof(G));

  for (int a = 1; a < argc; a++) {
    if (!strcmp(argv[a], "-i") && a + 1 < argc) athinput = argv[++a];
    else if (!strcmp(argv[a], "--steps") && a + 1 < argc) steps = atol(argv[++a]);
    else if (!strcmp(argv[a], "--dump") && a + 1 < argc) dump = argv[++a];
    else if (!strcmp(argv[a], "--init") && a + 1 < argc) g_init_file = argv[++a];
    else if (!strcmp(argv[a], "--l1")) want_l1 = 1;
    else if (!strcmp(argv[a], "--bench")) bench = 1;
    else if (!strcmp(argv[a], "--max-seconds") && a + 1 < argc) max_seconds = atof(argv[++a]);
    else if (!strcmp(argv[a], "--warmup") && a + 1 < argc) warmup = atol(argv[++a]);
    else if (!strcmp(argv[a], "--warmup-seconds") && a + 1 < argc) warmup_seconds = atof(argv[++a]);
    else if (!strcmp(argv[a], "--quiet")) ;
    else { fprintf(stderr, "unknown argument %s\n", argv[a]); return 2; }
  }
  if (!athinput) { fprintf(stderr, "-i <athinput> required\n"); return 2; }

  /* src/main.c:75-94 */
  par_open((char *)athinput);
  CourNo = par_getd("time", "cour_no");
  int nlim = par_geti_def("time", "nlim", -1);
  Real tlim = par_getd("time", "tlim");
  Gamma = par_getd("problem", "gamma");
  Gamma_1 = Gamma - 1.0;
  Gamma_2 = Gamma - 2.0;

  /* src/main.c:100-149 */
  init_grid(&G);
  problem(&G);
  set_bvals_init(&G);
  set_bvals(&G, 0);
  new_dt(&G);
  lr_states_init(G.Nx1, G.Nx2);
  integrate_init_2d(G.Nx1, G.Nx2);

  /* src/main.c:221-318, without output: untimed warm-up iterations first */
  long warm = 0;
  double tw = now_s();
  while (warm < warmup && G.time < tlim && (nlim < 0 || G.nstep < nlim)) {
    if ((tlim - G.time) < G.dt) G.dt = (tlim - G.time);
    integrate_2d(&G);
    G.nstep++;
    G.time += G.dt;
    new_dt(&G);
    set_bvals(&G, 0);
    warm++;
    if (warmup_seconds > 0.0 && now_s() - tw > warmup_seconds) break;
  }
  double t0 = now_s();
  long done = 0;
  while (G.time < tlim && (nlim < 0 || G.nstep < nlim) && (steps < 0 || done < steps)) {
    if ((tlim - G.time) < G.dt) G.dt = (tlim - G.time);
    integrate_2d(&G);
    G.nstep++;
    G.time += G.dt;
    new_dt(&G);
    set_bvals(&G, 0);
    done++;
    if (max_seconds > 0.0 && now_s() - t0 > max_seconds) break;
  }
  double t1 = now_s();

  if (want_l1) Userwork_after_loop(&G);
  if (dump) dump_state(&G, dump);
  if (bench) {
    double zc = (double)G.Nx1 * (double)G.Nx2 * (double)done;
    printf("{\"steps\": %ld, \"warmup\": %ld, \"seconds\": %.6f, \"zone_cycles_per_s\": %.6e, "
           "\"Nx1\": %d, \"Nx2\": %d}\n", done, warm, t1 - t0,
           (t1 > t0) ? zc / (t1 - t0) : 0.0, G.Nx1, G.Nx2);
  }
  lr_states_destruct();
  integrate_destruct_2d();
  return 0;
}
