/*
 * athena_b200.h -- C ABI of libathena_b200.so, a B200 (sm_100a) implementation
 * of the 2D adiabatic ideal-MHD CTU+CT step of Athena 3.1 as cut down in
 * awasiljew/athena-cuda.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the reference's names, signatures and Grid
 *     layout, so a program built against the reference CPU path links against
 *     this library instead of src/__integrate_2d__.c, src/lr_states_plm.c,
 *     src/set_bvals.c and src/new_dt.c.  They work on HOST Grid buffers: each
 *     call copies what it needs to the GPU and the result back.
 *
 *  2. The device-resident athb_* API: the grid lives in HBM between calls and
 *     a whole loop of steps runs without host round trips (CUDA graph).
 *
 * Every athb_* function returns ATHB_OK (0) or an ATHB_ERR_* code and never
 * exits the process; athb_last_error() gives the message of the calling
 * thread's last failure.  The drop-in functions keep the reference's
 * convention: a fatal error prints a message and exits (src/utils.c:111-127).
 *
 * Threading: one context is used by one host thread at a time.
 */
#ifndef ATHENA_B200_H
#define ATHENA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Reference data layout (src/athena.h:43-52 Gas, src/athena.h:106-120 Grid). */
/* Field order and types are identical, so a reference Grid* can be passed.   */
/* ------------------------------------------------------------------------ */
typedef struct athb_Gas {
  double d, M1, M2, M3, E, B1c, B2c, B3c;
} athb_Gas;

typedef struct athb_Grid {
  athb_Gas **U;                 /* [Nx2+8][Nx1+8] cell-centred conserved   */
  double **B1i, **B2i, **B3i;   /* [Nx2+8][Nx1+8] face-centred fields      */
  double x1_0, x2_0;
  double dx1, dx2;
  double dt, time;
  int nstep;
  int Nx1, Nx2;
  int is, ie, js, je;
  int idisp, jdisp;
  char *outfilename;
} athb_Grid;

typedef void (*athb_VBCFun_t)(athb_Grid *pG, int var_flag);

/* Reference globals (src/globals.h:18-20).  Defined weakly by the library so
 * a host program that defines them (src/main.c with MAIN_C) supplies them. */
extern double Gamma, Gamma_1, Gamma_2, CourNo;

/* ---- drop-in entry points (reference names) ----------------------------- */
/* replaces src/__integrate_2d__.c:573 integrate_init_2d(int nx1, int nx2)   */
void integrate_init_2d(int nx1, int nx2);
/* replaces src/__integrate_2d__.c:543 integrate_destruct_2d(void)           */
void integrate_destruct_2d(void);
/* replaces src/__integrate_2d__.c:100 integrate_2d(Grid *pG): one CTU+CT
 * step with pG->dt; writes U (interior), B1i (interior + column ie+1),
 * B2i (interior + row je+1) and B3i (interior), exactly as the reference.   */
void integrate_2d(athb_Grid *pG);
/* replaces src/lr_states_plm.c:253 / :270 (no state needed on the GPU)      */
void lr_states_init(int nx1, int nx2);
void lr_states_destruct(void);
/* replaces src/set_bvals.c:152 set_bvals_init(Grid*): reads grid/ibc_x1,
 * obc_x1, ibc_x2, obc_x2 through the host program's par_geti() (src/par.c)
 * unless athb_dropin_set_bc() set them first.                               */
void set_bvals_init(athb_Grid *pG);
/* replaces src/set_bvals.c:114 set_bvals(Grid*, int var_flag)               */
void set_bvals(athb_Grid *pG, int var_flag);
/* replaces src/set_bvals.c:269 set_bvals_fun(enum Direction, VBCFun_t):
 * dir 0..3 = left_x1, right_x1, left_x2, right_x2.  A user function runs on
 * the host Grid at its place in the x1-then-x2 order.                       */
void set_bvals_fun(int dir, athb_VBCFun_t prob_bc);
/* replaces src/new_dt.c:25 new_dt(Grid*): CFL reduction on the GPU, then the
 * reference dt rule (first step / at most 2x growth) on pG->dt.             */
void new_dt(athb_Grid *pG);

/* ---- status codes -------------------------------------------------------- */
#define ATHB_OK 0
#define ATHB_ERR_ARG 1      /* invalid argument or size                      */
#define ATHB_ERR_CUDA 2     /* CUDA runtime error (message has the detail)   */
#define ATHB_ERR_STATE 3    /* device flagged a non-finite / negative 1/dt   */
#define ATHB_ERR_PARSE 4    /* athinput file or parameter error              */
#define ATHB_ERR_NOMEM 5    /* allocation failure                            */
#define ATHB_ERR_NOTFOUND 6 /* unknown problem generator / parameter         */
#define ATHB_ERR_IO 7       /* file open / write error                       */

#define ATHB_FLUX_ROE 0     /* reference default (flux_roe, HLLE fallback)   */
#define ATHB_FLUX_HLLE 1    /* flux_hlle everywhere                          */

#define ATHB_BC_REFLECT 1   /* src/set_bvals.c:166-181 flag values           */
#define ATHB_BC_OUTFLOW 2
#define ATHB_BC_PERIODIC 4

#define ATHB_NPLANES 11     /* d M1 M2 M3 E B1c B2c B3c B1i B2i B3i          */

typedef struct athb_ctx athb_ctx;

typedef struct athb_config {
  int nx1, nx2;                 /* interior cells, each >= 4                 */
  double x1min, x1max, x2min, x2max;
  int bc_ix1, bc_ox1, bc_ix2, bc_ox2;  /* ATHB_BC_*                          */
  double gamma;                 /* Gamma_1 = gamma-1, Gamma_2 = gamma-2      */
  double cour_no;               /* CFL number                                */
  double tlim;                  /* loop ends when time >= tlim               */
  int nlim;                     /* ... or nstep >= nlim (nlim < 0: no limit) */
  int flux;                     /* ATHB_FLUX_*                               */
  int device;                   /* CUDA device ordinal                       */
} athb_config;

const char *athb_error_string(int code);
const char *athb_last_error(void);

int athb_create(const athb_config *cfg, athb_ctx **out);
void athb_destroy(athb_ctx *ctx);

/* Host layout of a state: ATHB_NPLANES planes of (nx2+8) x (nx1+8) doubles,
 * row-major, ghosts included, plane order d M1 M2 M3 E B1c B2c B3c B1i B2i B3i. */
int athb_shape(const athb_ctx *ctx, int *sx, int *sy);
int athb_upload(athb_ctx *ctx, const double *planes, double dt, double time, int nstep);
int athb_download(athb_ctx *ctx, double *planes, double *dt, double *time, int *nstep);

/* Ghost fill of the resident state (src/set_bvals.c:114).                   */
int athb_set_bvals(athb_ctx *ctx);
/* CFL dt of the resident state with the reference rule; stores and returns
 * it and applies the tlim clamp for the next step (src/main.c:230-232).     */
int athb_new_dt(athb_ctx *ctx, double *dt);
/* Run up to nsteps iterations of the reference main loop (clamp, step,
 * time += dt, new_dt, set_bvals) on the device; stops early at tlim/nlim.   */
int athb_run(athb_ctx *ctx, int nsteps, int *steps_done);
/* time, dt as the reference Grid holds it between iterations (new_dt's value;
 * the next step takes it after the tlim clamp, src/main.c:230-232), nstep,
 * done (0 running, 1 ended at tlim/nlim, 2 paused, see athb_set_pause).      */
int athb_status(athb_ctx *ctx, double *time, double *dt, int *nstep, int *done);
int athb_synchronize(athb_ctx *ctx);
/* Launch-only variant of athb_run for timing (no synchronisation).          */
int athb_run_async(athb_ctx *ctx, int nsteps);
/* Run nsteps loop iterations with CUDA events between the kernels and return
 * the mean time per step of each kernel in ms_out[7]: predict, emf (half
 * step), correct, emf (full step), update (+CFL), finalize, ghost.          */
int athb_profile_steps(athb_ctx *ctx, int nsteps, double *ms_out);
/* Tuning knob: rows per y-sweep march segment (work decomposition only; the
 * results do not depend on it).                                             */
int athb_set_ly(athb_ctx *ctx, int ly);
int athb_get_ly(const athb_ctx *ctx);
/* The CUDA stream the context launches on (as a cudaStream_t).               */
void *athb_stream(athb_ctx *ctx);
/* Pause the device loop at the first iteration that starts at time >= tpause
 * (on != 0; athb_run then returns there and athb_status reports done = 2),
 * or run freely (on = 0).  For host work due at a given simulation time,
 * such as the reference's data_output (src/main.c:239), without a host
 * round trip per step.                                                      */
int athb_set_pause(athb_ctx *ctx, double tpause, int on);

/* ---- pieces of an iteration, for a grid split over several contexts ------ */
/* A slab decomposition along x2 (one context per GPU, athena_cuda_b200/
 * decomp.py) runs each iteration as: athb_integrate_local; a max across the
 * contexts of athb_max_dti_bits; athb_finish_step(global max, 1); x1 ghosts
 * (athb_ghost_fill mode 1); the exchange of 4 ghost rows with the
 * neighbours (athb_rows_get / athb_rows_put); x2 ghosts at the global ends
 * (mode 2).  No reference counterpart: the reference grid is one process
 * (MPI_SERIAL).                                                             */
int athb_set_geometry(athb_ctx *ctx, double dx1, double dx2, double x1_0, double x2_0);
int athb_integrate_local(athb_ctx *ctx);
int athb_cfl_local(athb_ctx *ctx);
int athb_max_dti_bits(athb_ctx *ctx, unsigned long long *bits);
int athb_finish_step(athb_ctx *ctx, unsigned long long max_dti_bits, int after_step);
int athb_ghost_fill(athb_ctx *ctx, int mode, int sides);
int athb_rows_get(athb_ctx *ctx, int j0, int nrows, double *host);
int athb_rows_put(athb_ctx *ctx, int j0, int nrows, const double *host);
/* The same exchange on device buffers (no host copy per iteration): rows
 * [j0, j0+nrows) of the 11 planes packed into / unpacked from a contiguous
 * device buffer [plane][row][Nx1+8] by a kernel on the context's stream;
 * the running max of 1/dt written to a device word, and the step finished
 * with the max over n device words (after an NCCL all-reduce: n = 1; read
 * through IPC mappings of every rank's word: n = ranks).                    */
int athb_rows_pack(athb_ctx *ctx, int j0, int nrows, double *dev);
int athb_rows_unpack(athb_ctx *ctx, int j0, int nrows, const double *dev);
/* The same for the rectangle columns [i0, i0+ni) x rows [j0, j0+nj) (array
 * indices, ghosts included), buffer [plane][row][column]: the x1 exchange of
 * a 2D block decomposition.                                                 */
int athb_rect_pack(athb_ctx *ctx, int i0, int ni, int j0, int nj, double *dev);
int athb_rect_unpack(athb_ctx *ctx, int i0, int ni, int j0, int nj, const double *dev);
int athb_max_dti_bits_device(athb_ctx *ctx, unsigned long long *dev);
int athb_finish_step_device(athb_ctx *ctx, const unsigned long long *dev_bits, int n, int after_step);
/* Device buffers shared between processes: cudaMalloc'd (zeroed) on the
 * context's device, a CUDA-IPC handle (64 bytes) for another process, which
 * opens it as a device pointer; athb_copy_async copies on the context's
 * stream (cudaMemcpyAsync, plain peer stores when dst is a mapping).        */
void *athb_device_alloc(athb_ctx *ctx, unsigned long long bytes);
void athb_device_free(athb_ctx *ctx, void *dev);
int athb_ipc_handle(athb_ctx *ctx, void *dev, unsigned char handle[64]);
int athb_ipc_open(athb_ctx *ctx, const unsigned char handle[64], void **dev);
int athb_ipc_close(athb_ctx *ctx, void *dev);
int athb_copy_async(athb_ctx *ctx, void *dst, const void *src, unsigned long long bytes);

/* Data dumps of the resident state, byte-identical to the reference's:
 * athb_dump_bin writes dump_binary's file (src/dump_binary.c:25-134; the
 * interior is converted to float on the GPU), athb_dump_tab dump_tab's
 * (src/dump_tab.c:28-235; the middle row j = (js+je)/2; dat_fmt NULL for
 * the default " %12.8e").  The caller forms the file name
 * (src/ath_files.c:31-65: <problem_id>.<4-digit number>.<bin|tab>).        */
int athb_dump_bin(athb_ctx *ctx, const char *path);
int athb_dump_tab(athb_ctx *ctx, const char *path, const char *dat_fmt);

/* Single-variable ppm image of the resident state, the reference's
 * output_ppm (src/output_ppm.c:37-143) of an expression of src/output.c
 * (d M1 M2 M3 E B1c B2c B3c ME V1 V2 V3 P cs2 S) or, with usr_expr, of the
 * field-loop problem's get_usr_expr (J3, Bp2; src/field_loop.c:161-179).
 * The expression is evaluated on the GPU and only the float image comes
 * down.  The image is the first nx1 x nx2 interior cells (0: the grid's),
 * as the reference's subset2.  rgb: a 256x3 palette in 0..1 (NULL: black /
 * white at dmax); sdmin/sdmax fix the scale.  gmin/gmax carry the running
 * extremes between the outputs of one <output> block (num 0 resets them).   */
typedef struct athb_ppm_opts {
  const char *expr;
  int usr_expr;
  int nx1, nx2;
  const float *rgb;
  int sdmin, sdmax;
  float dmin, dmax;
  int num;                      /* output number (0: first image)           */
} athb_ppm_opts;
int athb_output_ppm(athb_ctx *ctx, const char *path, const athb_ppm_opts *opts, float *gmin, float *gmax);
/* Palette `name` (256 x 3 floats) from a file of colour tables, either in
 * the C form of the reference's palette.h or as lines "<name> v0 .. v767". */
int athb_palette_load(const char *path, const char *name, float rgb[768]);

/* Diagnostics of the resident state, computed on the GPU over the interior:
 * out[0] mass, out[1] total energy, out[2] magnetic energy (sum of
 * (B1c^2+B2c^2+B3c^2)/2 dV), out[3] sum of Bp2 = B1c^2+B2c^2 dV (the
 * field-loop expression, src/field_loop.c:167-171), out[4] max |div B| from
 * the face fields (constrained transport keeps it at round-off), out[5] max
 * |J3| (src/field_loop.c:161-165).  Deterministic (fixed reduction order).  */
int athb_diagnostics(athb_ctx *ctx, double out[6]);

/* Pinned host memory for fast transfers. */
void *athb_host_alloc(unsigned long long bytes);
void athb_host_free(void *p);

/* ---- athinput (src/par.c format) and problem generators ---------------- */
typedef struct athb_params athb_params;
int athb_params_open(const char *path, athb_params **out);
/* the same from the text of an athinput file                               */
int athb_params_from_string(const char *text, athb_params **out);
/* "block/name=value" overrides of existing keys (src/par.c:170-209)         */
int athb_params_override(athb_params *p, const char *arg);
int athb_params_getd(const athb_params *p, const char *block, const char *name, double *v);
int athb_params_geti(const athb_params *p, const char *block, const char *name, int *v);
/* the value text, or NULL when block/name does not exist (src/par.c:par_exist) */
const char *athb_params_gets(const athb_params *p, const char *block, const char *name);
void athb_params_close(athb_params *p);
/* config from the <grid>, <time> and <problem> blocks */
int athb_config_from_params(const athb_params *p, athb_config *cfg);

/* Problem generator hook: fill the interior cells and the interior faces
 * (including B1i column ie+1 and B2i row je+1) of a host state laid out as
 * in athb_upload.  Built in: "blast" (src/blast.c:25-72), "field_loop"
 * (src/field_loop.c:40-137), "cpaw2d" (src/cpaw2d.c:56-185).                */
typedef struct athb_grid_info {
  int nx1, nx2, sx, sy, is, ie, js, je;
  double dx1, dx2, x1_0, x2_0;
  int idisp, jdisp;
  double gamma, gamma_1, gamma_2;
} athb_grid_info;
typedef int (*athb_problem_fn)(const athb_grid_info *g, const athb_params *p,
                               double *planes, void *user);
int athb_register_problem(const char *name, athb_problem_fn fn, void *user);
int athb_grid_info_of(const athb_ctx *ctx, athb_grid_info *g);
int athb_problem_generate(const char *name, const athb_grid_info *g, const athb_params *p,
                          double *planes);

/* Replace the resident state with problem `name`'s initial condition (clock
 * reset to dt = time = nstep = 0; no set_bvals).  The built-in "blast" and
 * "field_loop" generators run on the GPU in the state buffer (no host array,
 * no upload; per cell they need only + - * / and sqrt, so the state is
 * bit-identical to the host generators'); "cpaw2d" (libm sin/cos per cell)
 * and registered generators run on the host and are uploaded.               */
int athb_generate(athb_ctx *ctx, const char *name, const athb_params *p);
/* Every built-in generator on the GPU, "cpaw2d" included: its per-cell
 * sin/cos are CUDA's (within 2 ulp of the exact values, where libm's are
 * within 1), so the cpaw2d state agrees with athb_generate's to a few ulp of
 * each term (face fields: of the vector potential over dx), not bit for bit.
 * ATHB_ERR_NOTFOUND for registered (non-built-in) generators.               */
int athb_generate_device(athb_ctx *ctx, const char *name, const athb_params *p);

/* Parse an athinput file (+ overrides), create the context, run the problem
 * generator (athb_generate), set_bvals and the first new_dt: the state
 * src/main.c:75-149 holds on entry to its main loop.                        */
int athb_create_from_athinput(const char *path, int noverride, const char *const *overrides,
                              const char *problem, athb_ctx **out);

/* cpaw2d L1 errors against the initial state (src/cpaw2d.c:222-302,
 * Userwork_after_loop): err[0]=RMS, err[1..8] = d M1 M2 M3 E B1c B2c B3c,
 * each divided by Nx1*Nx2.  Only for contexts created by cpaw2d.  The sums
 * run on the GPU in the reference's order against the initial state kept on
 * the device (8 doubles come back): equal to the reference's host loop.     */
int athb_cpaw2d_errors(athb_ctx *ctx, double err[9]);

/* ---- batched ensembles ---------------------------------------------------- */
/* Many independent grids (any sizes, own dt and end time, shared flux and
 * device) advanced by one persistent cooperative kernel launch per step.
 * Every instance is bit-identical to a single-grid run of the same problem. */
typedef struct athb_batch athb_batch;
int athb_batch_create(int n, const athb_config *cfgs, athb_batch **out);
void athb_batch_destroy(athb_batch *b);
int athb_batch_size(const athb_batch *b);
/* instance state in the athb_upload layout, and its clock                   */
int athb_batch_upload(athb_batch *b, int k, const double *planes, double dt, double time, int nstep);
int athb_batch_download(athb_batch *b, int k, double *planes, double *dt, double *time, int *nstep);
/* instance k's initial condition formed on the GPU (built-in generators
 * only, as athb_generate_device), clock reset                               */
int athb_batch_generate(athb_batch *b, int k, const char *name, const athb_params *p);
/* set_bvals and the first new_dt of every instance (src/main.c:139-149)      */
int athb_batch_prepare(athb_batch *b);
/* steps until every instance is done or max_steps launches                  */
int athb_batch_run(athb_batch *b, int max_steps, int *launches);
int athb_batch_run_async(athb_batch *b, int nsteps);
int athb_batch_synchronize(athb_batch *b);
void *athb_batch_stream(athb_batch *b);
/* tuning: y-march segment length of instance k (applied by _commit) and the
 * number of persistent blocks (at most the co-resident maximum)             */
int athb_batch_set_ly(athb_batch *b, int k, int ly);
int athb_batch_commit(athb_batch *b);
int athb_batch_set_grid(athb_batch *b, int blocks);
/* threads per work unit of the phased launches: 64, 128 (default) or 256;
 * applied by athb_batch_commit; the persistent mode keeps 128.  Results do
 * not depend on it.                                                         */
int athb_batch_set_threads(athb_batch *b, int nt);
int athb_batch_threads(const athb_batch *b);
int athb_batch_grid(const athb_batch *b);
/* per-phase time, accumulated in ms_out[6]: predict, emf (half step),
 * correct, emf (full step), update, ghost + finalize (persistent mode: block
 * 0's view, each phase ending at its grid barrier; phased mode: between
 * device time stamps after each phase).  enable: 1 start recording (resets),
 * 0 stop, -1 leave as is; ms_out may be NULL.                              */
int athb_batch_timing(athb_batch *b, int enable, double *ms_out);
/* execution mode: one launch per phase with the hardware block scheduler
 * (default: each phase keeps its single-grid kernel's register budget), or
 * one persistent cooperative launch per step; identical results             */
#define ATHB_BATCH_PERSISTENT 0
#define ATHB_BATCH_PHASED 1
int athb_batch_set_mode(athb_batch *b, int mode);
int athb_batch_mode(const athb_batch *b);
/* A grid barrier that times out in the persistent kernel (a block that never
 * arrived) sets a sticky ATHB_ERR_STATE on the batch and leaves the barrier's
 * arrival count inconsistent: every later athb_batch_run on that batch
 * reports the time-out again.  Destroy the batch and create a new one.      */
/* Failure-path self-test of the persistent kernel's grid barrier: one block
 * waits for two, gives up after `spins` polls (~64 ns each), and the time-out
 * is reported in *timed_out (1 expected) with the device still usable.      */
int athb_batch_selftest_barrier(int device, long long spins, int *timed_out);

/* ---- tangent-linear model and adjoint of the main loop --------------------- */
/* No reference counterpart (the reference has no derivatives).  Both run the
 * reference main loop (src/main.c:229-307: tlim clamp, integrate_2d,
 * time += dt, new_dt, set_bvals) for nsteps iterations, or until tlim, from
 * the context's resident state taken as the loop-entry state: set_bvals and
 * new_dt (nstep 0 rule, src/new_dt.c:93-97) are applied to it first, so dt
 * depends on the state as in the reference and is differentiated through
 * the CFL max (the cell attaining it, lowest index on ties), the 2x growth cap
 * and the tlim clamp.  Objective J = sum over interior cells of
 * (B1c^2 + B2c^2)/2 at the final state.  Branches (limiters, upwinding,
 * supersonic faces, the HLLE fallback of flux_roe) are those of the forward
 * step.  The resident state and clock are left untouched.
 * Host arrays use the athb_upload layout; only the cells a step writes are
 * independent inputs (interior cells, B1i column ie+1, B2i row je+1): ghost
 * entries of a direction are ignored and those of a gradient are zero.      */
typedef struct athb_adjoint_stats {
  int steps;                  /* iterations differentiated                    */
  int snapshots;              /* state snapshots held in device memory        */
  long long advances;         /* forward steps run (first sweep + recompute)  */
  long long taped;            /* recorded forward steps (one per reverse step)*/
  long long workspace_bytes;  /* device memory used, snapshots included       */
  double seconds;             /* wall time of the call                        */
  int tape_mode;              /* 1: every step's intermediates were kept by the
                                 first sweep (no recorded re-step)            */
} athb_adjoint_stats;
/* Tangent-linear model: J and its directional derivative dJ along dstate0
 * (host); dstate_out (host, may be NULL) receives the tangent of the final
 * state, ghosts included.                                                   */
int athb_tlm_run(athb_ctx *ctx, int nsteps, const double *dstate0, double *J, double *dJ, double *dstate_out);
/* Adjoint: J and dJ/d(state) of the loop-entry state into grad (host, may be
 * NULL).  Checkpointing: snapshot_bytes of device memory for snapshots
 * (<= 0: 85% of the free memory less 1 GiB).  With room for every step's
 * state and intermediates (the "tape", ~89 planes a step) the first sweep
 * keeps them all and the reverse sweep recomputes nothing; with room for the
 * states only the loop runs forward once and each reversed step is
 * re-recorded from its state; with less, binomial checkpointing (Griewank
 * 1992) recomputes the fewest forward steps the room allows.                */
int athb_adjoint_gradient(athb_ctx *ctx, int nsteps, long long snapshot_bytes, double *J, double *grad,
                          athb_adjoint_stats *stats);
/* The same for any objective of the final state: seed is dJ/dS^N in the
 * athb_upload layout (its entries on the cells a step writes are used: the
 * interior, B1i to column ie+1, B2i to row je+1), grad = (dS^N/dS^0)^T seed
 * and J = <seed, S^N>.  A user objective J(S^N) passes its gradient; with
 * athb_tlm_run's final tangent state this gives any directional derivative.
 * No reference counterpart.                                                 */
int athb_adjoint_vjp(athb_ctx *ctx, int nsteps, long long snapshot_bytes, const double *seed, double *J,
                     double *grad, athb_adjoint_stats *stats);
/* Keep the device workspace of athb_adjoint_gradient / athb_tlm_run on this
 * context between calls (on = 1: a repeated call of the same size reuses it
 * instead of allocating and freeing up to most of the GPU's memory; the
 * default budget counts the kept blocks as free), or free it now (on = 0,
 * the default state).  athb_destroy frees it too.  No reference counterpart. */
int athb_adjoint_keep_workspace(athb_ctx *ctx, int on);

/* ---- allocation-free step ------------------------------------------------ */
/* No counterpart in the reference.  One integrate_2d step (the cells
 * integrate_2d writes) from d_in into d_out, both caller-owned device buffers
 * in the athb_upload layout ((nx2+8) x (nx1+8) doubles per plane, 11 planes,
 * ghosts of d_in filled), with time step dt, on `stream` (a cudaStream_t, NULL
 * for the default stream).  For callers that cannot allocate device memory:
 * code running while a CUDA graph is captured, programs that reserve the whole
 * device memory budget up front, allocation-free real-time loops.  It calls
 * no cudaMalloc/cudaFree: its scratch is a fixed __device__ array in the
 * library (~2.4 MB, present on every GPU that loads the library until the
 * process exits), so it accepts only grids with (Nx1+8)*(Nx2+8) <= 5184
 * (64 x 64, or any shape with as many cells) and rejects larger ones with
 * ATHB_ERR_ARG.  All calls share that array: calls that overlap on the GPU
 * race.  The array's device address is looked up on the first call made on
 * each device (that device current); make that first call before any stream
 * capture.  The step runs on the calling thread's current device, which must
 * be cfg->device (ATHB_ERR_ARG otherwise).  It does no non-finite check: a
 * step that produces NaN or a negative pressure returns ATHB_OK.            */
int athb_integrate_noalloc(const athb_config *cfg, const double *d_in, double *d_out, double dt,
                           void *stream);

/* Drop-in configuration without the host program's par.c.                  */
void athb_dropin_set_bc(int ibc_x1, int obc_x1, int ibc_x2, int obc_x2);
/* GPU used by the drop-in calls (before the first call; default: the
 * ATHB_DEVICE environment variable, else 0).                                */
void athb_dropin_set_device(int device);
void athb_dropin_set_flux(int flux);
/* Opt-in for programs that do not modify the Grid between the drop-in calls
 * (the reference main loop between outputs, src/main.c:229-307): after the
 * first full upload the device copy is authoritative, integrate_2d uploads
 * nothing and new_dt reuses the CFL max its step already reduced; every call
 * still leaves the host Grid exactly as the reference would (integrate_2d
 * downloads the cells it writes, set_bvals the ghost frame).  Default off;
 * the environment variable ATHB_DROPIN_HOST_UNCHANGED=1 turns it on.  A
 * caller that writes the Grid must call this again (with 0 or 1) first.     */
void athb_dropin_set_host_unchanged(int on);
/* Bytes the drop-in entry points have copied host->device / device->host.  */
void athb_dropin_bytes(unsigned long long *h2d, unsigned long long *d2h);

/* Measured FP64 issue rate of this GPU: add/mul operations per second from
 * independent chains of DADD and DMUL (no fused multiply-add, like the step),
 * timed with CUDA events.  The roofline denominator of the FP64-bound step.  */
int athb_fp64_peak(int device, double *ops_per_s);

#ifdef __cplusplus
}
#endif
#endif /* ATHENA_B200_H */
