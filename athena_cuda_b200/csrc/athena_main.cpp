// athena_main.cpp -- command-line driver: the reference's main program
// (src/main.c:27-318) with the whole main loop on the device.
//
//   athena_b200 [-i athinput] [-p problem] [-d dir] [-q] [block/par=value ...]
//
// Same steps as the reference: read the athinput file and the command-line
// overrides (src/par.c:170-209), build the grid, run the problem generator,
// set_bvals, new_dt, register the <outputN> blocks (src/output.c:143-360),
// then loop: write the outputs that are due (src/output.c:362-441), clamp dt
// at tlim, integrate, time += dt, new_dt, set_bvals, print the cycle line.
// The step runs on the GPU through libathena_b200; between outputs the loop
// runs as CUDA graphs without a host round trip per step (with -q; without
// it, every cycle line is printed as the reference does, which reads the
// clock once per step).  Outputs: the "bin" and "tab" dumps (out = all) and
// the ppm images of one expression (out = d, M1, ..., S, or a problem's own
// expression with usr_expr_flag = 1), byte-identical to the reference's.
// The ppm palettes are read at run time from a file of colour tables (-P or
// ATHB_PALETTES): the reference's palette.h itself, or lines
// "<name> v0 .. v767".
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "athena_b200.h"

namespace {

struct Output {
  int n = 0;             // N of <outputN>
  std::string fmt;       // bin | tab | ppm
  std::string dat_fmt;   // tab only (empty: default)
  double t = 0.0, dt = 0.0;
  int num = 0;
  // single-variable outputs (fmt ppm)
  std::string expr, id;  // expression; file name id (default "outN")
  int usr_expr = 0;
  bool sliced = false;   // ix1 / ix2 given: the image is not 2D
  int sdmin = 0, sdmax = 0;
  double dmin = 0.0, dmax = 0.0;
  std::vector<float> rgb;
  float gmin = 0.0f, gmax = 0.0f;
};

void usage(const char* prog) {
  fprintf(stderr,
          "\nUsage: %s [options] [block/par=value ...]\n\nOptions:\n"
          "  -i <file>       Alternate input file [athinput]\n"
          "  -p <problem>    Problem generator: blast, field_loop, cpaw2d [<job>/problem, or\n"
          "                  the --with-problem= of <comment>/config]\n"
          "  -d <directory>  Directory the outputs are written to [.]\n"
          "  -q              Print no cycle lines; run between outputs without host round trips\n"
          "  -P <file>       Palettes of the ppm outputs [ATHB_PALETTES]: the reference's\n"
          "                  palette.h, or lines \"<name> v0 .. v767\"\n"
          "  -h              This help\n",
          prog);
  exit(0);
}

[[noreturn]] void die(const char* where) {
  fprintf(stderr, "[%s]: %s\n", where, athb_last_error());
  exit(1);
}

// <problem_id>.<num as 4 digits>.<ext> (src/ath_files.c:31-65, num_digit = 4).
std::string dump_name(const std::string& dir, const std::string& base, int num, const char* ext) {
  char buf[64];
  snprintf(buf, sizeof buf, ".%04d.%s", num, ext);
  return (dir.empty() ? std::string() : dir + "/") + base + buf;
}

// <problem_id>.<num as 4 digits>.<id>.<ext> (fname_construct with an id).
std::string output_name(const std::string& dir, const std::string& base, int num, const std::string& id,
                        const char* ext) {
  char buf[64];
  snprintf(buf, sizeof buf, ".%04d.", num);
  return (dir.empty() ? std::string() : dir + "/") + base + buf + id + "." + ext;
}

// The expressions a problem generator adds for single-variable outputs
// (get_usr_expr: src/field_loop.c:174-179; blast and cpaw2d have none).
bool usr_expr_known(const std::string& problem, const std::string& e) {
  return problem == "field_loop" && (e == "J3" || e == "Bp2");
}

bool expr_known(const std::string& e) {
  static const char* names[] = {"d", "M1", "M2", "M3", "E", "B1c", "B2c", "B3c", "ME", "V1", "V2", "V3", "P",
                                "cs2", "S"};
  for (const char* n : names)
    if (e == n) return true;
  return false;
}

// <outputN> blocks for N = 1 .. job/maxout (src/output.c:143-360).
std::vector<Output> read_outputs(const athb_params* p, double time0, const std::string& problem,
                                 const char* palettes) {
  std::vector<Output> outs;
  int maxout = 10;
  if (athb_params_gets(p, "job", "maxout")) athb_params_geti(p, "job", "maxout", &maxout);
  for (int n = 1; n <= maxout; n++) {
    char block[32];
    snprintf(block, sizeof block, "output%d", n);
    const char* fmt = athb_params_gets(p, block, "out_fmt");
    if (!fmt) continue;
    Output o;
    o.n = n;
    o.fmt = fmt;
    o.t = time0;
    if (athb_params_gets(p, block, "time")) athb_params_getd(p, block, "time", &o.t);
    if (athb_params_gets(p, block, "num")) athb_params_geti(p, block, "num", &o.num);
    if (athb_params_getd(p, block, "dt", &o.dt)) die("init_output");
    const char* out = athb_params_gets(p, block, "out");
    const std::string what = out ? out : "all";
    if (what != "all") {
      // single variable (src/output.c:229-345): the expression, the slice
      // bounds, the fixed scale, the palette
      o.expr = what;
      char defid[16];
      snprintf(defid, sizeof defid, "out%d", n);
      const char* id = athb_params_gets(p, block, "id");
      o.id = id ? id : defid;
      if (athb_params_gets(p, block, "usr_expr_flag")) athb_params_geti(p, block, "usr_expr_flag", &o.usr_expr);
      if (o.usr_expr ? !usr_expr_known(problem, what) : !expr_known(what)) {
        fprintf(stderr, "Could not parse expression %s, skipping it\n", what.c_str());
        continue;
      }
      o.sliced = athb_params_gets(p, block, "ix1") || athb_params_gets(p, block, "ix2");
      if (athb_params_gets(p, block, "dmin")) { o.sdmin = 1; athb_params_getd(p, block, "dmin", &o.dmin); }
      if (athb_params_gets(p, block, "dmax")) { o.sdmax = 1; athb_params_getd(p, block, "dmax", &o.dmax); }
      if (o.fmt != "ppm") {
        fprintf(stderr, "Unsupported %s/out_fmt=%s\n", block, o.fmt.c_str());
        exit(1);
      }
      const char* pal = athb_params_gets(p, block, "palette");
      const std::string name = pal ? pal : "rainbow";
      if (!palettes) {
        fprintf(stderr, "[init_output]: %s: the ppm palettes are read from a file: give -P <file> or "
                        "ATHB_PALETTES\n", block);
        exit(1);
      }
      o.rgb.resize(768);
      if (athb_palette_load(palettes, name.c_str(), o.rgb.data())) {
        fprintf(stderr, "Fatal error: could not find palette=%s (%s)\n", name.c_str(), athb_last_error());
        exit(1);
      }
      outs.push_back(o);
      continue;
    }
    if (o.fmt != "bin" && o.fmt != "tab") {
      fprintf(stderr, "Unsupported dump mode for %s/out_fmt=%s for out=all\n", block, o.fmt.c_str());
      exit(1);
    }
    if (o.fmt == "tab")
      if (const char* df = athb_params_gets(p, block, "dat_fmt")) o.dat_fmt = df;
    outs.push_back(o);
  }
  return outs;
}

// data_output(pGrid, 0): every output whose time has come is written once
// and its next time advanced by one interval (src/output.c:372-380, 432-439).
void data_output(athb_ctx* g, std::vector<Output>& outs, double time, const std::string& dir,
                 const std::string& base) {
  for (Output& o : outs) {
    if (!(time >= o.t)) continue;
    o.t += o.dt;
    if (o.fmt == "ppm") {
      if (o.sliced) {
        fprintf(stderr, "[output_ppm:] Data must be 2D\n");
        exit(1);
      }
      athb_ppm_opts po = {};
      po.expr = o.expr.c_str();
      po.usr_expr = o.usr_expr;
      po.rgb = o.rgb.data();
      po.sdmin = o.sdmin;
      po.sdmax = o.sdmax;
      po.dmin = (float)o.dmin;   // the reference assigns the Real scale to a float
      po.dmax = (float)o.dmax;
      po.num = o.num;
      const std::string path = output_name(dir, base, o.num, o.id, "ppm");
      if (athb_output_ppm(g, path.c_str(), &po, &o.gmin, &o.gmax)) die("output_ppm");
      o.num++;
      continue;
    }
    const std::string path = dump_name(dir, base, o.num, o.fmt.c_str());
    const int rc = o.fmt == "bin" ? athb_dump_bin(g, path.c_str())
                                  : athb_dump_tab(g, path.c_str(), o.dat_fmt.empty() ? nullptr : o.dat_fmt.c_str());
    if (rc) die(o.fmt == "bin" ? "dump_binary" : "dump_tab");
    o.num++;
  }
}

}  // namespace

int main(int argc, char** argv) {
  const char* athinput = "athinput";
  std::string problem, dir;
  bool quiet = false;
  const char* palettes = getenv("ATHB_PALETTES");
  for (int i = 1; i < argc; i++) {
    const char* a = argv[i];
    if (a[0] == '-' && a[1] != '\0' && a[2] == '\0') {
      switch (a[1]) {
      case 'i': if (i + 1 < argc) athinput = argv[++i]; break;
      case 'p': if (i + 1 < argc) problem = argv[++i]; break;
      case 'd': if (i + 1 < argc) dir = argv[++i]; break;
      case 'q': quiet = true; break;
      case 'P': if (i + 1 < argc) palettes = argv[++i]; break;
      default: usage(argv[0]);
      }
    }
  }
  std::vector<const char*> overrides;
  for (int i = 1; i < argc; i++)
    if (strchr(argv[i], '/') && strchr(strchr(argv[i], '/'), '=')) overrides.push_back(argv[i]);

  athb_params* p = nullptr;
  if (athb_params_open(athinput, &p)) die("par_open");
  for (const char* o : overrides)
    if (athb_params_override(p, o)) die("par_cmdline");
  if (problem.empty()) {
    // <job>/problem, else the configure line the reference's own athinput
    // files carry in <comment> ("config = --with-problem=blast")
    if (const char* pj = athb_params_gets(p, "job", "problem")) {
      problem = pj;
    } else if (const char* cf = athb_params_gets(p, "comment", "config")) {
      const char* w = strstr(cf, "--with-problem=");
      if (w) {
        w += strlen("--with-problem=");
        problem.assign(w, strcspn(w, " \t"));
      }
    }
    if (problem.empty()) {
      fprintf(stderr, "[main]: no problem generator: give -p <problem>, <job>/problem or "
                      "<comment>/config = --with-problem=<name>\n");
      return 1;
    }
  }
  const char* pid = athb_params_gets(p, "job", "problem_id");
  if (!pid) {
    fprintf(stderr, "[main]: job/problem_id not found\n");
    return 1;
  }
  const std::string base = pid;

  athb_ctx* g = nullptr;  // grid, problem, set_bvals, first new_dt
  if (athb_create_from_athinput(athinput, (int)overrides.size(), overrides.data(), problem.c_str(), &g))
    die("main");
  double time = 0.0, dt = 0.0;
  int nstep = 0, done = 0;
  if (athb_status(g, &time, &dt, &nstep, &done)) die("main");
  std::vector<Output> outs = read_outputs(p, time, problem, palettes);
  athb_params_close(p);

  printf("\nSetup complete, entering main loop...\n\n");
  printf("cycle=%i time=%e dt=%e\n", nstep, time, dt);
  fflush(stdout);
  while (done != 1) {
    data_output(g, outs, time, dir, base);
    if (quiet) {
      // run on the device until the next output is due or the run ends; an
      // output still due now (interval shorter than a step) waits one step,
      // as it does in the reference's loop
      double next = 0.0;
      bool any = false;
      for (const Output& o : outs)
        if (!any || o.t < next) { next = o.t; any = true; }
      const bool one = any && next <= time;
      if (athb_set_pause(g, next, any && !one ? 1 : 0)) die("main");
      int steps = 0;
      if (athb_run(g, one ? 1 : INT_MAX, &steps)) die("main");
    } else {
      int steps = 0;
      if (athb_run(g, 1, &steps)) die("main");
    }
    if (athb_status(g, &time, &dt, &nstep, &done)) die("main");
    if (!quiet) {
      printf("cycle=%i time=%e dt=%e\n", nstep, time, dt);
      fflush(stdout);
    }
  }
  if (quiet) printf("cycle=%i time=%e dt=%e\n", nstep, time, dt);
  printf("\nEnd of main loop\n\n");
  athb_destroy(g);
  return 0;
}
