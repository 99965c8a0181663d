// problems.cpp -- problem-generator hooks (initial conditions) and the cpaw2d
// error diagnostic.  The host generators use the reference's libm calls
// (sqrt/sin/cos/atan), so a state they produce is bit-identical to the
// reference's; athb_generate forms blast and field-loop states on the GPU
// instead (athb_problems_dev.cu) and uses these for the rest.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "athb_internal.h"

const char* athb_params_gets(const athb_params* p, const char* block, const char* name);

namespace {

constexpr double kPi = 3.14159265358979323846;  // PI, src/defs.h:97

enum { D = 0, M1, M2, M3, E, B1C, B2C, B3C, B1I, B2I, B3I };

struct View {
  const athb_grid_info& g;
  double* planes;
  double& at(int p, int j, int i) const {
    return planes[((size_t)p * g.sy + j) * g.sx + i];
  }
  // cell-centre position, src/cc_pos.c:25-31
  void cc_pos(int i, int j, double* x1, double* x2) const {
    *x1 = g.x1_0 + ((i + g.idisp) + 0.5) * g.dx1;
    *x2 = g.x2_0 + ((j + g.jdisp) + 0.5) * g.dx2;
  }
};

int getd(const athb_params* p, const char* b, const char* n, double* v) {
  return athb_params_getd(p, b, n, v);
}

// src/blast.c:25-72
int problem_blast(const athb_grid_info* gi, const athb_params* p, double* planes, void*) {
  View v{*gi, planes};
  const athb_grid_info& g = *gi;
  double rin, pa, prat, b0, angle;
  if (getd(p, "problem", "radius", &rin) || getd(p, "problem", "pamb", &pa) ||
      getd(p, "problem", "prat", &prat) || getd(p, "problem", "b0", &b0) ||
      getd(p, "problem", "angle", &angle))
    return ATHB_ERR_PARSE;
  const double theta = (kPi / 180.0) * angle;
  const double da = 1.0, ua = 0.0, va = 0.0, wa = 0.0;
  const double bxa = b0 * cos(theta), bya = b0 * sin(theta), bza = 0.0;
  for (int j = g.js; j <= g.je; j++) {
    for (int i = g.is; i <= g.ie; i++) {
      v.at(D, j, i) = da;
      v.at(M1, j, i) = da * ua;
      v.at(M2, j, i) = da * va;
      v.at(M3, j, i) = da * wa;
      v.at(B1I, j, i) = bxa;
      v.at(B2I, j, i) = bya;
      v.at(B3I, j, i) = bza;
      v.at(B1C, j, i) = bxa;
      v.at(B2C, j, i) = bya;
      v.at(B3C, j, i) = bza;
      if (i == g.ie && g.ie > g.is) v.at(B1I, j, i + 1) = bxa;
      if (j == g.je && g.je > g.js) v.at(B2I, j + 1, i) = bya;
      double x1, x2;
      v.cc_pos(i, j, &x1, &x2);
      const double rad = sqrt(x1 * x1 + x2 * x2);
      double pressure = pa;
      if (rad < rin) pressure = prat * pa;
      v.at(E, j, i) = pressure / g.gamma_1 + 0.5 * (bxa * bxa + bya * bya + bza * bza) +
                      0.5 * da * (ua * ua + va * va + wa * wa);
    }
  }
  return ATHB_OK;
}

// src/field_loop.c:40-137 (iprob = 1: loop in the x1-x2 plane)
int problem_field_loop(const athb_grid_info* gi, const athb_params* p, double* planes, void*) {
  View v{*gi, planes};
  const athb_grid_info& g = *gi;
  double rad, amp, vflow, iprob_d;
  if (getd(p, "problem", "rad", &rad) || getd(p, "problem", "amp", &amp) ||
      getd(p, "problem", "vflow", &vflow) || getd(p, "problem", "iprob", &iprob_d))
    return ATHB_ERR_PARSE;
  const int iprob = (int)iprob_d;
  std::vector<double> az((size_t)g.sx * g.sy, 0.0);
  auto AZ = [&](int j, int i) -> double& { return az[(size_t)j * g.sx + i]; };
  for (int j = g.js; j <= g.je + 1; j++) {
    for (int i = g.is; i <= g.ie + 1; i++) {
      double x1c, x2c;
      v.cc_pos(i, j, &x1c, &x2c);
      const double x1f = x1c - 0.5 * g.dx1;
      const double x2f = x2c - 0.5 * g.dx2;
      if (iprob == 1) {
        if ((x1f * x1f + x2f * x2f) < rad * rad) AZ(j, i) = amp * (rad - sqrt(x1f * x1f + x2f * x2f));
      }
    }
  }
  const double x1size = g.dx1 * (double)g.nx1;
  const double x2size = g.dx2 * (double)g.nx2;
  const double diag = sqrt(x1size * x1size + x2size * x2size);
  for (int j = g.js; j <= g.je; j++) {
    for (int i = g.is; i <= g.ie; i++) {
      v.at(D, j, i) = 1.0;
      v.at(M1, j, i) = v.at(D, j, i) * vflow * x1size / diag;
      v.at(M2, j, i) = v.at(D, j, i) * vflow * x2size / diag;
      v.at(M3, j, i) = 0.0;
      v.at(B1I, j, i) = (AZ(j + 1, i) - AZ(j, i)) / g.dx2;
      v.at(B2I, j, i) = -(AZ(j, i + 1) - AZ(j, i)) / g.dx1;
      v.at(B3I, j, i) = 0.0;
    }
  }
  for (int j = g.js; j <= g.je; j++) v.at(B1I, j, g.ie + 1) = (AZ(j + 1, g.ie + 1) - AZ(j, g.ie + 1)) / g.dx2;
  for (int i = g.is; i <= g.ie; i++) v.at(B2I, g.je + 1, i) = -(AZ(g.je + 1, i + 1) - AZ(g.je + 1, i)) / g.dx1;
  for (int j = g.js; j <= g.je; j++) {
    for (int i = g.is; i <= g.ie; i++) {
      const double b1 = 0.5 * (v.at(B1I, j, i) + v.at(B1I, j, i + 1));
      const double b2 = 0.5 * (v.at(B2I, j, i) + v.at(B2I, j + 1, i));
      const double b3 = v.at(B3I, j, i);
      v.at(B1C, j, i) = b1;
      v.at(B2C, j, i) = b2;
      v.at(B3C, j, i) = b3;
      const double m1 = v.at(M1, j, i), m2 = v.at(M2, j, i), m3 = v.at(M3, j, i);
      v.at(E, j, i) = 1.0 / g.gamma_1 + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) +
                      0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / v.at(D, j, i);
    }
  }
  return ATHB_OK;
}

// src/cpaw2d.c:56-185 and the vector potential A3 of src/cpaw2d.c:310-314
struct Cpaw {
  double sin_a, cos_a, b_par, b_perp, k_par;
  double A3(double x1, double x2) const {
    return b_par * (x1 * sin_a - x2 * cos_a) - (b_perp / k_par) * cos(k_par * (x1 * cos_a + x2 * sin_a));
  }
};

int problem_cpaw2d(const athb_grid_info* gi, const athb_params* p, double* planes, void*) {
  View v{*gi, planes};
  const athb_grid_info& g = *gi;
  athb_cpaw_wave q;
  if (athb_cpaw2d_wave(p, g.nx1, g.nx2, g.dx1, g.dx2, &q)) return ATHB_ERR_PARSE;
  Cpaw w{q.sin_a, q.cos_a, q.b_par, q.b_perp, q.k_par};
  const double den = q.den, v_par = q.v_par, v_perp = q.v_perp, b_perp = q.b_perp, pres = q.pres;
  const double dx1 = g.dx1, dx2 = g.dx2;
  for (int j = g.js; j <= g.je + 1; j++) {
    for (int i = g.is; i <= g.ie + 1; i++) {
      double x1, x2;
      v.cc_pos(i, j, &x1, &x2);
      const double cs = cos(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
      x1 -= 0.5 * g.dx1;
      x2 -= 0.5 * g.dx2;
      v.at(B1I, j, i) = -(w.A3(x1, x2 + dx2) - w.A3(x1, x2)) / dx2;
      v.at(B2I, j, i) = (w.A3(x1 + dx1, x2) - w.A3(x1, x2)) / dx1;
      v.at(B3I, j, i) = b_perp * cs;
    }
  }
  for (int j = g.js; j <= g.je; j++) {
    for (int i = g.is; i <= g.ie; i++) {
      double x1, x2;
      v.cc_pos(i, j, &x1, &x2);
      const double sn = sin(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
      const double cs = cos(w.k_par * (x1 * w.cos_a + x2 * w.sin_a));
      v.at(D, j, i) = den;
      v.at(M1, j, i) = den * (v_par * w.cos_a - v_perp * sn * w.sin_a);
      v.at(M2, j, i) = den * (v_par * w.sin_a + v_perp * sn * w.cos_a);
      v.at(M3, j, i) = den * v_perp * cs;
      const double b1 = 0.5 * (v.at(B1I, j, i) + v.at(B1I, j, i + 1));
      const double b2 = 0.5 * (v.at(B2I, j, i) + v.at(B2I, j + 1, i));
      const double b3 = b_perp * cs;
      v.at(B1C, j, i) = b1;
      v.at(B2C, j, i) = b2;
      v.at(B3C, j, i) = b3;
      const double m1 = v.at(M1, j, i), m2 = v.at(M2, j, i), m3 = v.at(M3, j, i);
      v.at(E, j, i) = pres / g.gamma_1 + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) +
                      0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / den;
    }
  }
  return ATHB_OK;
}

struct Entry { athb_problem_fn fn; void* user; };
std::map<std::string, Entry>& registry() {
  static std::map<std::string, Entry> r = {
      {"blast", {problem_blast, nullptr}},
      {"field_loop", {problem_field_loop, nullptr}},
      {"cpaw2d", {problem_cpaw2d, nullptr}},
  };
  return r;
}

}  // namespace

// The wave's scalars (src/cpaw2d.c:56-120): the direction of propagation
// from the grid's aspect, the wavelength along it, and the amplitudes.
int athb_cpaw2d_wave(const athb_params* p, int nx1, int nx2, double dx1, double dx2, athb_cpaw_wave* w) {
  double angle, b_par, b_perp, pres, v_par;
  if (getd(p, "problem", "angle", &angle) || getd(p, "problem", "b_par", &b_par) ||
      getd(p, "problem", "b_perp", &b_perp) || getd(p, "problem", "pres", &pres) ||
      getd(p, "problem", "v_par", &v_par))
    return ATHB_ERR_PARSE;
  double lambda;
  if (angle == 0.0) {
    w->sin_a = 0.0; w->cos_a = 1.0;
    lambda = nx1 * dx1;
  } else if (angle == 90.0) {
    w->sin_a = 1.0; w->cos_a = 0.0;
    lambda = nx2 * dx2;
  } else {
    if ((nx1 * dx1) == (nx2 * dx2)) {
      w->cos_a = w->sin_a = sqrt(0.5);
    } else {
      angle = atan((double)(nx1 * dx1) / (nx2 * dx2));
      w->sin_a = sin(angle);
      w->cos_a = cos(angle);
    }
    if (w->cos_a >= w->sin_a) lambda = nx1 * dx1 * w->cos_a;
    else lambda = nx2 * dx2 * w->sin_a;
  }
  w->k_par = 2.0 * kPi / lambda;
  w->b_par = b_par;
  w->den = 1.0;
  w->b_perp = b_perp;
  w->v_perp = b_perp / sqrt((double)w->den);
  w->v_par = v_par;
  w->pres = pres;
  return ATHB_OK;
}

extern "C" int athb_register_problem(const char* name, athb_problem_fn fn, void* user) {
  if (!name || !fn) return athb_fail(ATHB_ERR_ARG, "null argument");
  registry()[name] = Entry{fn, user};
  return ATHB_OK;
}

extern "C" int athb_problem_generate(const char* name, const athb_grid_info* g, const athb_params* p,
                                     double* planes) {
  if (!name || !g || !planes) return athb_fail(ATHB_ERR_ARG, "null argument");
  auto it = registry().find(name);
  if (it == registry().end()) return athb_fail(ATHB_ERR_NOTFOUND, "unknown problem \"%s\"", name);
  int rc = it->second.fn(g, p, planes, it->second.user);
  if (rc) return athb_fail(rc, "problem \"%s\" failed (missing <problem> parameter?)", name);
  return ATHB_OK;
}

// Kind of the generator registered under `name` when it is a built-in one
// (a user registration under the same name replaces it).
int athb_builtin_problem(const char* name) {
  auto it = registry().find(name ? name : "");
  if (it == registry().end()) return kProblemNone;
  if (it->second.fn == problem_blast) return kProblemBlast;
  if (it->second.fn == problem_field_loop) return kProblemFieldLoop;
  if (it->second.fn == problem_cpaw2d) return kProblemCpaw2d;
  return kProblemNone;
}

// The host path of athb_generate: run the registered generator on a host
// array and upload it (clock reset to dt = time = nstep = 0).
int athb_generate_host(athb_ctx* c, const char* name, const athb_params* p) {
  athb_grid_info gi;
  int rc = athb_grid_info_of(c, &gi);
  if (rc) return rc;
  std::vector<double> planes((size_t)ATHB_NPLANES * gi.sx * gi.sy, 0.0);
  rc = athb_problem_generate(name, &gi, p, planes.data());
  if (rc) return rc;
  rc = athb_upload(c, planes.data(), 0.0, 0.0, 0);
  // keep the initial cell-centred state: src/cpaw2d.c:160-180 (Soln)
  if (rc == ATHB_OK && athb_builtin_problem(name) == kProblemCpaw2d) rc = athb_keep_cpaw_soln(c);
  return rc;
}

extern "C" int athb_create_from_athinput(const char* path, int noverride, const char* const* overrides,
                                         const char* problem, athb_ctx** out) {
  if (!out) return athb_fail(ATHB_ERR_ARG, "null output pointer");
  *out = nullptr;
  athb_params* p = nullptr;
  int rc = athb_params_open(path, &p);
  if (rc) return rc;
  for (int k = 0; k < noverride && rc == ATHB_OK; k++) rc = athb_params_override(p, overrides[k]);
  athb_config cfg;
  if (rc == ATHB_OK) rc = athb_config_from_params(p, &cfg);
  athb_ctx* c = nullptr;
  if (rc == ATHB_OK) rc = athb_create(&cfg, &c);
  // src/main.c:124-149: problem -> set_bvals -> new_dt
  if (rc == ATHB_OK) rc = athb_generate(c, problem, p);
  athb_params_close(p);
  if (rc == ATHB_OK) rc = athb_set_bvals(c);
  if (rc == ATHB_OK) rc = athb_new_dt(c, nullptr);
  if (rc) { athb_destroy(c); return rc; }
  *out = c;
  return ATHB_OK;
}
