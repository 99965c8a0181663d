// athb_output.cu -- the reference's data dumps written from the device state.
//
// Binary dump (src/dump_binary.c:25-134): the interior of the eight cell
// variables is converted to float on the GPU and only those 32 bytes per cell
// cross PCIe (instead of the 88 bytes per cell of a full-state download);
// the header and cell-centre coordinates are formed on the host.  Table dump
// (src/dump_tab.c:28-235): one row of the grid (j = (js+je)/2), so only that
// row of each plane is copied.  Both files are byte-identical to the
// reference's, because the values are bit-identical and they are formatted
// by the same conversions and printf formats.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "athb_internal.h"
#include "step_kernels.cuh"

using namespace athb;

namespace {

// Interior of planes d M1 M2 M3 E B1c B2c B3c as float, variable-major, rows
// of nx1 (the order dump_binary writes them).
__global__ void __launch_bounds__(kThreads) k_interior_float(const double* s, long long ps, int pitch, int is,
                                                           int js, int nx1, int nx2, float* out) {
  const long long n = (long long)nx1 * nx2;
  for (long long t = blockIdx.x * (long long)kThreads + threadIdx.x; t < 8 * n;
       t += (long long)gridDim.x * kThreads) {
    const int v = (int)(t / n);
    const long long c = t - v * n;
    const int j = (int)(c / nx1), i = (int)(c - (long long)j * nx1);
    out[t] = (float)s[v * ps + (long long)(j + js) * pitch + (i + is)];
  }
}

#define CUDA_TRY(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return athb_fail(ATHB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                               \
  } while (0)

// Cell-centre coordinate of index i (src/cc_pos.c:21-27, with idisp = -is).
double cc_x(double x0, int i, int is, double dx) { return x0 + ((double)(i - is) + 0.5) * dx; }

}  // namespace

extern "C" int athb_dump_bin(athb_ctx* c, const char* path) {
  if (!c || !path) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  const int nx1 = c->cfg.nx1, nx2 = c->cfg.nx2;
  const size_t n = (size_t)nx1 * nx2;
  // 8 floats per cell fit in the first 4 scratch planes, which hold nothing
  // between steps (the dump runs on the context's stream, after the step)
  float* dbuf = reinterpret_cast<float*>(c->scr);
  std::vector<float> data(8 * n);
  const long long blocks = std::min<long long>((8 * (long long)n + kThreads - 1) / kThreads, 148LL * 16);
  k_interior_float<<<(int)blocks, kThreads, 0, c->stream>>>(c->state[c->cur], c->ps, c->pitch, c->is, c->js, nx1,
                                                            nx2, dbuf);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(data.data(), dbuf, data.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "athb_dump_bin: %s", cudaGetErrorString(e));

  FILE* f = fopen(path, "wb");
  if (!f) return athb_fail(ATHB_ERR_IO, "[dump_binary]: Unable to open binary dump file %s", path);
  const int ndata[6] = {nx1, nx2, 0, 8, 0, 0};  // zones, NVAR = 8, NSCALARS = 0
  const float gam[2] = {(float)(c->cfg.gamma - 1.0), 0.0f};
  const float clock[2] = {(float)h.time, (float)h.dt_new};  // pGrid->dt before the tlim clamp
  std::vector<float> x1(nx1), x2(nx2);
  for (int i = 0; i < nx1; i++) x1[i] = (float)cc_x(c->x1_0, i + c->is, c->is, c->dx1);
  for (int j = 0; j < nx2; j++) x2[j] = (float)cc_x(c->x2_0, j + c->js, c->js, c->dx2);
  bool ok = fwrite(ndata, sizeof(int), 6, f) == 6 && fwrite(gam, sizeof(float), 2, f) == 2 &&
            fwrite(clock, sizeof(float), 2, f) == 2 && fwrite(x1.data(), sizeof(float), nx1, f) == (size_t)nx1 &&
            fwrite(x2.data(), sizeof(float), nx2, f) == (size_t)nx2 &&
            fwrite(data.data(), sizeof(float), data.size(), f) == data.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) return athb_fail(ATHB_ERR_IO, "[dump_binary]: write error on %s", path);
  return ATHB_OK;
}

extern "C" int athb_dump_tab(athb_ctx* c, const char* path, const char* dat_fmt) {
  if (!c || !path) return athb_fail(ATHB_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  StepState h;
  int rc = athb_read_clock(c, &h);
  if (rc) return rc;
  const int nx1 = c->cfg.nx1, nx2 = c->cfg.nx2;
  const int il = c->is, iu = c->ie, jl = c->js, ju = c->je;
  const int j = (ju + jl) / 2;
  // row j, columns [il, iu], of all 11 planes: one strided 2D copy
  std::vector<double> row((size_t)NSTATE * nx1);
  CUDA_TRY(cudaMemcpy2DAsync(row.data(), sizeof(double) * nx1,
                             c->state[c->cur] + (size_t)j * c->pitch + il, sizeof(double) * c->ps,
                             sizeof(double) * nx1, NSTATE, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  auto at = [&](int plane, int i) { return row[(size_t)plane * nx1 + (i - il)]; };

  char fmt[96];
  if (dat_fmt && *dat_fmt) {
    if (strlen(dat_fmt) > 80) return athb_fail(ATHB_ERR_ARG, "dat_fmt too long");
    snprintf(fmt, sizeof fmt, " %s", dat_fmt);
  } else {
    snprintf(fmt, sizeof fmt, " %%12.8e");
  }
  FILE* f = fopen(path, "w");
  if (!f) return athb_fail(ATHB_ERR_IO, "[dump_tab]: File Open Error Occured (%s)", path);
  const double gamma_1 = c->cfg.gamma - 1.0;
  // header (the reference tests Nx2 > 2 for the j and x2 column names)
  if (nx1 > 1) {
    fprintf(f, "# Nx1 = %d\n", iu - il + 1);
    fprintf(f, "# x1-size = %g\n", (iu - il + 1) * c->dx1);
  }
  if (nx2 > 1) {
    fprintf(f, "# Nx2 = %d\n", ju - jl + 1);
    fprintf(f, "# x2-size = %g\n", (ju - jl + 1) * c->dx2);
  }
  fprintf(f, "# Time = %g\n", h.time);
  fprintf(f, "#\n#");
  int col = 1;
  if (nx1 > 1) fprintf(f, " [%d]=i-zone", col++);
  if (nx2 > 2) fprintf(f, " [%d]=j-zone", col++);
  if (nx1 > 1) fprintf(f, " [%d]=x1", col++);
  if (nx2 > 2) fprintf(f, " [%d]=x2", col++);
  static const char* const names[] = {"d", "M1", "M2", "M3", "P", "E", "B1c", "B2c", "B3c", "B1i", "B1i", "B1i"};
  for (const char* nm : names) fprintf(f, " [%d]=%s", col++, nm);
  fprintf(f, "\n#\n");
  for (int i = il; i <= iu; i++) {
    const double x1 = cc_x(c->x1_0, i, c->is, c->dx1), x2 = cc_x(c->x2_0, j, c->js, c->dx2);
    if (nx1 > 1) fprintf(f, "%d ", i);
    if (nx2 > 1) fprintf(f, "%d ", j);
    if (nx1 > 1) fprintf(f, fmt, x1);
    if (nx2 > 1) fprintf(f, fmt, x2);
    const double d = at(P_D, i), m1 = at(P_M1, i), m2 = at(P_M2, i), m3 = at(P_M3, i), en = at(P_E, i);
    const double b1 = at(P_B1C, i), b2 = at(P_B2C, i), b3 = at(P_B3C, i);
    fprintf(f, fmt, d);
    fprintf(f, fmt, m1);
    fprintf(f, fmt, m2);
    fprintf(f, fmt, m3);
    const double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / d;
    const double me = 0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
    fprintf(f, fmt, (en - ke - me) * gamma_1);
    fprintf(f, fmt, en);
    fprintf(f, fmt, b1);
    fprintf(f, fmt, b2);
    fprintf(f, fmt, b3);
    fprintf(f, fmt, at(P_B1I, i));
    fprintf(f, fmt, at(P_B2I, i));
    fprintf(f, fmt, at(P_B3I, i));
    fprintf(f, "\n");
  }
  if (fclose(f) != 0) return athb_fail(ATHB_ERR_IO, "[dump_tab]: write error on %s", path);
  return ATHB_OK;
}

// ---------------------------------------------------------------------------
// Single-variable ppm images (src/output_ppm.c:37-143, src/output.c:111-123
// and the problem expressions of src/field_loop.c:161-179).
//
// The expression is evaluated on the GPU over the image's cells and stored as
// float (the reference's float **data, src/output.c:subset2), so 4 bytes per
// pixel cross PCIe; minmax2 (src/utils.c:148-162: serial MIN/MAX, whose NaN
// behaviour depends on the order) and the palette interpolation
// (compute_rgb, float arithmetic as the reference's) run on the host.
// ---------------------------------------------------------------------------
namespace {

enum PpmExpr { X_D, X_M1, X_M2, X_M3, X_E, X_B1C, X_B2C, X_B3C, X_ME, X_V1, X_V2, X_V3, X_P, X_CS2, X_S,
               X_J3, X_BP2, X_NONE };

int ppm_expr_of(const char* e, int usr) {
  if (!e) return X_NONE;
  if (usr) {   // get_usr_expr of the field-loop problem (src/field_loop.c:174-179)
    if (!strcmp(e, "J3")) return X_J3;
    if (!strcmp(e, "Bp2")) return X_BP2;
    return X_NONE;
  }
  static const char* names[] = {"d", "M1", "M2", "M3", "E", "B1c", "B2c", "B3c", "ME", "V1", "V2", "V3", "P",
                                "cs2", "S"};
  for (int k = 0; k <= X_S; k++)
    if (!strcmp(e, names[k])) return k;
  return X_NONE;
}

// data[j][i] = (float) expr(i + is, j + js), j < nx2, i < nx1 (subset2 takes
// the first cells of the interior whatever the slice bounds).
__global__ void __launch_bounds__(kThreads) k_ppm_expr(const double* s, long long ps, int pitch, int is, int js,
                                                      int nx1, int nx2, int expr, double gamma, double gamma_1,
                                                      double dx1, double dx2, float* out) {
  const long long n = (long long)nx1 * nx2;
  for (long long t = blockIdx.x * (long long)kThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kThreads) {
    const int j = (int)(t / nx1), i = (int)(t - (long long)j * nx1);
    const long long o = (long long)(j + js) * pitch + (i + is);
    const double d = s[P_D * ps + o], m1 = s[P_M1 * ps + o], m2 = s[P_M2 * ps + o], m3 = s[P_M3 * ps + o];
    const double e = s[P_E * ps + o], b1 = s[P_B1C * ps + o], b2 = s[P_B2C * ps + o], b3 = s[P_B3C * ps + o];
    double v;
    switch (expr) {
    case X_D: v = d; break;
    case X_M1: v = m1; break;
    case X_M2: v = m2; break;
    case X_M3: v = m3; break;
    case X_E: v = e; break;
    case X_B1C: v = b1; break;
    case X_B2C: v = b2; break;
    case X_B3C: v = b3; break;
    case X_ME: v = 0.5 * (b1 * b1 + b2 * b2 + b3 * b3); break;
    case X_V1: v = m1 / d; break;
    case X_V2: v = m2 / d; break;
    case X_V3: v = m3 / d; break;
    case X_P: v = gamma_1 * (e - 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / d); break;
    case X_CS2:
      v = (gamma * gamma_1 * (e - 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / d) / d);
      break;
    case X_S: {
      const double p = gamma_1 * (e - 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / d);
      v = p / pow(d, gamma);
      break;
    }
    case X_J3:
      v = ((s[P_B2I * ps + o] - s[P_B2I * ps + o - 1]) / dx1 - (s[P_B1I * ps + o] - s[P_B1I * ps + o - pitch]) / dx2);
      break;
    default: v = b1 * b1 + b2 * b2; break;   // X_BP2
    }
    out[t] = (float)v;
  }
}

// compute_rgb of src/output_ppm.c:147-180: float x, the palette's rgb and its
// forward differences der, scaled to 0..255 and truncated.
void ppm_rgb(double data, double mn, double mx, const float* rgb, const float* der, int* R, int* G, int* B) {
  if (!rgb || mn == mx) {
    *R = *G = *B = (data > mx ? 255 : 0);
    return;
  }
  const float x = (float)((data - mn) * 255.0 / (mx - mn));
  if (x <= 0.0 || x >= 255.0) {
    const int i = (x <= 0.0 ? 0 : 255);
    *R = (int)(rgb[i * 3 + 0] * 255.0);
    *G = (int)(rgb[i * 3 + 1] * 255.0);
    *B = (int)(rgb[i * 3 + 2] * 255.0);
    return;
  }
  const int i = (int)x;
  const float f = x - (float)i;
  *R = (int)((rgb[i * 3 + 0] + f * der[i * 3 + 0]) * 255.0);
  *G = (int)((rgb[i * 3 + 1] + f * der[i * 3 + 1]) * 255.0);
  *B = (int)((rgb[i * 3 + 2] + f * der[i * 3 + 2]) * 255.0);
}

}  // namespace

extern "C" int athb_output_ppm(athb_ctx* c, const char* path, const athb_ppm_opts* o, float* gmin, float* gmax) {
  if (!c || !path || !o || !gmin || !gmax) return athb_fail(ATHB_ERR_ARG, "null argument");
  const int expr = ppm_expr_of(o->expr, o->usr_expr);
  if (expr == X_NONE) return athb_fail(ATHB_ERR_NOTFOUND, "Could not parse expression %s", o->expr ? o->expr : "");
  const int nx1 = o->nx1 > 0 ? o->nx1 : c->cfg.nx1, nx2 = o->nx2 > 0 ? o->nx2 : c->cfg.nx2;
  if (nx1 > c->cfg.nx1 || nx2 > c->cfg.nx2) return athb_fail(ATHB_ERR_ARG, "image larger than the grid");
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const size_t n = (size_t)nx1 * nx2;
  // the image fits in the first scratch plane (free between steps; the call
  // runs on the context's stream after the step)
  float* dbuf = reinterpret_cast<float*>(c->scr);
  std::vector<float> data(n);
  const long long blocks = std::min<long long>(((long long)n + kThreads - 1) / kThreads, 148LL * 16);
  k_ppm_expr<<<(int)std::max(1LL, blocks), kThreads, 0, c->stream>>>(
      c->state[c->cur], c->ps, c->pitch, c->is, c->js, nx1, nx2, expr, c->cfg.gamma, c->cfg.gamma - 1.0, c->dx1,
      c->dx2, dbuf);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(data.data(), dbuf, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return athb_fail(ATHB_ERR_CUDA, "athb_output_ppm: %s", cudaGetErrorString(e));
  // minmax2 (src/utils.c:148-162), then the running extremes of the output
  float dmin = data[0], dmax = data[0];
  for (size_t k = 0; k < n; k++) {
    dmin = (dmin < data[k]) ? dmin : data[k];
    dmax = (dmax > data[k]) ? dmax : data[k];
  }
  if (o->num == 0) {
    *gmin = dmin;
    *gmax = dmax;
  } else {
    *gmin = (dmin < *gmin) ? dmin : *gmin;
    *gmax = (dmax > *gmax) ? dmax : *gmax;
  }
  FILE* f = fopen(path, "w");
  if (!f) return athb_fail(ATHB_ERR_IO, "[output_ppm]: Unable to open ppm file %s", path);
  fprintf(f, "P6\n");
  fprintf(f, "# dmin = %.7e, dmax = %.7e, gmin = %.7e, gmax = %.7e\n", dmin, dmax, *gmin, *gmax);
  fprintf(f, "%d %d\n255\n", nx1, nx2);
  if (o->sdmin) dmin = o->dmin;
  if (o->sdmax) dmax = o->dmax;
  float der[768];
  if (o->rgb)
    for (int ch = 0; ch < 3; ch++)
      for (int i = 0; i < 255; i++) der[3 * i + ch] = o->rgb[3 * (i + 1) + ch] - o->rgb[3 * i + ch];
  std::vector<unsigned char> row((size_t)3 * nx1);
  for (int j = nx2 - 1; j >= 0; j--) {
    for (int i = 0; i < nx1; i++) {
      const float v = data[(size_t)j * nx1 + i];
      int r, g, b;
      ppm_rgb(std::isnan(v) ? 0.0f : v, dmin, dmax, o->rgb, der, &r, &g, &b);
      row[3 * i + 0] = (unsigned char)r;
      row[3 * i + 1] = (unsigned char)g;
      row[3 * i + 2] = (unsigned char)b;
    }
    fwrite(row.data(), 1, row.size(), f);
  }
  const bool ok = fclose(f) == 0;
  if (!ok) return athb_fail(ATHB_ERR_IO, "[output_ppm]: write error on %s", path);
  return ATHB_OK;
}

// Palettes: a file of colour tables in either of two text forms, read by
// name: the C initialiser form "static float <name>[256*3] = { v, v, ... };"
// of the reference's palette.h, or one line per table "<name> v0 ... v767".
extern "C" int athb_palette_load(const char* path, const char* name, float rgb[768]) {
  if (!path || !name || !rgb) return athb_fail(ATHB_ERR_ARG, "null argument");
  FILE* f = fopen(path, "r");
  if (!f) return athb_fail(ATHB_ERR_IO, "cannot open palette file %s", path);
  std::string text;
  char buf[65536];
  size_t got;
  while ((got = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
  fclose(f);
  const size_t nlen = strlen(name);
  size_t pos = 0;
  while ((pos = text.find(name, pos)) != std::string::npos) {
    const bool start = pos == 0 || !(isalnum((unsigned char)text[pos - 1]) || text[pos - 1] == '_');
    const char after = pos + nlen < text.size() ? text[pos + nlen] : '\0';
    const bool end = !(isalnum((unsigned char)after) || after == '_');
    if (!(start && end)) { pos += nlen; continue; }
    size_t p = pos + nlen;
    const bool cform = text.compare(p, 1, "[") == 0;
    if (cform) {   // skip to the opening brace
      p = text.find('{', p);
      if (p == std::string::npos) break;
      p++;
    }
    const char* s = text.c_str() + p;
    int k = 0;
    for (; k < 768; k++) {
      while (*s && (isspace((unsigned char)*s) || *s == ',')) s++;
      char* endp = nullptr;
      // a C compiler converts the literal to double, then to float
      const double v = strtod(s, &endp);
      if (endp == s) break;
      rgb[k] = (float)v;
      s = endp;
    }
    if (cform && k > 0 && *s == '}')   // a short initialiser: the rest is zero
      for (; k < 768; k++) rgb[k] = 0.0f;
    if (k == 768) return ATHB_OK;
    pos += nlen;
  }
  return athb_fail(ATHB_ERR_NOTFOUND, "palette %s not found in %s", name, path);
}
