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
