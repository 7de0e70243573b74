// Instantaneous-field files in the reference's layout, read and written
// straight from device state.
//
// Format (WRT_INSTANT_VARS_TG, src/processing/WRT_VARS_TG.f90:1-91, read by
// READ_3D_VARS, src/processing/READ_INTP_3D_VARS.f90:1-84): one file per
// variable; 4 x int32 (nx, ny, nz, iteration), 3 x float64 (time, Re, dt),
// then the global interior array F(1:nx, 1:ny, 1:nz) in Fortran order (no
// ghost layers), native byte order.  The MPI-IO subarray view of the
// reference writes exactly this byte stream for any number of ranks.
//
// File names: <dir>DNS_perixz_INSTANT_T<time as ES15.9>_<var>.D with var
// U, V, W, P (TG: Q_tg and PR_tg; IO: G_io and PR_io, src/processing/
// WRT_VARS_IO.f90:22-150) and, for a thermal IO section, T, D, E
// (TEMPERATURE, DENSITY, ENTHALPY).  An IO section that runs beside a TG
// section writes DNS_perioz_INSTANT_T... instead (WRT_VARS_IO.f90:24-28,
// RESTART_io.f90:25-29), so the two sections never overwrite each other.
// The coupled inflow / outflow section (x ghost columns) writes and reads
// I = 1..NCL1E = NCL1_io + 1, its outlet ghost column included, with NCL1E in
// the header (WRT_VARS_IO.f90:21-60, RESTART_io.f90:16-47).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "chapsim_internal.cuh"

using namespace chapsim;

namespace {

// Fortran ES15.9 of a time value: d.ddddddddd E+xx (two-digit exponent).
std::string es15_9(double t) {
  char b[64];
  snprintf(b, sizeof(b), "%.9E", t);
  return std::string(b);
}

std::string file_name(const char *dir, double time, const char *var, bool tg_and_io) {
  std::string s = dir ? dir : "";
  s += tg_and_io ? "DNS_perioz_INSTANT_T" : "DNS_perixz_INSTANT_T";
  s += es15_9(time);
  s += "_";
  s += var;
  s += ".D";
  return s;
}

}  // namespace

extern "C" {

int chapsim_instant_file_name(char *buf, int buflen, const char *dir, double time, const char *var, int tg_and_io) {
  if (!buf || buflen < 1 || !var) return CHAPSIM_ERR_ARG;
  const std::string s = file_name(dir, time, var, tg_and_io != 0);
  if ((int)s.size() + 1 > buflen) return CHAPSIM_ERR_ARG;
  memcpy(buf, s.c_str(), s.size() + 1);
  return CHAPSIM_OK;
}

int chapsim_instant_file_write(const char *path, int nx, int ny, int nz, int iteration, double time, double ren,
                               double dt, const double *field) {
  if (!path || !field || nx < 1 || ny < 1 || nz < 1) return CHAPSIM_ERR_ARG;
  FILE *f = fopen(path, "wb");
  if (!f) return CHAPSIM_ERR_ARG;
  const int32_t hi[4] = {nx, ny, nz, iteration};
  const double hr[3] = {time, ren, dt};
  bool ok = fwrite(hi, sizeof(int32_t), 4, f) == 4 && fwrite(hr, sizeof(double), 3, f) == 3;
  for (int k = 0; k < nz && ok; ++k)
    for (int j = 1; j <= ny && ok; ++j)
      ok = fwrite(field + (size_t)nx * (j + (size_t)(ny + 2) * k), sizeof(double), nx, f) == (size_t)nx;
  ok = (fclose(f) == 0) && ok;
  return ok ? CHAPSIM_OK : CHAPSIM_ERR_ARG;
}

int chapsim_instant_file_read(const char *path, int nx, int ny, int nz, int *iteration, double *time, double *ren,
                              double *dt, double *field) {
  if (!path || !field || nx < 1 || ny < 1 || nz < 1) return CHAPSIM_ERR_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) return CHAPSIM_ERR_ARG;
  int32_t hi[4];
  double hr[3];
  bool ok = fread(hi, sizeof(int32_t), 4, f) == 4 && fread(hr, sizeof(double), 3, f) == 3;
  // a different mesh would need READ_INTP_3D_VARS's interpolation (not built)
  ok = ok && hi[0] == nx && hi[1] == ny && hi[2] == nz;
  for (int k = 0; k < nz && ok; ++k)
    for (int j = 1; j <= ny && ok; ++j)
      ok = fread(field + (size_t)nx * (j + (size_t)(ny + 2) * k), sizeof(double), nx, f) == (size_t)nx;
  fclose(f);
  if (!ok) return CHAPSIM_ERR_ARG;
  if (iteration) *iteration = hi[3];
  if (time) *time = hr[0];
  if (ren) *ren = hr[1];
  if (dt) *dt = hr[2];
  return CHAPSIM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ contexts
namespace {

int download(chapsim_ctx *c, const double *dev, std::vector<double> &host) {
  host.resize((size_t)c->d.sz * c->d.nz);
  if (cudaMemcpyAsync(host.data(), dev, host.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    c->err = "instant-field download failed";
    cudaGetLastError();
    return CHAPSIM_ERR_CUDA;
  }
  return CHAPSIM_OK;
}

int upload(chapsim_ctx *c, double *dev, const std::vector<double> &host) {
  if (cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    c->err = "instant-field upload failed";
    cudaGetLastError();
    return CHAPSIM_ERR_CUDA;
  }
  return CHAPSIM_OK;
}

// BC_WALL_Q / BC_WALL_G (u, w ghosts 0; v = 0 on and beyond the walls) and
// BC_WALL_PR (zero normal gradient) on host copies.
void wall_bc_vec(const TGDev &d, std::vector<double> *q) {
  for (int k = 0; k < d.nz; ++k)
    for (int i = 0; i < d.nx; ++i) {
      const size_t b = i + d.sz * (size_t)k, top = b + d.sy * (size_t)(d.ny + 1);
      q[0][b] = 0.0; q[2][b] = 0.0; q[1][b] = 0.0; q[1][b + d.sy] = 0.0;
      q[0][top] = 0.0; q[2][top] = 0.0; q[1][top] = 0.0;
    }
}
void wall_bc_copy(const TGDev &d, std::vector<double> &p) {
  for (int k = 0; k < d.nz; ++k)
    for (int i = 0; i < d.nx; ++i) {
      const size_t b = i + d.sz * (size_t)k;
      p[b] = p[b + d.sy];
      p[b + d.sy * (size_t)(d.ny + 1)] = p[b + d.sy * (size_t)d.ny];
    }
}

}  // namespace

extern "C" {

int chapsim_write_instant(chapsim_ctx *ctx, const char *dir, int iteration, double time) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return CHAPSIM_ERR_CUDA;
  TGDev &d = ctx->d;
  const bool io = ctx->domain == CHAPSIM_IIO;
  const int xo = ctx->xoff, nxf = d.nx + xo;  // the file's x extent: NCL1E
  std::vector<const double *> src = io ? std::vector<const double *>{ctx->io.g[ctx->io_cur][0],
                                                                   ctx->io.g[ctx->io_cur][1],
                                                                   ctx->io.g[ctx->io_cur][2], d.p}
                                       : std::vector<const double *>{d.u, d.v, d.w, d.p};
  std::vector<const char *> names = {"U", "V", "W", "P"};
  if (io && ctx->io.thermal) {
    src.insert(src.end(), {ctx->io.T, ctx->io.D, ctx->io.h});
    names.insert(names.end(), {"T", "D", "E"});
  }
  std::vector<double> host, cols;
  for (size_t q = 0; q < src.size(); ++q) {
    int rc = download(ctx, src[q] - xo, host);
    if (rc) return rc;
    if (xo) {  // columns IC = 1 .. NCL1_io + 1 of every row
      cols.resize((size_t)nxf * (d.ny + 2) * d.nz);
      for (size_t r = 0; r < (size_t)(d.ny + 2) * d.nz; ++r)
        memcpy(cols.data() + r * nxf, host.data() + r * d.sy + 1, (size_t)nxf * sizeof(double));
    }
    const std::string path = file_name(dir, time, names[q], io && (ctx->iocfg.coupled || ctx->xnp));
    rc = chapsim_instant_file_write(path.c_str(), nxf, d.ny, d.nz, iteration, time, ctx->cfg.ren, ctx->cfg.dt,
                                    xo ? cols.data() : host.data());
    if (rc) {
      ctx->err = "cannot write " + path;
      return rc;
    }
  }
  return CHAPSIM_OK;
}

int chapsim_read_instant(chapsim_ctx *ctx, const char *dir, double time, int *iteration, double *time_out) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return CHAPSIM_ERR_CUDA;
  TGDev &d = ctx->d;
  const bool io = ctx->domain == CHAPSIM_IIO;
  const size_t n = (size_t)d.sz * d.nz;
  const int xo = ctx->xoff, nxf = d.nx + xo;  // the file's x extent: NCL1E
  if (xo && !ctx->inlet) {
    ctx->err = "coupled IO restart needs its TG inlet source (chapsim_io_set_inlet)";
    return CHAPSIM_ERR_STATE;
  }
  std::vector<double> f[7];
  const char *names[7] = {"U", "V", "W", "P", "T", "D", "E"};
  const int nf = (io && ctx->io.thermal) ? 7 : 4;
  if (io && ctx->io.thermal && !ctx->has_table) {
    ctx->err = "thermal IO restart needs the property table";
    return CHAPSIM_ERR_STATE;
  }
  int it = 0;
  double tm = 0.0;
  std::vector<double> cols;
  for (int q = 0; q < nf; ++q) {
    f[q].assign(n, 0.0);
    const std::string path = file_name(dir, time, names[q], io && (ctx->iocfg.coupled || ctx->xnp));
    if (xo) cols.assign((size_t)nxf * (d.ny + 2) * d.nz, 0.0);
    const int rc = chapsim_instant_file_read(path.c_str(), nxf, d.ny, d.nz, &it, &tm, nullptr, nullptr,
                                             xo ? cols.data() : f[q].data());
    if (rc) {
      ctx->err = "cannot read " + path + " (missing, or written for another mesh)";
      return rc;
    }
    if (xo)  // into columns IC = 1 .. NCL1_io + 1 of the ghost-column rows
      for (size_t r = 0; r < (size_t)(d.ny + 2) * d.nz; ++r)
        memcpy(f[q].data() + r * d.sy + 1, cols.data() + r * nxf, (size_t)nxf * sizeof(double));
  }
  // wall rows over every stored column (from the first one of the allocation)
  TGDev dw = d;
  dw.nx = (int)d.sy;
  wall_bc_vec(dw, f);
  wall_bc_copy(dw, f[3]);
  int rc;
  const size_t bytes = n * sizeof(double);
  if (!io) {
    // RESTART_INSTANT_VARS_TG + FLOWSTART's wall BCs; CONVH0 starts at zero
    double *dst[4] = {d.u, d.v, d.w, d.p};
    for (int q = 0; q < 4; ++q)
      if ((rc = upload(ctx, dst[q], f[q]))) return rc;
    for (int c = 0; c < 3; ++c)
      if (cudaMemsetAsync(d.h0[c], 0, n * (ctx->cfg.precision == CHAPSIM_MIXED ? sizeof(float) : sizeof(double)),
                          ctx->stream) != cudaSuccess)
        return CHAPSIM_ERR_CUDA;
  } else {
    // RESTART_INSTANT_VARS_IO (src/processing/RESTART_io.f90:1-140): G and
    // PR from U, V, W, P; T, D, E, RHOH = D E; then the wall ghosts, the
    // property update and u = G / rho_stag.  G0_io, EXPLT0_io and
    // RHS_ENERGY0 start at zero as after the reference's allocation.
    // The coupled section's arrays are addressed from their first (ghost)
    // column; its BC_CONV0 terms restart at zero too.
    IODev &iv = ctx->io;
    ctx->io_cur = 0;
    for (int q = 0; q < 3; ++q) {
      if ((rc = upload(ctx, iv.g[0][q] - xo, f[q]))) return rc;
      if (cudaMemsetAsync(iv.g[1][q] - xo, 0, bytes, ctx->stream) != cudaSuccess) return CHAPSIM_ERR_CUDA;
      if (cudaMemsetAsync((double *)d.h0[q] - xo, 0, bytes, ctx->stream) != cudaSuccess) return CHAPSIM_ERR_CUDA;
    }
    if ((rc = upload(ctx, d.p - xo, f[3]))) return rc;
    double *zero[] = {d.phi, d.rhsphi, iv.drho, iv.rhse0};
    for (double *z : zero)
      if (cudaMemsetAsync(z - xo, 0, bytes, ctx->stream) != cudaSuccess) return CHAPSIM_ERR_CUDA;
    if (iv.visc)
      for (int q = 0; q < 3; ++q)
        if (cudaMemsetAsync(iv.drhoi[q], 0, bytes, ctx->stream) != cudaSuccess) return CHAPSIM_ERR_CUDA;
    if (xo && cudaMemsetAsync(iv.bcp + (size_t)iv.bps * CHAPSIM_P_CONV0_X, 0, (size_t)iv.bps * 4 * sizeof(double),
                              ctx->stream) != cudaSuccess)
      return CHAPSIM_ERR_CUDA;
    if (iv.thermal) {
      std::vector<double> rhoh(n, 0.0);
      for (size_t t = 0; t < n; ++t) rhoh[t] = f[5][t] * f[6][t];
      if ((rc = upload(ctx, iv.T - xo, f[4])) || (rc = upload(ctx, iv.D - xo, f[5])) ||
          (rc = upload(ctx, iv.h - xo, f[6])) || (rc = upload(ctx, iv.rhoh - xo, rhoh)))
        return rc;
    }
    if ((rc = xo ? io_np_restart(ctx) : io_restart_fields(ctx))) return rc;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return CHAPSIM_ERR_CUDA;
  }
  for (auto &g : ctx->io_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (iteration) *iteration = it;
  if (time_out) *time_out = tm;
  return CHAPSIM_OK;
}

}  // extern "C"
