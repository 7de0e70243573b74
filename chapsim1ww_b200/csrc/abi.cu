// C ABI of libchapsim: context life cycle, host-side set-up (mesh, RK and
// line-solve coefficient tables, FFT plans), field transfer and the substep
// entry points.  Set-up restates, in host C++, the reference's initialisation
// routines: CONSPARA (src/CONSPARA.f90:41-73), COORDJR
// (src/COORDJR.f90:27-143,427-450,495-520), TDMA_COEF
// (src/TDMA_COEF.f90:53-119), CONS_RKCOEF (src/CONS_RKCOEF.f90:24-54) and
// FFT99_POIS3D_INIT (src/possion3d_FFT99.f90:54-220).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "chapsim_internal.cuh"

using namespace chapsim;

#define CKC(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);       \
      return CHAPSIM_ERR_CUDA;                                             \
    }                                                                      \
  } while (0)

#define REQUIRE(cond, code, msg)   \
  do {                             \
    if (!(cond)) {                 \
      if (ctx) ctx->err = (msg);   \
      return (code);               \
    }                              \
  } while (0)

namespace {

uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Uniform draw in [-1, 1) keyed by (seed, component, i, j, k), all 1-based.
double rnd_pm1(uint64_t seed, int comp, int i, int j, int k) {
  uint64_t ctr = ((uint64_t)comp << 60) ^ ((uint64_t)k << 40) ^ ((uint64_t)j << 20) ^ (uint64_t)i;
  uint64_t x = splitmix64(splitmix64(seed) ^ ctr);
  return -1.0 + 2.0 * ((double)(x >> 11) * (1.0 / 9007199254740992.0));
}

bool factor_plan(int n, FFTPlan &pl) {
  pl.n = n;
  pl.nrad = 0;
  int m = n;
  const int radices[] = {8, 4, 2, 3, 5, 7, 11};
  for (int r : radices)
    while (m % r == 0) {
      if (pl.nrad >= 16) return false;
      pl.rad[pl.nrad++] = r;
      m /= r;
    }
  for (int s = pl.nrad; s < 16; ++s) pl.rad[s] = 1;
  return m == 1;
}

// Cyclic factor tables for (1 - beta delta) with constant a = c, b = 1 - 2a
// (TDMAIJI_CYC coefficient-only recurrences, src/TDMAIJI_CYC.f90:100-146).
void cyc_tables(int n, double a, double *pp, double *h0, double *g2, double &b, double &qq) {
  const double c = a;
  b = 1.0 - 2.0 * a;
  h0[0] = c / b;
  g2[0] = -a / b;
  pp[0] = 1.0 / b;
  for (int i = 1; i <= n - 3; ++i) {
    pp[i] = 1.0 / (b - h0[i - 1] * a);
    h0[i] = c * pp[i];
    g2[i] = -(g2[i - 1] * a) * pp[i];
  }
  {
    const int i = n - 2;
    pp[i] = 1.0 / (b - h0[i - 1] * a);
    h0[i] = 0.0;
    g2[i] = (-c - g2[i - 1] * a) * pp[i];
  }
  pp[n - 1] = 0.0;
  h0[n - 1] = 0.0;
  g2[n - 1] = 0.0;
  for (int i = n - 3; i >= 0; --i) g2[i] = -h0[i] * g2[i + 1] + g2[i];
  qq = b + c * g2[0] + a * g2[n - 2];
}

// x = A^{-1} r for the cyclic tridiagonal (a, b, a) with the tables above
// (the same sweeps as the device routine cyc_line).
void cyc_apply(int n, double a, double b, double qq, const double *pp, const double *h0, const double *g2,
               double *r) {
  std::vector<double> g(n);
  g[0] = r[0] / b;
  for (int m = 1; m <= n - 2; ++m) g[m] = (r[m] - g[m - 1] * a) * pp[m];
  double gn = g[n - 2];
  for (int m = n - 3; m >= 0; --m) {
    gn = g[m] - h0[m] * gn;
    g[m] = gn;
  }
  const double xn = (r[n - 1] - a * g[0] - a * g[n - 2]) / qq;
  r[n - 1] = xn;
  for (int m = 0; m <= n - 2; ++m) r[m] = g[m] + g2[m] * xn;
}

// First row of the circulant inverse and the width past which its entries sum
// to less than 2^-60 of the central one (-1 when wider than wmax).
int circulant_band(int n, double a, double b, double qq, const double *pp, const double *h0, const double *g2,
                   int wmax, std::vector<double> &g) {
  g.assign(n, 0.0);
  g[0] = 1.0;
  cyc_apply(n, a, b, qq, pp, h0, g2, g.data());
  const double tol = ldexp(fabs(g[0]), -60);
  for (int w = 0; w <= wmax && 2 * w + 1 <= n; ++w) {
    double tail = 0.0;
    for (int m = w + 1; m <= n / 2; ++m) tail += fabs(g[m]) + (m != n - m ? fabs(g[n - m]) : 0.0);
    if (tail <= tol) return w;
  }
  return -1;
}

}  // namespace

extern "C" {

int chapsim_config_default(chapsim_config *cfg) {
  if (!cfg) return CHAPSIM_ERR_ARG;
  memset(cfg, 0, sizeof(*cfg));
  cfg->struct_size = (int32_t)sizeof(chapsim_config);
  cfg->nx = 64;
  cfg->ny = 64;
  cfg->nz = 64;
  cfg->lx = 4.0 * M_PI;
  cfg->lz = 4.0 * M_PI / 3.0;
  cfg->str2 = 2.0;
  cfg->istr2 = 1;
  cfg->flowdrvtp = 1;
  cfg->ren = 2800.0;
  cfg->dt = 1e-3;
  cfg->cfgv = 0.0;
  cfg->precision = CHAPSIM_FP64;
  cfg->device = 0;
  return CHAPSIM_OK;
}

// Captured graphs go stale when a launch parameter or a table they point to
// changes; a TG context's change also stales the pair graphs of the coupled
// sections it feeds (they hold its kernels).
static void drop_graphs(chapsim_ctx *ctx) {
  if (ctx->step_graph) { cudaGraphExecDestroy(ctx->step_graph); ctx->step_graph = nullptr; }
  for (auto &g : ctx->io_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto &g : ctx->pair_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (chapsim_ctx *io : ctx->fed)
    for (auto &g : io->pair_graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static void free_all(chapsim_ctx *ctx) {
  drop_graphs(ctx);
  for (void *p : ctx->table_allocs) cudaFree(p);
  ctx->table_allocs.clear();
  for (void *p : ctx->allocs) cudaFree(p);
  ctx->allocs.clear();
  for (auto &e : ctx->ev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  for (auto &e : ctx->evpool)
    if (e) cudaEventDestroy(e);
  ctx->evpool.clear();
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  ctx->own_stream = nullptr;
  ctx->stream = nullptr;
}

static int dalloc(chapsim_ctx *ctx, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    ctx->err = std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e);
    cudaGetLastError();
    return CHAPSIM_ERR_NOMEM;
  }
  ctx->allocs.push_back(*p);
  return CHAPSIM_OK;
}

static void setup_mesh(chapsim_ctx *ctx) {
  const chapsim_config &cf = ctx->cfg;
  const int ny = cf.ny, nnd2 = ny + 1;
  auto &ynd = ctx->ynd, &ycc = ctx->ycc, &dyfi = ctx->dyfi, &dyci = ctx->dyci, &wff = ctx->wff,
       &wfb = ctx->wfb;
  ynd.assign(ny + 2, 0.0); ycc.assign(ny + 2, 0.0); dyfi.assign(ny + 2, 0.0);
  dyci.assign(ny + 2, 0.0); wff.assign(ny + 2, 0.0); wfb.assign(ny + 2, 0.0);
  for (int j = 1; j <= nnd2; ++j) {
    if (cf.istr2 == 1)
      ynd[j] = tanh(cf.str2 * ((double)(j - 1) / (double)(nnd2 - 1) - 0.5)) / tanh(cf.str2 * 0.5);
    else
      ynd[j] = -1.0 + (double)(j - 1) * (2.0 / (double)ny);
  }
  for (int j = 1; j <= ny; ++j) {
    if (cf.istr2 == 1)
      ycc[j] = tanh(cf.str2 * (((double)(j - 1) + 0.5) / (double)(nnd2 - 1) - 0.5)) / tanh(cf.str2 * 0.5);
    else
      ycc[j] = 0.5 * (ynd[j] + ynd[j + 1]);
  }
  for (int j = 1; j <= ny; ++j) dyfi[j] = 1.0 / (ynd[j + 1] - ynd[j]);
  for (int j = 2; j <= nnd2 - 1; ++j) dyci[j] = 1.0 / ((ynd[j + 1] - ynd[j - 1]) * 0.5);
  dyci[1] = 2.0 / (ynd[2] - ynd[1]);
  dyci[nnd2] = 2.0 / (ynd[nnd2] - ynd[ny]);
  for (int jc = 2; jc <= ny; ++jc) {
    wff[jc] = (ynd[jc] - ycc[jc - 1]) / (ycc[jc] - ycc[jc - 1]);
    wfb[jc] = (ycc[jc] - ynd[jc]) / (ycc[jc] - ycc[jc - 1]);
  }
  wfb[1] = 1.0; wff[1] = 0.0; wfb[nnd2] = 0.0; wff[nnd2] = 1.0;
}

// Build every coefficient table into ctx->hcoef and return offsets through
// the lambda-set pointers after upload.
static int build_tables(chapsim_ctx *ctx) {
  const chapsim_config &cf = ctx->cfg;
  const int nx = cf.nx, ny = cf.ny, nz = cf.nz, lh = nx / 2 + 1, nnd2 = ny + 1;
  const double dxi = nx / cf.lx, dzi = nz / cf.lz, dxqi = dxi * dxi, dzqi = dzi * dzi;
  const double cvisc = 1.0 / cf.ren;
  const std::vector<double> &dyfi = ctx->dyfi, &dyci = ctx->dyci;
  std::vector<double> &H = ctx->hcoef;
  H.clear();
  auto alloc = [&](size_t n) { size_t o = H.size(); H.resize(o + ((n + 1) & ~(size_t)1), 0.0); return o; };
  const int Y = ny + 2;
  size_t o_dyfi = alloc(Y), o_dyci = alloc(Y), o_wff = alloc(Y), o_wfb = alloc(Y);
  for (int j = 0; j < Y; ++j) {
    H[o_dyfi + j] = dyfi[j]; H[o_dyci + j] = dyci[j]; H[o_wff + j] = ctx->wff[j]; H[o_wfb + j] = ctx->wfb[j];
  }
  size_t o_am[3], o_ac[3], o_ap[3];
  for (int c = 0; c < 3; ++c) { o_am[c] = alloc(Y); o_ac[c] = alloc(Y); o_ap[c] = alloc(Y); }
  // TDMA_COEF viscous y-operators (src/TDMA_COEF.f90:76-116)
  for (int c = 0; c < 3; ++c) {
    double *am = &H[o_am[c]], *ac = &H[o_ac[c]], *ap = &H[o_ap[c]];
    if (c != 1) {
      for (int jc = 2; jc <= ny - 1; ++jc) {
        am[jc] = dyfi[jc] * dyci[jc];
        ap[jc] = dyfi[jc] * dyci[jc + 1];
        ac[jc] = -(am[jc] + ap[jc]);
      }
      double ucaj = 4.0 / (2.0 / dyci[2] + 1.0 / dyfi[1]);
      am[1] = 0.0; ap[1] = ucaj * dyci[2]; ac[1] = -ucaj * (dyci[2] + 2.0 * dyfi[1]);
      ucaj = 4.0 / (2.0 / dyci[ny] + 1.0 / dyfi[ny]);
      am[ny] = ucaj * dyci[ny]; ap[ny] = 0.0; ac[ny] = -ucaj * (2.0 * dyfi[ny] + dyci[ny]);
    } else {
      for (int jc = 2; jc <= ny; ++jc) {
        am[jc] = dyfi[jc - 1] * dyci[jc];
        ap[jc] = dyfi[jc] * dyci[jc];
        ac[jc] = -(am[jc] + ap[jc]);
      }
      am[1] = 0.0; ap[1] = 0.0; ac[1] = 1.0;
      am[nnd2] = 0.0; ap[nnd2] = 0.0; ac[nnd2] = 1.0;
    }
  }
  // Poisson y-operator with Neumann folding (src/TDMA_COEF.f90:53-74)
  size_t o_amph = alloc(Y), o_acph = alloc(Y), o_apph = alloc(Y);
  {
    double *am = &H[o_amph], *ac = &H[o_acph], *ap = &H[o_apph];
    for (int jc = 1; jc <= ny; ++jc) {
      am[jc] = dyfi[jc] * dyci[jc];
      ap[jc] = dyfi[jc] * dyci[jc + 1];
      if (jc == 1) am[jc] = dyfi[jc] * dyci[jc] * 0.5;
      if (jc + 1 == nnd2) ap[jc] = dyfi[jc] * dyci[jc + 1] * 0.5;
    }
    for (int jc = 1; jc <= ny; ++jc) ac[jc] = -(am[jc] + ap[jc]);
    ac[1] = am[1] + ac[1]; am[1] = 0.0;
    ac[ny] = ap[ny] + ac[ny]; ap[ny] = 0.0;
  }
  // modified wavenumbers (src/possion3d_FFT99.f90:155-179)
  size_t o_ak1 = alloc(lh), o_ak3 = alloc(nz);
  for (int i = 0; i < lh; ++i) H[o_ak1 + i] = 2.0 * (1.0 - cos(2.0 * M_PI * (double)i / (double)nx)) * dxqi;
  for (int k = 0; k < nz; ++k) {
    // AN(K) = (K-1) 2 pi for K <= nz/2, -(nz-K+1) 2 pi beyond; cos is even.
    const int kk = k < nz / 2 ? k : -(nz - k);
    H[o_ak3 + k] = 2.0 * (1.0 - cos(2.0 * M_PI * (double)kk / (double)nz)) * dzqi;
  }
  // RK coefficients (src/CONS_RKCOEF.f90:28-54)
  const double tgam[4] = {1.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
  const double troh[4] = {0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0};
  size_t o_ya[4][3], o_ypp[4][3], o_yh[4][3], o_x[4][3], o_z[4][3];
  double xb[4], xa[4], xqq[4], zb[4], za[4], zqq[4];
  for (int ns = 0; ns < 4; ++ns) {
    const double alp = tgam[ns] + troh[ns];
    const double facoe = 0.5 * alp * cf.dt * cvisc;  // MOMFA_tg.f90:30
    for (int c = 0; c < 3; ++c) {
      o_ya[ns][c] = alloc(Y); o_ypp[ns][c] = alloc(Y); o_yh[ns][c] = alloc(Y);
      double *ya = &H[o_ya[ns][c]], *ypp = &H[o_ypp[ns][c]], *yh = &H[o_yh[ns][c]];
      const double *am = &H[o_am[c]], *ac = &H[o_ac[c]], *ap = &H[o_ap[c]];
      double hprev = 0.0;
      for (int j = 1; j <= ny; ++j) {
        const double a = -facoe * am[j], b = 1.0 - facoe * ac[j], cc = -facoe * ap[j];
        ya[j] = a;
        ypp[j] = j == 1 ? 1.0 / b : 1.0 / (b - hprev * a);
        yh[j] = cc * ypp[j];
        hprev = yh[j];
      }
    }
    for (int t = 0; t < 3; ++t) { o_x[ns][t] = alloc(nx); o_z[ns][t] = alloc(nz); }
    xa[ns] = -facoe * dxqi;
    za[ns] = -facoe * dzqi;
    cyc_tables(nx, xa[ns], &H[o_x[ns][0]], &H[o_x[ns][1]], &H[o_x[ns][2]], xb[ns], xqq[ns]);
    cyc_tables(nz, za[ns], &H[o_z[ns][0]], &H[o_z[ns][1]], &H[o_z[ns][2]], zb[ns], zqq[ns]);
  }
  // banded inverses of the y factors: (A^{-1})_{j, j+m}, |m| <= wy
  const int YW = 16;  // AYB_WMAX in tg_kernels.cu
  size_t o_yg[4][3];
  int wy[4];
  for (int ns = 0; ns < 4; ++ns) {
    wy[ns] = 0;
    std::vector<std::vector<double>> inv(3);
    for (int c = 0; c < 3; ++c) {
      const double *ya = &H[o_ya[ns][c]], *ypp = &H[o_ypp[ns][c]], *yh = &H[o_yh[ns][c]];
      std::vector<double> &A = inv[c];
      A.assign((size_t)(ny + 1) * (ny + 1), 0.0);  // A[j*(ny+1)+col], 1-based
      std::vector<double> x(ny + 2);
      for (int col = 1; col <= ny; ++col) {
        // Thomas on e_col with the precomputed pivots (same sweeps as the device)
        double g = (col == 1 ? 1.0 : 0.0) * ypp[1];
        x[1] = g;
        for (int j = 2; j <= ny; ++j) { g = ((j == col ? 1.0 : 0.0) - ya[j] * g) * ypp[j]; x[j] = g; }
        double xv = g;
        for (int j = ny - 1; j >= 1; --j) { xv = x[j] - yh[j] * xv; x[j] = xv; }
        for (int j = 1; j <= ny; ++j) A[(size_t)j * (ny + 1) + col] = x[j];
      }
      std::vector<double> dm(ny + 1);
      for (int j = 1; j <= ny; ++j) {
        double rmax = 0.0;
        for (int col = 1; col <= ny; ++col) rmax = fmax(rmax, fabs(A[(size_t)j * (ny + 1) + col]));
        const double tol = ldexp(rmax, -60);
        // dm[m] = |A(j, j+m)| + |A(j, j-m)|; smallest w whose tail sum is below tol
        for (int m = 0; m <= ny; ++m) {
          double v = 0.0;
          if (j + m <= ny) v += fabs(A[(size_t)j * (ny + 1) + j + m]);
          if (m > 0 && j - m >= 1) v += fabs(A[(size_t)j * (ny + 1) + j - m]);
          dm[m] = v;
        }
        double tail = 0.0;
        int w = ny;
        for (int m = ny; m >= 1; --m) {
          tail += dm[m];
          if (tail > tol) break;
          w = m - 1;
        }
        wy[ns] = w > wy[ns] ? w : wy[ns];
      }
    }
    if (wy[ns] > YW) wy[ns] = -1;
    for (int c = 0; c < 3; ++c) {
      o_yg[ns][c] = alloc((size_t)(ny + 1) * (2 * YW + 1));
      if (wy[ns] < 0) continue;
      const std::vector<double> &A = inv[c];
      for (int j = 1; j <= ny; ++j)
        for (int m = -wy[ns]; m <= wy[ns]; ++m) {
          const int col = j + m;
          if (col >= 1 && col <= ny)
            H[o_yg[ns][c] + (size_t)j * (2 * YW + 1) + YW + m] = A[(size_t)j * (ny + 1) + col];
        }
    }
  }
  // truncated circulant inverses of the x and z factors
  size_t o_gx[4], o_gz[4];
  int wx[4], wz[4];
  for (int ns = 0; ns < 4; ++ns) {
    std::vector<double> g;
    const int band_max = BAND_ROWS - 1;  // BAND_WMAX in tg_kernels.cu
    wx[ns] = circulant_band(nx, xa[ns], xb[ns], xqq[ns], &H[o_x[ns][0]], &H[o_x[ns][1]], &H[o_x[ns][2]], band_max, g);
    o_gx[ns] = alloc(band_max + 1);
    if (wx[ns] >= 0) for (int m = 0; m <= wx[ns]; ++m) H[o_gx[ns] + m] = g[m];
    wz[ns] = circulant_band(nz, za[ns], zb[ns], zqq[ns], &H[o_z[ns][0]], &H[o_z[ns][1]], &H[o_z[ns][2]], band_max, g);
    o_gz[ns] = alloc(band_max + 1);
    if (wz[ns] >= 0) for (int m = 0; m <= wz[ns]; ++m) H[o_gz[ns] + m] = g[m];
  }
  // FFT twiddles exp(-2 pi i m / n)
  size_t o_twx = alloc(2 * (size_t)nx), o_twz = alloc(2 * (size_t)nz);
  for (int m = 0; m < nx; ++m) {
    H[o_twx + 2 * m] = cos(2.0 * M_PI * (double)m / nx);
    H[o_twx + 2 * m + 1] = -sin(2.0 * M_PI * (double)m / nx);
  }
  for (int m = 0; m < nz; ++m) {
    H[o_twz + 2 * m] = cos(2.0 * M_PI * (double)m / nz);
    H[o_twz + 2 * m + 1] = -sin(2.0 * M_PI * (double)m / nz);
  }
  // float twiddles packed after the doubles (2 floats per double slot)
  size_t o_twx32 = alloc(nx), o_twz32 = alloc(nz);
  {
    float *fx = reinterpret_cast<float *>(&H[o_twx32]);
    for (int m = 0; m < 2 * nx; ++m) fx[m] = (float)H[o_twx + m];
    float *fz = reinterpret_cast<float *>(&H[o_twz32]);
    for (int m = 0; m < 2 * nz; ++m) fz[m] = (float)H[o_twz + m];
  }

  // upload
  void *p = nullptr;
  int rc = dalloc(ctx, &p, H.size() * sizeof(double));
  if (rc) return rc;
  ctx->dcoef = (double *)p;
  CKC(cudaMemcpy(ctx->dcoef, H.data(), H.size() * sizeof(double), cudaMemcpyHostToDevice));
  const double *D = ctx->dcoef;
  TGDev &d = ctx->d;
  d.dyfi = D + o_dyfi; d.dyci = D + o_dyci; d.wff = D + o_wff; d.wfb = D + o_wfb;
  for (int c = 0; c < 3; ++c) { d.amvr[c] = D + o_am[c]; d.acvr[c] = D + o_ac[c]; d.apvr[c] = D + o_ap[c]; }
  d.amph = D + o_amph; d.acph = D + o_acph; d.apph = D + o_apph;
  d.ak1 = D + o_ak1; d.ak3 = D + o_ak3;
  d.dxi = dxi; d.dzi = dzi; d.dxqi = dxqi; d.dzqi = dzqi; d.cvisc = cvisc; d.dt = cf.dt;
  double volm = 0.0, area = 0.0;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      area += 1.0 / dyfi[j] / dzi;
      for (int i = 1; i <= nx; ++i) volm += 1.0 / dyfi[j];
    }
  d.volm = volm;
  ctx->area_inlet = area;
  for (int ns = 0; ns < 4; ++ns) {
    SubParams &sp = ctx->sp[ns];
    sp.ns = ns;
    sp.gam = tgam[ns]; sp.roh = troh[ns]; sp.alp = tgam[ns] + troh[ns];
    for (int c = 0; c < 3; ++c) { sp.ya[c] = D + o_ya[ns][c]; sp.ypp[c] = D + o_ypp[ns][c]; sp.yh[c] = D + o_yh[ns][c]; }
    sp.xpp = D + o_x[ns][0]; sp.xh0 = D + o_x[ns][1]; sp.xg2 = D + o_x[ns][2];
    sp.xa = xa[ns]; sp.xb = xb[ns]; sp.xqq = xqq[ns];
    sp.zpp = D + o_z[ns][0]; sp.zh0 = D + o_z[ns][1]; sp.zg2 = D + o_z[ns][2];
    sp.za = za[ns]; sp.zb = zb[ns]; sp.zqq = zqq[ns];
    sp.flowdrvtp = cf.flowdrvtp;
    sp.dp_const = -0.5 * cf.cfgv * sp.alp * cf.dt;
    sp.gx = D + o_gx[ns];
    sp.gz = D + o_gz[ns];
    sp.wx = wx[ns];
    sp.wz = wz[ns];
    for (int m = 0; m < BAND_ROWS; ++m) {
      sp.bgx[m] = (wx[ns] >= 0 && m <= wx[ns]) ? H[o_gx[ns] + m] : 0.0;
      sp.bgz[m] = (wz[ns] >= 0 && m <= wz[ns]) ? H[o_gz[ns] + m] : 0.0;
    }
    sp.band = (wx[ns] >= 0 && wz[ns] >= 0 && ctx->allow_band) ? 1 : 0;
    for (int c = 0; c < 3; ++c) sp.yg[c] = D + o_yg[ns][c];
    sp.wy = ctx->allow_band ? wy[ns] : -1;
  }
  ctx->fx.tw64 = reinterpret_cast<const double2 *>(D + o_twx);
  ctx->fz.tw64 = reinterpret_cast<const double2 *>(D + o_twz);
  ctx->fx.tw32 = reinterpret_cast<const float2 *>(D + o_twx32);
  ctx->fz.tw32 = reinterpret_cast<const float2 *>(D + o_twz32);
  return CHAPSIM_OK;
}

// FISHPACK's x roots and transforms for Dirichlet / Neumann ends
// (src/possion3d_fishpack_reform.f90:104-163): XRT(I) = -4 DXQI sin^2((I - DI)
// DX) with DX = pi / (2 (L + LRDEL)); the transforms are FFTPACK's SINT,
// SINQF / SINQB, COST and COSQF / COSQB (libs/fishpack4.1/fftpack.f, from
// their documented sums), built as dense matrices, the forward one divided
// by the final SCALX, both stored transposed for the device kernels.  The
// spectral descriptor dnp has nx lines with shifts -XRT(I).
static int xnp_setup(chapsim_ctx *ctx, int lp) {
  const int n = ctx->cfg.nx;
  const int lrdel = ((lp - 1) * (lp - 3) * (lp - 5)) / 3;
  const double sc = (double)(n + lrdel), dx = M_PI / (2.0 * sc);
  const double di = lp == 2 ? 0.0 : (lp == 4 ? 1.0 : 0.5);
  const double scalx = (lp == 3 || lp == 5) ? 4.0 * sc : 2.0 * sc;
  std::vector<double> ak1(n), ft((size_t)n * n), bt((size_t)n * n);
  for (int i = 1; i <= n; ++i) {
    const double sn = sin(((double)i - di) * dx);
    ak1[i - 1] = 4.0 * ctx->d.dxqi * sn * sn;  // -XRT(I)
  }
  if (lp == 4) ak1[0] = 0.0;  // sin(0): the zero mode, exactly
  auto fwd = [&](int i, int k) -> double {  // coefficient of X(K) in the forward output I, 1-based
    switch (lp) {
      case 2: return 2.0 * sin((double)k * i * M_PI / (n + 1));
      case 3: return k == n ? ((i - 1) % 2 ? -1.0 : 1.0) : 2.0 * sin((2.0 * i - 1.0) * k * M_PI / (2.0 * n));
      case 4:
        if (k == 1) return 1.0;
        if (k == n) return (i - 1) % 2 ? -1.0 : 1.0;
        return 2.0 * cos((double)(k - 1) * (i - 1) * M_PI / (n - 1));
      default: return k == 1 ? 1.0 : 2.0 * cos((2.0 * i - 1.0) * (k - 1) * M_PI / (2.0 * n));
    }
  };
  auto bwd = [&](int i, int k) -> double {  // coefficient of X(K) in the backward output I
    switch (lp) {
      case 3: return 4.0 * sin((2.0 * k - 1.0) * i * M_PI / (2.0 * n));
      case 5: return 4.0 * cos((2.0 * k - 1.0) * (i - 1) * M_PI / (2.0 * n));
      default: return fwd(i, k);  // SINT and COST are their own inverses
    }
  };
  for (int i = 1; i <= n; ++i)
    for (int k = 1; k <= n; ++k) {
      ft[(size_t)(k - 1) * n + (i - 1)] = fwd(i, k) / scalx;
      bt[(size_t)(k - 1) * n + (i - 1)] = bwd(i, k);
    }
  chapsim::TGDev &s = ctx->dnp;
  s = ctx->d;
  s.lh = n;
  s.lp = n + (n & 1);
  void *p = nullptr;
  int rc;
  const size_t nsp = (size_t)s.lp * ctx->cfg.ny * ctx->cfg.nz;
  if ((rc = dalloc(ctx, &p, nsp * sizeof(double2)))) return rc;
  s.spec = p;
  if ((rc = dalloc(ctx, &p, nsp * sizeof(double2)))) return rc;
  s.ypiv = (double2 *)p;
  if ((rc = dalloc(ctx, &p, (size_t)n * sizeof(double)))) return rc;
  s.ak1 = (const double *)p;
  CKC(cudaMemcpyAsync(p, ak1.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = dalloc(ctx, &p, (size_t)n * n * sizeof(double)))) return rc;
  ctx->xnp_f = (double *)p;
  CKC(cudaMemcpyAsync(p, ft.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = dalloc(ctx, &p, (size_t)n * n * sizeof(double)))) return rc;
  ctx->xnp_b = (double *)p;
  CKC(cudaMemcpyAsync(p, bt.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = chapsim::xnp_pivots(ctx))) return rc;
  std::vector<double2> qw;
  if (lp == 3 || lp == 5) {
    // the quarter-wave pairs through the complex FFT: exp(-i pi m / (2 N))
    qw.resize(n);
    for (int m = 0; m < n; ++m) qw[m] = make_double2(cos(M_PI * m / (2.0 * n)), -sin(M_PI * m / (2.0 * n)));
    if ((rc = dalloc(ctx, &p, (size_t)n * sizeof(double2)))) return rc;
    ctx->xnp_qw = (double2 *)p;
    CKC(cudaMemcpyAsync(p, qw.data(), (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    ctx->xnp_rscal = 1.0 / scalx;
    if ((rc = chapsim::xnp_q_setup(ctx))) return rc;
  }
  CKC(cudaStreamSynchronize(ctx->stream));  // the host vectors go out of scope
  ctx->xnp = lp;
  return CHAPSIM_OK;
}

static int create_ctx(const chapsim_config *cfg, const chapsim_io_config *iocfg, chapsim_ctx **out) {
  chapsim_ctx *ctx = nullptr;
  if (!cfg || !out) return CHAPSIM_ERR_ARG;
  *out = nullptr;
  if (cfg->struct_size != (int32_t)sizeof(chapsim_config)) return CHAPSIM_ERR_ARG;
  if (cfg->nx < 8 || cfg->nz < 8 || cfg->ny < 4 || (cfg->nx & 1) || (cfg->nz & 1)) return CHAPSIM_ERR_ARG;
  if (!(cfg->lx > 0) || !(cfg->lz > 0) || !(cfg->ren > 0) || !(cfg->dt > 0)) return CHAPSIM_ERR_ARG;
  if (cfg->istr2 != 0 && cfg->istr2 != 1) return CHAPSIM_ERR_ARG;
  if (cfg->flowdrvtp != 1 && cfg->flowdrvtp != 2) return CHAPSIM_ERR_ARG;
  if (cfg->precision != CHAPSIM_FP64 && cfg->precision != CHAPSIM_MIXED) return CHAPSIM_ERR_ARG;
  if (cfg->nx > 4096 || cfg->nz > 4096 || cfg->ny > 4096) return CHAPSIM_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CHAPSIM_ERR_NODEVICE;
  }
  if (cfg->device < 0 || cfg->device >= ndev) return CHAPSIM_ERR_ARG;
  ctx = new chapsim_ctx();
  ctx->cfg = *cfg;
  ctx->device = cfg->device;
  if (iocfg) {
    ctx->domain = CHAPSIM_IIO;
    ctx->iocfg = *iocfg;
  }
  int rc = CHAPSIM_OK;
  FFTPlan px{}, pz{};
  if (!factor_plan(cfg->nx, px) || !factor_plan(cfg->nz, pz)) {
    delete ctx;
    return CHAPSIM_ERR_UNSUPPORTED;  // lengths with prime factors > 11
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) { delete ctx; return CHAPSIM_ERR_CUDA; }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return CHAPSIM_ERR_CUDA;
  }
  ctx->own_stream = ctx->stream;
  for (auto &e : ctx->ev)
    if (cudaEventCreate(&e) != cudaSuccess) { free_all(ctx); delete ctx; return CHAPSIM_ERR_CUDA; }
  ctx->evpool.assign((size_t)chapsim_ctx::kEvSub * (CHAPSIM_PH_COUNT + 1), nullptr);
  for (auto &e : ctx->evpool)
    if (cudaEventCreate(&e) != cudaSuccess) { free_all(ctx); delete ctx; return CHAPSIM_ERR_CUDA; }
  setup_mesh(ctx);
  TGDev &d = ctx->d;
  d.nx = cfg->nx; d.ny = cfg->ny; d.nz = cfg->nz; d.lh = cfg->nx / 2 + 1;
  d.lp = (d.lh + 1) & ~1;
  d.sy = cfg->nx;
  if (iocfg && iocfg->bcx_in != 3) {
    // the coupled inflow / outflow section: x ghost columns IC = 0 and
    // NCL1_io + 1 in every field (NCL1S:NCL1E, src/MEMALLOCT.f90:154-168);
    // field pointers address IC = 1
    d.xnp = 1;
    d.sy = cfg->nx + 2;
    ctx->xoff = 1;
  }
  d.sz = d.sy * (cfg->ny + 2);
  const size_t n = (size_t)d.sz * cfg->nz;
  // every field allocation carries two values of slack past its n, so that
  // a whole-array pass from the offset pointer stays inside it
  const size_t nal = n + 2;
  const int xo = ctx->xoff;
  void *p = nullptr;
  {
    const bool mixed = cfg->precision == CHAPSIM_MIXED;
    // TG temporaries follow the precision form; the IO kernels keep EXPLT0 and
    // RHS_io in FP64 (their mixed form narrows only the Poisson spectra)
    const size_t tsz = (mixed && !iocfg) ? sizeof(float) : sizeof(double);
    double **f64[] = {&d.u, &d.v, &d.w, &d.p, &d.phi, &d.rhsphi, &d.res};
    for (double **f : f64) {
      if ((rc = dalloc(ctx, &p, nal * sizeof(double)))) goto fail;
      *f = (double *)p + xo;
      cudaMemsetAsync(p, 0, nal * sizeof(double), ctx->stream);
    }
    for (int c = 0; c < 3; ++c) {
      void **tmp[] = {&d.h0[c], &d.rhs[c], &d.dq[c]};
      for (void **f : tmp) {
        // the explicit IO substep needs EXPLT0 only; the semi-implicit one
        // also keeps RHS_io per component
        if (iocfg && (f == &d.dq[c] || (f == &d.rhs[c] && !iocfg->visc_scheme))) continue;
        if ((rc = dalloc(ctx, &p, nal * tsz))) goto fail;
        *f = (char *)p + xo * tsz;
        cudaMemsetAsync(p, 0, nal * tsz, ctx->stream);
      }
    }
    if (iocfg) {
      IODev &io = ctx->io;
      double **f64io[] = {&io.g[0][0], &io.g[0][1], &io.g[0][2], &io.g[1][0], &io.g[1][1], &io.g[1][2],
                          &io.drho, &io.rhoh, &io.h, &io.T, &io.D, &io.D0, &io.mu, &io.mu0, &io.kap, &io.rhse0,
                          &io.msum};
      for (double **f : f64io) {
        if ((rc = dalloc(ctx, &p, nal * sizeof(double)))) goto fail;
        *f = (double *)p + xo;
        cudaMemsetAsync(p, 0, nal * sizeof(double), ctx->stream);
      }
      io.visc = iocfg->visc_scheme ? 1 : 0;
      if (io.visc) {
        for (int c = 0; c < 3; ++c)
          for (double **f : {&io.drhoi[c], &io.stg[c], &io.stg[c + 3]}) {
            if ((rc = dalloc(ctx, &p, n * sizeof(double)))) goto fail;
            *f = (double *)p;
            cudaMemsetAsync(p, 0, n * sizeof(double), ctx->stream);
          }
        // AMVR1 and APVRN of TDMA_COEF (src/TDMA_COEF.f90:87-96)
        const int ny = cfg->ny;
        double ucaj = 4.0 / (2.0 / ctx->dyci[2] + 1.0 / ctx->dyfi[1]);
        io.amvr1 = ucaj * (2.0 * ctx->dyfi[1]);
        ucaj = 4.0 / (2.0 / ctx->dyci[ny] + 1.0 / ctx->dyfi[ny]);
        io.apvrn = ucaj * (2.0 * ctx->dyfi[ny]);
      }
      io.bps = (int64_t)(cfg->ny + 2) * cfg->nz;
      if ((rc = dalloc(ctx, &p, ((size_t)io.bps * chapsim::P_ALL + 8) * sizeof(double)))) goto fail;
      io.bcp = (double *)p;
      io.bcs = io.bcp + (size_t)io.bps * chapsim::P_ALL;
      cudaMemsetAsync(p, 0, ((size_t)io.bps * chapsim::P_ALL + 8) * sizeof(double), ctx->stream);
      if ((rc = dalloc(ctx, &p, 2 * sizeof(unsigned long long)))) goto fail;
      io.bad = (unsigned long long *)p;
      io.model_again = io.bad + 1;
      cudaMemsetAsync(p, 0, 2 * sizeof(unsigned long long), ctx->stream);
      io.thermal = iocfg->thermal ? 1 : 0;
      io.cthecd = 1.0 / cfg->ren / iocfg->prt;  // CTHECD, src/Flow_State.f90:87
      io.qw_bot = iocfg->qw_bot;
      io.qw_top = iocfg->qw_top;
      io.isothermal = iocfg->thermal ? iocfg->isothermal : 0;
      io.gravdir = iocfg->gravdir;
      io.f_a = iocfg->f_a;
      io.cfgv = cfg->cfgv;
      io.flowdrvtp = cfg->flowdrvtp;
      d.pin_last = 1;  // FISHPACK's TRID0 pins the mean mode at the last row
    }
    const size_t ns = (size_t)d.lp * cfg->ny * cfg->nz;
    if ((rc = dalloc(ctx, &p, ns * (mixed ? sizeof(float2) : sizeof(double2))))) goto fail;
    d.spec = p;
    if ((rc = dalloc(ctx, &p, ns * sizeof(double2)))) goto fail;
    d.ypiv = (double2 *)p;
  }
  {
    // block partials: one per 32x8 tile of the (x, y) plane per z plane
    ctx->npart = ((cfg->nx + 31) / 32) * ((cfg->ny + 7) / 8) * cfg->nz;
    if ((rc = dalloc(ctx, &p, (size_t)ctx->npart * sizeof(double)))) goto fail;
    d.partials = (double *)p;
    if ((rc = dalloc(ctx, &p, 16 * sizeof(double)))) goto fail;
    d.scal = (double *)p;
    cudaMemsetAsync(p, 0, 16 * sizeof(double), ctx->stream);
    if ((rc = dalloc(ctx, &p, 16 * sizeof(int)))) goto fail;
    d.err = (int *)p;
    cudaMemsetAsync(p, 0, 16 * sizeof(int), ctx->stream);
    ctx->io.dpg = d.scal;
    ctx->io.part = d.partials;
  }
  if ((rc = build_tables(ctx))) goto fail;
  px.tw64 = ctx->fx.tw64; px.tw32 = ctx->fx.tw32;
  pz.tw64 = ctx->fz.tw64; pz.tw32 = ctx->fz.tw32;
  ctx->fx = px;
  ctx->fz = pz;
  if ((rc = init_kernels(ctx))) goto fail;
  if (iocfg && iocfg->bcx_in != 3) {
    const int b0 = iocfg->bcx_in, b1 = iocfg->bcx_out;
    const int lp = b0 == 1 ? (b1 == 1 ? 2 : 3) : (b1 == 2 ? 4 : 5);  // LPEROD + 1
    if ((rc = xnp_setup(ctx, lp))) goto fail;
  }
  if (iocfg && (rc = io_init_maps(ctx))) goto fail;
  if (iocfg) {
    // reference property values (thermal off, or before the table is set)
    IODev &io = ctx->io;
    double *ones[] = {io.T, io.D, io.D0, io.mu, io.mu0, io.kap};
    for (double *f : ones)
      if ((rc = fill_value(ctx, f - xo, nal, 1.0))) goto fail;
    if ((rc = fill_value(ctx, io.msum - xo, nal, 2.0))) goto fail;
    if ((rc = fill_value(ctx, io.bcp + (size_t)io.bps * CHAPSIM_P_IN_RHO, (size_t)io.bps, 1.0))) goto fail;
  }
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { rc = CHAPSIM_ERR_CUDA; goto fail; }
  *out = ctx;
  return CHAPSIM_OK;
fail:
  free_all(ctx);
  delete ctx;
  return rc;
}

int chapsim_create(const chapsim_config *cfg, chapsim_ctx **out) { return create_ctx(cfg, nullptr, out); }

int chapsim_io_config_default(chapsim_io_config *io) {
  if (!io) return CHAPSIM_ERR_ARG;
  memset(io, 0, sizeof(*io));
  io->struct_size = (int32_t)sizeof(chapsim_io_config);
  io->thermal = 1;
  io->prt = 0.71;
  io->qw_bot = 1.0;
  io->qw_top = 1.0;
  io->gravdir = 0;
  io->visc_scheme = 0;
  io->f_a = 0.0;
  io->coupled = 0;
  io->isothermal = 0;
  io->bcx_in = 3;
  io->bcx_out = 3;
  return CHAPSIM_OK;
}

int chapsim_create_io(const chapsim_config *cfg, const chapsim_io_config *io, chapsim_ctx **out) {
  if (!cfg || !io || !out) return CHAPSIM_ERR_ARG;
  if (io->struct_size != (int32_t)sizeof(chapsim_io_config)) return CHAPSIM_ERR_ARG;
  if (cfg->precision == CHAPSIM_MIXED && io->visc_scheme != 0) return CHAPSIM_ERR_UNSUPPORTED;
  if (!(io->prt > 0) || io->gravdir < 0 || io->gravdir > 3) return CHAPSIM_ERR_ARG;
  if (io->visc_scheme != 0 && io->visc_scheme != 1) return CHAPSIM_ERR_ARG;
  if (io->coupled != 0 && io->coupled != 1) return CHAPSIM_ERR_ARG;
  if (io->isothermal < 0 || io->isothermal > 3 || (io->isothermal && !io->thermal)) return CHAPSIM_ERR_ARG;
  if (io->bcx_in < 1 || io->bcx_in > 3 || io->bcx_out < 1 || io->bcx_out > 3 ||
      ((io->bcx_in == 3) != (io->bcx_out == 3)))
    return CHAPSIM_ERR_ARG;
  // the coupled section (non-periodic x): FP64, explicit viscous terms (the
  // reference's semi-implicit inlet terms BC_CBC_TDMA are unfinished,
  // src/SOLVERRK3_MOM_IO.f90:22), iso-flux walls (BC_COUTLET_ENEG_RK3's
  // outlet-plane walls)
  if (io->bcx_in != 3 && (cfg->precision != CHAPSIM_FP64 || cfg->nx < 4 || io->visc_scheme != 0 || io->isothermal))
    return CHAPSIM_ERR_UNSUPPORTED;
  return create_ctx(cfg, io, out);
}

// A coupled section leaves its TG source: back on its own stream.
static void detach_inlet(chapsim_ctx *io) {
  chapsim_ctx *tg = io->inlet;
  if (!tg) return;
  cudaStreamSynchronize(io->stream);
  for (auto it = tg->fed.begin(); it != tg->fed.end(); ++it)
    if (*it == io) { tg->fed.erase(it); break; }
  drop_graphs(io);
  io->inlet = nullptr;
  io->stream = io->own_stream;
}

int chapsim_destroy(chapsim_ctx *ctx) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  detach_inlet(ctx);
  while (!ctx->fed.empty()) detach_inlet(ctx->fed.back());
  free_all(ctx);
  delete ctx;
  return CHAPSIM_OK;
}

const char *chapsim_last_error(const chapsim_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// Read and clear the device error word (bounded waits that gave up).
static int check_device_error(chapsim_ctx *ctx) {
  int e = 0;
  CKC(cudaMemcpyAsync(&e, ctx->d.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CKC(cudaStreamSynchronize(ctx->stream));
  if (e != 0) {
    CKC(cudaMemsetAsync(ctx->d.err, 0, sizeof(int), ctx->stream));
    ctx->err = "device-side wait gave up (error word " + std::to_string(e) + ")";
    return CHAPSIM_ERR_CUDA;
  }
  return CHAPSIM_OK;
}

int chapsim_sync(chapsim_ctx *ctx) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  CKC(cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);
}

int chapsim_set_refinement(chapsim_ctx *ctx, int sweeps) {
  if (!ctx || (sweeps != 0 && sweeps != 1)) return CHAPSIM_ERR_ARG;
  CKC(cudaSetDevice(ctx->device));
  CKC(cudaStreamSynchronize(ctx->stream));
  ctx->refine = sweeps == 1;
  drop_graphs(ctx);
  return CHAPSIM_OK;
}

int chapsim_inject_wait_timeout(chapsim_ctx *ctx, int polls) {
  if (!ctx || polls < 1 || polls > (1 << 20)) return CHAPSIM_ERR_ARG;
  CKC(cudaSetDevice(ctx->device));
  return chapsim::launch_wait_probe(ctx, polls);
}

int64_t chapsim_field_len(const chapsim_ctx *ctx) {
  return ctx ? ctx->d.sz * (int64_t)ctx->d.nz : -1;
}

static double *field_ptr(chapsim_ctx *ctx, int domain, int field) {
  if (domain != ctx->domain) return nullptr;
  TGDev &d = ctx->d;
  if (domain == CHAPSIM_IIO) {
    IODev &io = ctx->io;
    const int cur = ctx->io_cur;
    switch (field) {
      case CHAPSIM_F_GX: return io.g[cur][0];
      case CHAPSIM_F_GY: return io.g[cur][1];
      case CHAPSIM_F_GZ: return io.g[cur][2];
      case CHAPSIM_F_G0X: return io.g[1 - cur][0];
      case CHAPSIM_F_G0Y: return io.g[1 - cur][1];
      case CHAPSIM_F_G0Z: return io.g[1 - cur][2];
      case CHAPSIM_F_H: return io.h;
      case CHAPSIM_F_T: return io.T;
      case CHAPSIM_F_RHO: return io.D;
      case CHAPSIM_F_MU: return io.mu;
      case CHAPSIM_F_K: return io.kap;
      case CHAPSIM_F_RHOH: return io.rhoh;
      case CHAPSIM_F_RHO0: return io.D0;
      case CHAPSIM_F_MU0: return io.mu0;
      case CHAPSIM_F_DRHO: return io.drho;
      case CHAPSIM_F_RHSE0: return io.rhse0;
    }
  }
  switch (field) {
    case CHAPSIM_F_U: return d.u;
    case CHAPSIM_F_V: return d.v;
    case CHAPSIM_F_W: return d.w;
    case CHAPSIM_F_P: return d.p;
    case CHAPSIM_F_PHI: return d.phi;
    case CHAPSIM_F_RHSPHI: return d.rhsphi;
    case CHAPSIM_F_H0U: return (double *)d.h0[0];
    case CHAPSIM_F_H0V: return (double *)d.h0[1];
    case CHAPSIM_F_H0W: return (double *)d.h0[2];
  }
  return nullptr;
}

static int xfer(chapsim_ctx *ctx, int domain, int field, void *dst_or_src, int64_t n, cudaMemcpyKind kind,
                bool to_dev, bool async = false) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  double *f = field_ptr(ctx, domain, field);
  REQUIRE(f, CHAPSIM_ERR_ARG, "unknown domain/field id");
  REQUIRE(dst_or_src, CHAPSIM_ERR_ARG, "null buffer");
  REQUIRE(n == chapsim_field_len(ctx), CHAPSIM_ERR_ARG, "field length mismatch");
  CKC(cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)n * sizeof(double);
  const bool h0f = field >= CHAPSIM_F_H0U && field <= CHAPSIM_F_H0W;
  if (h0f && ctx->cfg.precision == CHAPSIM_MIXED && ctx->domain == CHAPSIM_ITG) {
    // CONVH0 is held in FP32 in the TG mixed form: convert through the host
    REQUIRE(kind != cudaMemcpyDeviceToDevice, CHAPSIM_ERR_UNSUPPORTED, "device copies of FP32 H0 fields");
    REQUIRE(!async, CHAPSIM_ERR_UNSUPPORTED, "stream-ordered copies of FP32 H0 fields");
    std::vector<float> tmp((size_t)n);
    if (to_dev) {
      const double *src = (const double *)dst_or_src;
      for (int64_t t = 0; t < n; ++t) tmp[t] = (float)src[t];
      CKC(cudaMemcpyAsync(f, tmp.data(), (size_t)n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
      CKC(cudaStreamSynchronize(ctx->stream));
    } else {
      CKC(cudaMemcpyAsync(tmp.data(), f, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
      CKC(cudaStreamSynchronize(ctx->stream));
      double *dst = (double *)dst_or_src;
      for (int64_t t = 0; t < n; ++t) dst[t] = (double)tmp[t];
    }
    return CHAPSIM_OK;
  }
  // the whole array, from its first value (the inlet ghost column of the
  // first row in the coupled section)
  double *base = f - ctx->xoff;
  if (to_dev)
    CKC(cudaMemcpyAsync(base, dst_or_src, bytes, kind, ctx->stream));
  else
    CKC(cudaMemcpyAsync(dst_or_src, base, bytes, kind, ctx->stream));
  if (to_dev && domain == CHAPSIM_IIO && (field == CHAPSIM_F_MU || field == CHAPSIM_F_MU0)) {
    const int rc = io_refresh_msum(ctx);  // keep mu0 + mu in step
    if (rc) return rc;
  }
  if (kind != cudaMemcpyDeviceToDevice && !async) CKC(cudaStreamSynchronize(ctx->stream));
  return CHAPSIM_OK;
}

int chapsim_set_field(chapsim_ctx *ctx, int domain, int field, const double *host, int64_t n) {
  return xfer(ctx, domain, field, (void *)host, n, cudaMemcpyHostToDevice, true);
}
int chapsim_get_field(chapsim_ctx *ctx, int domain, int field, double *host, int64_t n) {
  return xfer(ctx, domain, field, host, n, cudaMemcpyDeviceToHost, false);
}
int chapsim_set_field_async(chapsim_ctx *ctx, int domain, int field, const double *host, int64_t n) {
  return xfer(ctx, domain, field, (void *)host, n, cudaMemcpyHostToDevice, true, true);
}
int chapsim_get_field_async(chapsim_ctx *ctx, int domain, int field, double *host, int64_t n) {
  return xfer(ctx, domain, field, host, n, cudaMemcpyDeviceToHost, false, true);
}
int chapsim_set_field_device(chapsim_ctx *ctx, int domain, int field, const double *dev, int64_t n) {
  return xfer(ctx, domain, field, (void *)dev, n, cudaMemcpyDeviceToDevice, true);
}
int chapsim_get_field_device(chapsim_ctx *ctx, int domain, int field, double *dev, int64_t n) {
  return xfer(ctx, domain, field, dev, n, cudaMemcpyDeviceToDevice, false);
}

int chapsim_get_mesh(const chapsim_ctx *ctx, int what, double *out, int64_t n) {
  if (!ctx || !out) return CHAPSIM_ERR_ARG;
  const int ny = ctx->cfg.ny;
  const std::vector<double> *v = nullptr;
  int hi = ny;
  switch (what) {
    case 0: v = &ctx->ynd; hi = ny + 1; break;
    case 1: v = &ctx->ycc; break;
    case 2: v = &ctx->dyfi; break;
    case 3: v = &ctx->dyci; hi = ny + 1; break;
    default: return CHAPSIM_ERR_ARG;
  }
  if (n != hi) return CHAPSIM_ERR_ARG;
  for (int j = 1; j <= hi; ++j) out[j - 1] = (*v)[j];
  return CHAPSIM_OK;
}

// The seeded initial velocity of RANDOM_FL_FLD_TG (also used for the IO
// domain): perturbation, xz-mean removal, laminar profile, v = 0 on the
// wall, unit bulk velocity, zero wall ghosts.
static void seeded_velocity(chapsim_ctx *ctx, uint64_t seed, double amp, std::vector<double> *q) {
  const int nx = ctx->cfg.nx, ny = ctx->cfg.ny, nz = ctx->cfg.nz;
  const int64_t sy = nx, sz = (int64_t)nx * (ny + 2), n = sz * nz;
  for (int c = 0; c < 3; ++c) q[c].assign((size_t)n, 0.0);
  auto id = [&](int i, int j, int k) { return (size_t)((i - 1) + sy * j + sz * (k - 1)); };
  // RANDOM_FL_FLD_TG (src/INITIAL_FL_FLD_TG.f90:2-72) with a counter-based
  // generator in place of gfortran's random_number.
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i)
        for (int c = 0; c < 3; ++c) q[c][id(i, j, k)] = amp * rnd_pm1(seed, c + 1, i, j, k);
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) q[1][id(i, 1, k)] = 0.0;
  for (int c = 0; c < 3; ++c)
    for (int j = 1; j <= ny; ++j) {
      double s = 0.0;
      for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= nz; ++k) s += q[c][id(i, j, k)];
      s /= (double)nx * (double)nz;
      for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= nz; ++k) q[c][id(i, j, k)] -= s;
    }
  for (int j = 1; j <= ny; ++j) {
    const double vini = 1.5 * (1.0 - ctx->ycc[j] * ctx->ycc[j]);  // LAMPOISLPROF.f90:49-56
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) q[0][id(i, j, k)] += vini;
  }
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) q[1][id(i, 1, k)] = 0.0;
  // bulk velocity rescale (BULK_VELOCITY_TG, src/INITIAL_FL_FLD_TG.f90:122-149)
  double s = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 1; k <= nz; ++k) s += q[0][id(i, j, k)] / ctx->dyfi[j];
  s = s / (nz / ctx->cfg.lz);
  const double ub = s / (ctx->area_inlet * (double)nx);
  for (auto &x : q[0]) x /= ub;
  // wall ghosts
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i)
      for (int c = 0; c < 3; ++c) { q[c][id(i, 0, k)] = 0.0; q[c][id(i, ny + 1, k)] = 0.0; }
}

// Host spline look-up with the reference's search (table set-up only).
static bool host_spline_eval(const std::vector<double> &x, const std::vector<double> &y, const std::vector<double> &b,
                             const std::vector<double> &c, const std::vector<double> &dd, double u, double &out) {
  const int n = (int)x.size();
  if (u <= x[0] || u >= x[n - 1]) return false;
  int i = 0, j = n;
  while (j > i + 1) {
    const int k = (i + j) / 2;
    if (u < x[k]) j = k; else i = k;
  }
  const double dx = u - x[i];
  out = y[i] + dx * (b[i] + dx * (c[i] + dx * dd[i]));
  return true;
}

struct HostSpline {
  std::vector<double> x, y, b, c, d;
  HostSpline(const std::vector<double> &xs, const std::vector<double> &ys) : x(xs), y(ys) {
    const int n = (int)x.size();
    b.assign(n, 0.0); c.assign(n, 0.0); d.assign(n, 0.0);
    chapsim_spl::fmm_spline(n, x.data(), y.data(), b.data(), c.data(), d.data());
  }
  bool eval(double u, double &out) const { return host_spline_eval(x, y, b, c, d, u, out); }
};

// IO initial field (RANDOM_FL_THEML_FLD_io + CALC_INITIALIZATION_io with the
// seeded velocity of the TG recipe).
static int io_init_random(chapsim_ctx *ctx, uint64_t seed, double amp, int project) {
  IODev &io = ctx->io;
  REQUIRE(!io.thermal || ctx->has_table, CHAPSIM_ERR_STATE, "thermal IO domain without a property table");
  REQUIRE(!ctx->xnp || ctx->inlet, CHAPSIM_ERR_STATE,
          "coupled IO section without its TG inlet source (chapsim_io_set_inlet)");
  const int nx = ctx->cfg.nx, ny = ctx->cfg.ny, nz = ctx->cfg.nz;
  // the seeded field is built on the interior columns (sy = nx), then laid
  // out in the context's fields (with the coupled section's ghost columns)
  const int64_t sy = nx, sz = (int64_t)nx * (ny + 2), n = sz * nz;
  const int64_t nf = ctx->d.sz * nz;
  auto id = [&](int i, int j, int k) { return (size_t)((i - 1) + sy * j + sz * (k - 1)); };
  std::vector<double> q[3], g[3];
  for (auto &f : q) f.assign((size_t)n, 0.0);
  for (auto &f : g) f.assign((size_t)n, 0.0);
  seeded_velocity(ctx, seed, amp, q);
  // properties at h = 0: the table's values, or the reference state 1 when the
  // table keeps the reference shortcuts (INIFIELD_THERMAL_io)
  double T0 = 1.0, D0 = 1.0, M0 = 1.0, K0 = 1.0;
  if (io.thermal && !io.shortcuts) {
    const HostSpline ht(ctx->tab[0], ctx->tab[1]), td(ctx->tab[1], ctx->tab[2]), tm(ctx->tab[1], ctx->tab[3]),
        tk(ctx->tab[1], ctx->tab[4]);
    REQUIRE(ht.eval(0.0, T0) && td.eval(T0, D0) && tm.eval(T0, M0) && tk.eval(T0, K0), CHAPSIM_ERR_RANGE,
            "h = 0 lies outside the property table");
  }
  // RHO_STG of the uniform initial density (DENSITY_Staggered)
  const double rx = io.thermal ? (D0 + D0 + D0 + D0) * 0.5 * 0.5 : 1.0;
  std::vector<double> ry(ny + 2, 1.0);
  if (io.thermal)
    for (int j = 2; j <= ny; ++j) ry[j] = (ctx->wff[j] * (D0 + D0) + ctx->wfb[j] * (D0 + D0)) * 0.5;
  auto velo2massflux = [&]() {  // VELO2MASSFLUX (src/INITIAL_FL_THEML_FLD_io.f90:481-560)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          const size_t c = id(i, j, k);
          g[0][c] = q[0][c] * rx;
          g[2][c] = q[2][c] * rx;
          if (j >= 2) g[1][c] = q[1][c] * ry[j];
        }
  };
  velo2massflux();
  // Unified_massflux (:653-682): unit bulk mass flux
  double s = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 1; k <= nz; ++k) s += g[0][id(i, j, k)] / ctx->dyfi[j];
  s = s / (nz / ctx->cfg.lz);
  const double gm = s / (ctx->area_inlet * (double)nx);
  for (int c = 0; c < 3; ++c)
    for (auto &x : q[c]) x /= gm;
  velo2massflux();
  if (ctx->xnp) {
    // coupled section: the interior into the ghost-column layout, and the
    // outlet ghost column IC = NCL1_io + 1 a copy of the last interior column
    // (the inlet column comes from the TG section in the projection's
    // BC_TINLET_FLOW)
    const int64_t fy = ctx->d.sy, fz = ctx->d.sz;
    for (auto *set : {q, g})
      for (int c = 0; c < 3; ++c) {
        std::vector<double> e((size_t)nf, 0.0);
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j <= ny + 1; ++j) {
            const double *src = set[c].data() + sy * j + sz * k;
            double *dst = e.data() + 1 + fy * j + fz * k;
            for (int i = 0; i < nx; ++i) dst[i] = src[i];
            dst[nx] = src[nx - 1];
          }
        set[c].swap(e);
      }
  }
  int rc;
  const size_t fbytes = (size_t)nf * sizeof(double);
  const int xo = ctx->xoff;
  for (int c = 0; c < 3; ++c) {
    if ((rc = chapsim_set_field(ctx, CHAPSIM_IIO, CHAPSIM_F_U + c, q[c].data(), nf))) return rc;
    CKC(cudaMemcpyAsync(io.g[0][c] - xo, g[c].data(), fbytes, cudaMemcpyHostToDevice, ctx->stream));
    CKC(cudaMemsetAsync(io.g[1][c] - xo, 0, fbytes, ctx->stream));  // G0_io = 0 until MOM_IO
    CKC(cudaMemsetAsync((double *)ctx->d.h0[c] - xo, 0, fbytes, ctx->stream));
  }
  CKC(cudaStreamSynchronize(ctx->stream));
  ctx->io_cur = 0;
  TGDev &d = ctx->d;
  double *zero[] = {d.p, d.phi, d.rhsphi, io.drho, io.rhoh, io.h, io.rhse0};
  for (double *f : zero) CKC(cudaMemsetAsync(f - xo, 0, fbytes, ctx->stream));
  if (io.visc)  // DRHOI_STG is zero until the first DENSITY_implicit_add
    for (int c = 0; c < 3; ++c) CKC(cudaMemsetAsync(io.drhoi[c] - xo, 0, fbytes, ctx->stream));
  CKC(cudaMemsetAsync(io.bad, 0, sizeof(unsigned long long), ctx->stream));
  if (ctx->xnp)  // the boundary operators' RK3 memory terms BC_CONV0, BC_CONV0_ENG
    CKC(cudaMemsetAsync(io.bcp + (size_t)io.bps * CHAPSIM_P_CONV0_X, 0, (size_t)io.bps * 4 * sizeof(double),
                        ctx->stream));
  const double M2 = M0 + M0;
  const double *vals[] = {&T0, &D0, &D0, &M0, &M0, &K0, &M2};
  double *arrs[] = {io.T, io.D, io.D0, io.mu, io.mu0, io.kap, io.msum};
  for (int a = 0; a < 7; ++a)
    if ((rc = fill_value(ctx, arrs[a] - xo, (size_t)nf, *vals[a]))) return rc;
  if (project) {  // CALC_INITIALIZATION_io
    if (io.thermal) {
      if ((rc = io_thermal_bc(ctx))) return rc;
      if ((rc = io_eng(ctx, 0))) return rc;
    }
    if ((rc = io_mom(ctx, 0, false))) return rc;
  }
  CKC(cudaStreamSynchronize(ctx->stream));
  return CHAPSIM_OK;
}

int chapsim_init_random(chapsim_ctx *ctx, uint64_t seed, double amp, int project) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  CKC(cudaSetDevice(ctx->device));
  if (ctx->domain == CHAPSIM_IIO) return io_init_random(ctx, seed, amp, project);
  const int nx = ctx->cfg.nx, ny = ctx->cfg.ny, nz = ctx->cfg.nz;
  const int64_t n = (int64_t)nx * (ny + 2) * nz;
  std::vector<double> q[3];
  for (auto &f : q) f.assign((size_t)n, 0.0);
  seeded_velocity(ctx, seed, amp, q);
  int rc;
  for (int c = 0; c < 3; ++c)
    if ((rc = chapsim_set_field(ctx, CHAPSIM_ITG, CHAPSIM_F_U + c, q[c].data(), n))) return rc;
  TGDev &d = ctx->d;
  const size_t bytes = (size_t)n * sizeof(double);
  CKC(cudaMemsetAsync(d.p, 0, bytes, ctx->stream));
  const size_t tbytes = (size_t)n * (ctx->cfg.precision == CHAPSIM_MIXED ? sizeof(float) : sizeof(double));
  for (int c = 0; c < 3; ++c) CKC(cudaMemsetAsync(d.h0[c], 0, tbytes, ctx->stream));
  if (project) {
    rc = launch_substep(ctx, 0);  // CALC_INITIALIZATION_tg: SOLVERRK3_MOM_tg(0)
    if (rc) return rc;
  }
  CKC(cudaStreamSynchronize(ctx->stream));
  return CHAPSIM_OK;
}

int chapsim_rk3_mom_tg(chapsim_ctx *ctx, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_ITG, CHAPSIM_ERR_STATE, "not a TG context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  CKC(cudaSetDevice(ctx->device));
  return launch_substep(ctx, ns);
}

int chapsim_step_tg(chapsim_ctx *ctx, int nsteps) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_ITG, CHAPSIM_ERR_STATE, "not a TG context");
  REQUIRE(nsteps >= 0, CHAPSIM_ERR_ARG, "nsteps must be >= 0");
  CKC(cudaSetDevice(ctx->device));
  if (ctx->timing) {
    for (int s = 0; s < nsteps; ++s)
      for (int ns = 1; ns <= 3; ++ns) {
        int rc = launch_substep(ctx, ns);
        if (rc) return rc;
      }
    return CHAPSIM_OK;
  }
  if (!ctx->step_graph) {
    cudaGraph_t g = nullptr;
    const int64_t before = ctx->launches;
    CKC(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = CHAPSIM_OK;
    for (int ns = 1; ns <= 3 && rc == CHAPSIM_OK; ++ns) rc = launch_substep(ctx, ns);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) { ctx->err = cudaGetErrorString(e); return CHAPSIM_ERR_CUDA; }
    e = cudaGraphInstantiate(&ctx->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { ctx->step_graph = nullptr; ctx->err = cudaGetErrorString(e); return CHAPSIM_ERR_CUDA; }
    ctx->kernels_per_step = ctx->launches - before;  // kernels inside one replay
    ctx->launches = before;
  }
  for (int s = 0; s < nsteps; ++s) {
    CKC(cudaGraphLaunch(ctx->step_graph, ctx->stream));
    ctx->launches += ctx->kernels_per_step;
  }
  return CHAPSIM_OK;
}

int chapsim_divg(chapsim_ctx *ctx, int domain, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(domain == ctx->domain, CHAPSIM_ERR_ARG, "domain does not match the context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  CKC(cudaSetDevice(ctx->device));
  if (ctx->xnp) return chapsim::io_np_divg(ctx, ns, ctx->io_cur);  // coupled section: RHSLLPHI only
  if (domain == CHAPSIM_IIO) {
    // DIVG_io (src/DIVG.f90:60-150) of the current G and DrhoDtP
    const TGDev saved = ctx->d;
    const int cur = ctx->io_cur;
    ctx->d.u = ctx->io.g[cur][0]; ctx->d.v = ctx->io.g[cur][1]; ctx->d.w = ctx->io.g[cur][2];
    ctx->d.drho = ctx->io.thermal ? ctx->io.drho : nullptr;
    const int rc = launch_divg(ctx, ns);
    ctx->d = saved;
    return rc;
  }
  return launch_divg(ctx, ns);
}

int chapsim_pois3d(chapsim_ctx *ctx, int domain) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(domain == ctx->domain, CHAPSIM_ERR_ARG, "domain does not match the context");
  CKC(cudaSetDevice(ctx->device));
  if (ctx->xnp) return xnp_pois3d(ctx);  // Dirichlet / Neumann x ends
  return launch_pois3d(ctx);  // FISHPACK_POIS3D_SIMPLE on an IO context (mean mode pinned last)
}

int chapsim_velo_correction(chapsim_ctx *ctx, int domain, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(domain == ctx->domain, CHAPSIM_ERR_ARG, "domain does not match the context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  CKC(cudaSetDevice(ctx->device));
  if (domain == CHAPSIM_IIO) return io_correction(ctx, ns);
  return launch_correction(ctx, ns);
}

int chapsim_stats(chapsim_ctx *ctx, int accumulate) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(!ctx->xnp, CHAPSIM_ERR_UNSUPPORTED,
          "the IO statistics are PP_MEAN_ZX_FLOW_Xperiodic_IO's: x-periodic sections only");
  CKC(cudaSetDevice(ctx->device));
  return stats_run(ctx, accumulate);
}

int chapsim_get_stats(chapsim_ctx *ctx, int which, double *out, int64_t n, int64_t *nstatis) {
  REQUIRE(ctx && out, CHAPSIM_ERR_ARG, "null argument");
  REQUIRE(which == 0 || which == 1, CHAPSIM_ERR_ARG, "which: 0 xz average, 1 time average");
  REQUIRE(ctx->stats_buf, CHAPSIM_ERR_STATE, "chapsim_stats has not run");
  REQUIRE(n == (int64_t)ctx->cfg.ny * (ctx->domain == CHAPSIM_IIO ? CHAPSIM_STATS_IO_NV : CHAPSIM_STATS_NV),
          CHAPSIM_ERR_ARG, "n must be ny * CHAPSIM_STATS_NV (TG) or ny * CHAPSIM_STATS_IO_NV (IO)");
  CKC(cudaSetDevice(ctx->device));
  if (nstatis) *nstatis = ctx->nstatis;
  return stats_get(ctx, which, out, n);
}

int chapsim_stats_reset(chapsim_ctx *ctx) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  CKC(cudaSetDevice(ctx->device));
  return stats_reset(ctx);
}

int chapsim_set_dt(chapsim_ctx *ctx, double dt) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(dt > 0 && dt < 1e3, CHAPSIM_ERR_ARG, "dt must be positive");
  CKC(cudaSetDevice(ctx->device));
  CKC(cudaStreamSynchronize(ctx->stream));
  // every coefficient table that depends on dt (RK factors, Crank-Nicolson
  // factors and their banded inverses) is rebuilt; captured graphs go stale
  double *old = ctx->dcoef;
  const double dt_old = ctx->cfg.dt;
  ctx->cfg.dt = dt;
  int rc = build_tables(ctx);
  if (rc) {
    ctx->cfg.dt = dt_old;
    return rc;
  }
  if (ctx->xnp) {
    // the non-periodic Poisson descriptor points into the coefficient tables
    // too: refresh it, keeping its own spectral array, pivots and x shifts
    chapsim::TGDev &s = ctx->dnp;
    void *spec = s.spec;
    double2 *ypiv = s.ypiv;
    const double *ak1 = s.ak1;
    const int lh = s.lh, lp = s.lp;
    s = ctx->d;
    s.spec = spec; s.ypiv = ypiv; s.ak1 = ak1; s.lh = lh; s.lp = lp;
  }
  for (auto it = ctx->allocs.begin(); it != ctx->allocs.end(); ++it)
    if (*it == (void *)old) {
      cudaFree(old);
      ctx->allocs.erase(it);
      break;
    }
  drop_graphs(ctx);
  return CHAPSIM_OK;
}

int chapsim_set_table(chapsim_ctx *ctx, const double *H, const double *T, const double *D, const double *M,
                      const double *K, int n, int shortcuts) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "property tables belong to IO contexts");
  REQUIRE(H && T && D && M && K && n >= 4, CHAPSIM_ERR_ARG, "table needs 5 columns of n >= 4 points");
  for (int i = 1; i < n; ++i)
    REQUIRE(H[i] > H[i - 1] && T[i] > T[i - 1], CHAPSIM_ERR_ARG, "H and T must increase strictly");
  CKC(cudaSetDevice(ctx->device));
  CKC(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  for (void *p : ctx->table_allocs) cudaFree(p);
  ctx->table_allocs.clear();
  const double *cols[5] = {H, T, D, M, K};
  for (int q = 0; q < 5; ++q) ctx->tab[q].assign(cols[q], cols[q] + n);
  IODev &io = ctx->io;
  const std::pair<int, int> xy[4] = {{0, 1}, {1, 2}, {1, 3}, {1, 4}};
  chapsim_spl::Spline *dst[4] = {&io.ht, &io.td, &io.tm, &io.tk};
  for (int q = 0; q < 4; ++q) {
    const cudaError_t e = chapsim_spl::upload_spline(ctx->table_allocs, ctx->tab[xy[q].first], ctx->tab[xy[q].second],
                                                     *dst[q]);
    if (e != cudaSuccess) {
      ctx->err = std::string("property table upload: ") + cudaGetErrorString(e);
      cudaGetLastError();
      return CHAPSIM_ERR_NOMEM;
    }
  }
  io.shortcuts = shortcuts ? 1 : 0;
  // RHOHmax (src/Flow_State.f90:963-990): max of rho(h) h over 3n - 1 samples
  const HostSpline hd(ctx->tab[0], ctx->tab[2]);
  double rm = -1e-14;
  for (int i = 2; i <= 3 * n; ++i) {
    const double h = H[0] + (double)(i - 1) * (H[n - 1] - H[0]) / (double)(3 * n);
    double dv = 0.0;
    hd.eval(h, dv);
    if (io.shortcuts && fabs(h) < 1.0e-10) dv = 1.0;
    if (dv * h > rm) rm = dv * h;
  }
  io.rhohmax = rm;
  // iso-thermal walls (WALL_ISOTHERMAL_GIVEN, src/Flow_State.f90:603-645):
  // h, rho, mu, k at the wall temperature from the T-splines of the table
  for (int side = 0; side < 2; ++side) {
    if (!(io.isothermal & (1 << side))) continue;
    const double tw = side == 0 ? io.qw_bot : io.qw_top;
    double v[4];
    bool ok = true;
    for (int q = 0; q < 4; ++q) {
      const int col = q == 0 ? 0 : q + 1;  // H, D, M, K against T
      const HostSpline sp(ctx->tab[1], ctx->tab[col]);
      ok = ok && sp.eval(tw, v[q]);
    }
    REQUIRE(ok, CHAPSIM_ERR_ARG, "iso-thermal wall temperature outside the property table");
    io.wall[side][0] = tw;
    for (int q = 0; q < 4; ++q) io.wall[side][q + 1] = v[q];
  }
  ctx->has_table = true;
  ctx->props_mode = CHAPSIM_PROPS_TABLE;  // a model trained on another table no longer applies
  return CHAPSIM_OK;
}

int chapsim_io_wall_values(const chapsim_ctx *ctx, double *out, int n) {
  if (!ctx || !out || n != 10 || ctx->domain != CHAPSIM_IIO) return CHAPSIM_ERR_ARG;
  for (int side = 0; side < 2; ++side)
    for (int q = 0; q < 5; ++q) out[5 * side + q] = (ctx->io.isothermal & (1 << side)) ? ctx->io.wall[side][q] : 0.0;
  return CHAPSIM_OK;
}

int chapsim_set_props_mode(chapsim_ctx *ctx, int mode, const chapsim_props *pe) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO && ctx->io.thermal, CHAPSIM_ERR_STATE,
          "property modes belong to IO contexts with the energy equation");
  REQUIRE(ctx->has_table, CHAPSIM_ERR_STATE, "no property table: call chapsim_set_table first");
  REQUIRE(!ctx->xnp || mode == CHAPSIM_PROPS_TABLE, CHAPSIM_ERR_UNSUPPORTED,
          "the learned property kernel walks x-periodic fields (no ghost columns)");
  REQUIRE(mode == CHAPSIM_PROPS_TABLE || mode == CHAPSIM_PROPS_MLP, CHAPSIM_ERR_ARG, "unknown property mode");
  CKC(cudaSetDevice(ctx->device));
  CKC(cudaStreamSynchronize(ctx->stream));
  if (mode == CHAPSIM_PROPS_MLP) {
    REQUIRE(pe, CHAPSIM_ERR_ARG, "the learned mode needs a property engine with a trained model");
    chapsim_mlp::MlpDev src{};
    int dev = -1;
    const int rc = chapsim::props_model(pe, &src, &dev);
    REQUIRE(rc == CHAPSIM_OK, rc, "the property engine has no trained model");
    REQUIRE(dev == ctx->device, CHAPSIM_ERR_ARG, "property engine and context on different devices");
    REQUIRE(chapsim::props_same_table(pe, ctx->tab), CHAPSIM_ERR_ARG,
            "the model was trained on another table than the context's");
    // the three parts of the copy start on 256-byte boundaries: the kernels
    // read the weight tiles with 16-byte vector loads
    const size_t npar_b = chapsim_mlp::NP * sizeof(float);
    const size_t nwt_b = (2 * chapsim_mlp::NH * chapsim_mlp::NH + 2 * chapsim_mlp::NOP * chapsim_mlp::NH) *
                         sizeof(uint16_t);
    const size_t npar = (npar_b + 255) & ~(size_t)255, nwt = (nwt_b + 255) & ~(size_t)255;
    if (!ctx->mlp_buf) {
      void *p = nullptr;
      if (cudaMalloc(&p, npar + nwt + chapsim_mlp::kMaxGateBins) != cudaSuccess) {
        cudaGetLastError();
        ctx->err = "cannot allocate the model's buffers";
        return CHAPSIM_ERR_NOMEM;
      }
      ctx->mlp_buf = p;
      ctx->allocs.push_back(p);
    }
    char *b = static_cast<char *>(ctx->mlp_buf);
    CKC(cudaMemcpyAsync(b, src.par, npar_b, cudaMemcpyDeviceToDevice, ctx->stream));
    CKC(cudaMemcpyAsync(b + npar, src.wt, nwt_b, cudaMemcpyDeviceToDevice, ctx->stream));
    CKC(cudaMemcpyAsync(b + npar + nwt, src.gate, chapsim_mlp::kMaxGateBins, cudaMemcpyDeviceToDevice, ctx->stream));
    CKC(cudaStreamSynchronize(ctx->stream));
    ctx->mlp = src;
    ctx->mlp.par = reinterpret_cast<const float *>(b);
    ctx->mlp.wt = reinterpret_cast<const uint16_t *>(b + npar);
    ctx->mlp.gate = reinterpret_cast<const uint8_t *>(b + npar + nwt);
    REQUIRE(((uintptr_t)ctx->mlp.wt & 15) == 0, CHAPSIM_ERR_STATE, "model weight tiles not 16-byte aligned");
  }
  ctx->props_mode = mode;
  drop_graphs(ctx);  // the captured steps hold the other property kernel
  return CHAPSIM_OK;
}

int chapsim_therm_prop_update(chapsim_ctx *ctx, int iregion, int mode) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(!ctx->xnp, CHAPSIM_ERR_UNSUPPORTED,
          "THERM_PROP_UPDATE alone walks x-periodic fields (the coupled section updates inside its substeps)");
  REQUIRE(ctx->domain == CHAPSIM_IIO && ctx->io.thermal && ctx->has_table, CHAPSIM_ERR_STATE,
          "THERM_PROP_UPDATE needs an IO context with the energy equation and a table");
  REQUIRE(iregion == CHAPSIM_IMAIND || iregion == CHAPSIM_IALLDM, CHAPSIM_ERR_UNSUPPORTED,
          "region: the outlet plane (IOULET) is updated by chapsim_io_bc_outlet_eng");
  REQUIRE(mode == CHAPSIM_PROPS_TABLE || mode == CHAPSIM_PROPS_MLP, CHAPSIM_ERR_ARG, "unknown property mode");
  REQUIRE(mode == CHAPSIM_PROPS_TABLE || ctx->mlp.par, CHAPSIM_ERR_STATE,
          "no model on the context: call chapsim_set_props_mode with a trained engine first");
  CKC(cudaSetDevice(ctx->device));
  return chapsim::io_therm_props(ctx, mode);
}

int chapsim_rk3_eng_io(chapsim_ctx *ctx, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  REQUIRE(ctx->io.thermal, CHAPSIM_ERR_STATE, "thermal is off on this IO context");
  REQUIRE(ctx->has_table, CHAPSIM_ERR_STATE, "no property table");
  CKC(cudaSetDevice(ctx->device));
  return io_eng(ctx, ns);
}

int chapsim_rk3_mom_io(chapsim_ctx *ctx, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  CKC(cudaSetDevice(ctx->device));
  return io_mom(ctx, ns, ns >= 1);
}

// Coupled inflow/outflow boundary planes (BC_TINLET_FLOW, BC_COUTLET_MOM_RK3,
// BC_COUTLET_ENEG_RK3): io_kernels.cu.
static const char *kCoupledBc = "the coupled section runs its boundary operators inside its substeps";

int chapsim_io_bc_inlet(chapsim_ctx *ctx, chapsim_ctx *tg) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(!ctx->xnp, CHAPSIM_ERR_UNSUPPORTED, kCoupledBc);
  REQUIRE(tg, CHAPSIM_ERR_ARG, "null TG context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(tg->domain == CHAPSIM_ITG, CHAPSIM_ERR_ARG, "the inlet source must be a TG context");
  REQUIRE(tg->device == ctx->device, CHAPSIM_ERR_UNSUPPORTED, "the TG and IO contexts are on different devices");
  REQUIRE(tg->cfg.ny == ctx->cfg.ny && tg->cfg.nz == ctx->cfg.nz, CHAPSIM_ERR_ARG,
          "the TG and IO sections differ in ny or nz");
  CKC(cudaSetDevice(ctx->device));
  CKC(cudaStreamSynchronize(tg->stream));  // the TG fields are final
  const int rc = io_bc_inlet(ctx, tg);
  if (rc) return rc;
  CKC(cudaStreamSynchronize(ctx->stream));  // the TG fields may change after return
  return CHAPSIM_OK;
}

int chapsim_io_bc_outlet_mom(chapsim_ctx *ctx, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(!ctx->xnp, CHAPSIM_ERR_UNSUPPORTED, kCoupledBc);
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  CKC(cudaSetDevice(ctx->device));
  return io_bc_outlet_mom(ctx, ns);
}

int chapsim_io_bc_outlet_eng(chapsim_ctx *ctx, int ns) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(!ctx->xnp, CHAPSIM_ERR_UNSUPPORTED, kCoupledBc);
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(ns >= 0 && ns <= 3, CHAPSIM_ERR_ARG, "NS must be in 0..3");
  REQUIRE(ctx->io.thermal && ctx->has_table, CHAPSIM_ERR_STATE,
          "the outlet energy condition needs the energy equation and a property table");
  REQUIRE(!ctx->io.isothermal, CHAPSIM_ERR_UNSUPPORTED,
          "the outlet plane's wall ghost rows are built for iso-flux walls only");
  CKC(cudaSetDevice(ctx->device));
  return io_bc_outlet_eng(ctx, ns);
}

static int plane_copy(chapsim_ctx *ctx, int plane, void *host, int64_t n, bool to_dev) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(plane >= 0 && plane < CHAPSIM_P_COUNT, CHAPSIM_ERR_ARG, "unknown plane id");
  REQUIRE(host, CHAPSIM_ERR_ARG, "null buffer");
  REQUIRE(n == ctx->io.bps, CHAPSIM_ERR_ARG, "plane length must be (ny + 2) * nz");
  CKC(cudaSetDevice(ctx->device));
  double *p = ctx->io.bcp + (size_t)plane * ctx->io.bps;
  if (to_dev)
    CKC(cudaMemcpyAsync(p, host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  else
    CKC(cudaMemcpyAsync(host, p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CKC(cudaStreamSynchronize(ctx->stream));
  return CHAPSIM_OK;
}
int chapsim_io_set_plane(chapsim_ctx *ctx, int plane, const double *host, int64_t n) {
  return plane_copy(ctx, plane, (void *)host, n, true);
}
int chapsim_io_get_plane(chapsim_ctx *ctx, int plane, double *host, int64_t n) {
  return plane_copy(ctx, plane, host, n, false);
}

int chapsim_io_bc_scalars(chapsim_ctx *ctx, double *out, int n) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(out && n >= 7, CHAPSIM_ERR_ARG, "need 7 values");
  CKC(cudaSetDevice(ctx->device));
  CKC(cudaMemcpyAsync(out, ctx->io.bcs, 7 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CKC(cudaStreamSynchronize(ctx->stream));
  return CHAPSIM_OK;
}

static int io_substeps(chapsim_ctx *ctx) {
  for (int ns = 1; ns <= 3; ++ns) {
    int rc;
    if (ctx->io.thermal && (rc = io_eng(ctx, ns))) return rc;
    if ((rc = io_mom(ctx, ns, true))) return rc;
  }
  return CHAPSIM_OK;
}

int chapsim_step_io(chapsim_ctx *ctx, int nsteps) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(ctx->domain == CHAPSIM_IIO, CHAPSIM_ERR_STATE, "not an IO context");
  REQUIRE(nsteps >= 0, CHAPSIM_ERR_ARG, "nsteps must be >= 0");
  REQUIRE(!ctx->io.thermal || ctx->has_table, CHAPSIM_ERR_STATE, "no property table");
  CKC(cudaSetDevice(ctx->device));
  if (ctx->timing) {
    for (int s = 0; s < nsteps; ++s) {
      int rc = io_substeps(ctx);
      if (rc) return rc;
    }
    return CHAPSIM_OK;
  }
  for (int s = 0; s < nsteps; ++s) {
    // three substeps flip the G buffers three times: one graph per starting parity
    const int par = ctx->io_cur;
    if (!ctx->io_graph[par]) {
      cudaGraph_t g = nullptr;
      const int64_t before = ctx->launches;
      CKC(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      int rc = io_substeps(ctx);
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      ctx->io_cur = par;  // captured, not run
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) { ctx->err = cudaGetErrorString(e); return CHAPSIM_ERR_CUDA; }
      e = cudaGraphInstantiate(&ctx->io_graph[par], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { ctx->io_graph[par] = nullptr; ctx->err = cudaGetErrorString(e); return CHAPSIM_ERR_CUDA; }
      ctx->kernels_per_step = ctx->launches - before;
      ctx->launches = before;
    }
    CKC(cudaGraphLaunch(ctx->io_graph[par], ctx->stream));
    ctx->launches += ctx->kernels_per_step;
    ctx->io_cur = 1 - par;
  }
  return CHAPSIM_OK;
}

int chapsim_io_set_inlet(chapsim_ctx *io, chapsim_ctx *tg) {
  chapsim_ctx *ctx = io;  // error messages go to the IO context
  REQUIRE(io, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(io->domain == CHAPSIM_IIO && io->xnp, CHAPSIM_ERR_STATE,
          "not a coupled IO section (create it with non-periodic bcx_in / bcx_out)");
  CKC(cudaSetDevice(io->device));
  detach_inlet(io);
  if (!tg) return CHAPSIM_OK;
  REQUIRE(tg->domain == CHAPSIM_ITG, CHAPSIM_ERR_ARG, "the inlet source must be a TG context");
  REQUIRE(tg->device == io->device, CHAPSIM_ERR_UNSUPPORTED, "the TG and IO contexts are on different devices");
  REQUIRE(tg->cfg.ny == io->cfg.ny && tg->cfg.nz == io->cfg.nz, CHAPSIM_ERR_ARG,
          "the TG and IO sections differ in ny or nz");
  CKC(cudaStreamSynchronize(io->stream));
  CKC(cudaStreamSynchronize(tg->stream));
  // the section's kernels run in the TG stream's order from now on: its
  // BC_TINLET_FLOW reads the TG fields between the TG's substeps
  io->inlet = tg;
  io->stream = tg->stream;
  tg->fed.push_back(io);
  drop_graphs(io);
  return CHAPSIM_OK;
}

// SOLVE.f90's substep loop (src/SOLVE.f90:119-134) over both sections:
// SOLVERRK3_MOM_tg(NS), then SOLVERRK3_ENG_IO(NS) with the density terms,
// VELOCITY_CALC_io and SOLVERRK3_MOM_IO(NS), which reads the TG's new fields.
static int pair_substeps(chapsim_ctx *tg, chapsim_ctx *io) {
  for (int ns = 1; ns <= 3; ++ns) {
    int rc;
    if ((rc = launch_substep(tg, ns))) return rc;
    if (io->io.thermal && (rc = io_eng(io, ns))) return rc;
    if ((rc = io_mom(io, ns, true))) return rc;
  }
  return CHAPSIM_OK;
}

int chapsim_step_coupled(chapsim_ctx *tg, chapsim_ctx *io, int nsteps) {
  chapsim_ctx *ctx = io;  // error messages go to the IO context
  REQUIRE(tg && io, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(io->domain == CHAPSIM_IIO && io->xnp && io->inlet == tg, CHAPSIM_ERR_STATE,
          "the IO section is not coupled to this TG context (chapsim_io_set_inlet)");
  REQUIRE(nsteps >= 0, CHAPSIM_ERR_ARG, "nsteps must be >= 0");
  REQUIRE(!io->io.thermal || io->has_table, CHAPSIM_ERR_STATE, "no property table");
  CKC(cudaSetDevice(io->device));
  if (tg->timing || io->timing) {
    for (int s = 0; s < nsteps; ++s) {
      int rc = pair_substeps(tg, io);
      if (rc) return rc;
    }
    return CHAPSIM_OK;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int par = io->io_cur;
    if (!io->pair_graph[par]) {
      cudaGraph_t g = nullptr;
      const int64_t bt = tg->launches, bi = io->launches;
      CKC(cudaStreamBeginCapture(io->stream, cudaStreamCaptureModeThreadLocal));
      int rc = pair_substeps(tg, io);
      cudaError_t e = cudaStreamEndCapture(io->stream, &g);
      io->io_cur = par;  // captured, not run
      io->pair_kernels = (tg->launches - bt) + (io->launches - bi);
      tg->launches = bt;
      io->launches = bi;
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) { io->err = cudaGetErrorString(e); return CHAPSIM_ERR_CUDA; }
      e = cudaGraphInstantiate(&io->pair_graph[par], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { io->pair_graph[par] = nullptr; io->err = cudaGetErrorString(e); return CHAPSIM_ERR_CUDA; }
    }
    CKC(cudaGraphLaunch(io->pair_graph[par], io->stream));
    io->launches += io->pair_kernels;
    io->io_cur = 1 - par;
  }
  return CHAPSIM_OK;
}

int chapsim_reduce(chapsim_ctx *ctx, int domain, int what, double *out) {
  REQUIRE(ctx, CHAPSIM_ERR_ARG, "null context");
  REQUIRE(!ctx->xnp || what != CHAPSIM_R_DIVMAX_Q, CHAPSIM_ERR_UNSUPPORTED,
          "max|div u| of the coupled section: use CHAPSIM_R_DIVMAX (div G + DrhoDtP)");
  REQUIRE(out, CHAPSIM_ERR_ARG, "null output");
  REQUIRE(domain == ctx->domain, CHAPSIM_ERR_ARG, "domain does not match the context");
  CKC(cudaSetDevice(ctx->device));
  if (domain == CHAPSIM_IIO) {
    if (what == CHAPSIM_R_BADCELLS || what == CHAPSIM_R_MODEL_AGAIN) {
      unsigned long long b = 0;
      CKC(cudaMemcpyAsync(&b, what == CHAPSIM_R_BADCELLS ? ctx->io.bad : ctx->io.model_again, sizeof(b),
                          cudaMemcpyDeviceToHost, ctx->stream));
      CKC(cudaStreamSynchronize(ctx->stream));
      *out = (double)b;
      return CHAPSIM_OK;
    }
    if (what == CHAPSIM_R_DIVMAX_Q || what == CHAPSIM_R_NANCOUNT)
      return launch_reduce(ctx, what == CHAPSIM_R_DIVMAX_Q ? 0 : 2, out);  // on u, v, w (, p)
    REQUIRE(what == CHAPSIM_R_DIVMAX || what == CHAPSIM_R_BULK || what == CHAPSIM_R_BULK_G ||
                what == CHAPSIM_R_BULK_H || what == CHAPSIM_R_CFL,
            CHAPSIM_ERR_ARG, "unknown reduction");
    return io_reduce(ctx, what, out);
  }
  if (what == CHAPSIM_R_CFL) return launch_reduce(ctx, 3, out);
  REQUIRE(what >= 0 && what <= 2, CHAPSIM_ERR_ARG, "unknown reduction");
  double v = 0.0;
  int rc = launch_reduce(ctx, what, &v);
  if (rc) return rc;
  if (what == CHAPSIM_R_BULK) v = v / (ctx->cfg.nz / ctx->cfg.lz) / (ctx->area_inlet * (double)ctx->cfg.nx);
  *out = v;
  return CHAPSIM_OK;
}

int chapsim_get_stream(const chapsim_ctx *ctx, void **stream) {
  if (!ctx || !stream) return CHAPSIM_ERR_ARG;
  *stream = (void *)ctx->stream;
  return CHAPSIM_OK;
}

int chapsim_phase_timing(chapsim_ctx *ctx, int enable) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  if (!enable && ctx->timing) {
    int rc = flush_phase_events(ctx);
    if (rc) return rc;
  }
  ctx->timing = enable != 0;
  return CHAPSIM_OK;
}
int chapsim_phase_times(chapsim_ctx *ctx, double *ms, int n, int64_t *substeps) {
  if (!ctx || !ms || n < CHAPSIM_PH_COUNT) return CHAPSIM_ERR_ARG;
  int rc = flush_phase_events(ctx);
  if (rc) return rc;
  for (int i = 0; i < CHAPSIM_PH_COUNT; ++i) ms[i] = ctx->phase_ms[i];
  if (substeps) *substeps = ctx->timed_substeps;
  return CHAPSIM_OK;
}
int chapsim_phase_reset(chapsim_ctx *ctx) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  int rc = flush_phase_events(ctx);
  if (rc) return rc;
  for (double &m : ctx->phase_ms) m = 0.0;
  ctx->timed_substeps = 0;
  return CHAPSIM_OK;
}

int chapsim_set_tuning(chapsim_ctx *ctx, int rhs_nzc, int fft_lb) {
  if (!ctx || rhs_nzc < 1 || fft_lb < 0 || fft_lb > 64 || (fft_lb & 1)) return CHAPSIM_ERR_ARG;
  ctx->rhs_nzc = rhs_nzc;
  ctx->io_nzc = rhs_nzc;  // the IO momentum RHS marches the same way
  ctx->fft_lb = fft_lb;
  drop_graphs(ctx);
  return CHAPSIM_OK;
}

int chapsim_set_line_tuning(chapsim_ctx *ctx, int ysolve_bx) {
  if (!ctx || (ysolve_bx != 64 && ysolve_bx != 128 && ysolve_bx != 256)) return CHAPSIM_ERR_ARG;
  ctx->ys_bx = ysolve_bx;
  drop_graphs(ctx);
  return CHAPSIM_OK;
}

int chapsim_get_line_tuning(const chapsim_ctx *ctx, int *ysolve_bx) {
  if (!ctx || !ysolve_bx) return CHAPSIM_ERR_ARG;
  *ysolve_bx = ctx->ys_bx;
  return CHAPSIM_OK;
}

int chapsim_get_tuning(const chapsim_ctx *ctx, int *rhs_nzc, int *fft_lb) {
  if (!ctx || !rhs_nzc || !fft_lb) return CHAPSIM_ERR_ARG;
  *rhs_nzc = ctx->rhs_nzc;
  *fft_lb = ctx->fft_lb;
  return CHAPSIM_OK;
}

int chapsim_launch_count(const chapsim_ctx *ctx, int64_t *count) {
  if (!ctx || !count) return CHAPSIM_ERR_ARG;
  *count = ctx->launches;
  return CHAPSIM_OK;
}
int chapsim_launch_count_reset(chapsim_ctx *ctx) {
  if (!ctx) return CHAPSIM_ERR_ARG;
  ctx->launches = 0;
  return CHAPSIM_OK;
}

}  // extern "C"
