// IO-domain kernels: one RK3 substep of the inflow/outflow channel section,
// x-periodic or coupled to a TG section (x ghost columns, the inlet and
// convective outlet operators; the io_np_* functions at the end), with the
// explicit viscous scheme, variable density and viscosity, and the energy
// equation with table properties.
//
// Reference (CHAPSim1WW, paths relative to the project root), channel branch
// (RCCI1 = RCCI2 = RNDI1 = 1), x periodic (IPV_io/IMV_io wrap) or not
// (TGFLOWFLG, src/INDEXSET.f90:25-32):
//   SOLVERRK3_ENG_IO        src/SOLVERRK3_ENG_IO.f90:1-77
//   RHS_ENERGY_EXPLICIT     src/RHS_ENERGY_EXPLICIT.f90:1-150
//   ENTHALPY/DENSITY_UPDATE, THERM_PROP_UPDATE, DENSITY_TIME_DERIVATION
//                           src/THERM_PROP_UPDATE.f90:2-291
//   BC_WALL_ISOFLUX         src/BC_WALL.f90:522-627
//   DENSITY_/MU_Staggered, VELOCITY_CALC_io, MASSFLUX_CALC_IO
//                           src/MASSFLUX_CALC_IO.f90:1-311
//   CONVECTION_X/Y/Z_io     src/CONVECTION_X.f90:77-176, CONVECTION_Y.f90:125-230,
//                           src/CONVECTION_Z.f90:113-200
//   DIVG_U_io               src/DIVG.f90:153-259
//   VISCOUS_ALL_EXPLT_X/Y/Z_io  src/VISCOUS_X_EXPLICIT_io.f90:1-112 and the
//                           ICHANL branches of VISCOUS_Y/Z_EXPLICIT_io.f90
//   RHS_MOM_EXPLICIT_io     src/RHS_MOM_EXPLICIT_io.f90:1-297
//   PRCALC_io, MASSFLUX_UPDATE_IO  src/PRESSURE_CORRECTION.f90:86-122,
//                           src/VELO_CORRECTION.f90:107-185
//   DIVGCK_io               src/DIVGCK.f90:60-190
//
// Layout and fusion:
//  * fields are F(1:nx, 0:ny+1, 1:nz) in HBM (x fastest, one y ghost layer);
//  * the staggered viscosities MU_STG and densities RHO_STG are never stored:
//    each kernel forms the ones it needs from mu, mu0, rho, rho0, and the
//    cell divergence DivU_io is formed from u where the stress needs it;
//  * the three momentum RHS, the RK3 combination with EXPLT0, the pressure
//    gradient and MASSFLUX_CALC_IO are one kernel (k_io_rhs) writing the
//    provisional mass flux G* into the buffer that held G0 (its old value is
//    no longer needed once DrhoDtP is formed); the x mass-flux forcing
//    DPGRNS, a constant over the domain, leaves the divergence unchanged and
//    is subtracted in the correction kernel;
//  * DIVG_io rides on the Poisson solver's forward x-transform (the shared
//    k_fftx with DrhoDtP added), and the spectral y-solve pins the mean mode
//    at the last row as FISHPACK's TRID0 does.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>

#include <string.h>

#include <string>

#include "chapsim_internal.cuh"
#include "tma.cuh"

namespace chapsim {
namespace {

using chapsim_spl::Spline;

constexpr int IO_BX = 32, IO_BY = 8;

#define CK(call)                                                          \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      return CHAPSIM_ERR_CUDA;                                            \
    }                                                                     \
  } while (0)

#define LAUNCHED()                                                        \
  do {                                                                    \
    ++c->launches;                                                        \
    cudaError_t e_ = cudaGetLastError();                                  \
    if (e_ != cudaSuccess) {                                              \
      c->err = std::string("kernel launch: ") + cudaGetErrorString(e_);   \
      return CHAPSIM_ERR_CUDA;                                            \
    }                                                                     \
  } while (0)

__device__ __forceinline__ int wrapp(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int wrapm(int i, int n) { return i == 0 ? n - 1 : i - 1; }
// x-neighbour offsets: the periodic wrap (IPV_io / IMV_io of the x-periodic
// section), or the coupled section's ghost columns (IPV_io(NCL1_io) =
// NCL1_io + 1, IMV_io(1) = 0, src/INDEXSET.f90:25-32)
__device__ __forceinline__ int64_t xplus(const TGDev &d, int i) { return d.xnp ? 1 : (int64_t)(wrapp(i, d.nx) - i); }
__device__ __forceinline__ int64_t xminus(const TGDev &d, int i) { return d.xnp ? -1 : (int64_t)(wrapm(i, d.nx) - i); }

// ---------------------------------------------------------------- table look-ups
// NIST_SLEVAL_HT (src/Flow_State.f90:1015-1070): false outside the table.
__device__ __forceinline__ bool look_ht(const IODev &io, double h, double &T) {
  if (!chapsim_spl::inside(io.ht, h)) return false;
  T = chapsim_spl::spline_eval(io.ht, h);
  if (io.shortcuts && fabs(h) < 1.0e-10) T = 1.0;
  return true;
}
// NIST_SLEVAL_TD (src/Flow_State.f90:1528-1581).
__device__ __forceinline__ bool look_td(const IODev &io, double T, double &D) {
  if (!chapsim_spl::inside(io.td, T)) return false;
  D = chapsim_spl::spline_eval(io.td, T);
  if (io.shortcuts && fabs(T - 1.0) < 1.0e-10) D = 1.0;
  return true;
}
// NIST_SLEVAL_TM / TK / TD: the three T-splines share the T grid, so one
// search serves all of them.
__device__ __forceinline__ bool look_tprops(const IODev &io, double T, double &D, double &M, double &K) {
  if (!chapsim_spl::inside(io.tm, T)) return false;
  const int it = chapsim_spl::spline_find(io.tm, T);
  M = chapsim_spl::spline_at(io.tm, it, T);
  K = chapsim_spl::spline_at(io.tk, it, T);
  D = chapsim_spl::spline_at(io.td, it, T);
  if (io.shortcuts && fabs(T - 1.0) < 1.0e-10) { M = 1.0; K = 1.0; D = 1.0; }
  return true;
}

// ---------------------------------------------------------------- energy
// RHS_ENERGY_EXPLICIT and the RHOH update of SOLVERRK3_ENG_IO (:22-35):
// rhoh += gam dt R + zeta dt R_old, limited to RHOHmax + REALMIN.  Six blocks
// per SM (40 registers): latency-bound on its neighbour loads, it gains from
// the extra resident warps (measured 0.536 -> 0.510 ms at 512x192x256).
__global__ void __launch_bounds__(IO_BX *IO_BY, 6) k_io_eng_rhs(TGDev d, IODev io, double cdt1, double cdt0, int cur) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
  const int64_t oxp = xplus(d, i), oxm = xminus(d, i);
  const int64_t ozp = d.sz * (wrapp(k, d.nz) - k), ozm = d.sz * (wrapm(k, d.nz) - k);
  const double *__restrict__ gx = io.g[cur][0], *__restrict__ gy = io.g[cur][1], *__restrict__ gz = io.g[cur][2];
  const double *__restrict__ hx = io.g[1 - cur][0], *__restrict__ hy = io.g[1 - cur][1],
               *__restrict__ hz = io.g[1 - cur][2];  // G0_io
  const double *__restrict__ H = io.h, *__restrict__ T = io.T, *__restrict__ K = io.kap;
  const double coe1 = d.dxi * 0.5 * 0.5, coe11 = d.dxqi * 0.5 * io.cthecd;
  const double coe2 = d.dyfi[j] * 0.5, coe3 = d.dzi * 0.5 * 0.5;
  const double coe33 = d.dzqi * 0.5 * io.cthecd, coe22 = d.dyfi[j] * io.cthecd;
  // the wall rows: an iso-flux wall takes its flux with coefficient 1, an
  // iso-thermal wall the conduction to its ghost row (the wall values, half a
  // cell away: DYCI of the wall node), src/RHS_ENERGY_EXPLICIT.f90:41-72
  const bool iso_bot = io.isothermal & 1, iso_top = io.isothermal & 2;
  double coe221, coe222;
  if (j == 1) {
    coe221 = d.dyci[j + 1];
    coe222 = iso_bot ? d.dyci[j] : 1.0;
  } else if (j == ny) {
    coe222 = d.dyci[j];
    coe221 = iso_top ? d.dyci[j + 1] : 1.0;
  } else {
    coe221 = d.dyci[j + 1];
    coe222 = d.dyci[j];
  }
  const double wffp = d.wff[j + 1], wfbp = d.wfb[j + 1], wff = d.wff[j], wfb = d.wfb[j];
  const double hc = H[c];
  double dx_rhohu = (H[c + oxp] + hc) * (hx[c + oxp] + gx[c + oxp]) - (hc + H[c + oxm]) * (hx[c] + gx[c]);
  dx_rhohu *= coe1;
  double dy_rhohv = (wffp * H[c + sy] + wfbp * hc) * (hy[c + sy] + gy[c + sy]) -
                    (wff * hc + wfb * H[c - sy]) * (hy[c] + gy[c]);
  dy_rhohv *= coe2;
  double dz_rhohw = (H[c + ozp] + hc) * (hz[c + ozp] + gz[c + ozp]) - (hc + H[c + ozm]) * (hz[c] + gz[c]);
  dz_rhohw *= coe3;
  const double tc = T[c], kc = K[c];
  double dx_kdt = (K[c + oxp] + kc) * (T[c + oxp] - tc) - (kc + K[c + oxm]) * (tc - T[c + oxm]);
  dx_kdt *= coe11;
  double kdty1 = (wffp * K[c + sy] + wfbp * kc) * (T[c + sy] - tc) * coe221;
  double kdty2 = (wff * kc + wfb * K[c - sy]) * (tc - T[c - sy]) * coe222;
  if (j == 1 && !iso_bot)
    kdty2 = -io.qw_bot * coe222;  // WALLFLUX(bottom) = +qw
  else if (j == ny && !iso_top)
    kdty1 = io.qw_top * coe221;   // -WALLFLUX(top), WALLFLUX(top) = -qw
  const double dy_kdt = (kdty1 - kdty2) * coe22;
  double dz_kdt = (K[c + ozp] + kc) * (T[c + ozp] - tc) - (K[c + ozm] + kc) * (tc - T[c + ozm]);
  dz_kdt *= coe33;
  const double R = -dx_rhohu - dy_rhohv - dz_rhohw + dx_kdt + dy_kdt + dz_kdt;
  double r = io.rhoh[c] + cdt1 * R + cdt0 * io.rhse0[c];
  r = fmin(io.rhohmax + 1.0e-14, r);
  io.rhoh[c] = r;
  io.rhse0[c] = R;
}

// VISCOUSITY0 <- VISCOUSITY, DENSITY0 <- DENSITY over the whole array (ghost
// rows included), then for interior cells ENTHALPY_UPDATE, DENSITY_UPDATE,
// ENTHALPY_UPDATE, THERM_PROP_UPDATE.  A look-up outside the table leaves the
// value unchanged and is counted (the reference STOPs).
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_eng_props(TGDev d, IODev io) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y;  // 0 .. ny+1
  const int k = blockIdx.z;
  if (i >= nx || j > ny + 1) return;
  const int64_t c = i + d.sy * j + d.sz * k;
  const double dold = io.D[c], muold = io.mu[c];
  io.mu0[c] = muold;
  io.D0[c] = dold;
  if (j < 1 || j > ny) {
    io.msum[c] = muold + muold;  // ghost rows: the ghost kernel sets the new value
    return;
  }
  const double rh = io.rhoh[c];
  int bad = 0;
  double h = rh / dold, T, D = dold;
  if (look_ht(io, h, T) && look_td(io, T, D)) {
  } else {
    D = dold;
    ++bad;
  }
  h = rh / D;
  io.h[c] = h;
  bool keep = io.shortcuts && fabs(h) < 1.0e-10;
  double munew = muold;
  if (!keep) {
    double M, K, D2;
    if (look_ht(io, h, T) && look_tprops(io, T, D2, M, K)) {
      io.T[c] = T;
      io.mu[c] = M;
      io.kap[c] = K;
      D = D2;
      munew = M;
    } else {
      ++bad;
    }
  }
  io.D[c] = D;
  io.msum[c] = muold + munew;  // VISCOUSITY0 + VISCOUSITY
  if (bad) atomicAdd(io.bad, (unsigned long long)bad);
}

// BC_WALL_ISOFLUX: ghost enthalpy extrapolated from the first two cells, the
// ghost properties from the table.  blockIdx.y: 0 bottom, 1 top.
__global__ void k_io_eng_ghost(TGDev d, IODev io) {
  const int nx = d.nx, ny = d.ny;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * d.nz) return;
  const int k = t / nx, i = t - k * nx;
  const int64_t sy = d.sy, base = i + d.sz * k;
  const bool top = blockIdx.y == 1;
  const int j = top ? ny + 1 : 0;
  const int64_t c = base + sy * j;
  const int side = top ? 1 : 0;
  double h, T, D, M, K;
  if (io.isothermal & (1 << side)) {
    // BC_WALL_ISOTHERMAL (src/BC_WALL.f90:462-515): the wall values
    T = io.wall[side][0];
    h = io.wall[side][1];
    D = io.wall[side][2];
    M = io.wall[side][3];
    K = io.wall[side][4];
    io.h[c] = h;
  } else {
    if (!top)
      h = 2.0 * io.h[base + sy] - d.wff[2] * io.h[base + 2 * sy] - d.wfb[2] * io.h[base + sy];
    else
      h = 2.0 * io.h[base + sy * ny] - d.wff[ny] * io.h[base + sy * ny] - d.wfb[ny] * io.h[base + sy * (ny - 1)];
    io.h[c] = h;
    if (!look_ht(io, h, T) || !look_tprops(io, T, D, M, K)) {
      atomicAdd(io.bad, 1ull);
      return;
    }
  }
  io.D[c] = D;
  io.T[c] = T;
  io.mu[c] = M;
  io.kap[c] = K;
  io.rhoh[c] = h * D;
  io.msum[c] = io.mu0[c] + M;
}

// THERM_PROP_UPDATE on the interior after a restart (h read from the file),
// then mu0 = mu, rho0 = rho and mu0 + mu over every row (the ghost rows
// already hold BC_WALL_ISOFLUX's values).
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_props_only(TGDev d, IODev io) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y;  // 0 .. ny+1
  const int k = blockIdx.z;
  if (i >= nx || j > ny + 1) return;
  const int64_t c = i + d.sy * j + d.sz * k;
  if (io.thermal && j >= 1 && j <= ny) {
    const double h = io.h[c];
    if (!(io.shortcuts && fabs(h) < 1.0e-10)) {
      double T, D, M, K;
      if (look_ht(io, h, T) && look_tprops(io, T, D, M, K)) {
        io.T[c] = T;
        io.mu[c] = M;
        io.kap[c] = K;
        io.D[c] = D;
      } else {
        atomicAdd(io.bad, 1ull);
      }
    }
  }
  const double mu = io.mu[c];
  io.mu0[c] = mu;
  io.D0[c] = io.D[c];
  io.msum[c] = mu + mu;
}

// ------------------------------------------------------ learned properties
// The property update of SOLVERRK3_ENG_IO (:46-55) with the learned model
// (mlp_tc.cuh) in place of the table splines: VISCOUSITY0 / DENSITY0 <-
// VISCOUSITY / DENSITY, then DENSITY_UPDATE on h1 = rho h / rho_old (the
// model's rho), ENTHALPY_UPDATE h2 = rho h / rho_new, and THERM_PROP_UPDATE
// on h2 (the model's T, rho, mu, k).  Cells whose h-bin the error gate has
// not cleared for all four take the table splines, as do out-of-table
// checks.  The field is walked as a flat array in 128-cell tiles (ghost rows
// keep the plain kernel's treatment: mu0, rho0 and mu0 + mu only).
// The model is evaluated once per tile, at h1, with its derivative (forward
// mode on the tensor cores, tile_eval_d); the properties at h2 come from the
// first-order expansion of the network's residual around h1 plus the exact
// polynomial base at h2.  h2 differs from h1 by the density change of one
// substep (|dx| ~ 1e-4); a tile in which any model cell moves further than
// kTaylorMax evaluates the model a second time at h2.  This halves the tanh
// evaluations; the elementwise work between the layers runs on packed FP32
// pairs, and the kernel is bound by its instruction issue rate.
__global__ void __launch_bounds__(chapsim_mlp::TILE, 3) k_io_eng_props_mlp(TGDev d, IODev io, chapsim_mlp::MlpDev M) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  chapsim_mlp::SmemD &s = chapsim_mlp::smem_of<chapsim_mlp::SmemD>(smem_raw);
  chapsim_mlp::cta_setup_d(s, M);
  uint32_t phase = 0;
  const int64_t n = d.sz * d.nz;
  const int64_t ntiles = (n + chapsim_mlp::TILE - 1) / chapsim_mlp::TILE;
  const int64_t rows = d.ny + 2;
  const double hinv = 1.0 / M.hhalf;
  // The thread's cell advances by a fixed stride per tile: its x index and
  // row j follow incrementally instead of by two 64-bit divisions per cell.
  const int64_t stride = (int64_t)gridDim.x * chapsim_mlp::TILE;
  const int sx = (int)(stride % d.nx), sj = (int)((stride / d.nx) % rows);
  int64_t c = (int64_t)blockIdx.x * chapsim_mlp::TILE + threadIdx.x;
  int ix = (int)(c % d.nx), j = (int)((c / d.nx) % rows);
  // the next tile's inputs are loaded while the current one is evaluated
  double nD = 1.0, nmu = 0.0, nrh = 0.0;
  if (c < n) {
    nD = io.D[c];
    nmu = io.mu[c];
    nrh = io.rhoh[c];
  }
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, c += stride) {
    const bool valid = c < n;
    const bool interior = valid && j >= 1 && j <= d.ny;
    const double dold = nD, muold = nmu, rh = interior ? nrh : 0.0;
    if (c + stride < n) {
      nD = io.D[c + stride];
      nmu = io.mu[c + stride];
      nrh = io.rhoh[c + stride];
    }
    ix += sx;
    const int carry = ix >= d.nx;
    ix -= carry ? d.nx : 0;
    j += sj + carry;
    j -= j >= rows ? (int)rows : 0;
    if (valid) {
      io.mu0[c] = muold;
      io.D0[c] = dold;
      if (!interior) io.msum[c] = muold + muold;  // ghost rows: the ghost kernel sets the new value
    }
    // DENSITY_UPDATE
    const double h1 = rh / dold;
    const double x1 = (h1 - M.hmid) * hinv;
    float y[chapsim_mlp::NO], dy[chapsim_mlp::NO];
    chapsim_mlp::tile_eval_d(s, (float)x1, y, dy, phase, d.err);  // a failed wait: s.fail, read below
    int bad = 0;
    double D = dold;
    if (interior) {
      double T;
      if (!chapsim_spl::inside(io.ht, h1)) {
        ++bad;
      } else if (chapsim_mlp::gate_step(s, M, h1)) {
        D = chapsim_mlp::assemble(M, 1, x1, y[1]);
      } else if (!(look_ht(io, h1, T) && look_td(io, T, D))) {
        D = dold;
        ++bad;
      }
    }
    // ENTHALPY_UPDATE; the model at h2 by expansion or, for a far step, anew
    const double h2 = rh / D;
    const double x2 = (h2 - M.hmid) * hinv;
    const bool keep = io.shortcuts && fabs(h2) < 1.0e-10;
    const bool model2 = interior && !keep && chapsim_spl::inside(io.ht, h2) &&
                        chapsim_mlp::gate_step(s, M, h2);
    const bool again = __syncthreads_or(model2 && fabs(x2 - x1) > chapsim_mlp::kTaylorMax);
    if (s.fail) break;  // block-uniform after the barrier
    float y2[chapsim_mlp::NO];
    if (again && threadIdx.x == 0) atomicAdd(io.model_again, 1ull);
    if (again) {
      if (!chapsim_mlp::tile_eval(s, (float)x2, y2, phase, d.err)) break;
    } else {
#pragma unroll
      for (int q = 0; q < chapsim_mlp::NO; ++q) y2[q] = y[q] + dy[q] * (float)(x2 - x1);
    }
    if (!interior) continue;
    io.h[c] = h2;
    double munew = muold;
    if (!keep) {
      double T, M2, K, D2;
      bool ok = model2;
      if (model2) {
        T = chapsim_mlp::assemble(M, 0, x2, y2[0]);
        D2 = chapsim_mlp::assemble(M, 1, x2, y2[1]);
        M2 = chapsim_mlp::assemble(M, 2, x2, y2[2]);
        K = chapsim_mlp::assemble(M, 3, x2, y2[3]);
      } else {
        ok = look_ht(io, h2, T) && look_tprops(io, T, D2, M2, K);
      }
      if (ok) {
        io.T[c] = T;
        io.mu[c] = M2;
        io.kap[c] = K;
        D = D2;
        munew = M2;
      } else {
        ++bad;
      }
    }
    io.D[c] = D;
    io.msum[c] = muold + munew;
    if (bad) atomicAdd(io.bad, (unsigned long long)bad);
  }
  chapsim_mlp::cta_teardown(s);
}

// THERM_PROP_UPDATE(IMAIND) on its own (src/THERM_PROP_UPDATE.f90:129-205):
// h -> T, mu, k, rho on the interior rows, by the table splines
// (use_mlp = 0, one thread per cell) or the learned model with the table
// where the gate has not cleared the bin; mu0 + mu follows the new mu.
__global__ void __launch_bounds__(chapsim_mlp::TILE, 4) k_io_therm_props(TGDev d, IODev io, chapsim_mlp::MlpDev M,
                                                                         int use_mlp) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  chapsim_mlp::Smem *sp = nullptr;
  uint32_t phase = 0;
  if (use_mlp) {
    sp = &chapsim_mlp::smem_of(smem_raw);
    chapsim_mlp::cta_setup(*sp, M);
  }
  const int64_t n = d.sz * d.nz;
  const int64_t ntiles = (n + chapsim_mlp::TILE - 1) / chapsim_mlp::TILE;
  const int64_t rows = d.ny + 2;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t c = tile * chapsim_mlp::TILE + threadIdx.x;
    const bool valid = c < n;
    const int j = valid ? (int)((c / d.nx) % rows) : 0;
    const bool interior = valid && j >= 1 && j <= d.ny;
    const double h = interior ? io.h[c] : 0.0;
    const double x = use_mlp ? (h - M.hmid) / M.hhalf : 0.0;
    float y[chapsim_mlp::NO];
    if (use_mlp && !chapsim_mlp::tile_eval(*sp, (float)x, y, phase, d.err)) break;
    if (!interior || (io.shortcuts && fabs(h) < 1.0e-10)) continue;
    double T, D, Mu, K;
    bool ok = chapsim_spl::inside(io.ht, h);
    if (ok && use_mlp && chapsim_mlp::gate_step(*sp, M, h)) {
      T = chapsim_mlp::assemble(M, 0, x, y[0]);
      D = chapsim_mlp::assemble(M, 1, x, y[1]);
      Mu = chapsim_mlp::assemble(M, 2, x, y[2]);
      K = chapsim_mlp::assemble(M, 3, x, y[3]);
    } else {
      ok = ok && look_ht(io, h, T) && look_tprops(io, T, D, Mu, K);
    }
    if (!ok) {
      atomicAdd(io.bad, 1ull);
      continue;
    }
    io.T[c] = T;
    io.D[c] = D;
    io.mu[c] = Mu;
    io.kap[c] = K;
    io.msum[c] = io.mu0[c] + Mu;
  }
  if (use_mlp) chapsim_mlp::cta_teardown(*sp);
}

// msum = mu0 + mu over the whole array (after the host replaces mu or mu0).
__global__ void k_io_msum(IODev io, size_t n) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    io.msum[t] = io.mu0[t] + io.mu[t];
}

// ---------------------------------------------------------------- momentum
// DENSITY_TIME_DERIVATION (gamma - 2 divisor as written) and VELOCITY_CALC_io
// with its wall BC.  RHO_STG is formed from rho, rho0 (DENSITY_Staggered).
// Eight blocks per SM for the explicit scheme (32 registers, measured 0.459
// -> 0.410 ms at 512x192x256): latency-bound, it gains from the extra
// resident warps.  The DRHOI variant keeps its register count (a cap spills).
// DENSITY_TIME_DERIVATION and VELOCITY_CALC_io of one cell; returns its DrhoDtP
// (zero without do_drho)
template <bool VISC>
__device__ __forceinline__ double io_prep_cell(TGDev d, IODev io, double gp, double zr, double den, int cur,
                                               int do_drho, int i, int j, int k) {
  const int ny = d.ny;
  double drho_c = 0.0;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
  const int64_t oxp = xplus(d, i), oxm = xminus(d, i);
  const int64_t ozp = d.sz * (wrapp(k, d.nz) - k), ozm = d.sz * (wrapm(k, d.nz) - k);
  const double *__restrict__ gx = io.g[cur][0], *__restrict__ gy = io.g[cur][1], *__restrict__ gz = io.g[cur][2];
  if (do_drho) {
    const double *__restrict__ hx = io.g[1 - cur][0], *__restrict__ hy = io.g[1 - cur][1],
                 *__restrict__ hz = io.g[1 - cur][2];
    const double divx = (gx[c + oxp] - gx[c]) * d.dxi, divx0 = (hx[c + oxp] - hx[c]) * d.dxi;
    const double divy = (gy[c + sy] - gy[c]) * d.dyfi[j], divy0 = (hy[c + sy] - hy[c]) * d.dyfi[j];
    const double divz = (gz[c + ozp] - gz[c]) * d.dzi, divz0 = (hz[c + ozp] - hz[c]) * d.dzi;
    drho_c = (gp * (divx + divy + divz) + zr * (divx0 + divy0 + divz0)) / den;
    io.drho[c] = drho_c;
  }
  double rx = 1.0, ry = 1.0, rz = 1.0;
  if (io.thermal) {
    const double *__restrict__ D = io.D, *__restrict__ D0 = io.D0;
    rx = (D[c] + D[c + oxm] + D0[c] + D0[c + oxm]) * 0.5 * 0.5;
    rz = (D[c] + D[c + ozm] + D0[c] + D0[c + ozm]) * 0.5 * 0.5;
    if (j >= 2) ry = (d.wff[j] * (D[c] + D0[c]) + d.wfb[j] * (D[c - sy] + D0[c - sy])) * 0.5;
  }
  if (VISC && do_drho) {
    // DENSITY_implicit_add (src/MASSFLUX_CALC_IO.f90:316-399): 1/RHO_STG minus
    // 1/(the old density on the face); other rows stay zero
    const double *__restrict__ D0 = io.D0;
    io.drhoi[0][c] = 1.0 / rx - 1.0 / ((D0[c] + D0[c + oxm]) * 0.5);
    io.drhoi[2][c] = 1.0 / rz - 1.0 / ((D0[c] + D0[c + ozm]) * 0.5);
    if (j >= 2) io.drhoi[1][c] = 1.0 / ry - 1.0 / (d.wff[j] * D0[c] + d.wfb[j] * D0[c - sy]);
  }
  d.u[c] = gx[c] / rx;
  d.w[c] = gz[c] / rz;
  if (j >= 2) d.v[c] = gy[c] / ry;
  if (j == 1) {
    d.u[c - sy] = 0.0; d.w[c - sy] = 0.0; d.v[c - sy] = 0.0; d.v[c] = 0.0;
  }
  if (j == ny) {
    d.u[c + sy] = 0.0; d.w[c + sy] = 0.0; d.v[c + sy] = 0.0;
  }
  return drho_c;
}

// mass_part (the coupled section): the block sums of DrhoDtP / DYFI, which
// CHK_MassConsv_io's mass rate needs, go to d.partials in the order of
// k_io_red_part (same bits), saving that kernel's pass over DrhoDtP.
template <bool VISC>
__global__ void __launch_bounds__(IO_BX *IO_BY, VISC ? 1 : 8) k_io_prep(TGDev d, IODev io, double gp, double zr, double den,
                                                        int cur, int do_drho, int mass_part) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (mass_part) {
    __shared__ double red[IO_BX * IO_BY / 32];
    double v = 0.0;
    if (i < nx && j <= ny) v = io_prep_cell<VISC>(d, io, gp, zr, den, cur, do_drho, i, j, k) / d.dyfi[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int tid = threadIdx.x + IO_BX * threadIdx.y;
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
      double sum = 0.0;
      for (int q = 0; q < IO_BX * IO_BY / 32; ++q) sum += red[q];
      d.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = sum;
    }
    return;
  }
  if (i >= nx || j > ny) return;
  io_prep_cell<VISC>(d, io, gp, zr, den, cur, do_drho, i, j, k);
}


// Staggered viscosities of MU_Staggered, formed on demand.  mustg1: x-face /
// y-face edge, rows 2..ny, wall rows 1 and ny+1 from the ghost cells;
// mustg2: x-face / z-face edge, rows 1..ny; mustg3: y-face / z-face edge.
struct MuView {
  const double *__restrict__ mu;
  const double *__restrict__ mu0;
  const double *__restrict__ wff;
  const double *__restrict__ wfb;
  int64_t sy;
  int ny, thermal;
  __device__ __forceinline__ double cell(int64_t c) const { return thermal ? 0.5 * (mu0[c] + mu[c]) : 1.0; }
  // c: the cell (i, jj, k); oxm: offset to i-1
  __device__ __forceinline__ double s1(int64_t c, int jj, int64_t oxm) const {
    if (!thermal) return 1.0;
    if (jj == 1) return 0.5 * (mu0[c - sy] + mu[c - sy]);
    if (jj == ny + 1) return 0.5 * (mu0[c] + mu[c]);
    return ((mu[c] + mu[c + oxm] + mu0[c] + mu0[c + oxm]) * wff[jj] +
            (mu[c - sy] + mu[c - sy + oxm] + mu0[c - sy] + mu0[c - sy + oxm]) * wfb[jj]) * 0.5 * 0.5;
  }
  __device__ __forceinline__ double s2(int64_t c, int64_t oxm, int64_t ozm) const {
    if (!thermal) return 1.0;
    return (mu[c] + mu[c + oxm] + mu0[c] + mu0[c + oxm] + mu[c + ozm] + mu[c + oxm + ozm] + mu0[c + ozm] +
            mu0[c + oxm + ozm]) * 0.5 * 0.5 * 0.5;
  }
  __device__ __forceinline__ double s3(int64_t c, int jj, int64_t ozm) const {
    if (!thermal) return 1.0;
    if (jj == 1) return 0.5 * (mu0[c - sy] + mu[c - sy]);
    if (jj == ny + 1) return 0.5 * (mu0[c] + mu[c]);
    return ((mu[c + ozm] + mu[c] + mu0[c + ozm] + mu0[c]) * wff[jj] +
            (mu[c - sy + ozm] + mu[c - sy] + mu0[c - sy + ozm] + mu0[c - sy]) * wfb[jj]) * 0.5 * 0.5;
  }
};

// Convection, DivU, viscous stresses, RHS_MOM_EXPLICIT_io and
// MASSFLUX_CALC_IO for all three components of one cell; G* goes to the
// buffer g[1 - cur].  Per-block sums of RHS_x / DYFI feed DPGRNS.
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_rhs(TGDev d, IODev io, double gam, double roh, double alp,
                                                       int cur) {
  __shared__ double red[IO_BX * IO_BY / 32];
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  double part = 0.0;
  if (i < nx && j <= ny) {
    const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
    const int64_t oxp = xplus(d, i), oxm = xminus(d, i);
    const int64_t ozp = d.sz * (wrapp(k, d.nz) - k), ozm = d.sz * (wrapm(k, d.nz) - k);
    const double *__restrict__ u = d.u, *__restrict__ v = d.v, *__restrict__ w = d.w, *__restrict__ p = d.p;
    const double *__restrict__ gx = io.g[cur][0], *__restrict__ gy = io.g[cur][1], *__restrict__ gz = io.g[cur][2];
    double *__restrict__ nxg = io.g[1 - cur][0];
    double *__restrict__ nyg = io.g[1 - cur][1];
    double *__restrict__ nzg = io.g[1 - cur][2];
    const MuView mv{io.mu, io.mu0, d.wff, d.wfb, sy, ny, io.thermal};
    const double dxi = d.dxi, dzi = d.dzi, cv = d.cvisc, dt = d.dt;
    const double dyfj = d.dyfi[j], dycj = d.dyci[j], dycp = d.dyci[j + 1];
    const double wff = d.wff[j], wfb = d.wfb[j], wffp = d.wff[j + 1], wfbp = d.wfb[j + 1];
    // DIVG_U_io at cell (ii, jj, kk) = cc
    auto divu = [&](int64_t cc, int ii, int jj, int kk) {
      const int64_t op = (!d.xnp && ii + 1 == nx) ? -(int64_t)(nx - 1) : 1;
      const int64_t oz = (kk + 1 == d.nz) ? -(int64_t)d.sz * (d.nz - 1) : d.sz;
      return ((u[cc + op] - u[cc]) * dxi + (v[cc + sy] - v[cc]) * d.dyfi[jj] + (w[cc + oz] - w[cc]) * dzi) / 3.0;
    };
    const double divc = divu(c, i, j, k);
    // the coupled section's staggered viscosities MU_STG on the outlet ghost
    // face keep their initial value 1 (MU_Staggered covers IC = 1..NCL1_io,
    // src/MASSFLUX_CALC_IO.f90:147-237, MEMALLOCT.f90:201)
    const bool xout = d.xnp && i == nx - 1;
    // ---------------- x: CONVECTION_X_io + VISCOUS_ALL_EXPLT_X_io; the coupled
    // section's inlet face (NXI = 2) keeps its value (copied by k_np_gbound)
    if (!d.xnp || i > 0) {
      double h11f = (gx[c + oxp] + gx[c]) * (u[c + oxp] + u[c]);
      double h11b = (gx[c] + gx[c + oxm]) * (u[c] + u[c + oxm]);
      double h11 = (h11f - h11b) * (dxi * 0.5 * 0.5);
      double h12f = (gy[c + sy] + gy[c + sy + oxm]) * (wffp * u[c + sy] + wfbp * u[c]);
      double h12b = (gy[c] + gy[c + oxm]) * (wff * u[c] + wfb * u[c - sy]);
      double h12 = (h12f - h12b) * (dyfj * 0.5);
      double h13f = (gz[c + ozp] + gz[c + ozp + oxm]) * (u[c + ozp] + u[c]);
      double h13b = (gz[c] + gz[c + oxm]) * (u[c] + u[c + ozm]);
      double h13 = (h13f - h13b) * (dzi * 0.5 * 0.5);
      double ex = -(h11 + h12 + h13);
      double dudx = (u[c + oxp] - u[c]) * dxi;
      const double tau11f = mv.cell(c) * (dudx - divc);
      dudx = (u[c] - u[c + oxm]) * dxi;
      const double tau11b = mv.cell(c + oxm) * (dudx - divu(c + oxm, wrapm(i, nx), j, k));
      const double d11 = (tau11f - tau11b) * (2.0 * dxi * cv);
      double dudy = (u[c + sy] - u[c]) * dycp;
      double dvdx = (v[c + sy] - v[c + sy + oxm]) * dxi;
      const double tau12f = mv.s1(c + sy, j + 1, oxm) * (dudy + dvdx);
      dudy = (u[c] - u[c - sy]) * dycj;
      dvdx = (v[c] - v[c + oxm]) * dxi;
      const double tau12b = mv.s1(c, j, oxm) * (dudy + dvdx);
      const double d12 = (tau12f - tau12b) * (dyfj * cv);
      double dudz = (u[c + ozp] - u[c]) * dzi;
      double dwdx = (w[c + ozp] - w[c + ozp + oxm]) * dxi;
      const double tau13f = mv.s2(c + ozp, oxm, -ozp) * (dudz + dwdx);
      dudz = (u[c] - u[c + ozm]) * dzi;
      dwdx = (w[c] - w[c + oxm]) * dxi;
      const double tau13b = mv.s2(c, oxm, ozm) * (dudz + dwdx);
      const double d13 = (tau13f - tau13b) * (dzi * cv);
      ex = ex + d11 + d12 + d13;
      double *e0 = (double *)d.h0[0];
      double r = (gam * ex + roh * e0[c]) * dt;
      e0[c] = ex;
      r -= (p[c] - p[c + oxm]) * (alp * dt * dxi);
      if (io.gravdir == 1) {
        const double rs = io.thermal ? (io.D[c] + io.D[c + oxm] + io.D0[c] + io.D0[c + oxm]) * 0.5 * 0.5 : 1.0;
        r += rs * (alp * dt * io.f_a);
      }
      part = r / dyfj;
      nxg[c] = gx[c] + r;
    }
    // ---------------- y (rows 2..ny): CONVECTION_Y_io + VISCOUS_ALL_EXPLT_Y_io
    if (j >= 2) {
      double h21f = (wff * gx[c + oxp] + wfb * gx[c + oxp - sy]) * (v[c + oxp] + v[c]);
      double h21b = (wff * gx[c] + wfb * gx[c - sy]) * (v[c] + v[c + oxm]);
      double h21 = (h21f - h21b) * (dxi * 0.5);
      double h22f = (gy[c + sy] + gy[c]) * (v[c + sy] + v[c]);
      double h22b = (gy[c] + gy[c - sy]) * (v[c] + v[c - sy]);
      double h22 = (h22f - h22b) * (dycj * 0.5 * 0.5);
      double h23f = (wff * gz[c + ozp] + wfb * gz[c + ozp - sy]) * (v[c + ozp] + v[c]);
      double h23b = (wff * gz[c] + wfb * gz[c - sy]) * (v[c] + v[c + ozm]);
      double h23 = (h23f - h23b) * (dzi * 0.5);
      double ey = -(h21 + h22 + h23);
      double dvdy = (v[c + sy] - v[c]) * dyfj;
      const double tau22f = mv.cell(c) * (dvdy - divc);
      dvdy = (v[c] - v[c - sy]) * d.dyfi[j - 1];
      const double tau22b = mv.cell(c - sy) * (dvdy - divu(c - sy, i, j - 1, k));
      const double d22 = (tau22f - tau22b) * (2.0 * dycj * cv);
      double dvdx = (v[c + oxp] - v[c]) * dxi;
      double dudy = (u[c + oxp] - u[c + oxp - sy]) * dycj;
      const double tau21f = (xout ? 1.0 : mv.s1(c + oxp, j, -oxp)) * (dvdx + dudy);
      dvdx = (v[c] - v[c + oxm]) * dxi;
      dudy = (u[c] - u[c - sy]) * dycj;
      const double tau21b = mv.s1(c, j, oxm) * (dvdx + dudy);
      const double d21 = (tau21f - tau21b) * (dxi * cv);
      double dvdz = (v[c + ozp] - v[c]) * dzi;
      double dwdy = (w[c + ozp] - w[c + ozp - sy]) * dycj;
      const double tau23f = mv.s3(c + ozp, j, -ozp) * (dvdz + dwdy);
      dvdz = (v[c] - v[c + ozm]) * dzi;
      dwdy = (w[c] - w[c - sy]) * dycj;
      const double tau23b = mv.s3(c, j, ozm) * (dvdz + dwdy);
      const double d23 = (tau23f - tau23b) * (dzi * cv);
      ey = ey + d21 + d22 + d23;
      double *e0 = (double *)d.h0[1];
      double r = (gam * ey + roh * e0[c]) * dt;
      e0[c] = ey;
      r -= (p[c] - p[c - sy]) * (alp * dt * dycj);
      if (io.gravdir == 2) {
        const double rs = io.thermal ? (wff * (io.D[c] + io.D0[c]) + wfb * (io.D[c - sy] + io.D0[c - sy])) * 0.5 : 1.0;
        r += rs * (alp * dt * io.f_a);
      }
      nyg[c] = gy[c] + r;
    }
    // ---------------- z: CONVECTION_Z_io + VISCOUS_ALL_EXPLT_Z_io
    {
      double h31f = (gx[c + oxp] + gx[c + oxp + ozm]) * (w[c + oxp] + w[c]);
      double h31b = (gx[c] + gx[c + ozm]) * (w[c] + w[c + oxm]);
      double h31 = (h31f - h31b) * (dxi * 0.5 * 0.5);
      double h32f = (gy[c + sy] + gy[c + sy + ozm]) * (wffp * w[c + sy] + wfbp * w[c]);
      double h32b = (gy[c] + gy[c + ozm]) * (wff * w[c] + wfb * w[c - sy]);
      double h32 = (h32f - h32b) * (dyfj * 0.5);
      double h33f = (gz[c + ozp] + gz[c]) * (w[c + ozp] + w[c]);
      double h33b = (gz[c] + gz[c + ozm]) * (w[c] + w[c + ozm]);
      double h33 = (h33f - h33b) * (dzi * 0.5 * 0.5);
      double ez = -(h31 + h32 + h33);
      double dwdz = (w[c + ozp] - w[c]) * dzi;
      const double tau33f = mv.cell(c) * (dwdz - divc);
      dwdz = (w[c] - w[c + ozm]) * dzi;
      const double tau33b = mv.cell(c + ozm) * (dwdz - divu(c + ozm, i, j, wrapm(k, d.nz)));
      const double d33 = (tau33f - tau33b) * (2.0 * dzi * cv);
      double dwdx = (w[c + oxp] - w[c]) * dxi;
      double dudz = (u[c + oxp] - u[c + oxp + ozm]) * dzi;
      const double tau31f = (xout ? 1.0 : mv.s2(c + oxp, -oxp, ozm)) * (dwdx + dudz);
      dwdx = (w[c] - w[c + oxm]) * dxi;
      dudz = (u[c] - u[c + ozm]) * dzi;
      const double tau31b = mv.s2(c, oxm, ozm) * (dwdx + dudz);
      const double d31 = (tau31f - tau31b) * (dxi * cv);
      double dwdy = (w[c + sy] - w[c]) * dycp;
      double dvdz = (v[c + sy] - v[c + sy + ozm]) * dzi;
      const double tau32f = mv.s3(c + sy, j + 1, ozm) * (dwdy + dvdz);
      dwdy = (w[c] - w[c - sy]) * dycj;
      dvdz = (v[c] - v[c + ozm]) * dzi;
      const double tau32b = mv.s3(c, j, ozm) * (dwdy + dvdz);
      const double d32 = (tau32f - tau32b) * (dyfj * cv);
      ez = ez + d31 + d32 + d33;
      double *e0 = (double *)d.h0[2];
      double r = (gam * ez + roh * e0[c]) * dt;
      e0[c] = ez;
      r -= (p[c] - p[c + ozm]) * (alp * dt * dzi);
      if (io.gravdir == 3) {
        const double rs = io.thermal ? (io.D[c] + io.D[c + ozm] + io.D0[c] + io.D0[c + ozm]) * 0.5 * 0.5 : 1.0;
        r += rs * (alp * dt * io.f_a);
      }
      nzg[c] = gz[c] + r;
    }
  }
  // fixed-order block sum of RHS_x / DYFI
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  const int tid = threadIdx.x + IO_BX * threadIdx.y;
  if ((tid & 31) == 0) red[tid >> 5] = part;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int q = 0; q < IO_BX * IO_BY / 32; ++q) s += red[q];
    io.part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
  }
}

// The same per-cell arithmetic as k_io_rhs, as a 2.5-D stencil: a block owns
// a 32 x 8 (x, y) tile and marches along z over nzc planes.  Each plane of u,
// v, w, G (three components), p and, with thermal on, M = mu0 + mu arrives in
// shared memory as one TMA box of 36 x 10 doubles (x0-2 .. x0+33,
// j0-1 .. j0+8; the x start is 16-byte aligned) in a ring of four plane
// slots, so plane k+2 is in flight while plane k is computed.  Periodic x
// neighbours outside the box are patched in from global memory on the first
// and last x tiles; z wraps by plane index.  p travels with the plane, and
// mu, mu0 as their sum M (the only combination MU_STG and the cell viscosity
// use); EXPLT0 of the tile's own cells comes by 32 x 8 boxes in a two-slot
// ring one plane ahead.
constexpr int IT_BXW = 36, IT_BYW = 10, IT_PLANE = IT_BXW * IT_BYW, IT_PST = 368, IT_NF = 8;
// halo fields of a plane slot; M = mu0 + mu (thermal only, last)
constexpr int F_U = 0, F_V = 1, F_W = 2, F_GX = 3, F_GY = 4, F_GZ = 5, F_P = 6, F_M = 7;
constexpr int IT_EBOX = IO_BX * IO_BY;  // EXPLT0 boxes: the tile's own 32 x 8 cells
constexpr size_t IT_SLOT = (size_t)IT_NF * IT_PST * sizeof(double);
constexpr size_t IT_ESLOT = (size_t)3 * IT_EBOX * sizeof(double);
static_assert((IT_PST * 8) % 128 == 0 && IT_PST >= IT_PLANE, "TMA destinations must stay 128-byte aligned");
static_assert(IT_SLOT % 128 == 0 && IT_ESLOT % 128 == 0 && (IT_EBOX * 8) % 128 == 0, "128-byte aligned slots");
struct IoMaps {
  CUtensorMap m[14];  // u, v, w, p, msum, g[0][0..2], g[1][0..2], EXPLT0[0..2]
};

// EXPLT0 of the tile's own cells: plain loads into registers, issued at the
// top of each plane's iteration ahead of the plane waits (measured faster
// than the two-slot TMA ring: 0.260 against 0.274 ms per launch at
// 512x192x64, x-periodic, energy equation on), or the ring.
constexpr bool IT_EREG = true;

// Plane geometry.  The coupled section's fields start one value before
// column 0 (its inlet ghost column), and its maps start there: the box that
// covers columns x0 - 2 .. x0 + 33 must start at an even map coordinate, so
// it starts at column x0 - 3 (map x0 - 2) and is 38 wide.  Its EXPLT0 is
// always read with plain loads (a 32-wide box at column x0 would start at an
// odd map coordinate).
template <bool CPL> struct ItGeo {
  static constexpr int BXW = CPL ? 38 : IT_BXW, PLANE = BXW * IT_BYW, PST = CPL ? 384 : IT_PST, XO = CPL ? 3 : 2;
  static constexpr bool EREG = CPL || IT_EREG;  // EXPLT0 through registers
  static constexpr size_t SLOT = (size_t)IT_NF * PST * sizeof(double);
  static constexpr size_t ESLOTS = EREG ? 0 : 2 * IT_ESLOT;
  static constexpr size_t SMEM = 4 * SLOT + ESLOTS + 6 * sizeof(uint64_t);
};
static_assert((ItGeo<true>::PST * 8) % 128 == 0 && ItGeo<true>::PST >= ItGeo<true>::PLANE &&
                  (ItGeo<true>::BXW * 8) % 16 == 0,
              "coupled TMA boxes: 128-byte aligned destinations, 16-byte rows");

template <bool TH, bool CPL>
__global__ void __launch_bounds__(IO_BX *IO_BY, 2)
k_io_rhs_tma(const __grid_constant__ IoMaps maps, TGDev d, IODev io, double gam, double roh, double alp, int cur,
             int nzc) {
  typedef ItGeo<CPL> G;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto slot = [&](int sl) { return reinterpret_cast<double *>(smem_raw + (size_t)sl * G::SLOT); };
  auto eslot = [&](int sl) { return reinterpret_cast<double *>(smem_raw + 4 * G::SLOT + (size_t)sl * IT_ESLOT); };
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + 4 * G::SLOT + G::ESLOTS);
  uint64_t *ebar = bar + 4;
  __shared__ double red[IO_BX * IO_BY / 32];
  __shared__ double ycoef[IO_BY][9];
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + IO_BX * ty;
  const int x0 = blockIdx.x * IO_BX, j0 = 1 + blockIdx.y * IO_BY;
  const int kbeg = blockIdx.z * nzc;
  const int kend = min(kbeg + nzc, nz);
  const int i = x0 + tx, j = j0 + ty;
  const bool active = (i < nx) && (j <= ny);
  const bool left_edge = (x0 == 0), right_edge = (x0 + IO_BX >= nx);
  const int right_col = nx - x0 + 2;  // smem column of x = nx (wraps to 0)
  const int nf = io.thermal ? 8 : 7;
  const uint32_t tx_bytes = (uint32_t)(nf * G::PLANE * sizeof(double));
  const CUtensorMap *mp[IT_NF] = {&maps.m[0], &maps.m[1], &maps.m[2], &maps.m[5 + 3 * cur], &maps.m[6 + 3 * cur],
                                  &maps.m[7 + 3 * cur], &maps.m[3], &maps.m[4]};
  const double *gsrc[IT_NF] = {d.u, d.v, d.w, io.g[cur][0], io.g[cur][1], io.g[cur][2], d.p, io.msum};
  if (tid == 0) {
    for (int q = 0; q < 6; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  if (tid < IO_BY * 9) {
    const int r = tid / 9, q = tid - 9 * r, jr = j0 + r;
    double v = 0.0;
    if (jr <= ny) {
      switch (q) {
        case 0: v = d.wff[jr]; break;
        case 1: v = d.wfb[jr]; break;
        case 2: v = d.wff[jr + 1]; break;
        case 3: v = d.wfb[jr + 1]; break;
        case 4: v = d.dyfi[jr]; break;
        case 5: v = d.dyci[jr]; break;
        case 6: v = d.dyci[jr + 1]; break;
        case 7: v = d.dyfi[jr - 1]; break;
        case 8: v = 1.0 / d.dyfi[jr]; break;
      }
    }
    ycoef[r][q] = v;
  }
  __syncthreads();
  auto slot_of = [&](int k) { return (k - kbeg + 1) & 3; };
  auto issue = [&](int k) {
    const int sl = slot_of(k);
    const int kz = k < 0 ? k + nz : (k >= nz ? k - nz : k);
    mbar_expect_tx(&bar[sl], tx_bytes);
#pragma unroll
    for (int f = 0; f < IT_NF; ++f)
      if (f < nf) tma_load_3d(slot(sl) + f * G::PST, mp[f], x0 - 2, j0 - 1, kz, &bar[sl]);
  };
  uint32_t par = 0;
  auto wait_plane = [&](int k) -> bool {
    const int sl = slot_of(k);
    const bool ok = mbar_wait(&bar[sl], (par >> sl) & 1u, d.err);
    par ^= 1u << sl;
    const int kz = k < 0 ? k + nz : (k >= nz ? k - nz : k);
    if (CPL) return ok;  // the coupled section's ghost columns came with the box
    if (left_edge && tid < 10 * IT_NF) {
      const int f = tid / 10, r = tid - f * 10, jr = j0 - 1 + r;
      if (f < nf && jr <= ny + 1) slot(sl)[f * IT_PST + r * IT_BXW + 1] = gsrc[f][(nx - 1) + d.sy * jr + d.sz * kz];
    }
    if (right_edge && tid >= 128 && tid < 128 + 10 * IT_NF) {
      const int q = tid - 128, f = q / 10, r = q - f * 10, jr = j0 - 1 + r;
      if (f < nf && jr <= ny + 1) slot(sl)[f * IT_PST + r * IT_BXW + right_col] = gsrc[f][d.sy * jr + d.sz * kz];
    }
    return ok;
  };
  // EXPLT0 of the tile's own cells, two-slot ring one plane ahead
  auto issue_e = [&](int k) {
    const int sl = (k - kbeg) & 1;
    mbar_expect_tx(&ebar[sl], (uint32_t)(3 * IT_EBOX * sizeof(double)));
#pragma unroll
    for (int q = 0; q < 3; ++q) tma_load_3d(eslot(sl) + q * IT_EBOX, &maps.m[11 + q], x0, j0, k, &ebar[sl]);
  };
  uint32_t epar = 0;
  if (tid == 0) {
    issue(kbeg - 1);
    issue(kbeg);
    issue(kbeg + 1);
    if (!G::EREG) issue_e(kbeg);
  }
  bool ok = wait_plane(kbeg - 1);
  ok = wait_plane(kbeg) && ok;
  double part = 0.0;
  const double dxi = d.dxi, dzi = d.dzi, cv = d.cvisc, dt = d.dt;
  const double *yc = ycoef[ty];
  const int xx = tx + G::XO, yy = ty + 1;
  constexpr bool th = TH;
  // EXPLT0 of the cell by plain loads (G::EREG), issued before the plane
  // waits so that their latency hides behind them (the stores of the plane's
  // results may alias them, so they could not move later)
  double e0r[3] = {0.0, 0.0, 0.0};
  for (int k = kbeg; k < kend; ++k) {
    if (G::EREG && active) {
      const int64_t ce = i + d.sy * j + d.sz * k;
#pragma unroll
      for (int q = 0; q < 3; ++q) e0r[q] = ((const double *)d.h0[q])[ce];
    }
    if (tid == 0) {
      fence_proxy_async();
      if (k + 2 <= kend) issue(k + 2);
      if (!G::EREG && k + 1 < kend) issue_e(k + 1);
    }
    ok = wait_plane(k + 1) && ok;
    if (!G::EREG) {
      const int esl = (k - kbeg) & 1;
      ok = mbar_wait(&ebar[esl], (epar >> esl) & 1u, d.err) && ok;
      epar ^= 1u << esl;
    }
    __syncthreads();
    const double *Es = eslot((k - kbeg) & 1);
    if (active && ok) {
      const double *Sm = slot(slot_of(k - 1));
      const double *Sc = slot(slot_of(k));
      const double *Sp = slot(slot_of(k + 1));
#define A(S, f, dx, dy) S[(f) * G::PST + (yy + (dy)) * G::BXW + xx + (dx)]
      const double wff = yc[0], wfb = yc[1], wffp = yc[2], wfbp = yc[3], dyfj = yc[4], dycj = yc[5], dycp = yc[6];
      // cell-centred 0.5 (mu0 + mu), M = mu0 + mu
      auto muc = [&](const double *S, int dx, int dy) { return th ? 0.5 * A(S, F_M, dx, dy) : 1.0; };
      // MU_STG(.,.,.,1) at the cell (dx, dy) of plane S, row jj = j + dy
      auto s1 = [&](const double *S, int dx, int dy, double wf, double wb) {
        if (!th) return 1.0;
        const int jj = j + dy;
        if (jj == 1) return 0.5 * A(S, F_M, dx, dy - 1);
        if (jj == ny + 1) return 0.5 * A(S, F_M, dx, dy);
        return ((A(S, F_M, dx, dy) + A(S, F_M, dx - 1, dy)) * wf + (A(S, F_M, dx, dy - 1) + A(S, F_M, dx - 1, dy - 1)) * wb) *
               0.5 * 0.5;
      };
      // MU_STG(.,.,.,2) at the cell (dx) of plane S (its z-minus plane Sb)
      auto s2 = [&](const double *S, const double *Sb, int dx) {
        if (!th) return 1.0;
        return (A(S, F_M, dx, 0) + A(S, F_M, dx - 1, 0) + A(Sb, F_M, dx, 0) + A(Sb, F_M, dx - 1, 0)) * 0.5 * 0.5 * 0.5;
      };
      // MU_STG(.,.,.,3) at row jj = j + dy of plane S (z-minus plane Sb)
      auto s3 = [&](const double *S, const double *Sb, int dy, double wf, double wb) {
        if (!th) return 1.0;
        const int jj = j + dy;
        if (jj == 1) return 0.5 * A(S, F_M, 0, dy - 1);
        if (jj == ny + 1) return 0.5 * A(S, F_M, 0, dy);
        return ((A(Sb, F_M, 0, dy) + A(S, F_M, 0, dy)) * wf + (A(Sb, F_M, 0, dy - 1) + A(S, F_M, 0, dy - 1)) * wb) * 0.5 *
               0.5;
      };
      // DIVG_U_io at (dx, dy) of plane S (its z-plus plane Sn), row jj
      auto divu = [&](const double *S, const double *Sn, int dx, int dy, double dyf) {
        return ((A(S, F_U, dx + 1, dy) - A(S, F_U, dx, dy)) * dxi + (A(S, F_V, dx, dy + 1) - A(S, F_V, dx, dy)) * dyf +
                (A(Sn, F_W, dx, dy) - A(S, F_W, dx, dy)) * dzi) * (1.0 / 3.0);
      };
      const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
      const int64_t oxm = CPL ? -1 : (i == 0 ? nx - 1 : i - 1) - i, ozm = d.sz * ((k == 0 ? nz - 1 : k - 1) - k);
      const double p0 = A(Sc, F_P, 0, 0);
      const double divc = divu(Sc, Sp, 0, 0, dyfj);
      // EXPLT0 of the cell: the staged box, or (coupled) a plain load
      auto e0of = [&](int q) { return G::EREG ? e0r[q] : Es[q * IT_EBOX + tid]; };
      // the coupled outlet ghost face keeps MU_STG = 1 (MU_Staggered covers IC <= NCL1_io)
      const bool xout = CPL && i == nx - 1;
      // ---------------- x (the coupled inlet face, NXI = 2, keeps its value: k_np_gbound)
      if (!CPL || i > 0) {
        const double u0 = A(Sc, F_U, 0, 0);
        double h11f = (A(Sc, F_GX, 1, 0) + A(Sc, F_GX, 0, 0)) * (A(Sc, F_U, 1, 0) + u0);
        double h11b = (A(Sc, F_GX, 0, 0) + A(Sc, F_GX, -1, 0)) * (u0 + A(Sc, F_U, -1, 0));
        double h11 = (h11f - h11b) * (dxi * 0.5 * 0.5);
        double h12f = (A(Sc, F_GY, 0, 1) + A(Sc, F_GY, -1, 1)) * (wffp * A(Sc, F_U, 0, 1) + wfbp * u0);
        double h12b = (A(Sc, F_GY, 0, 0) + A(Sc, F_GY, -1, 0)) * (wff * u0 + wfb * A(Sc, F_U, 0, -1));
        double h12 = (h12f - h12b) * (dyfj * 0.5);
        double h13f = (A(Sp, F_GZ, 0, 0) + A(Sp, F_GZ, -1, 0)) * (A(Sp, F_U, 0, 0) + u0);
        double h13b = (A(Sc, F_GZ, 0, 0) + A(Sc, F_GZ, -1, 0)) * (u0 + A(Sm, F_U, 0, 0));
        double h13 = (h13f - h13b) * (dzi * 0.5 * 0.5);
        double ex = -(h11 + h12 + h13);
        double dudx = (A(Sc, F_U, 1, 0) - u0) * dxi;
        const double tau11f = muc(Sc, 0, 0) * (dudx - divc);
        dudx = (u0 - A(Sc, F_U, -1, 0)) * dxi;
        const double tau11b = muc(Sc, -1, 0) * (dudx - divu(Sc, Sp, -1, 0, dyfj));
        const double d11 = (tau11f - tau11b) * (2.0 * dxi * cv);
        double dudy = (A(Sc, F_U, 0, 1) - u0) * dycp;
        double dvdx = (A(Sc, F_V, 0, 1) - A(Sc, F_V, -1, 1)) * dxi;
        const double tau12f = s1(Sc, 0, 1, wffp, wfbp) * (dudy + dvdx);
        dudy = (u0 - A(Sc, F_U, 0, -1)) * dycj;
        dvdx = (A(Sc, F_V, 0, 0) - A(Sc, F_V, -1, 0)) * dxi;
        const double tau12b = s1(Sc, 0, 0, wff, wfb) * (dudy + dvdx);
        const double d12 = (tau12f - tau12b) * (dyfj * cv);
        double dudz = (A(Sp, F_U, 0, 0) - u0) * dzi;
        double dwdx = (A(Sp, F_W, 0, 0) - A(Sp, F_W, -1, 0)) * dxi;
        const double tau13f = s2(Sp, Sc, 0) * (dudz + dwdx);
        dudz = (u0 - A(Sm, F_U, 0, 0)) * dzi;
        dwdx = (A(Sc, F_W, 0, 0) - A(Sc, F_W, -1, 0)) * dxi;
        const double tau13b = s2(Sc, Sm, 0) * (dudz + dwdx);
        const double d13 = (tau13f - tau13b) * (dzi * cv);
        ex = ex + d11 + d12 + d13;
        double r = (gam * ex + roh * e0of(0)) * dt;
        ((double *)d.h0[0])[c] = ex;
        r -= (p0 - A(Sc, F_P, -1, 0)) * (alp * dt * dxi);
        if (io.gravdir == 1) {
          const double rs = th ? (io.D[c] + io.D[c + oxm] + io.D0[c] + io.D0[c + oxm]) * 0.5 * 0.5 : 1.0;
          r += rs * (alp * dt * io.f_a);
        }
        part += r * yc[8];  // RHS_x / DYFI
        io.g[1 - cur][0][c] = A(Sc, F_GX, 0, 0) + r;
      }
      // ---------------- y (rows 2..ny)
      if (j >= 2) {
        const double v0 = A(Sc, F_V, 0, 0);
        double h21f = (wff * A(Sc, F_GX, 1, 0) + wfb * A(Sc, F_GX, 1, -1)) * (A(Sc, F_V, 1, 0) + v0);
        double h21b = (wff * A(Sc, F_GX, 0, 0) + wfb * A(Sc, F_GX, 0, -1)) * (v0 + A(Sc, F_V, -1, 0));
        double h21 = (h21f - h21b) * (dxi * 0.5);
        double h22f = (A(Sc, F_GY, 0, 1) + A(Sc, F_GY, 0, 0)) * (A(Sc, F_V, 0, 1) + v0);
        double h22b = (A(Sc, F_GY, 0, 0) + A(Sc, F_GY, 0, -1)) * (v0 + A(Sc, F_V, 0, -1));
        double h22 = (h22f - h22b) * (dycj * 0.5 * 0.5);
        double h23f = (wff * A(Sp, F_GZ, 0, 0) + wfb * A(Sp, F_GZ, 0, -1)) * (A(Sp, F_V, 0, 0) + v0);
        double h23b = (wff * A(Sc, F_GZ, 0, 0) + wfb * A(Sc, F_GZ, 0, -1)) * (v0 + A(Sm, F_V, 0, 0));
        double h23 = (h23f - h23b) * (dzi * 0.5);
        double ey = -(h21 + h22 + h23);
        double dvdy = (A(Sc, F_V, 0, 1) - v0) * dyfj;
        const double tau22f = muc(Sc, 0, 0) * (dvdy - divc);
        dvdy = (v0 - A(Sc, F_V, 0, -1)) * yc[7];
        const double tau22b = muc(Sc, 0, -1) * (dvdy - divu(Sc, Sp, 0, -1, yc[7]));
        const double d22 = (tau22f - tau22b) * (2.0 * dycj * cv);
        double dvdx = (A(Sc, F_V, 1, 0) - v0) * dxi;
        double dudy = (A(Sc, F_U, 1, 0) - A(Sc, F_U, 1, -1)) * dycj;
        const double tau21f = (xout ? 1.0 : s1(Sc, 1, 0, wff, wfb)) * (dvdx + dudy);
        dvdx = (v0 - A(Sc, F_V, -1, 0)) * dxi;
        dudy = (A(Sc, F_U, 0, 0) - A(Sc, F_U, 0, -1)) * dycj;
        const double tau21b = s1(Sc, 0, 0, wff, wfb) * (dvdx + dudy);
        const double d21 = (tau21f - tau21b) * (dxi * cv);
        double dvdz = (A(Sp, F_V, 0, 0) - v0) * dzi;
        double dwdy = (A(Sp, F_W, 0, 0) - A(Sp, F_W, 0, -1)) * dycj;
        const double tau23f = s3(Sp, Sc, 0, wff, wfb) * (dvdz + dwdy);
        dvdz = (v0 - A(Sm, F_V, 0, 0)) * dzi;
        dwdy = (A(Sc, F_W, 0, 0) - A(Sc, F_W, 0, -1)) * dycj;
        const double tau23b = s3(Sc, Sm, 0, wff, wfb) * (dvdz + dwdy);
        const double d23 = (tau23f - tau23b) * (dzi * cv);
        ey = ey + d21 + d22 + d23;
        double r = (gam * ey + roh * e0of(1)) * dt;
        ((double *)d.h0[1])[c] = ey;
        r -= (p0 - A(Sc, F_P, 0, -1)) * (alp * dt * dycj);
        if (io.gravdir == 2) {
          const double rs = th ? (wff * (io.D[c] + io.D0[c]) + wfb * (io.D[c - sy] + io.D0[c - sy])) * 0.5 : 1.0;
          r += rs * (alp * dt * io.f_a);
        }
        io.g[1 - cur][1][c] = A(Sc, F_GY, 0, 0) + r;
      }
      // ---------------- z
      {
        const double w0 = A(Sc, F_W, 0, 0);
        double h31f = (A(Sc, F_GX, 1, 0) + A(Sm, F_GX, 1, 0)) * (A(Sc, F_W, 1, 0) + w0);
        double h31b = (A(Sc, F_GX, 0, 0) + A(Sm, F_GX, 0, 0)) * (w0 + A(Sc, F_W, -1, 0));
        double h31 = (h31f - h31b) * (dxi * 0.5 * 0.5);
        double h32f = (A(Sc, F_GY, 0, 1) + A(Sm, F_GY, 0, 1)) * (wffp * A(Sc, F_W, 0, 1) + wfbp * w0);
        double h32b = (A(Sc, F_GY, 0, 0) + A(Sm, F_GY, 0, 0)) * (wff * w0 + wfb * A(Sc, F_W, 0, -1));
        double h32 = (h32f - h32b) * (dyfj * 0.5);
        double h33f = (A(Sp, F_GZ, 0, 0) + A(Sc, F_GZ, 0, 0)) * (A(Sp, F_W, 0, 0) + w0);
        double h33b = (A(Sc, F_GZ, 0, 0) + A(Sm, F_GZ, 0, 0)) * (w0 + A(Sm, F_W, 0, 0));
        double h33 = (h33f - h33b) * (dzi * 0.5 * 0.5);
        double ez = -(h31 + h32 + h33);
        double dwdz = (A(Sp, F_W, 0, 0) - w0) * dzi;
        const double tau33f = muc(Sc, 0, 0) * (dwdz - divc);
        dwdz = (w0 - A(Sm, F_W, 0, 0)) * dzi;
        const double tau33b = muc(Sm, 0, 0) * (dwdz - divu(Sm, Sc, 0, 0, dyfj));
        const double d33 = (tau33f - tau33b) * (2.0 * dzi * cv);
        double dwdx = (A(Sc, F_W, 1, 0) - w0) * dxi;
        double dudz = (A(Sc, F_U, 1, 0) - A(Sm, F_U, 1, 0)) * dzi;
        const double tau31f = (xout ? 1.0 : s2(Sc, Sm, 1)) * (dwdx + dudz);
        dwdx = (w0 - A(Sc, F_W, -1, 0)) * dxi;
        dudz = (A(Sc, F_U, 0, 0) - A(Sm, F_U, 0, 0)) * dzi;
        const double tau31b = s2(Sc, Sm, 0) * (dwdx + dudz);
        const double d31 = (tau31f - tau31b) * (dxi * cv);
        double dwdy = (A(Sc, F_W, 0, 1) - w0) * dycp;
        double dvdz = (A(Sc, F_V, 0, 1) - A(Sm, F_V, 0, 1)) * dzi;
        const double tau32f = s3(Sc, Sm, 1, wffp, wfbp) * (dwdy + dvdz);
        dwdy = (w0 - A(Sc, F_W, 0, -1)) * dycj;
        dvdz = (A(Sc, F_V, 0, 0) - A(Sm, F_V, 0, 0)) * dzi;
        const double tau32b = s3(Sc, Sm, 0, wff, wfb) * (dwdy + dvdz);
        const double d32 = (tau32f - tau32b) * (dyfj * cv);
        ez = ez + d31 + d32 + d33;
        double r = (gam * ez + roh * e0of(2)) * dt;
        ((double *)d.h0[2])[c] = ez;
        r -= (p0 - A(Sm, F_P, 0, 0)) * (alp * dt * dzi);
        if (io.gravdir == 3) {
          const double rs = th ? (io.D[c] + io.D[c + ozm] + io.D0[c] + io.D0[c + ozm]) * 0.5 * 0.5 : 1.0;
          r += rs * (alp * dt * io.f_a);
        }
        io.g[1 - cur][2][c] = A(Sc, F_GZ, 0, 0) + r;
      }
#undef A
    }
    __syncthreads();
  }
  // every issued plane has been waited for, so no bulk copy is in flight at exit
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((tid & 31) == 0) red[tid >> 5] = part;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int q = 0; q < IO_BX * IO_BY / 32; ++q) s += red[q];
    io.part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
  }
}

// DPGRNS (src/RHS_MOM_EXPLICIT_io.f90:200-240): constant mass flux from the
// block partials in a fixed order, or the constant pressure gradient.
__global__ void __launch_bounds__(1024) k_io_dpgrns(TGDev d, IODev io, double alp, int npart) {
  __shared__ double sh[32];
  if (io.flowdrvtp != 1) {
    if (threadIdx.x == 0) *io.dpg = io.flowdrvtp == 2 ? -0.5 * io.cfgv * alp * d.dt : 0.0;
    return;
  }
  double s = 0.0;
  for (int t = threadIdx.x; t < npart; t += blockDim.x) s += io.part[t];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < 32; ++q) r += sh[q];
    *io.dpg = r / d.volm;
  }
}

// PRCALC_io and MASSFLUX_UPDATE_IO on g[buf], with the deferred DPGRNS on
// G_x when use_dpg; pressure ghosts by copy (BC_WALL_PR).
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_corr(TGDev d, IODev io, double alp, int buf, int use_dpg,
                                                        double be) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
  const int64_t oxm = xminus(d, i), ozm = d.sz * (wrapm(k, d.nz) - k);
  double *gx = io.g[buf][0], *gy = io.g[buf][1], *gz = io.g[buf][2];
  const double phi = d.phi[c];
  double gxv = gx[c];
  if (use_dpg) gxv -= *io.dpg;
  // the coupled section corrects the x flux from NXI = 2 to NXE = NCL1_io + 1:
  // the inlet face keeps its value, the outlet face takes the ghost
  // DPH_io(NCL1_io + 1), which no routine writes (zero)
  if (!d.xnp || i > 0) gx[c] = gxv - (phi - d.phi[c + oxm]) * (d.dt * alp * d.dxi);
  if (d.xnp && i == nx - 1) gx[c + 1] -= (0.0 - phi) * (d.dt * alp * d.dxi);
  gz[c] -= (phi - d.phi[c + ozm]) * (d.dt * alp * d.dzi);
  if (j >= 2) gy[c] -= (phi - d.phi[c - sy]) * (d.dt * alp * d.dyci[j]);
  // semi-implicit PRCALC_io (src/PRESSURE_CORRECTION.f90:100-110) with the
  // physical Poisson right-hand side; be = 0 for the explicit scheme
  const double pn = be != 0.0 ? d.p[c] + phi - be * d.rhsphi[c] : d.p[c] + phi;
  d.p[c] = pn;
  if (j == 1) d.p[c - sy] = pn;
  if (j == ny) d.p[c + sy] = pn;
}

// ---------------------------------------------------------------- reductions
// what 0: max|div G + DrhoDtP| (DIVGCK_io); 1: sum of f / DYFI (bulk values);
// 2: max CFL of G plus the explicit viscous limit (CFL_io + CFL_VISCOUS,
// src/CFL.f90:42-133).
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_red_part(TGDev d, IODev io, int what, int cur, const double *f) {
  __shared__ double sh[IO_BX * IO_BY / 32];
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  double v = 0.0;
  if (i < nx && j <= ny) {
    const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
    if (what == 0) {
      const int64_t oxp = xplus(d, i), ozp = d.sz * (wrapp(k, d.nz) - k);
      const double *gx = io.g[cur][0], *gy = io.g[cur][1], *gz = io.g[cur][2];
      const double dv = (gx[c + oxp] - gx[c]) * d.dxi + (gy[c + sy] - gy[c]) * d.dyfi[j] +
                        (gz[c + ozp] - gz[c]) * d.dzi + io.drho[c];
      v = fabs(dv);
      if (dv != dv) v = __longlong_as_double(0x7ff0000000000000ll);
    } else if (what == 2) {
      const int64_t oxp = xplus(d, i), ozp = d.sz * (wrapp(k, d.nz) - k);
      const double *gx = io.g[cur][0], *gy = io.g[cur][1], *gz = io.g[cur][2];
      v = (fabs((gx[c] + gx[c + oxp]) * d.dxi) + fabs((gy[c] + gy[c + sy]) * d.dyfi[j]) +
           fabs((gz[c] + gz[c + ozp]) * d.dzi)) * 0.5;
      if (!io.visc) v = v + 2.0 * d.cvisc * (d.dxqi + d.dzqi + d.dyfi[j] * d.dyfi[j]);  // zero when implicit
    } else {
      v = f[c] / d.dyfi[j];
    }
  }
  const bool mx = what != 1;
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, v, o);
    v = mx ? fmax(v, x) : v + x;
  }
  const int tid = threadIdx.x + IO_BX * threadIdx.y;
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int q = 0; q < IO_BX * IO_BY / 32; ++q) s = mx ? fmax(s, sh[q]) : s + sh[q];
    d.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
  }
}

__global__ void __launch_bounds__(1024) k_io_red_final(TGDev d, int what, int npart) {
  __shared__ double sh[32];
  const bool mx = what != 1;
  double s = 0.0;
  for (int t = threadIdx.x; t < npart; t += blockDim.x) s = mx ? fmax(s, d.partials[t]) : s + d.partials[t];
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, s, o);
    s = mx ? fmax(s, x) : s + x;
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < 32; ++q) r = mx ? fmax(r, sh[q]) : r + sh[q];
    d.scal[1] = r;
  }
}

__global__ void k_fill(double *p, size_t n, double v) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) p[t] = v;
}

inline dim3 cell_grid(const TGDev &d) { return dim3((d.nx + IO_BX - 1) / IO_BX, (d.ny + IO_BY - 1) / IO_BY, d.nz); }

}  // namespace

int fill_value(chapsim_ctx *c, double *p, size_t n, double v) {
  k_fill<<<148 * 8, 256, 0, c->stream>>>(p, n, v);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_thermal_bc(chapsim_ctx *c) {
  TGDev &d = c->d;
  k_io_eng_ghost<<<dim3((d.nx * d.nz + 127) / 128, 2), 128, 0, c->stream>>>(d, c->io);
  LAUNCHED();
  return CHAPSIM_OK;
}

// The learned-property kernels take more than 48 KB of dynamic shared memory
// (set once per context) and run persistently, three (energy substep, with
// the derivative tile) or four CTAs of 128 threads per SM; each CTA holds 128
// of the SM's 512 tensor-memory columns.
int mlp_kernel_setup(chapsim_ctx *c) {
  if (c->mlp_smem_set) return CHAPSIM_OK;
  const void *fns[] = {(const void *)k_io_eng_props_mlp, (const void *)k_io_therm_props};
  const size_t bytes[] = {chapsim_mlp::kSmemDBytes, chapsim_mlp::kSmemBytes};
  for (int q = 0; q < 2; ++q)
    if (cudaFuncSetAttribute(fns[q], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes[q]) != cudaSuccess) {
      cudaGetLastError();
      c->err = "learned properties: cannot raise the shared-memory limit";
      return CHAPSIM_ERR_CUDA;
    }
  c->mlp_smem_set = true;
  return CHAPSIM_OK;
}

int mlp_grid(const chapsim_ctx *c, int per_sm) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int64_t tiles = (c->d.sz * c->d.nz + chapsim_mlp::TILE - 1) / chapsim_mlp::TILE;
  return (int)std::min<int64_t>(tiles, (int64_t)nsm * per_sm);
}

int io_np_eng_bc(chapsim_ctx *c, int ns);
int io_np_mom(chapsim_ctx *c, int ns, bool mass_parts);

// Phase-timer slots of an IO substep, in execution order: 0 energy RHS,
// 1 property update + wall ghosts, 2 prep (DrhoDtP, u = G / rho), 3 momentum
// RHS + DPGRNS, 4-8 the Poisson transforms and y-solve, 9 correction.
int io_eng(chapsim_ctx *c, int ns) {
  TGDev &d = c->d;
  const SubParams &sp = c->sp[ns];
  phase_mark(c, 0);
  k_io_eng_rhs<<<cell_grid(d), dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io, sp.gam * d.dt, sp.roh * d.dt, c->io_cur);
  LAUNCHED();
  dim3 g2((d.nx + IO_BX - 1) / IO_BX, (d.ny + 2 + IO_BY - 1) / IO_BY, d.nz);
  phase_mark(c, 1);
  if (c->props_mode == CHAPSIM_PROPS_MLP) {
    int rc = mlp_kernel_setup(c);
    if (rc) return rc;
    k_io_eng_props_mlp<<<mlp_grid(c, 3), chapsim_mlp::TILE, chapsim_mlp::kSmemDBytes, c->stream>>>(d, c->io, c->mlp);
  } else {
    k_io_eng_props<<<g2, dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io);
  }
  LAUNCHED();
  if (c->xnp) {
    const int rc = io_np_eng_bc(c, ns);
    if (rc) return rc;
  }
  return io_thermal_bc(c);
}

int io_therm_props(chapsim_ctx *c, int mode) {
  int rc = mlp_kernel_setup(c);
  if (rc) return rc;
  const bool mlp = mode == CHAPSIM_PROPS_MLP;
  k_io_therm_props<<<mlp_grid(c, 4), chapsim_mlp::TILE, mlp ? chapsim_mlp::kSmemBytes : 0, c->stream>>>(
      c->d, c->io, c->mlp, mlp ? 1 : 0);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_mom(chapsim_ctx *c, int ns, bool prep) {
  TGDev &d = c->d;
  IODev &io = c->io;
  const SubParams &sp = c->sp[ns];
  const int cur = c->io_cur, nxt = 1 - cur;
  const dim3 grid = cell_grid(d), blk(IO_BX, IO_BY);
  if (!io.thermal) {
    phase_mark(c, 0);
    phase_mark(c, 1);
  }
  phase_mark(c, 2);
  if (prep) {
    if (io.visc)
      k_io_prep<true><<<grid, blk, 0, c->stream>>>(d, io, sp.gam + sp.roh, sp.roh, sp.gam - 2.0, cur, io.thermal, 0);
    else
      k_io_prep<false><<<grid, blk, 0, c->stream>>>(d, io, sp.gam + sp.roh, sp.roh, sp.gam - 2.0, cur, io.thermal,
                                                     c->xnp ? 1 : 0);
    LAUNCHED();
  }
  phase_mark(c, 3);
  if (c->xnp) return io_np_mom(c, ns, prep);
  int npart = (int)(grid.x * grid.y * grid.z);
  if (io.visc) {
    // semi-implicit scheme: RHS_io of the three components, DPGRNS, factored
    // solves into G*
    int rc = io_mom_si(c, ns, &npart);
    if (rc) return rc;
    k_io_dpgrns<<<1, 1024, 0, c->stream>>>(d, io, sp.alp, npart);
    LAUNCHED();
    if ((rc = io_factor_si(c, ns))) return rc;
    // the semi-implicit PRCALC_io reads RHSLLPHI
    rc = launch_pois_io(c, ns, io.g[nxt][0], io.g[nxt][1], io.g[nxt][2], io.thermal ? io.drho : nullptr, true);
    if (rc) return rc;
    phase_mark(c, CHAPSIM_PH_CORR);
    k_io_corr<<<grid, blk, 0, c->stream>>>(d, io, sp.alp, nxt, 0, 0.5 * sp.alp * d.dt * d.cvisc);
    LAUNCHED();
    c->io_cur = nxt;
    if (c->timing) {
      phase_mark(c, CHAPSIM_PH_COUNT);
      if (++c->ev_pending == chapsim_ctx::kEvSub) return flush_phase_events(c);
    }
    return CHAPSIM_OK;
  }
  if (c->use_tma_io) {
    IoMaps maps;
    memcpy(maps.m, c->io_maps, sizeof(maps.m));
    dim3 g2(grid.x, grid.y, (d.nz + c->io_nzc - 1) / c->io_nzc);
    constexpr size_t sm = ItGeo<false>::SMEM;
    if (io.thermal)
      k_io_rhs_tma<true, false><<<g2, blk, sm, c->stream>>>(maps, d, io, sp.gam, sp.roh, sp.alp, cur, c->io_nzc);
    else
      k_io_rhs_tma<false, false><<<g2, blk, sm, c->stream>>>(maps, d, io, sp.gam, sp.roh, sp.alp, cur, c->io_nzc);
    npart = (int)(g2.x * g2.y * g2.z);
  } else {
    k_io_rhs<<<grid, blk, 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, cur);
  }
  LAUNCHED();
  k_io_dpgrns<<<1, 1024, 0, c->stream>>>(d, io, sp.alp, npart);
  LAUNCHED();
  // the explicit PRCALC_io does not read RHSLLPHI: the transform skips storing it
  int rc = launch_pois_io(c, ns, io.g[nxt][0], io.g[nxt][1], io.g[nxt][2], io.thermal ? io.drho : nullptr, false);
  if (rc) return rc;
  phase_mark(c, CHAPSIM_PH_CORR);
  k_io_corr<<<grid, blk, 0, c->stream>>>(d, io, sp.alp, nxt, 1, 0.0);
  LAUNCHED();
  c->io_cur = nxt;
  if (c->timing) {
    phase_mark(c, CHAPSIM_PH_COUNT);
    if (++c->ev_pending == chapsim_ctx::kEvSub) return flush_phase_events(c);
  }
  return CHAPSIM_OK;
}

int io_init_maps(chapsim_ctx *c) {
  TGDev &d = c->d;
  c->use_tma_io = false;
  if (d.nx < IT_BXW || d.ny < 8) return CHAPSIM_OK;  // small grids use k_io_rhs
  const bool cpl = c->xnp != 0;  // the coupled layout: maps from the inlet ghost column
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&encode, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !encode) {
    cudaGetLastError();
    return CHAPSIM_OK;
  }
  IODev &io = c->io;
  const int xo = c->xoff;
  void *f[14] = {d.u - xo,        d.v - xo,        d.w - xo,        d.p - xo,        io.msum - xo,
                 io.g[0][0] - xo, io.g[0][1] - xo, io.g[0][2] - xo, io.g[1][0] - xo, io.g[1][1] - xo,
                 io.g[1][2] - xo, (double *)d.h0[0] - xo, (double *)d.h0[1] - xo, (double *)d.h0[2] - xo};
  cuuint64_t dims[3] = {(cuuint64_t)(d.nx + 2 * xo), (cuuint64_t)(d.ny + 2), (cuuint64_t)d.nz};
  cuuint64_t strides[2] = {(cuuint64_t)d.sy * sizeof(double), (cuuint64_t)d.sz * sizeof(double)};
  cuuint32_t box[3] = {(cuuint32_t)(cpl ? ItGeo<true>::BXW : ItGeo<false>::BXW), IT_BYW, 1};
  cuuint32_t ebox[3] = {IO_BX, IO_BY, 1};
  cuuint32_t es[3] = {1, 1, 1};
  if ((d.sy * sizeof(double)) % 16 != 0) return CHAPSIM_OK;  // TMA strides must be multiples of 16 bytes
  for (int m = 0; m < 14; ++m) {
    CUresult r = encode(&c->io_maps[m], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, f[m], dims, strides, m >= 11 ? ebox : box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      c->err = "cuTensorMapEncodeTiled failed";
      return CHAPSIM_ERR_CUDA;
    }
  }
  int dev = 0, optin = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t smem = cpl ? ItGeo<true>::SMEM : ItGeo<false>::SMEM;
  const void *fns[2] = {cpl ? (const void *)k_io_rhs_tma<true, true> : (const void *)k_io_rhs_tma<true, false>,
                        cpl ? (const void *)k_io_rhs_tma<false, true> : (const void *)k_io_rhs_tma<false, false>};
  for (const void *fn : fns) {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, fn));
    if ((size_t)optin < smem + fa.sharedSizeBytes) return CHAPSIM_OK;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
  }
  c->use_tma_io = true;
  return CHAPSIM_OK;
}

int io_refresh_msum(chapsim_ctx *c) {
  k_io_msum<<<148 * 8, 256, 0, c->stream>>>(c->io, (size_t)c->d.sz * c->d.nz);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_restart_fields(chapsim_ctx *c) {
  TGDev &d = c->d;
  int rc;
  if (c->io.thermal && (rc = io_thermal_bc(c))) return rc;
  dim3 g2((d.nx + IO_BX - 1) / IO_BX, (d.ny + 2 + IO_BY - 1) / IO_BY, d.nz);
  k_io_props_only<<<g2, dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io);
  LAUNCHED();
  k_io_prep<false><<<cell_grid(d), dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io, 0.0, 0.0, 1.0, c->io_cur, 0, 0);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_correction(chapsim_ctx *c, int ns) {
  // MASSFLUX_UPDATE_IO + PRCALC_io on the current G (no DPGRNS)
  const double be = c->io.visc ? 0.5 * c->sp[ns].alp * c->d.dt * c->d.cvisc : 0.0;
  k_io_corr<<<cell_grid(c->d), dim3(IO_BX, IO_BY), 0, c->stream>>>(c->d, c->io, c->sp[ns].alp, c->io_cur, 0, be);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_reduce(chapsim_ctx *c, int what, double *host_out) {
  TGDev &d = c->d;
  const dim3 grid = cell_grid(d), blk(IO_BX, IO_BY);
  const int npart = (int)(grid.x * grid.y * grid.z);
  const double *f = nullptr;
  int kind = 1;
  switch (what) {
    case CHAPSIM_R_DIVMAX: kind = 0; break;
    case CHAPSIM_R_CFL: kind = 2; break;
    case CHAPSIM_R_BULK: f = d.u; break;
    case CHAPSIM_R_BULK_G: f = c->io.g[c->io_cur][0]; break;
    case CHAPSIM_R_BULK_H: f = c->io.h; break;
    default: return CHAPSIM_ERR_ARG;
  }
  k_io_red_part<<<grid, blk, 0, c->stream>>>(d, c->io, kind, c->io_cur, f);
  LAUNCHED();
  k_io_red_final<<<1, 1024, 0, c->stream>>>(d, kind, npart);
  LAUNCHED();
  double v = 0.0;
  CK(cudaMemcpyAsync(&v, d.scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (kind == 1) v = v / d.dzi / (c->area_inlet * (double)d.nx);  // BULK_*_IO normalisation
  *host_out = v;
  return CHAPSIM_OK;
}


// ---------------------------------------------------------------- coupled inflow/outflow planes
// Ghost planes i = 0 and i = NCL1_io + 1 of the coupled IO section, each
// (nz, ny + 2) at [k * (ny + 2) + j]; the last interior column i = NCL1_io is
// the context's x index nx - 1.
namespace {

__device__ __forceinline__ double *bplane(const IODev &io, int q) { return io.bcp + (int64_t)q * io.bps; }

// BC_TINLET_FLOW + BC_TINLET_THERML (src/BC_INLET.f90:2-76), j = 0 .. ny+1
__global__ void k_bc_inlet(TGDev d, IODev io, const double *__restrict__ tu, const double *__restrict__ tv,
                           const double *__restrict__ tw, const double *__restrict__ tp, int nxt, int64_t tsy,
                           int64_t tsz, int cur) {
  const int ny = d.ny;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (ny + 2) * d.nz) return;
  const int k = t / (ny + 2), j = t - k * (ny + 2);
  const int64_t tl = (nxt - 1) + tsy * j + tsz * k, tf = tsy * j + tsz * k;
  const int64_t c0 = d.sy * j + d.sz * k;  // the first IO cell
  const double rin = 1.0;                   // DENSITY(0, J, K), BC_TINLET_THERML
  bplane(io, CHAPSIM_P_IN_RHO)[t] = rin;
  const double ul = tu[tl], uf = tu[tf], vl = tv[tl], wl = tw[tl];
  bplane(io, CHAPSIM_P_IN_U)[t] = ul;
  d.u[c0] = uf;
  bplane(io, CHAPSIM_P_IN_GX)[t] = ul * rin;
  io.g[cur][0][c0] = uf * (rin + io.D[c0]) * 0.5;  // * XND2CL
  bplane(io, CHAPSIM_P_IN_V)[t] = vl;
  bplane(io, CHAPSIM_P_IN_GY)[t] = vl * rin;
  bplane(io, CHAPSIM_P_IN_W)[t] = wl;
  bplane(io, CHAPSIM_P_IN_GZ)[t] = wl * rin;
  bplane(io, CHAPSIM_P_IN_P)[t] = tp[tl];
}

// CONVCTION_OUTLET_U (src/BC_COUTLET_MOM_RK3.f90:101-174): (max + min) / 2 of
// the outlet-face mean 0.5 (u(NCL1) + u(NCL1 + 1)) over j = 1..ny; one block.
__global__ void __launch_bounds__(1024) k_bc_umax(TGDev d, IODev io, int slot) {
  __shared__ double smx[32], smn[32];
  const int nx = d.nx, ny = d.ny;
  const double *uo = bplane(io, CHAPSIM_P_OUT_U);
  double mx = -1.0e20, mn = 1.0e20;
#pragma unroll 8
  for (int t = threadIdx.x; t < ny * d.nz; t += blockDim.x) {
    const int k = t / ny, j = t - k * ny + 1;
    const double ucc = (d.u[(nx - 1) + d.sy * j + d.sz * k] + uo[j + (ny + 2) * k]) * 0.5;
    mx = fmax(mx, ucc);
    mn = fmin(mn, ucc);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) {
    smx[threadIdx.x >> 5] = mx;
    smn[threadIdx.x >> 5] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      mx = fmax(mx, smx[q]);
      mn = fmin(mn, smn[q]);
    }
    io.bcs[slot] = 0.5 * (mx + mn);
  }
}

// BC_COUTLET_MOM_RK3, the convective update (:22-44), j = 1..ny (2..ny for v)
__global__ void k_bc_outlet_conv(TGDev d, IODev io, double gam, double roh, int cur) {
  const int nx = d.nx, ny = d.ny;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ny * d.nz) return;
  const int k = t / ny, j = t - k * ny + 1;
  const int64_t pc = j + (int64_t)(ny + 2) * k, c = (nx - 1) + d.sy * j + d.sz * k;
  const double coe1 = d.dxi * io.bcs[0];
  const double rho = (io.D[c] + bplane(io, CHAPSIM_P_OUT_RHO)[pc]) * 0.5;  // * XND2CL
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q == 1 && j == 1) continue;
    double *go = bplane(io, CHAPSIM_P_OUT_GX + q), *c0 = bplane(io, CHAPSIM_P_CONV0_X + q);
    const double conv = -(go[pc] - io.g[cur][q][c]) * coe1;
    const double rhs = gam * conv + roh * c0[pc];
    c0[pc] = conv;
    const double gn = go[pc] + d.dt * rhs;
    go[pc] = gn;
    bplane(io, CHAPSIM_P_OUT_U + q)[pc] = gn / rho;
  }
}

// CHK_MassConsv_io (src/processing/CHK_conservation.f90:2-71): inflow and
// outflow from the planes (fixed-order block sums), the mass rate from the
// grid reduction of DrhoDtP / DYFI in d.scal[1]; one block.
__global__ void __launch_bounds__(1024) k_bc_mass(TGDev d, IODev io, int cur) {
  __shared__ double sa[32], sb[32];
  const int ny = d.ny;
  const double *go = bplane(io, CHAPSIM_P_OUT_GX);
  double fin = 0.0, fout = 0.0;
#pragma unroll 8
  for (int t = threadIdx.x; t < ny * d.nz; t += blockDim.x) {
    const int k = t / ny, j = t - k * ny + 1;
    const double coe2 = 1.0 / d.dyfi[j];
    fin += io.g[cur][0][d.sy * j + d.sz * k] * coe2;
    fout += go[j + (int64_t)(ny + 2) * k] * coe2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    fin += __shfl_xor_sync(0xffffffffu, fin, o);
    fout += __shfl_xor_sync(0xffffffffu, fout, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = fin;
    sb[threadIdx.x >> 5] = fout;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      fin += sa[q];
      fout += sb[q];
    }
    fin /= d.dzi;
    fout /= d.dzi;
    const double mass = d.scal[1] / d.dzi / d.dxi;
    io.bcs[1] = (fin - mass) / fout;
    io.bcs[2] = fin - mass - fout;
    io.bcs[3] = fin;
    io.bcs[4] = fout;
    io.bcs[5] = mass;
  }
}

// BC_COUTLET_MOM_RK3 (:47-61): the outlet x-flux rescaled, then
// BC_WALL_G_io / BC_WALL_Q_io on the plane (src/BC_WALL.f90:233-256, 412-460)
__global__ void k_bc_outlet_scale(TGDev d, IODev io) {
  const int nx = d.nx, ny = d.ny;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (ny + 2) * d.nz) return;
  const int k = t / (ny + 2), j = t - k * (ny + 2);
  double *gx = bplane(io, CHAPSIM_P_OUT_GX), *gy = bplane(io, CHAPSIM_P_OUT_GY), *gz = bplane(io, CHAPSIM_P_OUT_GZ);
  double *u = bplane(io, CHAPSIM_P_OUT_U), *v = bplane(io, CHAPSIM_P_OUT_V), *w = bplane(io, CHAPSIM_P_OUT_W);
  if (j >= 1 && j <= ny) {
    const double s = io.bcs[1];
    const int64_t c = (nx - 1) + d.sy * j + d.sz * k;
    double g = gx[t];
    g = g * (s - 1.0) + g;
    gx[t] = g;
    u[t] = g / ((io.D[c] + bplane(io, CHAPSIM_P_OUT_RHO)[t]) * 0.5);
  }
  if (j == 0 || j == ny + 1) {
    gx[t] = 0.0; gy[t] = 0.0; gz[t] = 0.0;
    u[t] = 0.0; v[t] = 0.0; w[t] = 0.0;
  } else if (j == 1) {
    gy[t] = 0.0;
    v[t] = 0.0;
  }
}

// BC_COUTLET_ENEG_RK3 (src/BC_COUTLET_ENEG_RK3.f90:2-41): the convective
// update of rho h, then ENTHALPY_UPDATE, DENSITY_UPDATE, ENTHALPY_UPDATE and
// THERM_PROP_UPDATE of the outlet plane (the steps of k_io_eng_props without
// the old-value copies), j = 1..ny
__global__ void k_bc_outlet_eng(TGDev d, IODev io, double gam, double roh) {
  const int nx = d.nx, ny = d.ny;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ny * d.nz) return;
  const int k = t / ny, j = t - k * ny + 1;
  const int64_t pc = j + (int64_t)(ny + 2) * k, c = (nx - 1) + d.sy * j + d.sz * k;
  double *rh = bplane(io, CHAPSIM_P_OUT_RHOH), *c0 = bplane(io, CHAPSIM_P_CONV0_ENG);
  const double conv = -d.dxi * io.bcs[6] * (rh[pc] - io.rhoh[c]);
  const double rhs = gam * conv + roh * c0[pc];
  c0[pc] = conv;
  const double r = rh[pc] + d.dt * rhs;
  rh[pc] = r;
  double *dd = bplane(io, CHAPSIM_P_OUT_RHO);
  const double dold = dd[pc];
  int bad = 0;
  double h = r / dold, T, D = dold;
  if (look_ht(io, h, T) && look_td(io, T, D)) {
  } else {
    D = dold;
    ++bad;
  }
  h = r / D;
  bplane(io, CHAPSIM_P_OUT_H)[pc] = h;
  if (!(io.shortcuts && fabs(h) < 1.0e-10)) {
    double M, K, D2;
    if (look_ht(io, h, T) && look_tprops(io, T, D2, M, K)) {
      bplane(io, CHAPSIM_P_OUT_T)[pc] = T;
      bplane(io, CHAPSIM_P_OUT_MU)[pc] = M;
      bplane(io, CHAPSIM_P_OUT_K)[pc] = K;
      D = D2;
    } else {
      ++bad;
    }
  }
  dd[pc] = D;
  if (bad) atomicAdd(io.bad, (unsigned long long)bad);
}

// BC_WALL_ISOFLUX (src/BC_WALL.f90:522-627) on the outlet plane's ghost rows;
// blockIdx.y: 0 bottom, 1 top
__global__ void k_bc_outlet_eng_ghost(TGDev d, IODev io) {
  const int ny = d.ny;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.nz) return;
  const bool top = blockIdx.y == 1;
  const int64_t row = (int64_t)(ny + 2) * k;
  double *hh = bplane(io, CHAPSIM_P_OUT_H);
  double h;
  if (!top)
    h = 2.0 * hh[row + 1] - d.wff[2] * hh[row + 2] - d.wfb[2] * hh[row + 1];
  else
    h = 2.0 * hh[row + ny] - d.wff[ny] * hh[row + ny] - d.wfb[ny] * hh[row + ny - 1];
  const int64_t pc = row + (top ? ny + 1 : 0);
  hh[pc] = h;
  double T, D, M, K;
  if (!look_ht(io, h, T) || !look_tprops(io, T, D, M, K)) {
    atomicAdd(io.bad, 1ull);
    return;
  }
  bplane(io, CHAPSIM_P_OUT_RHO)[pc] = D;
  bplane(io, CHAPSIM_P_OUT_T)[pc] = T;
  bplane(io, CHAPSIM_P_OUT_MU)[pc] = M;
  bplane(io, CHAPSIM_P_OUT_K)[pc] = K;
  bplane(io, CHAPSIM_P_OUT_RHOH)[pc] = h * D;
}


// ---------------------------------------------------------------- coupled section (xnp)
// The coupled inflow / outflow section holds its x ghost columns in the
// fields (i = -1: IC = 0, i = nx: IC = NCL1_io + 1).  The boundary operators
// above work on planes: k_np_mom_pre / k_np_eng_pre copy the columns they
// read into the planes, k_np_mom_post / k_np_eng_post write their results
// back.  Every kernel runs one thread per (j, k), j = 0..ny+1.
__device__ __forceinline__ int64_t col(const TGDev &d, int i, int j, int k) {
  return (int64_t)i + d.sy * j + d.sz * k;
}

// Start of a coupled SOLVERRK3_MOM_IO (:15-21): G0_io = G_io happens by the
// buffer swap, except on the columns the boundary operators rewrite in
// place; their old G goes to the P_SAVE planes.  The outlet planes get u, v,
// w, G and rho of the outlet ghost column.
__global__ void k_np_mom_pre(TGDev d, IODev io, int cur) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int64_t ci = col(d, -1, j, k), c1 = col(d, 0, j, k), co = col(d, d.nx, j, k);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    bplane(io, P_SAVE_IN + q)[t] = io.g[cur][q][ci];
    bplane(io, P_SAVE_OUT + q)[t] = io.g[cur][q][co];
    bplane(io, CHAPSIM_P_OUT_GX + q)[t] = io.g[cur][q][co];
  }
  bplane(io, P_SAVE_FACE1)[t] = io.g[cur][0][c1];
  bplane(io, CHAPSIM_P_OUT_U)[t] = d.u[co];
  bplane(io, CHAPSIM_P_OUT_V)[t] = d.v[co];
  bplane(io, CHAPSIM_P_OUT_W)[t] = d.w[co];
  bplane(io, CHAPSIM_P_OUT_RHO)[t] = io.D[co];
}

// After BC_TINLET_FLOW and BC_COUTLET_MOM_RK3: the inlet planes into ghost
// column IC = 0 (u, v, w, G, p, rho; DPH_io(0) stays zero), the outlet
// planes into IC = NCL1_io + 1 (u, v, w, G).
__global__ void k_np_mom_post(TGDev d, IODev io, int cur) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int64_t ci = col(d, -1, j, k), co = col(d, d.nx, j, k);
  double *q3[3] = {d.u, d.v, d.w};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    q3[q][ci] = bplane(io, CHAPSIM_P_IN_U + q)[t];
    io.g[cur][q][ci] = bplane(io, CHAPSIM_P_IN_GX + q)[t];
    q3[q][co] = bplane(io, CHAPSIM_P_OUT_U + q)[t];
    io.g[cur][q][co] = bplane(io, CHAPSIM_P_OUT_GX + q)[t];
  }
  d.p[ci] = bplane(io, CHAPSIM_P_IN_P)[t];
  io.D[ci] = bplane(io, CHAPSIM_P_IN_RHO)[t];
}

// After the momentum RHS wrote G* into g[nxt]: the boundary columns the
// substep does not advance (the ghost columns and the inlet face) carry the
// boundary operators' G into G*, and g[cur], which becomes G0_io, gets back
// its values from the start of the substep.
__global__ void k_np_gbound(TGDev d, IODev io, int cur) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int nxt = 1 - cur;
  const int64_t ci = col(d, -1, j, k), c1 = col(d, 0, j, k), co = col(d, d.nx, j, k);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    io.g[nxt][q][ci] = io.g[cur][q][ci];
    io.g[nxt][q][co] = io.g[cur][q][co];
    io.g[cur][q][ci] = bplane(io, P_SAVE_IN + q)[t];
    io.g[cur][q][co] = bplane(io, P_SAVE_OUT + q)[t];
  }
  io.g[nxt][0][c1] = io.g[cur][0][c1];
  io.g[cur][0][c1] = bplane(io, P_SAVE_FACE1)[t];
}

// DIVG_io (src/DIVG.f90:60-150) of the coupled section: RHSLLPHI = (div G +
// DrhoDtP) / (dt alpha) on the interior, the outlet face from the ghost column.
__global__ void __launch_bounds__(IO_BX *IO_BY) k_np_divg(TGDev d, IODev io, int buf, double coe0) {
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= d.nx || j > d.ny) return;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k, ozp = d.sz * (wrapp(k, d.nz) - k);
  const double *gx = io.g[buf][0], *gy = io.g[buf][1], *gz = io.g[buf][2];
  const double dv = (gx[c + 1] - gx[c]) * d.dxi + (gy[c + sy] - gy[c]) * d.dyfi[j] + (gz[c + ozp] - gz[c]) * d.dzi;
  d.rhsphi[c] = (dv + (io.thermal ? io.drho[c] : 0.0)) * coe0;
}

// Coupled SOLVERRK3_ENG_IO after the interior property update: VISCOUSITY0 /
// DENSITY0 <- VISCOUSITY / DENSITY on both ghost columns (:13-16), then
// BC_TINLET_THERML (src/BC_INLET.f90:54-76: the reference state on IC = 0),
// and the outlet planes of BC_COUTLET_ENEG_RK3 from IC = NCL1_io + 1.
__global__ void k_np_eng_pre(TGDev d, IODev io) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int64_t ci = col(d, -1, j, k), co = col(d, d.nx, j, k);
  io.D0[ci] = io.D[ci];
  io.mu0[ci] = io.mu[ci];
  io.D0[co] = io.D[co];
  io.mu0[co] = io.mu[co];
  io.T[ci] = 1.0;
  io.kap[ci] = 1.0;
  io.D[ci] = 1.0;
  io.mu[ci] = 1.0;
  io.rhoh[ci] = 0.0;
  io.h[ci] = 0.0;
  io.msum[ci] = io.mu0[ci] + 1.0;
  bplane(io, CHAPSIM_P_OUT_U)[t] = d.u[co];
  bplane(io, CHAPSIM_P_OUT_RHO)[t] = io.D[co];
  bplane(io, CHAPSIM_P_OUT_RHOH)[t] = io.rhoh[co];
  bplane(io, CHAPSIM_P_OUT_H)[t] = io.h[co];
  bplane(io, CHAPSIM_P_OUT_T)[t] = io.T[co];
  bplane(io, CHAPSIM_P_OUT_MU)[t] = io.mu[co];
  bplane(io, CHAPSIM_P_OUT_K)[t] = io.kap[co];
}

// Restart of the coupled section: BC_TINLET_THERML's reference state on the
// inlet ghost column IC = 0 (src/BC_INLET.f90:54-76), with DENSITY0 and
// VISCOUSITY0 equal to it.
__global__ void k_np_restart_inlet(TGDev d, IODev io) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int64_t ci = col(d, -1, j, k);
  io.T[ci] = 1.0;
  io.kap[ci] = 1.0;
  io.D[ci] = 1.0;
  io.D0[ci] = 1.0;
  io.mu[ci] = 1.0;
  io.mu0[ci] = 1.0;
  io.msum[ci] = 2.0;
  io.h[ci] = 0.0;
  io.rhoh[ci] = 0.0;
}

// Restart of the coupled section: u, v, w of the outlet ghost column from its
// G and the outlet-face density 0.5 (rho(NCL1_io) + rho(NCL1_io + 1)), the
// relation BC_COUTLET_MOM_RK3 keeps between them; zero on the wall rows.  The
// reference leaves Q_io(NCL1_io + 1) at its allocation value here, which
// halves U_OUTLET in the first substep after a restart; this rebuilds it so
// that a restart continues the run.
__global__ void k_np_restart_outlet(TGDev d, IODev io, int cur) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int64_t co = col(d, d.nx, j, k), cl = col(d, d.nx - 1, j, k);
  double *q3[3] = {d.u, d.v, d.w};
  const bool wall = j == 0 || j == d.ny + 1;
  const double rho = (io.D[cl] + io.D[co]) * 0.5;
#pragma unroll
  for (int q = 0; q < 3; ++q) q3[q][co] = (wall || (q == 1 && j == 1)) ? 0.0 : io.g[cur][q][co] / rho;
}

__global__ void k_np_eng_post(TGDev d, IODev io) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (d.ny + 2) * d.nz) return;
  const int k = t / (d.ny + 2), j = t - k * (d.ny + 2);
  const int64_t co = col(d, d.nx, j, k);
  io.D[co] = bplane(io, CHAPSIM_P_OUT_RHO)[t];
  io.rhoh[co] = bplane(io, CHAPSIM_P_OUT_RHOH)[t];
  io.h[co] = bplane(io, CHAPSIM_P_OUT_H)[t];
  io.T[co] = bplane(io, CHAPSIM_P_OUT_T)[t];
  io.mu[co] = bplane(io, CHAPSIM_P_OUT_MU)[t];
  io.kap[co] = bplane(io, CHAPSIM_P_OUT_K)[t];
  io.msum[co] = io.mu0[co] + io.mu[co];
}
}  // namespace

int io_bc_inlet(chapsim_ctx *c, const chapsim_ctx *tg) {
  const TGDev &d = c->d, &t = tg->d;
  const int n = (d.ny + 2) * d.nz;
  k_bc_inlet<<<(n + 255) / 256, 256, 0, c->stream>>>(d, c->io, t.u, t.v, t.w, t.p, t.nx, t.sy, t.sz, c->io_cur);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_bc_outlet_mom(chapsim_ctx *c, int ns, bool mass_parts) {
  TGDev &d = c->d;
  const SubParams &sp = c->sp[ns];
  const int np = d.ny * d.nz, nall = (d.ny + 2) * d.nz;
  k_bc_umax<<<1, 1024, 0, c->stream>>>(d, c->io, 0);
  LAUNCHED();
  k_bc_outlet_conv<<<(np + 255) / 256, 256, 0, c->stream>>>(d, c->io, sp.gam, sp.roh, c->io_cur);
  LAUNCHED();
  // sum of DrhoDtP / DYFI over the interior into d.scal[1] (its block sums
  // already in d.partials when the substep's k_io_prep formed them)
  const dim3 grid = cell_grid(d), blk(IO_BX, IO_BY);
  if (!mass_parts) {
    k_io_red_part<<<grid, blk, 0, c->stream>>>(d, c->io, 1, c->io_cur, c->io.drho);
    LAUNCHED();
  }
  k_io_red_final<<<1, 1024, 0, c->stream>>>(d, 1, (int)(grid.x * grid.y * grid.z));
  LAUNCHED();
  k_bc_mass<<<1, 1024, 0, c->stream>>>(d, c->io, c->io_cur);
  LAUNCHED();
  k_bc_outlet_scale<<<(nall + 255) / 256, 256, 0, c->stream>>>(d, c->io);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_bc_outlet_eng(chapsim_ctx *c, int ns) {
  TGDev &d = c->d;
  const SubParams &sp = c->sp[ns];
  const int np = d.ny * d.nz;
  k_bc_umax<<<1, 1024, 0, c->stream>>>(d, c->io, 6);
  LAUNCHED();
  k_bc_outlet_eng<<<(np + 255) / 256, 256, 0, c->stream>>>(d, c->io, sp.gam, sp.roh);
  LAUNCHED();
  k_bc_outlet_eng_ghost<<<dim3((d.nz + 127) / 128, 2), 128, 0, c->stream>>>(d, c->io);
  LAUNCHED();
  return CHAPSIM_OK;
}


// Coupled SOLVERRK3_ENG_IO boundaries (:61-64) after the interior property
// update: ghost-column DENSITY0 / VISCOUSITY0, BC_TINLET_THERML, and
// BC_COUTLET_ENEG_RK3 on the outlet column.
int io_np_eng_bc(chapsim_ctx *c, int ns) {
  TGDev &d = c->d;
  const int nb = ((d.ny + 2) * d.nz + 255) / 256;
  k_np_eng_pre<<<nb, 256, 0, c->stream>>>(d, c->io);
  LAUNCHED();
  int rc = io_bc_outlet_eng(c, ns);
  if (rc) return rc;
  k_np_eng_post<<<nb, 256, 0, c->stream>>>(d, c->io);
  LAUNCHED();
  return CHAPSIM_OK;
}

// RESTART_INSTANT_VARS_IO of the coupled section (src/processing/RESTART_io.f90:
// 80-120 with TGFLOWFLG) once G, PR (and T, DENSITY, ENTHALPY, RHOH) of
// IC = 1 .. NCL1_io + 1 are in place: BC_WALL_THERMAL and THERM_PROP_UPDATE
// over those columns (rho0 = rho, mu0 = mu), BC_TINLET_THERML, BC_TINLET_FLOW
// from the TG context, the outlet column's velocity, then DENSITY_Staggered,
// MU_Staggered and VELOCITY_CALC_io on the interior.
int io_np_restart(chapsim_ctx *c) {
  TGDev &d = c->d;
  IODev &io = c->io;
  if (!c->inlet) {
    c->err = "coupled IO section without its TG inlet source (chapsim_io_set_inlet)";
    return CHAPSIM_ERR_STATE;
  }
  TGDev e = d;
  e.nx = d.nx + 1;  // IC = 1 .. NCL1_io + 1 from the field pointers
  if (io.thermal) {
    k_io_eng_ghost<<<dim3((e.nx * e.nz + 127) / 128, 2), 128, 0, c->stream>>>(e, io);
    LAUNCHED();
  }
  const dim3 blk(IO_BX, IO_BY), g2((e.nx + IO_BX - 1) / IO_BX, (d.ny + 2 + IO_BY - 1) / IO_BY, d.nz);
  k_io_props_only<<<g2, blk, 0, c->stream>>>(e, io);
  LAUNCHED();
  const int nb = ((d.ny + 2) * d.nz + 255) / 256, cur = c->io_cur;
  if (io.thermal) {
    k_np_restart_inlet<<<nb, 256, 0, c->stream>>>(d, io);
    LAUNCHED();
  }
  k_np_mom_pre<<<nb, 256, 0, c->stream>>>(d, io, cur);  // the outlet planes hold the outlet column
  LAUNCHED();
  int rc = io_bc_inlet(c, c->inlet);
  if (rc) return rc;
  k_np_mom_post<<<nb, 256, 0, c->stream>>>(d, io, cur);
  LAUNCHED();
  k_np_restart_outlet<<<nb, 256, 0, c->stream>>>(d, io, cur);
  LAUNCHED();
  k_io_prep<false><<<cell_grid(d), blk, 0, c->stream>>>(d, io, 0.0, 0.0, 1.0, cur, 0, 0);
  LAUNCHED();
  return CHAPSIM_OK;
}

int io_np_divg(chapsim_ctx *c, int ns, int buf) {
  TGDev &d = c->d;
  k_np_divg<<<cell_grid(d), dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io, buf, 1.0 / d.dt / c->sp[ns].alp);
  LAUNCHED();
  return CHAPSIM_OK;
}

// Coupled SOLVERRK3_MOM_IO(NS) after VELOCITY_CALC_io (src/SOLVERRK3_MOM_IO.f90:
// 15-168 with TGFLOWFLG): BC_TINLET_FLOW from the TG context and
// BC_COUTLET_MOM_RK3 on the ghost columns, the momentum RHS and
// MASSFLUX_CALC_IO from the second x face (no DPGRNS forcing, :218), DIVG_io
// into RHSLLPHI, FISHPACK_POIS3D_SIMPLE with the non-periodic x transform on
// the IO arrays (the coupled branch of :116-121 solves on the TG arrays; the
// IO-only branch's arrays are used), PRCALC_io and MASSFLUX_UPDATE_IO with
// the outlet face.
int io_np_mom(chapsim_ctx *c, int ns, bool mass_parts) {
  TGDev &d = c->d;
  IODev &io = c->io;
  if (!c->inlet) {
    c->err = "coupled IO section without its TG inlet source (chapsim_io_set_inlet)";
    return CHAPSIM_ERR_STATE;
  }
  const SubParams &sp = c->sp[ns];
  const int cur = c->io_cur, nxt = 1 - cur;
  const dim3 grid = cell_grid(d), blk(IO_BX, IO_BY);
  const int nb = ((d.ny + 2) * d.nz + 255) / 256;
  k_np_mom_pre<<<nb, 256, 0, c->stream>>>(d, io, cur);
  LAUNCHED();
  int rc = io_bc_inlet(c, c->inlet);
  if (rc) return rc;
  if ((rc = io_bc_outlet_mom(c, ns, mass_parts))) return rc;
  k_np_mom_post<<<nb, 256, 0, c->stream>>>(d, io, cur);
  LAUNCHED();
  if (c->use_tma_io) {
    IoMaps maps;
    memcpy(maps.m, c->io_maps, sizeof(maps.m));
    const dim3 g2(grid.x, grid.y, (d.nz + c->io_nzc - 1) / c->io_nzc);
    constexpr size_t sm = ItGeo<true>::SMEM;
    if (io.thermal)
      k_io_rhs_tma<true, true><<<g2, blk, sm, c->stream>>>(maps, d, io, sp.gam, sp.roh, sp.alp, cur, c->io_nzc);
    else
      k_io_rhs_tma<false, true><<<g2, blk, sm, c->stream>>>(maps, d, io, sp.gam, sp.roh, sp.alp, cur, c->io_nzc);
  } else {
    k_io_rhs<<<grid, blk, 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, cur);
  }
  LAUNCHED();
  k_np_gbound<<<nb, 256, 0, c->stream>>>(d, io, cur);
  LAUNCHED();
  phase_mark(c, CHAPSIM_PH_FFTX);
  if ((rc = io_np_divg(c, ns, nxt))) return rc;
  if ((rc = xnp_pois3d(c, true))) return rc;
  phase_mark(c, CHAPSIM_PH_CORR);
  k_io_corr<<<grid, blk, 0, c->stream>>>(d, io, sp.alp, nxt, 0, 0.0);
  LAUNCHED();
  c->io_cur = nxt;
  if (c->timing) {
    phase_mark(c, CHAPSIM_PH_COUNT);
    if (++c->ev_pending == chapsim_ctx::kEvSub) return flush_phase_events(c);
  }
  return CHAPSIM_OK;
}
}  // namespace chapsim
