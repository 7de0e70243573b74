// IO-domain kernels: one RK3 substep of the x-periodic inflow/outflow channel
// section with the explicit viscous scheme, variable density and viscosity,
// and the energy equation with table properties.
//
// Reference (CHAPSim1WW, paths relative to the project root), channel branch
// (RCCI1 = RCCI2 = RNDI1 = 1), x periodic (IPV_io/IMV_io wrap):
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
#include <math.h>

#include <string>

#include "chapsim_internal.cuh"

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
// rhoh += gam dt R + zeta dt R_old, limited to RHOHmax + REALMIN.
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_eng_rhs(TGDev d, IODev io, double cdt1, double cdt0, int cur) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
  const int64_t oxp = wrapp(i, nx) - i, oxm = wrapm(i, nx) - i;
  const int64_t ozp = d.sz * (wrapp(k, d.nz) - k), ozm = d.sz * (wrapm(k, d.nz) - k);
  const double *__restrict__ gx = io.g[cur][0], *__restrict__ gy = io.g[cur][1], *__restrict__ gz = io.g[cur][2];
  const double *__restrict__ hx = io.g[1 - cur][0], *__restrict__ hy = io.g[1 - cur][1],
               *__restrict__ hz = io.g[1 - cur][2];  // G0_io
  const double *__restrict__ H = io.h, *__restrict__ T = io.T, *__restrict__ K = io.kap;
  const double coe1 = d.dxi * 0.5 * 0.5, coe11 = d.dxqi * 0.5 * io.cthecd;
  const double coe2 = d.dyfi[j] * 0.5, coe3 = d.dzi * 0.5 * 0.5;
  const double coe33 = d.dzqi * 0.5 * io.cthecd, coe22 = d.dyfi[j] * io.cthecd;
  double coe221, coe222;
  if (j == 1) {
    coe221 = d.dyci[j + 1];
    coe222 = 1.0;
  } else if (j == ny) {
    coe222 = d.dyci[j];
    coe221 = 1.0;
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
  if (j == 1)
    kdty2 = -io.qw_bot * coe222;  // WALLFLUX(bottom) = +qw
  else if (j == ny)
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
  const double dold = io.D[c];
  io.mu0[c] = io.mu[c];
  io.D0[c] = dold;
  if (j < 1 || j > ny) return;
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
  if (!keep) {
    double M, K, D2;
    if (look_ht(io, h, T) && look_tprops(io, T, D2, M, K)) {
      io.T[c] = T;
      io.mu[c] = M;
      io.kap[c] = K;
      D = D2;
    } else {
      ++bad;
    }
  }
  io.D[c] = D;
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
  double h;
  if (!top)
    h = 2.0 * io.h[base + sy] - d.wff[2] * io.h[base + 2 * sy] - d.wfb[2] * io.h[base + sy];
  else
    h = 2.0 * io.h[base + sy * ny] - d.wff[ny] * io.h[base + sy * ny] - d.wfb[ny] * io.h[base + sy * (ny - 1)];
  io.h[c] = h;
  double T, D, M, K;
  if (!look_ht(io, h, T) || !look_tprops(io, T, D, M, K)) {
    atomicAdd(io.bad, 1ull);
    return;
  }
  io.D[c] = D;
  io.T[c] = T;
  io.mu[c] = M;
  io.kap[c] = K;
  io.rhoh[c] = h * D;
}

// ---------------------------------------------------------------- momentum
// DENSITY_TIME_DERIVATION (gamma - 2 divisor as written) and VELOCITY_CALC_io
// with its wall BC.  RHO_STG is formed from rho, rho0 (DENSITY_Staggered).
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_prep(TGDev d, IODev io, double gp, double zr, double den,
                                                        int cur, int do_drho) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
  const int64_t oxp = wrapp(i, nx) - i, oxm = wrapm(i, nx) - i;
  const int64_t ozp = d.sz * (wrapp(k, d.nz) - k), ozm = d.sz * (wrapm(k, d.nz) - k);
  const double *__restrict__ gx = io.g[cur][0], *__restrict__ gy = io.g[cur][1], *__restrict__ gz = io.g[cur][2];
  if (do_drho) {
    const double *__restrict__ hx = io.g[1 - cur][0], *__restrict__ hy = io.g[1 - cur][1],
                 *__restrict__ hz = io.g[1 - cur][2];
    const double divx = (gx[c + oxp] - gx[c]) * d.dxi, divx0 = (hx[c + oxp] - hx[c]) * d.dxi;
    const double divy = (gy[c + sy] - gy[c]) * d.dyfi[j], divy0 = (hy[c + sy] - hy[c]) * d.dyfi[j];
    const double divz = (gz[c + ozp] - gz[c]) * d.dzi, divz0 = (hz[c + ozp] - hz[c]) * d.dzi;
    io.drho[c] = (gp * (divx + divy + divz) + zr * (divx0 + divy0 + divz0)) / den;
  }
  double rx = 1.0, ry = 1.0, rz = 1.0;
  if (io.thermal) {
    const double *__restrict__ D = io.D, *__restrict__ D0 = io.D0;
    rx = (D[c] + D[c + oxm] + D0[c] + D0[c + oxm]) * 0.5 * 0.5;
    rz = (D[c] + D[c + ozm] + D0[c] + D0[c + ozm]) * 0.5 * 0.5;
    if (j >= 2) ry = (d.wff[j] * (D[c] + D0[c]) + d.wfb[j] * (D[c - sy] + D0[c - sy])) * 0.5;
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
    const int64_t oxp = wrapp(i, nx) - i, oxm = wrapm(i, nx) - i;
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
      const int64_t op = (ii + 1 == nx) ? -(int64_t)(nx - 1) : 1;
      const int64_t oz = (kk + 1 == d.nz) ? -(int64_t)d.sz * (d.nz - 1) : d.sz;
      return ((u[cc + op] - u[cc]) * dxi + (v[cc + sy] - v[cc]) * d.dyfi[jj] + (w[cc + oz] - w[cc]) * dzi) / 3.0;
    };
    const double divc = divu(c, i, j, k);
    // ---------------- x: CONVECTION_X_io + VISCOUS_ALL_EXPLT_X_io
    {
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
      const double tau21f = mv.s1(c + oxp, j, -oxp) * (dvdx + dudy);
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
      const double tau31f = mv.s2(c + oxp, -oxp, ozm) * (dwdx + dudz);
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

// PRCALC_io (explicit branch) and MASSFLUX_UPDATE_IO on g[buf], with the
// deferred DPGRNS on G_x when use_dpg; pressure ghosts by copy (BC_WALL_PR).
__global__ void __launch_bounds__(IO_BX *IO_BY) k_io_corr(TGDev d, IODev io, double alp, int buf, int use_dpg) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * IO_BX + threadIdx.x;
  const int j = blockIdx.y * IO_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy, c = i + sy * j + d.sz * k;
  const int64_t oxm = wrapm(i, nx) - i, ozm = d.sz * (wrapm(k, d.nz) - k);
  double *gx = io.g[buf][0], *gy = io.g[buf][1], *gz = io.g[buf][2];
  const double phi = d.phi[c];
  double gxv = gx[c];
  if (use_dpg) gxv -= *io.dpg;
  gx[c] = gxv - (phi - d.phi[c + oxm]) * (d.dt * alp * d.dxi);
  gz[c] -= (phi - d.phi[c + ozm]) * (d.dt * alp * d.dzi);
  if (j >= 2) gy[c] -= (phi - d.phi[c - sy]) * (d.dt * alp * d.dyci[j]);
  const double pn = d.p[c] + phi;
  d.p[c] = pn;
  if (j == 1) d.p[c - sy] = pn;
  if (j == ny) d.p[c + sy] = pn;
}

// ---------------------------------------------------------------- reductions
// what 0: max|div G + DrhoDtP| (DIVGCK_io); 1: sum of f / DYFI (bulk values).
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
      const int64_t oxp = wrapp(i, nx) - i, ozp = d.sz * (wrapp(k, d.nz) - k);
      const double *gx = io.g[cur][0], *gy = io.g[cur][1], *gz = io.g[cur][2];
      const double dv = (gx[c + oxp] - gx[c]) * d.dxi + (gy[c + sy] - gy[c]) * d.dyfi[j] +
                        (gz[c + ozp] - gz[c]) * d.dzi + io.drho[c];
      v = fabs(dv);
      if (dv != dv) v = __longlong_as_double(0x7ff0000000000000ll);
    } else {
      v = f[c] / d.dyfi[j];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, v, o);
    v = what == 0 ? fmax(v, x) : v + x;
  }
  const int tid = threadIdx.x + IO_BX * threadIdx.y;
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int q = 0; q < IO_BX * IO_BY / 32; ++q) s = what == 0 ? fmax(s, sh[q]) : s + sh[q];
    d.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
  }
}

__global__ void __launch_bounds__(1024) k_io_red_final(TGDev d, int what, int npart) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int t = threadIdx.x; t < npart; t += blockDim.x) s = what == 0 ? fmax(s, d.partials[t]) : s + d.partials[t];
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, s, o);
    s = what == 0 ? fmax(s, x) : s + x;
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < 32; ++q) r = what == 0 ? fmax(r, sh[q]) : r + sh[q];
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

int io_eng(chapsim_ctx *c, int ns) {
  TGDev &d = c->d;
  const SubParams &sp = c->sp[ns];
  k_io_eng_rhs<<<cell_grid(d), dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io, sp.gam * d.dt, sp.roh * d.dt, c->io_cur);
  LAUNCHED();
  dim3 g2((d.nx + IO_BX - 1) / IO_BX, (d.ny + 2 + IO_BY - 1) / IO_BY, d.nz);
  k_io_eng_props<<<g2, dim3(IO_BX, IO_BY), 0, c->stream>>>(d, c->io);
  LAUNCHED();
  return io_thermal_bc(c);
}

int io_mom(chapsim_ctx *c, int ns, bool prep) {
  TGDev &d = c->d;
  IODev &io = c->io;
  const SubParams &sp = c->sp[ns];
  const int cur = c->io_cur, nxt = 1 - cur;
  const dim3 grid = cell_grid(d), blk(IO_BX, IO_BY);
  if (prep) {
    k_io_prep<<<grid, blk, 0, c->stream>>>(d, io, sp.gam + sp.roh, sp.roh, sp.gam - 2.0, cur, io.thermal);
    LAUNCHED();
  }
  k_io_rhs<<<grid, blk, 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, cur);
  LAUNCHED();
  k_io_dpgrns<<<1, 1024, 0, c->stream>>>(d, io, sp.alp, (int)(grid.x * grid.y * grid.z));
  LAUNCHED();
  int rc = launch_pois_io(c, ns, io.g[nxt][0], io.g[nxt][1], io.g[nxt][2], io.thermal ? io.drho : nullptr);
  if (rc) return rc;
  k_io_corr<<<grid, blk, 0, c->stream>>>(d, io, sp.alp, nxt, 1);
  LAUNCHED();
  c->io_cur = nxt;
  return CHAPSIM_OK;
}

int io_correction(chapsim_ctx *c, int ns) {
  // MASSFLUX_UPDATE_IO + PRCALC_io on the current G (no DPGRNS)
  k_io_corr<<<cell_grid(c->d), dim3(IO_BX, IO_BY), 0, c->stream>>>(c->d, c->io, c->sp[ns].alp, c->io_cur, 0);
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

}  // namespace chapsim
