// Semi-implicit viscous scheme of the IO section (visthemflg = 1): the
// viscous terms split into an explicit part, a part treated by
// Crank-Nicolson factors and its density correction; then the factored
// variable-coefficient solves (1 - A_x)(1 - A_z)(1 - A_y) dG = RHS_io.
//
// Restates (paths relative to the CHAPSim1WW project root), channel branches:
//   VISCOUS_PAR_EXPLT_X/Y/Z_io  src/VISCOUS_X_EXPLICIT_io.f90:124-286,
//                           src/VISCOUS_Y_EXPLICIT_io.f90:264-424,
//                           src/VISCOUS_Z_EXPLICIT_io.f90:289-460
//   RHS_MOM_EXPLICIT_io     src/RHS_MOM_EXPLICIT_io.f90:79-95 (implicit branch)
//   MOMFA_io, MOMFA1_X_io, MOMFA2_Z_io, MOMFA3_Y_io  src/MOMFA_io.f90:17-377
//   TDMAIJI_CYC, TDMAIJJ_nonCYC  src/TDMAIJI_CYC.f90:67-157,
//                           src/TDMAIJJ_nonCYC.f90:67-123
//   DENSITY_implicit_add    src/MASSFLUX_CALC_IO.f90:316-399 (in k_io_prep)
//
// The three components' right-hand sides are formed by one kernel before any
// solve: VISCOUS_PAR_EXPLT_*_io and RHS_MOM_EXPLICIT_io of component c read
// Q_io, the convection terms (all formed first by the reference too), the
// pressure and G_io component c only, and MOMFA_io(c) changes G_io component
// c only, so the reference's interleaved order gives the same values.
//
// Line solves: one warp per line with the line in shared memory
// (warp_part_solve: chunked elimination, then parallel cyclic reduction of
// the chunk-end system over shuffles), staged by coalesced loads: x lines are
// rows, z and y lines come in tiles of consecutive x.  The coefficients are
// formed from VISCOUSITY and the MU_STG / RHO_STG fields k_si_stg forms once
// per substep (as MU_Staggered and DENSITY_Staggered do).  Nothing but the
// right-hand sides and the result crosses global memory.
#include <cuda_runtime.h>

#include <string>

#include "chapsim_internal.cuh"

#define LAUNCHED()                                                        \
  do {                                                                    \
    ++c->launches;                                                        \
    cudaError_t e_ = cudaGetLastError();                                  \
    if (e_ != cudaSuccess) {                                              \
      c->err = std::string("kernel launch: ") + cudaGetErrorString(e_);   \
      return CHAPSIM_ERR_CUDA;                                            \
    }                                                                     \
  } while (0)

namespace chapsim {
namespace {

constexpr int SI_BX = 32, SI_BY = 8;

__device__ __forceinline__ int wp(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int wm(int i, int n) { return i == 0 ? n - 1 : i - 1; }

// MU_Staggered and DENSITY_Staggered (src/MASSFLUX_CALC_IO.f90:147-311) at
// (i, j, k), periodic in i and k, formed from mu, mu0, rho, rho0.
struct StgForm {
  const double *__restrict__ mu;
  const double *__restrict__ mu0;
  const double *__restrict__ D;
  const double *__restrict__ D0;
  const double *__restrict__ wff;
  const double *__restrict__ wfb;
  int nx, ny, nz;
  int64_t sy, sz;
  __device__ __forceinline__ int64_t at(int i, int j, int k) const { return (int64_t)i + sy * j + sz * k; }
  // x-face / y-face edge; wall rows 1 and ny+1 from the ghost cells
  __device__ __forceinline__ double s1(int i, int j, int k) const {
    const int64_t c = at(i, j, k), m = at(wm(i, nx), j, k);
    if (j == 1) return 0.5 * (mu0[c - sy] + mu[c - sy]);
    if (j == ny + 1) return 0.5 * (mu0[c] + mu[c]);
    return ((mu[c] + mu[m] + mu0[c] + mu0[m]) * wff[j] + (mu[c - sy] + mu[m - sy] + mu0[c - sy] + mu0[m - sy]) * wfb[j]) *
           0.5 * 0.5;
  }
  // x-face / z-face edge
  __device__ __forceinline__ double s2(int i, int j, int k) const {
    const int im = wm(i, nx), km = wm(k, nz);
    const int64_t c = at(i, j, k), cx = at(im, j, k), cz = at(i, j, km), cxz = at(im, j, km);
    return (mu[c] + mu[cx] + mu0[c] + mu0[cx] + mu[cz] + mu[cxz] + mu0[cz] + mu0[cxz]) * 0.5 * 0.5 * 0.5;
  }
  // y-face / z-face edge; wall rows from the ghost cells
  __device__ __forceinline__ double s3(int i, int j, int k) const {
    const int64_t c = at(i, j, k), m = at(i, j, wm(k, nz));
    if (j == 1) return 0.5 * (mu0[c - sy] + mu[c - sy]);
    if (j == ny + 1) return 0.5 * (mu0[c] + mu[c]);
    return ((mu[m] + mu[c] + mu0[m] + mu0[c]) * wff[j] + (mu[m - sy] + mu[c - sy] + mu0[m - sy] + mu0[c - sy]) * wfb[j]) *
           0.5 * 0.5;
  }
  __device__ __forceinline__ double r1(int i, int j, int k) const {
    const int64_t c = at(i, j, k), m = at(wm(i, nx), j, k);
    return (D[c] + D[m] + D0[c] + D0[m]) * 0.5 * 0.5;
  }
  // v faces: row 0 keeps the allocation value 1 (never formed by
  // DENSITY_Staggered), rows 1 and ny+1 from the ghost cells
  __device__ __forceinline__ double r2(int i, int j, int k) const {
    if (j == 0) return 1.0;
    const int64_t c = at(i, j, k);
    if (j == 1) return 0.5 * (D0[c - sy] + D[c - sy]);
    if (j == ny + 1) return 0.5 * (D0[c] + D[c]);
    return (wff[j] * (D[c] + D0[c]) + wfb[j] * (D[c - sy] + D0[c - sy])) * 0.5;
  }
  __device__ __forceinline__ double r3(int i, int j, int k) const {
    const int64_t c = at(i, j, k), m = at(i, j, wm(k, nz));
    return (D[c] + D[m] + D0[c] + D0[m]) * 0.5 * 0.5;
  }
};

// MU_STG 1-3 and RHO_STG 1-3 of the substep into io.stg, once, for the
// right-hand sides and the factor solves: rows 0..ny+1 of the faces that
// have them (s1, s3: 1..ny+1; s2, r1, r3: 1..ny; r2: 0..ny+1).
__global__ void __launch_bounds__(SI_BX *SI_BY) k_si_stg(TGDev d, IODev io) {
  const int i = blockIdx.x * SI_BX + threadIdx.x;
  const int j = blockIdx.y * SI_BY + threadIdx.y;  // 0..ny+1
  const int k = blockIdx.z;
  if (i >= d.nx || j > d.ny + 1) return;
  const StgForm F{io.mu, io.mu0, io.D, io.D0, d.wff, d.wfb, d.nx, d.ny, d.nz, d.sy, d.sz};
  const int64_t c = F.at(i, j, k);
  if (j >= 1) {
    io.stg[0][c] = F.s1(i, j, k);
    io.stg[2][c] = F.s3(i, j, k);
  }
  if (j >= 1 && j <= d.ny) {
    io.stg[1][c] = F.s2(i, j, k);
    io.stg[3][c] = F.r1(i, j, k);
    io.stg[5][c] = F.r3(i, j, k);
  }
  io.stg[4][c] = F.r2(i, j, k);
}

// VISCOUSITY, MU_STG(1..3) and RHO_STG(1..3) at (i, j, k) from the fields
// k_si_stg formed; with the energy equation off all of them are 1.
struct Prop {
  const double *__restrict__ mu;
  const double *__restrict__ st1;
  const double *__restrict__ st2;
  const double *__restrict__ st3;
  const double *__restrict__ rs1;
  const double *__restrict__ rs2;
  const double *__restrict__ rs3;
  int nx, ny, nz, th;
  int64_t sy, sz;
  __device__ __forceinline__ int64_t at(int i, int j, int k) const { return (int64_t)i + sy * j + sz * k; }
  __device__ __forceinline__ double vis(int i, int j, int k) const { return th ? mu[at(i, j, k)] : 1.0; }
  __device__ __forceinline__ double s1(int i, int j, int k) const { return th ? st1[at(i, j, k)] : 1.0; }
  __device__ __forceinline__ double s2(int i, int j, int k) const { return th ? st2[at(i, j, k)] : 1.0; }
  __device__ __forceinline__ double s3(int i, int j, int k) const { return th ? st3[at(i, j, k)] : 1.0; }
  __device__ __forceinline__ double r1(int i, int j, int k) const { return th ? rs1[at(i, j, k)] : 1.0; }
  __device__ __forceinline__ double r2(int i, int j, int k) const { return th ? rs2[at(i, j, k)] : 1.0; }
  __device__ __forceinline__ double r3(int i, int j, int k) const { return th ? rs3[at(i, j, k)] : 1.0; }
};

__device__ __forceinline__ Prop make_prop(const TGDev &d, const IODev &io) {
  return Prop{io.mu, io.stg[0], io.stg[1], io.stg[2], io.stg[3], io.stg[4], io.stg[5],
              d.nx, d.ny, d.nz, io.thermal, d.sy, d.sz};
}

// Convection (CONVECTION_*_io), the split viscous terms (VISCOUS_PAR_EXPLT_*_io)
// and RHS_MOM_EXPLICIT_io's implicit branch for component C of one cell
// (one launch per component): RHS_io -> d.rhs[C], EXPLT0_io updated.  Per-block sums of RHS_x / DYFI
// feed DPGRNS.  Row 1 of the v right-hand side is zero (VISCOUS_PAR_EXPLT_Y_io
// clears RHS_io and nothing writes that row before MOMFA3_Y_io).
template <int C, bool TH>
__global__ void __launch_bounds__(SI_BX *SI_BY, 4) k_io_rhs_si(TGDev d, IODev io, double gam, double roh, double alp,
                                                          int cur) {
  __shared__ double red[SI_BX * SI_BY / 32];
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int i = blockIdx.x * SI_BX + threadIdx.x;
  const int j = blockIdx.y * SI_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  double part = 0.0;
  if (i < nx && j <= ny) {
    const int64_t sy = d.sy, sz = d.sz;
    const int ip = wp(i, nx), im = wm(i, nx), kp = wp(k, nz), km = wm(k, nz);
    Prop P = make_prop(d, io);
    P.th = TH;  // compile-time: the property loads and density parts fold away without the energy equation
    constexpr bool th = TH;
    const double *__restrict__ u = d.u, *__restrict__ v = d.v, *__restrict__ w = d.w, *__restrict__ p = d.p;
    const double *__restrict__ gx = io.g[cur][0], *__restrict__ gy = io.g[cur][1], *__restrict__ gz = io.g[cur][2];
    const double *__restrict__ r0 = io.drhoi[0], *__restrict__ r1 = io.drhoi[1], *__restrict__ r2 = io.drhoi[2];
    auto A = [&](const double *f, int ii, int jj, int kk) { return f[(int64_t)ii + sy * jj + sz * kk]; };
    // G_io * DRHOI_STG (and Q_io * DRHOI_STG where the reference writes it)
    auto AD = [&](const double *f, const double *r, int ii, int jj, int kk) {
      const int64_t q = (int64_t)ii + sy * jj + sz * kk;
      return f[q] * r[q];
    };
    const int64_t c = (int64_t)i + sy * j + sz * k;
    const double dxi = d.dxi, dzi = d.dzi, cv = d.cvisc, dt = d.dt, coe2a = alp * dt;
    const double dyfj = d.dyfi[j], dycj = d.dyci[j], dycp = d.dyci[j + 1];
    const double wff = d.wff[j], wfb = d.wfb[j], wffp = d.wff[j + 1], wfbp = d.wfb[j + 1];
    const int64_t oxp = ip - i, oxm = im - i, ozp = sz * (kp - k), ozm = sz * (km - k);
    // ------------------------------------------------ x
    if (C == 0) {
      const double h11 = ((gx[c + oxp] + gx[c]) * (u[c + oxp] + u[c]) - (gx[c] + gx[c + oxm]) * (u[c] + u[c + oxm])) *
                         (dxi * 0.5 * 0.5);
      const double h12 = ((gy[c + sy] + gy[c + sy + oxm]) * (wffp * u[c + sy] + wfbp * u[c]) -
                          (gy[c] + gy[c + oxm]) * (wff * u[c] + wfb * u[c - sy])) * (dyfj * 0.5);
      const double h13 = ((gz[c + ozp] + gz[c + ozp + oxm]) * (u[c + ozp] + u[c]) -
                          (gz[c] + gz[c + oxm]) * (u[c] + u[c + ozm])) * (dzi * 0.5 * 0.5);
      const double conv = -(h11 + h12 + h13);
      const double coe1 = -2.0 / 3.0 * dxi * cv, coe2 = dyfj * cv, coe32 = dzi * cv;
      const double muc = P.vis(i, j, k), mum = P.vis(im, j, k);
      double dudx = (A(u, ip, j, k) - A(u, i, j, k)) * dxi;
      double dvdy = (A(v, i, j + 1, k) - A(v, i, j, k)) * dyfj;
      double dwdz = (A(w, i, j, kp) - A(w, i, j, k)) * dzi;
      const double t11fe = muc * (dvdy + dwdz), t11fi = muc * dudx;
      const double t11fa = th ? muc * ((AD(gx, r0, ip, j, k) - AD(gx, r0, i, j, k)) * dxi) : 0.0;
      dudx = (A(u, i, j, k) - A(u, im, j, k)) * dxi;
      dvdy = (A(v, im, j + 1, k) - A(v, im, j, k)) * dyfj;
      dwdz = (A(w, im, j, kp) - A(w, im, j, k)) * dzi;
      const double t11be = mum * (dvdy + dwdz), t11bi = mum * dudx;
      const double t11ba = th ? mum * ((AD(gx, r0, i, j, k) - AD(gx, r0, im, j, k)) * dxi) : 0.0;
      const double d11e = (t11fe - t11be) * coe1, d11i = (t11fi - t11bi) * coe1 * (-2.0);
      const double d11a = (t11fa - t11ba) * coe1 * (-2.0);
      const double vis12p = P.s1(i, j + 1, k), vis12c = P.s1(i, j, k);
      double dvdx = (A(v, i, j + 1, k) - A(v, im, j + 1, k)) * dxi;
      double dudy = (A(u, i, j + 1, k) - A(u, i, j, k)) * dycp;
      const double t12fe = vis12p * dvdx, t12fi = vis12p * dudy;
      const double t12fa = th ? vis12p * ((AD(gx, r0, i, j + 1, k) - AD(gx, r0, i, j, k)) * dycp) : 0.0;
      dudy = (A(u, i, j, k) - A(u, i, j - 1, k)) * dycj;
      dvdx = (A(v, i, j, k) - A(v, im, j, k)) * dxi;
      const double t12be = vis12c * dvdx, t12bi = vis12c * dudy;
      const double t12ba = th ? vis12c * ((AD(gx, r0, i, j, k) - AD(gx, r0, i, j - 1, k)) * dycj) : 0.0;
      const double d12e = (t12fe - t12be) * coe2, d12i = (t12fi - t12bi) * coe2, d12a = (t12fa - t12ba) * coe2;
      const double vis13p = P.s2(i, j, kp), vis13c = P.s2(i, j, k);
      double dudz = (A(u, i, j, kp) - A(u, i, j, k)) * dzi;
      double dwdx = (A(w, i, j, kp) - A(w, im, j, kp)) * dxi;
      const double t13fe = vis13p * dwdx, t13fi = vis13p * dudz;
      // the density part of tau13 differences Q_io, as the reference writes it
      const double t13fa = th ? vis13p * ((AD(u, r0, i, j, kp) - AD(u, r0, i, j, k)) * dzi) : 0.0;
      dudz = (A(u, i, j, k) - A(u, i, j, km)) * dzi;
      dwdx = (A(w, i, j, k) - A(w, im, j, k)) * dxi;
      const double t13be = vis13c * dwdx, t13bi = vis13c * dudz;
      const double t13ba = th ? vis13c * ((AD(u, r0, i, j, k) - AD(u, r0, i, j, km)) * dzi) : 0.0;
      const double d13e = (t13fe - t13be) * coe32, d13i = (t13fi - t13bi) * coe32, d13a = (t13fa - t13ba) * coe32;
      const double explt = (d11e + d12e + d13e) + conv;
      const double imp = d11i + d12i + d13i, adv = d11a + d12a + d13a;
      double *e0 = (double *)d.h0[0];
      double r = (gam * explt + roh * e0[c]) * dt;
      r = r + coe2a * imp + 0.5 * coe2a * adv;
      e0[c] = explt;
      r -= (p[c] - p[c + oxm]) * (alp * dt * dxi);
      if (io.gravdir == 1) r += P.r1(i, j, k) * (alp * dt * io.f_a);
      part = r / dyfj;
      ((double *)d.rhs[0])[c] = r;
    }
    // ------------------------------------------------ y (rows 2..ny)
    if (C == 1 && j >= 2) {
      const double h21 = ((wff * gx[c + oxp] + wfb * gx[c + oxp - sy]) * (v[c + oxp] + v[c]) -
                          (wff * gx[c] + wfb * gx[c - sy]) * (v[c] + v[c + oxm])) * (dxi * 0.5);
      const double h22 = ((gy[c + sy] + gy[c]) * (v[c + sy] + v[c]) - (gy[c] + gy[c - sy]) * (v[c] + v[c - sy])) *
                         (dycj * 0.5 * 0.5);
      const double h23 = ((wff * gz[c + ozp] + wfb * gz[c + ozp - sy]) * (v[c + ozp] + v[c]) -
                          (wff * gz[c] + wfb * gz[c - sy]) * (v[c] + v[c + ozm])) * (dzi * 0.5);
      const double conv = -(h21 + h22 + h23);
      const double coe1 = dxi * cv, coe3 = dzi * cv, coe2 = -2.0 / 3.0 * dycj * cv;
      const double muc = P.vis(i, j, k), mub = P.vis(i, j - 1, k);
      double dudx = (A(u, ip, j, k) - A(u, i, j, k)) * dxi;
      double dvdy = (A(v, i, j + 1, k) - A(v, i, j, k)) * dyfj;
      double dwdz = (A(w, i, j, kp) - A(w, i, j, k)) * dzi;
      const double t22fe = muc * (dudx + dwdz), t22fi = muc * dvdy;
      const double t22fa = th ? muc * ((AD(gy, r1, i, j + 1, k) - AD(gy, r1, i, j, k)) * dyfj) : 0.0;
      dudx = (A(u, ip, j - 1, k) - A(u, i, j - 1, k)) * dxi;
      dvdy = (A(v, i, j, k) - A(v, i, j - 1, k)) * d.dyfi[j - 1];
      dwdz = (A(w, i, j - 1, kp) - A(w, i, j - 1, k)) * dzi;
      const double t22be = mub * (dudx + dwdz), t22bi = mub * dvdy;
      const double t22ba = th ? mub * ((AD(gy, r1, i, j, k) - AD(gy, r1, i, j - 1, k)) * d.dyfi[j - 1]) : 0.0;
      const double d22e = (t22fe - t22be) * coe2, d22i = (t22fi - t22bi) * coe2 * (-2.0);
      const double d22a = (t22fa - t22ba) * coe2 * (-2.0);
      const double vis21p = P.s1(ip, j, k), vis21c = P.s1(i, j, k);
      double dvdx = (A(v, ip, j, k) - A(v, i, j, k)) * dxi;
      double dudy = (A(u, ip, j, k) - A(u, ip, j - 1, k)) * dycj;
      const double t21fe = vis21p * dudy, t21fi = vis21p * dvdx;
      const double t21fa = th ? vis21p * ((AD(gy, r1, ip, j, k) - AD(gy, r1, i, j, k)) * dxi) : 0.0;
      dvdx = (A(v, i, j, k) - A(v, im, j, k)) * dxi;
      dudy = (A(u, i, j, k) - A(u, i, j - 1, k)) * dycj;
      const double t21be = vis21c * dudy, t21bi = vis21c * dvdx;
      const double t21ba = th ? vis21c * ((AD(gy, r1, i, j, k) - AD(gy, r1, im, j, k)) * dxi) : 0.0;
      const double d21e = (t21fe - t21be) * coe1, d21i = (t21fi - t21bi) * coe1, d21a = (t21fa - t21ba) * coe1;
      const double vis23p = P.s3(i, j, kp), vis23c = P.s3(i, j, k);
      double dvdz = (A(v, i, j, kp) - A(v, i, j, k)) * dzi;
      double dwdy = (A(w, i, j, kp) - A(w, i, j - 1, kp)) * dycj;
      const double t23fe = vis23p * dwdy, t23fi = vis23p * dvdz;
      const double t23fa = th ? vis23p * ((AD(gy, r1, i, j, kp) - AD(gy, r1, i, j, k)) * dzi) : 0.0;
      dvdz = (A(v, i, j, k) - A(v, i, j, km)) * dzi;
      dwdy = (A(w, i, j, k) - A(w, i, j - 1, k)) * dycj;
      const double t23be = vis23c * dwdy, t23bi = vis23c * dvdz;
      const double t23ba = th ? vis23c * ((AD(gy, r1, i, j, k) - AD(gy, r1, i, j, km)) * dzi) : 0.0;
      const double d23e = (t23fe - t23be) * coe3, d23i = (t23fi - t23bi) * coe3, d23a = (t23fa - t23ba) * coe3;
      const double explt = (d21e + d22e + d23e) + conv;
      const double imp = d21i + d22i + d23i, adv = d21a + d22a + d23a;
      double *e0 = (double *)d.h0[1];
      double r = (gam * explt + roh * e0[c]) * dt;
      r = r + coe2a * imp + 0.5 * coe2a * adv;
      e0[c] = explt;
      r -= (p[c] - p[c - sy]) * (alp * dt * dycj);
      if (io.gravdir == 2) r += P.r2(i, j, k) * (alp * dt * io.f_a);
      ((double *)d.rhs[1])[c] = r;
    } else if (C == 1) {
      ((double *)d.rhs[1])[c] = 0.0;
    }
    // ------------------------------------------------ z
    if (C == 2) {
      const double h31 = ((gx[c + oxp] + gx[c + oxp + ozm]) * (w[c + oxp] + w[c]) -
                          (gx[c] + gx[c + ozm]) * (w[c] + w[c + oxm])) * (dxi * 0.5 * 0.5);
      const double h32 = ((gy[c + sy] + gy[c + sy + ozm]) * (wffp * w[c + sy] + wfbp * w[c]) -
                          (gy[c] + gy[c + ozm]) * (wff * w[c] + wfb * w[c - sy])) * (dyfj * 0.5);
      const double h33 = ((gz[c + ozp] + gz[c]) * (w[c + ozp] + w[c]) - (gz[c] + gz[c + ozm]) * (w[c] + w[c + ozm])) *
                         (dzi * 0.5 * 0.5);
      const double conv = -(h31 + h32 + h33);
      const double coe1 = dxi * cv, coe3 = -2.0 / 3.0 * dzi * cv, coe2 = dyfj * cv;
      const double muc = P.vis(i, j, k), mub = P.vis(i, j, km);
      double dudx = (A(u, ip, j, k) - A(u, i, j, k)) * dxi;
      double dvdy = (A(v, i, j + 1, k) - A(v, i, j, k)) * dyfj;
      double dwdz = (A(w, i, j, kp) - A(w, i, j, k)) * dzi;
      const double t33fe = muc * (dudx + dvdy), t33fi = muc * dwdz;
      const double t33fa = th ? muc * ((AD(gz, r2, i, j, kp) - AD(gz, r2, i, j, k)) * dzi) : 0.0;
      dudx = (A(u, ip, j, km) - A(u, i, j, km)) * dxi;
      dvdy = (A(v, i, j + 1, km) - A(v, i, j, km)) * dyfj;
      dwdz = (A(w, i, j, k) - A(w, i, j, km)) * dzi;
      const double t33be = mub * (dudx + dvdy), t33bi = mub * dwdz;
      const double t33ba = th ? mub * ((AD(gz, r2, i, j, k) - AD(gz, r2, i, j, km)) * dzi) : 0.0;
      const double d33e = (t33fe - t33be) * coe3, d33i = (t33fi - t33bi) * coe3 * (-2.0);
      const double d33a = (t33fa - t33ba) * coe3 * (-2.0);
      const double vis31p = P.s2(ip, j, k), vis31c = P.s2(i, j, k);
      double dwdx = (A(w, ip, j, k) - A(w, i, j, k)) * dxi;
      double dudz = (A(u, ip, j, k) - A(u, ip, j, km)) * dzi;
      const double t31fe = vis31p * dudz, t31fi = vis31p * dwdx;
      const double t31fa = th ? vis31p * ((AD(gz, r2, ip, j, k) - AD(gz, r2, i, j, k)) * dxi) : 0.0;
      dwdx = (A(w, i, j, k) - A(w, im, j, k)) * dxi;
      dudz = (A(u, i, j, k) - A(u, i, j, km)) * dzi;
      const double t31be = vis31c * dudz, t31bi = vis31c * dwdx;
      const double t31ba = th ? vis31c * ((AD(gz, r2, i, j, k) - AD(gz, r2, im, j, k)) * dxi) : 0.0;
      const double d31e = (t31fe - t31be) * coe1, d31i = (t31fi - t31bi) * coe1, d31a = (t31fa - t31ba) * coe1;
      const double vis32p = P.s3(i, j + 1, k), vis32c = P.s3(i, j, k);
      double dwdy = (A(w, i, j + 1, k) - A(w, i, j, k)) * dycp;
      double dvdz = (A(v, i, j + 1, k) - A(v, i, j + 1, km)) * dzi;
      const double t32fe = vis32p * dvdz, t32fi = vis32p * dwdy;
      const double t32fa = th ? vis32p * ((AD(gz, r2, i, j + 1, k) - AD(gz, r2, i, j, k)) * dycp) : 0.0;
      dwdy = (A(w, i, j, k) - A(w, i, j - 1, k)) * dycj;
      dvdz = (A(v, i, j, k) - A(v, i, j, km)) * dzi;
      const double t32be = vis32c * dvdz, t32bi = vis32c * dwdy;
      const double t32ba = th ? vis32c * ((AD(gz, r2, i, j, k) - AD(gz, r2, i, j - 1, k)) * dycj) : 0.0;
      const double d32e = (t32fe - t32be) * coe2, d32i = (t32fi - t32bi) * coe2, d32a = (t32fa - t32ba) * coe2;
      const double explt = (d31e + d32e + d33e) + conv;
      const double imp = d31i + d32i + d33i, adv = d31a + d32a + d33a;
      double *e0 = (double *)d.h0[2];
      double r = (gam * explt + roh * e0[c]) * dt;
      r = r + coe2a * imp + 0.5 * coe2a * adv;
      e0[c] = explt;
      r -= (p[c] - p[c + ozm]) * (alp * dt * dzi);
      if (io.gravdir == 3) r += P.r3(i, j, k) * (alp * dt * io.f_a);
      ((double *)d.rhs[2])[c] = r;
    }
  }
  if (C == 0) {
    // fixed-order block sum of RHS_x / DYFI
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    const int tid = threadIdx.x + SI_BX * threadIdx.y;
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int q = 0; q < SI_BX * SI_BY / 32; ++q) s += red[q];
      io.part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
    }
  }
}

// MOMFA1_X_io / MOMFA2_Z_io coefficients at (i, j, k) of component C along
// axis X (true: x, false: z): a x(-1) + b x(0) + c x(+1).
template <int C, bool X>
__device__ __forceinline__ void cyc_coef(const Prop &P, int i, int j, int k, double coe1, double coe2, double &a,
                                         double &b, double &cc) {
  const int im = wm(i, P.nx), ip = wp(i, P.nx), km = wm(k, P.nz), kp = wp(k, P.nz);
  double amu, apu, rm, rp, rc;
  if (X) {
    if (C == 0) {
      amu = -coe1 * P.vis(im, j, k); apu = -coe1 * P.vis(i, j, k);
      rm = P.r1(im, j, k); rp = P.r1(ip, j, k); rc = P.r1(i, j, k);
    } else if (C == 1) {
      amu = -coe2 * P.s1(i, j, k); apu = -coe2 * P.s1(ip, j, k);
      rm = P.r2(im, j, k); rp = P.r2(ip, j, k); rc = P.r2(i, j, k);
    } else {
      amu = -coe2 * P.s2(i, j, k); apu = -coe2 * P.s2(ip, j, k);
      rm = P.r3(im, j, k); rp = P.r3(ip, j, k); rc = P.r3(i, j, k);
    }
  } else {
    if (C == 0) {
      amu = -coe2 * P.s2(i, j, k); apu = -coe2 * P.s2(i, j, kp);
      rm = P.r1(i, j, km); rp = P.r1(i, j, kp); rc = P.r1(i, j, k);
    } else if (C == 1) {
      amu = -coe2 * P.s3(i, j, k); apu = -coe2 * P.s3(i, j, kp);
      rm = P.r2(i, j, km); rp = P.r2(i, j, kp); rc = P.r2(i, j, k);
    } else {
      amu = -coe1 * P.vis(i, j, km); apu = -coe1 * P.vis(i, j, k);
      rm = P.r3(i, j, km); rp = P.r3(i, j, kp); rc = P.r3(i, j, k);
    }
  }
  a = amu / rm;
  cc = apu / rp;
  b = 1.0 - (amu + apu) / rc;
}

// MOMFA3_Y_io coefficients of row j (1..ny), component C.
template <int C>
__device__ __forceinline__ void y_coef(const TGDev &d, const IODev &io, const Prop &P, int i, int j, int k,
                                       double facoe, double &a, double &b, double &cc) {
  const int ny = d.ny;
  double amu, apu, den;
  if (C != 1) {
    // u (C = 0) with MU_STG(1), RHO_STG(1); w (C = 2) with MU_STG(3), RHO_STG(3)
    auto fmu = [&](int jj) { return C == 0 ? P.s1(i, jj, k) : P.s3(i, jj, k); };
    auto fden = [&](int jj) { return C == 0 ? P.r1(i, jj, k) : P.r3(i, jj, k); };
    if (j == 1) {
      const double muqt = (P.vis(i, 1, k) + P.vis(i, 0, k)) * 0.5;
      amu = -facoe * io.amvr1 * muqt;
      apu = -facoe * d.apvr[C][1] * fmu(2);
      a = 0.0;
      cc = apu / fden(2);
    } else if (j == ny) {
      const double muqt = (P.vis(i, ny, k) + P.vis(i, ny + 1, k)) * 0.5;
      amu = -facoe * d.amvr[C][ny] * fmu(ny);
      apu = -facoe * io.apvrn * muqt;
      a = amu / fden(ny - 1);
      cc = 0.0;
    } else {
      amu = -facoe * d.amvr[C][j] * fmu(j);
      apu = -facoe * d.apvr[C][j] * fmu(j + 1);
      a = amu / fden(j - 1);
      cc = apu / fden(j + 1);
    }
    den = fden(j);
  } else {
    const double coe1 = facoe * 4.0 / 3.0;
    amu = -coe1 * d.amvr[1][j] * P.vis(i, j - 1, k);
    apu = -coe1 * d.apvr[1][j] * P.vis(i, j, k);
    a = amu / P.r2(i, j - 1, k);
    cc = apu / P.r2(i, j == 1 ? 2 : j, k);  // rows >= 2 divide by the v face j itself, as written
    den = P.r2(i, j, k);
  }
  b = 1.0 - (amu + apu) / den;
}

// ------------------------------------------------------------ line solves
// Warp partition solver for one tridiagonal line of n unknowns,
// a x(i-1) + b x(i) + c x(i+1) = r, cyclic (CYC) or with a(0) = c(n-1) = 0.
// The line is split into P equal chunks of m = n / P (P a power of two, at
// most 32, m >= 2: part_count).  Lane p eliminates its chunk's first m-1
// unknowns in terms of the chunk-end values L(p-1) and L(p) (one Thomas sweep
// with three right-hand sides), which leaves a P-unknown tridiagonal system
// for the chunk ends, cyclic when the line is; parallel cyclic reduction over
// shuffles solves it; then every lane back-substitutes its chunk.  The
// arrays live in shared memory with element i = p m + t at t Q + p
// (Q = P + 1, part_slot), so the lanes' sweeps touch consecutive words.  The result overwrites R.
__host__ __device__ inline int part_count(int n) {
  int P = 1;
  while (P < 32 && n % (2 * P) == 0 && n / (2 * P) >= 2) P *= 2;
  return P;
}
// Shared-memory layout of one line: element i at (i % m) * Q + i / m, rows of
// pitch Q = P + 1, so the lanes' chunk walks (row t, lane p: t * Q + p) read
// consecutive words and the coalesced staging loops, whose lanes take
// consecutive i, spread over the banks instead of hitting one bank at stride P.
__device__ __forceinline__ int part_slot(int i, int m, int Q) { return (i % m) * Q + i / m; }
// values of one line array: m rows of pitch P + 1
__host__ __device__ inline int part_len(int n) {
  const int P = part_count(n);
  return (n / P) * (P + 1);
}
// stride of the lines of a z / y block (4 arrays), = 2 (mod 16) words: the
// staging loops' 8 lines x 2 elements per half-warp then fall in 16 banks
__host__ __device__ inline int zy_stride(int n) {
  const int s = 4 * part_len(n);
  return s + ((2 - s) % 16 + 16) % 16;
}

template <bool CYC>
__device__ void warp_part_solve(double *__restrict__ A, double *__restrict__ B, double *__restrict__ Cc,
                                double *__restrict__ R, int P, int Q, int m, int lane) {
  const bool act = lane < P;
  double yl = 0.0, vl = 0.0, wl = 0.0, yf = 0.0, vf = 0.0, wf = 0.0;
  double ae = 0.0, be = 1.0, ce = 0.0, re = 0.0;
  if (act) {
    double h = 0.0, y = 0.0, v = 0.0, w = 0.0;
    for (int t = 0; t <= m - 2; ++t) {
      const int q = t * Q + lane;
      const double a = A[q], b = B[q], c = Cc[q], r = R[q];
      const double al = t == 0 ? 0.0 : a;       // first row: a couples to L(p-1)
      const double cu = t == m - 2 ? 0.0 : c;   // last interior row: c couples to L(p)
      const double inv = 1.0 / (b - al * h);
      h = cu * inv;
      y = (r - al * y) * inv;
      v = ((t == 0 ? -a : 0.0) - al * v) * inv;
      w = ((t == m - 2 ? -c : 0.0) - al * w) * inv;
      Cc[q] = h; R[q] = y; A[q] = v; B[q] = w;
    }
    yl = y; vl = v; wl = w;
    for (int t = m - 3; t >= 0; --t) {
      const int q = t * Q + lane;
      const double hq = Cc[q];
      y = R[q] - hq * y;
      v = A[q] - hq * v;
      w = B[q] - hq * w;
      R[q] = y; A[q] = v; B[q] = w;
    }
    yf = y; vf = v; wf = w;
    const int qe = (m - 1) * Q + lane;
    ae = A[qe]; be = B[qe]; ce = Cc[qe]; re = R[qe];
  }
  const unsigned full = 0xffffffffu;
  const int nxt = act ? (lane + 1) % P : lane;
  const double yn = __shfl_sync(full, yf, nxt), vn = __shfl_sync(full, vf, nxt), wn = __shfl_sync(full, wf, nxt);
  // chunk-end equation: row e with x(e-1) = yl + vl L(p-1) + wl L(p) and
  // x(e+1) = yn + vn L(p) + wn L(p+1)
  double Ap = ae * vl, Bp = ae * wl + be + ce * vn, Cp = ce * wn, Rp = re - ae * yl - ce * yn;
  if (!act) { Ap = 0.0; Bp = 1.0; Cp = 0.0; Rp = 0.0; }
  for (int hs = 1; hs < P; hs <<= 1) {
    const int lm = act ? (lane - hs + P) % P : lane, lp = act ? (lane + hs) % P : lane;
    double Am = __shfl_sync(full, Ap, lm), Bm = __shfl_sync(full, Bp, lm), Cm = __shfl_sync(full, Cp, lm),
           Rm = __shfl_sync(full, Rp, lm);
    double Aq = __shfl_sync(full, Ap, lp), Bq = __shfl_sync(full, Bp, lp), Cq = __shfl_sync(full, Cp, lp),
           Rq = __shfl_sync(full, Rp, lp);
    if (!CYC) {
      if (lane - hs < 0) { Am = 0.0; Bm = 1.0; Cm = 0.0; Rm = 0.0; }
      if (lane + hs >= P) { Aq = 0.0; Bq = 1.0; Cq = 0.0; Rq = 0.0; }
    }
    if (act) {
      const double k1 = Ap / Bm, k2 = Cp / Bq;
      const double nA = -Am * k1, nC = -Cq * k2;
      const double nB = Bp - Cm * k1 - Aq * k2;
      const double nR = Rp - Rm * k1 - Rq * k2;
      Ap = nA; Bp = nB; Cp = nC; Rp = nR;
    }
  }
  // couplings now reach distance P: the unknown itself (cyclic) or nothing
  const double L = CYC ? Rp / (Ap + Bp + Cp) : Rp / Bp;
  double Lm = __shfl_sync(full, L, act ? (lane - 1 + P) % P : lane);
  if (!CYC && lane == 0) Lm = 0.0;
  if (act) {
    for (int t = 0; t <= m - 2; ++t) {
      const int q = t * Q + lane;
      R[q] = R[q] + A[q] * Lm + B[q] * L;
    }
    R[(m - 1) * Q + lane] = L;
  }
}

// MOMFA1_X_io (TDMAIJI_CYC along x) for component C: one warp per (j, k) row;
// the row and its coefficients are staged in shared memory with coalesced
// loads, solved by warp_part_solve and written back in place.  x-momentum
// subtracts DPGRNS from RHS_io as it is read.
template <int C>
__global__ void __launch_bounds__(256) k_si_x(TGDev d, IODev io, double coe1, double coe2, int use_dpg) {
  extern __shared__ double xs_smem[];
  const int nx = d.nx, j0 = C == 1 ? 2 : 1, nj = d.ny - j0 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int line = blockIdx.x * nw + warp;
  if (line >= nj * d.nz) return;  // whole warp leaves together
  const int j = j0 + line % nj, k = line / nj;
  const int P = part_count(nx), m = nx / P, Q = P + 1, len = m * Q;
  double *A = xs_smem + (size_t)warp * 4 * len, *B = A + len, *Cc = B + len, *Rs = Cc + len;
  const Prop Pr = make_prop(d, io);
  double *__restrict__ R = (double *)d.rhs[C] + d.sy * j + d.sz * k;
  const double sub = (C == 0 && use_dpg) ? *io.dpg : 0.0;
#pragma unroll 4
  for (int i = lane; i < nx; i += 32) {
    double a, b, cc;
    cyc_coef<C, true>(Pr, i, j, k, coe1, coe2, a, b, cc);
    const int q = part_slot(i, m, Q);
    A[q] = a; B[q] = b; Cc[q] = cc; Rs[q] = R[i] - sub;
  }
  __syncwarp();
  warp_part_solve<true>(A, B, Cc, Rs, P, Q, m, lane);
  __syncwarp();
  for (int i = lane; i < nx; i += 32) R[i] = Rs[part_slot(i, m, Q)];
}

// Lines along z (MOMFA2_Z_io, cyclic) or y (MOMFA3_Y_io, rows 1..ny, zero
// boundary values) for component C: a block stages LB lines of consecutive x
// (each row of the tile one coalesced load), its warps solve them in turn.
// The y solve ends with G* = G + dG in the other G buffer from row N2I.
// Four blocks per SM (64 registers, a few spilled words) with 8 lines each at
// n = 192: the blocks' stage / solve / store phases overlap better than two
// blocks of 16 lines (momentum stage of the heated 384x192x192 channel 8.35
// -> 7.35 ms per substep).
template <int C, bool Y>
__global__ void __launch_bounds__(256, 4) k_si_zy(TGDev d, IODev io, double coe1, double coe2, int LB, int cur) {
  extern __shared__ double zs_smem[];
  const int nx = d.nx, ny = d.ny;
  const int n = Y ? ny : d.nz;
  const int j0 = C == 1 ? 2 : 1;
  const int i0 = blockIdx.x * LB;
  const int nl = min(LB, nx - i0);
  // z lines: blockIdx.y = row j - j0; y lines: blockIdx.y = plane k
  const int jz = Y ? 0 : j0 + (int)blockIdx.y, ky = Y ? (int)blockIdx.y : 0;
  const int P = part_count(n), m = n / P, Q = P + 1, len = m * Q, S = zy_stride(n);
  const Prop Pr = make_prop(d, io);
  const int64_t st = Y ? d.sy : d.sz;
  const int64_t base = Y ? d.sz * ky : d.sy * jz;  // + i, + st * (index along the line)
  double *__restrict__ R = (double *)d.rhs[C];
#pragma unroll 4
  for (int t = threadIdx.x; t < n * nl; t += blockDim.x) {
    const int e = t / nl, l = t - e * nl, i = i0 + l;
    double a, b, cc;
    int64_t g;
    if (Y) {
      const int j = e + 1;
      y_coef<C>(d, io, Pr, i, j, ky, coe1, a, b, cc);
      if (j == 1) a = 0.0;    // zero boundary values: the end couplings drop
      if (j == ny) cc = 0.0;
      g = i + base + st * j;
    } else {
      cyc_coef<C, false>(Pr, i, jz, e, coe1, coe2, a, b, cc);
      g = i + base + st * e;
    }
    double *L = zs_smem + (size_t)l * S;
    const int q = part_slot(e, m, Q);
    L[q] = a; L[len + q] = b; L[2 * len + q] = cc; L[3 * len + q] = R[g];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int l = warp; l < nl; l += nw) {
    double *L = zs_smem + (size_t)l * S;
    warp_part_solve<!Y>(L, L + len, L + 2 * len, L + 3 * len, P, Q, m, lane);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < n * nl; t += blockDim.x) {
    const int e = t / nl, l = t - e * nl, i = i0 + l;
    const double x = zs_smem[(size_t)l * S + 3 * len + part_slot(e, m, Q)];
    if (Y) {
      const int j = e + 1;
      if (j >= j0) {
        const int64_t g = i + base + st * j;
        io.g[1 - cur][C][g] = x + io.g[cur][C][g];
      }
    } else {
      R[i + base + st * e] = x;
    }
  }
}

inline dim3 si_cell_grid(const TGDev &d) { return dim3((d.nx + SI_BX - 1) / SI_BX, (d.ny + SI_BY - 1) / SI_BY, d.nz); }

}  // namespace

// Right-hand sides of the semi-implicit momentum stage; *npart receives the
// number of block partials written for DPGRNS.
int io_mom_si(chapsim_ctx *c, int ns, int *npart) {
  TGDev &d = c->d;
  IODev &io = c->io;
  const SubParams &sp = c->sp[ns];
  const dim3 grid = si_cell_grid(d);
  if (io.thermal) {
    k_si_stg<<<dim3(grid.x, (d.ny + 2 + SI_BY - 1) / SI_BY, d.nz), dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io);
    LAUNCHED();
  }
  // one kernel per component: a third of the live values each
  if (io.thermal) {
    k_io_rhs_si<0, true><<<grid, dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, c->io_cur);
    LAUNCHED();
    k_io_rhs_si<1, true><<<grid, dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, c->io_cur);
    LAUNCHED();
    k_io_rhs_si<2, true><<<grid, dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, c->io_cur);
    LAUNCHED();
  } else {
    k_io_rhs_si<0, false><<<grid, dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, c->io_cur);
    LAUNCHED();
    k_io_rhs_si<1, false><<<grid, dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, c->io_cur);
    LAUNCHED();
    k_io_rhs_si<2, false><<<grid, dim3(SI_BX, SI_BY), 0, c->stream>>>(d, io, sp.gam, sp.roh, sp.alp, c->io_cur);
    LAUNCHED();
  }
  *npart = (int)(grid.x * grid.y * grid.z);
  return CHAPSIM_OK;
}

// MOMFA_io for the three components: x, z and y factor solves, G* into the
// other G buffer.
namespace {
int zy_lines_per_block(int n) {
  // lines of one z / y block: as many as fit in 50 KB (4 arrays of n values),
  // so that four blocks share an SM
  int lb = (int)(50 * 1024 / ((size_t)32 * n));
  return lb < 1 ? 1 : (lb > 32 ? 32 : lb);
}
template <int C>
int si_solves(chapsim_ctx *c, double facoe, double cx1, double cx2, double cz1, double cz2) {
  TGDev &d = c->d;
  IODev &io = c->io;
  const int j0 = C == 1 ? 2 : 1, nj = d.ny - j0 + 1;
  {
    // rows per block: as many as fit in 110 KB (4 arrays of nx values each)
    int wpb = (int)(110 * 1024 / ((size_t)32 * d.nx));
    wpb = wpb < 1 ? 1 : (wpb > 8 ? 8 : wpb);
    const size_t sm = (size_t)wpb * 4 * part_len(d.nx) * sizeof(double);
    k_si_x<C><<<(nj * d.nz + wpb - 1) / wpb, 32 * wpb, sm, c->stream>>>(d, io, cx1, cx2, 1);
    LAUNCHED();
  }
  {
    const int lb = zy_lines_per_block(d.nz);
    k_si_zy<C, false><<<dim3((d.nx + lb - 1) / lb, nj), 256, (size_t)lb * zy_stride(d.nz) * sizeof(double), c->stream>>>(
        d, io, cz1, cz2, lb, c->io_cur);
    LAUNCHED();
  }
  {
    const int lb = zy_lines_per_block(d.ny);
    k_si_zy<C, true><<<dim3((d.nx + lb - 1) / lb, d.nz), 256, (size_t)lb * zy_stride(d.ny) * sizeof(double), c->stream>>>(
        d, io, facoe, 0.0, lb, c->io_cur);
    LAUNCHED();
  }
  return CHAPSIM_OK;
}
}  // namespace

int io_factor_si(chapsim_ctx *c, int ns) {
  TGDev &d = c->d;
  const double facoe = 0.5 * c->sp[ns].alp * d.dt * d.cvisc;  // FACOE_io
  const double cx1 = facoe * 4.0 / 3.0 * d.dxqi, cx2 = facoe * d.dxqi;
  const double cz1 = facoe * 4.0 / 3.0 * d.dzqi, cz2 = facoe * d.dzqi;
  if (!c->si_smem_set) {
    // dynamic shared memory above 48 KB (k_si_zy at ny = 192 takes 51 KB):
    // the limit is set per device, with that device current, by every
    // context before its first solve; setting it again is harmless and it
    // involves no process-wide bookkeeping shared between host threads
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    const void *fns[] = {(const void *)k_si_x<0>, (const void *)k_si_x<1>, (const void *)k_si_x<2>,
                         (const void *)k_si_zy<0, false>, (const void *)k_si_zy<1, false>,
                         (const void *)k_si_zy<2, false>, (const void *)k_si_zy<0, true>,
                         (const void *)k_si_zy<1, true>, (const void *)k_si_zy<2, true>};
    for (const void *f : fns)
      if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess) {
        cudaGetLastError();
        c->err = "semi-implicit line solves: cannot raise the shared-memory limit";
        return CHAPSIM_ERR_CUDA;
      }
    c->si_smem_set = true;
  }
  int rc;
  if ((rc = si_solves<0>(c, facoe, cx1, cx2, cz1, cz2))) return rc;
  if ((rc = si_solves<1>(c, facoe, cx1, cx2, cz1, cz2))) return rc;
  return si_solves<2>(c, facoe, cx1, cx2, cz1, cz2);
}

}  // namespace chapsim
