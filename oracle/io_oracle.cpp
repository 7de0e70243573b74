// CPU FP64 oracle for the CHAPSim IO-section substep (the x-periodic channel
// section, and the section coupled to a TG section: x ghost columns, the
// inlet and convective outlet operators, non-periodic Poisson in x).
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA IO path.  The product
// never links or calls it.  Parity against reference outputs is unpinned (the
// Fortran reference cannot be built here and ships no golden data).
//
// Restates (paths relative to the CHAPSim1WW project root), channel branches
// only, so RCCI1 = RCCI2 = RNDI1 = RNDI2 = 1 (src/COORDJR.f90:20-23), the
// explicit viscous scheme (visthemflg = 0, src/readdata.ini:23), no weighted
// pressure, x periodic (BCX_io = 3: IPV_io/IMV_io wrap, src/INDEXSET.f90:24-32)
// or coupled (TGFLOWFLG: the ghost columns, NXI = 2, the boundary operators
// below; src/SOLVERRK3_MOM_IO.f90:15-21, src/SOLVERRK3_ENG_IO.f90:57-64,
// src/VELO_CORRECTION.f90:124-139, src/MEMALLOCT.f90:154-168):
//   SOLVERRK3_ENG_IO        src/SOLVERRK3_ENG_IO.f90:1-77
//   RHS_ENERGY_EXPLICIT     src/RHS_ENERGY_EXPLICIT.f90:1-150
//   ENTHALPY/DENSITY_UPDATE, THERM_PROP_UPDATE, DENSITY_TIME_DERIVATION
//                           src/THERM_PROP_UPDATE.f90:2-291
//   NIST_SLEVAL_*           src/Flow_State.f90:1015-1690 (binary search,
//                           cubic, out of range = error, reference shortcuts)
//   RHOHmax                 src/Flow_State.f90:963-990
//   BC_WALL_ISOFLUX         src/BC_WALL.f90:522-627
//   DENSITY/MU_Staggered, VELOCITY_CALC_io, MASSFLUX_CALC_IO
//                           src/MASSFLUX_CALC_IO.f90:1-311
//   SOLVERRK3_MOM_IO        src/SOLVERRK3_MOM_IO.f90:1-168
//   CONVECTION_X/Y/Z_io     src/CONVECTION_X.f90:77-176, CONVECTION_Y.f90:125-230,
//                           CONVECTION_Z.f90:113-200
//   DIVG_U_io, DIVG_io      src/DIVG.f90:58-259
//   VISCOUS_ALL_EXPLT_X/Y/Z_io  src/VISCOUS_X_EXPLICIT_io.f90:1-112,
//                           VISCOUS_Y_EXPLICIT_io.f90 (ICHANL branch),
//                           VISCOUS_Z_EXPLICIT_io.f90 (ICHANL branch)
//   RHS_MOM_EXPLICIT_io     src/RHS_MOM_EXPLICIT_io.f90:1-297
//   FISHPACK_POIS3D_SIMPLE  src/possion3d_fishpack_reform.f90:29-547 (RFFTF/
//                           RFFTB in x and z from FFTPACK's documented
//                           definitions, eigenvalues -4c sin^2, TRID0)
//   PRCALC_io, MASSFLUX_UPDATE_IO, BC_WALL_G/Q/PR/DPH
//                           src/PRESSURE_CORRECTION.f90:86-122,
//                           src/VELO_CORRECTION.f90:107-185, src/BC_WALL.f90
//   DIVGCK_io               src/DIVGCK.f90:60-190
//   BULK_*_IO               src/INITIAL_FL_THEML_FLD_io.f90:385-476
// and the semi-implicit viscous scheme (visthemflg = 1):
//   VISCOUS_PAR_EXPLT_X/Y/Z_io  src/VISCOUS_X_EXPLICIT_io.f90:124-286,
//                           VISCOUS_Y_EXPLICIT_io.f90:264-424,
//                           VISCOUS_Z_EXPLICIT_io.f90:289-460 (channel branches)
//   RHS_MOM_EXPLICIT_io     src/RHS_MOM_EXPLICIT_io.f90:79-95 (implicit branch)
//   MOMFA_io, MOMFA1_X_io, MOMFA2_Z_io, MOMFA3_Y_io
//                           src/MOMFA_io.f90:17-377
//   TDMAIJI_CYC, TDMAIJJ_nonCYC  src/TDMAIJI_CYC.f90:67-157, src/TDMAIJJ_nonCYC.f90:67-123
//   AMVR/APVR, AMVR1, APVRN src/TDMA_COEF.f90:77-116
//   DENSITY_implicit_add    src/MASSFLUX_CALC_IO.f90:316-399
//   PRCALC_io               src/PRESSURE_CORRECTION.f90:100-110 (implicit branch)
//
// Decisions (each also stated where it applies):
//  * The mean mode (x-slot 1, z-slot 1) of the Poisson y-solve is singular;
//    TRID0 takes its zero branch only when the last pivot falls under 1e-14,
//    which for that mode depends on round-off.  Here that mode always takes
//    the zero branch (phi(ny) = 0 for the mean), the other modes use the
//    threshold as written.
//  * The reference-state shortcuts of the table look-ups are kept only when
//    the table follows the reference normalisation (h = 0 <-> T = 1); the
//    flag is set per table.
//  * Initial field: the TG recipe (counter-based generator) for velocity,
//    h = 0 for enthalpy with the table's properties at h = 0 (the reference
//    writes T = rho = mu = k = 1, its normalised reference state), then the
//    reference's CALC_INITIALIZATION_io projection.
//  * Y ghosts of MU_STG, RHO_STG and DivU_io, filled by the periodic MPI halo
//    exchange in the reference, are never read in the channel branch and are
//    not formed.  The y ghosts of DRHOI_STG (periodic halo values there) are
//    only ever multiplied by wall ghosts of G, which are zero; they are zero
//    here.
//  * Coupled section: the Poisson solve runs on the IO arrays (the
//    reference's coupled branch passes the TG arrays,
//    src/SOLVERRK3_MOM_IO.f90:116-121, which leaves the IO velocity
//    unprojected); the initial outlet ghost column is a copy of the last
//    interior column and the boundary operators' RK3 memory starts at zero;
//    lines longer than 64 take the quarter-wave transforms (LP 3, 5)
//    through the DFT (qwave_fast), shorter ones the documented sums.
//  * Semi-implicit PRCALC_io subtracts BE * RHSLLPHI_io, but
//    FISHPACK_POIS3D_SIMPLE has by then written its x/z-transformed right-hand
//    side back into RHSLLPHI_io (src/possion3d_fishpack_reform.f90:456-463):
//    spectral coefficients used as a physical field.  Here the physical
//    right-hand side of the Poisson equation is used, as PRCALC_tg does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "chapsim_oracle.h"

extern "C" void oracle_cubic_spline(int n, const double *x, const double *y, double *b, double *c, double *d);

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Same counter-based draw as the TG oracle and the library's initial field.
inline double rnd_pm1(uint64_t seed, int comp, int i, int j, int k) {
  uint64_t ctr = ((uint64_t)comp << 60) ^ ((uint64_t)k << 40) ^ ((uint64_t)j << 20) ^ (uint64_t)i;
  uint64_t x = splitmix64(splitmix64(seed) ^ ctr);
  double u = (double)(x >> 11) * (1.0 / 9007199254740992.0);
  return -1.0 + 2.0 * u;
}

struct Spl {
  std::vector<double> x, y, b, c, d;
  int n = 0;
  void build(const double *xs, const double *ys, int n_) {
    n = n_;
    x.assign(xs, xs + n);
    y.assign(ys, ys + n);
    b.assign(n, 0.0); c.assign(n, 0.0); d.assign(n, 0.0);
    oracle_cubic_spline(n, x.data(), y.data(), b.data(), c.data(), d.data());
  }
  // NIST_SLEVAL_* (src/Flow_State.f90:1015-1070): false when u is outside
  // (x(1), x(n)) -- the reference STOPs there.
  bool eval(double u, double &out) const {
    if (u <= x[0] || u >= x[n - 1]) return false;
    int i = 0, j = n;
    while (j > i + 1) {
      int k = (i + j) / 2;
      if (u < x[k]) j = k; else i = k;
    }
    double dx = u - x[i];
    out = y[i] + dx * (b[i] + dx * (c[i] + dx * d[i]));
    return true;
  }
};

}  // namespace

struct oracle_io {
  int nx, ny, nz, istr2, flowdrvtp, thermal, gravdir;
  double lx, lz, str2, ren, dt, cfgv, prt, qw[2], f_a;
  double dxi, dzi, dxqi, dzqi, cvisc, cthecd, volm, area_inlet;
  std::vector<double> ynd, ycc, dyfi, dyci, wff, wfb, amph, acph, apph;  // 1-based, size ny+2
  double tgam[4], troh[4], talp[4];
  // table
  bool has_table = false;
  int shortcuts = 0;
  Spl ht, td, tm, tk, hd, th;
  // BCWALLHEAT: bit 0 bottom, bit 1 top iso-thermal; wall[side] = T, h, rho,
  // mu, k at the wall temperature (qw[side] holds it)
  int isothermal = 0;
  double wall[2][5] = {{0.0}};
  // x boundary type of the Poisson solve, FISHPACK's LP = LPEROD + 1
  // (src/possion3d_fishpack_reform.f90:342-346): 1 periodic, 2 Dirichlet
  // both ends (SINT), 3 Dirichlet-Neumann (SINQ), 4 Neumann both (COST), 5
  // Neumann-Dirichlet (COSQ)
  int lpx = 1;
  double rhohmax = 0.0;
  int64_t bad = 0;
  // flow fields (1..3 used)
  std::vector<double> q[4], g[4], g0[4], explt0[4], mustg[4], rhostg[4];
  std::vector<double> pr, dph, rhsllphi, qtmp, dphtmp, rhsz, divu, drho;
  // thermal fields
  std::vector<double> rhoh, hh, tt, dd, dd0, mu, mu0, kk, rhse, rhse0;
  oracle_dft *dftx = nullptr, *dftz = nullptr;
  // semi-implicit viscous scheme (visthemflg = 1)
  int implicit = 0;
  std::vector<double> rhsio[4], adv[4], drhoi[4];  // RHS_io per component, DIVU_io (density part), DRHOI_STG
  std::vector<double> amvr13, apvr13, amvr2, apvr2;  // TDMA_COEF y-operators, 1-based
  double amvr1 = 0.0, apvrn = 0.0;
  // coupled inflow/outflow ghost planes (i = 0 and i = NCL1_io + 1), each
  // (nz, ny + 2), ids ORC_P_*; bcs: U_OUTLET (momentum), scaling, balance,
  // inflow, outflow, mass rate, U_OUTLET (energy)
  std::vector<double> bcp[ORC_P_COUNT];
  double bcs[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

  // TGFLOWFLG (a TG section feeds the inlet; src/READINI.f90:127-131: any
  // non-periodic BCX_io): the arrays carry the x ghost columns i = 0 and
  // NCL1_io + 1 (NCL1S:NCL1E, src/MEMALLOCT.f90:154-168) and the x neighbours
  // do not wrap (IPV_io / IMV_io, src/INDEXSET.f90:25-32)
  int coupled = 0;
  int sx = 0;  // x extent of the arrays: nx, or nx + 2 with the ghost columns
  // TG arrays (nz, ny + 2, tg_nx) that feed BC_TINLET_FLOW during a coupled substep
  int tg_nx = 0;
  const double *tg_u = nullptr, *tg_v = nullptr, *tg_w = nullptr, *tg_p = nullptr;

  int64_t len() const { return (int64_t)sx * (ny + 2) * nz; }
  inline int64_t pj(int j, int k) const { return (int64_t)j + (int64_t)(ny + 2) * (k - 1); }
  inline int64_t id(int i, int j, int k) const {
    return (int64_t)(i - 1 + coupled) + (int64_t)sx * ((int64_t)j + (int64_t)(ny + 2) * (k - 1));
  }
  inline int ip(int i) const { return coupled ? i + 1 : (i == nx ? 1 : i + 1); }
  inline int im(int i) const { return coupled ? i - 1 : (i == 1 ? nx : i - 1); }
  // first x face the x-momentum equation advances (NXI of CONVECTION_X_io,
  // VISCOUS_ALL_EXPLT_X_io, RHS_MOM_EXPLICIT_io, MASSFLUX_CALC_IO): the
  // coupled inlet face keeps the value BC_TINLET_FLOW gives it
  inline int nxi() const { return coupled ? 2 : 1; }
  inline int kp(int k) const { return k == nz ? 1 : k + 1; }
  inline int km(int k) const { return k == 1 ? nz : k - 1; }
};

namespace {

constexpr double XND2CL = 0.5, YND2CL = 0.5, ZND2CL = 0.5;

#define F(arr, i, j, k) (o->arr[o->id(i, j, k)])
#define FC(arr, c, i, j, k) (o->arr[c][o->id(i, j, k)])

int nthreads() { return oracle_get_threads(); }

// ------------------------------------------------------------- table look-ups
// h -> T, then T -> rho (DENSITY_UPDATE path, src/THERM_PROP_UPDATE.f90:74-127).
bool lookup_ht(const oracle_io *o, double h, double &T) {
  if (!o->ht.eval(h, T)) return false;
  if (o->shortcuts && std::fabs(h) < 1.0e-10) T = 1.0;  // Flow_State.f90:1068
  return true;
}
bool lookup_t(const oracle_io *o, const Spl &s, double T, double &v) {
  if (!s.eval(T, v)) return false;
  if (o->shortcuts && std::fabs(T - 1.0) < 1.0e-10) v = 1.0;  // Flow_State.f90:1470,1524,1578
  return true;
}

// BC_WALL_ISOFLUX (src/BC_WALL.f90:522-627): ghost enthalpy extrapolated from
// the first two cells, ghost properties from the table; BC_WALL_ISOTHERMAL
// (src/BC_WALL.f90:462-515) on an iso-thermal wall: the wall values.
void bc_wall_thermal(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int side = 0; side < 2; ++side) {
    const int j = side == 0 ? 0 : ny + 1;
    if (o->isothermal & (1 << side)) {
      const double *w = o->wall[side];
      for (int k = 1; k <= nz; ++k)
        for (int i = 1; i <= nx; ++i) {
          F(tt, i, j, k) = w[0];
          F(hh, i, j, k) = w[1];
          F(dd, i, j, k) = w[2];
          F(mu, i, j, k) = w[3];
          F(kk, i, j, k) = w[4];
          F(rhoh, i, j, k) = w[1] * w[2];
        }
      continue;
    }
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) {
        double h;
        if (side == 0)
          h = 2.0 * F(hh, i, 1, k) - o->wff[2] * F(hh, i, 2, k) - o->wfb[2] * F(hh, i, 1, k);
        else
          h = 2.0 * F(hh, i, ny, k) - o->wff[ny] * F(hh, i, ny, k) - o->wfb[ny] * F(hh, i, ny - 1, k);
        F(hh, i, j, k) = h;
        double T, M, K, D;
        if (!lookup_ht(o, h, T) || !lookup_t(o, o->tm, T, M) || !lookup_t(o, o->tk, T, K) ||
            !lookup_t(o, o->td, T, D)) {
          ++o->bad;
          continue;
        }
        F(dd, i, j, k) = D;
        F(tt, i, j, k) = T;
        F(mu, i, j, k) = M;
        F(kk, i, j, k) = K;
        F(rhoh, i, j, k) = h * D;
      }
  }
}

// RHS_ENERGY_EXPLICIT (src/RHS_ENERGY_EXPLICIT.f90:1-150), iso-flux or
// iso-thermal walls (:41-72, :118-123).
void rhs_energy(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double coe1 = o->dxi * XND2CL * 0.5, coe11 = o->dxqi * XND2CL * o->cthecd;
  const double wallflux_bot = o->qw[0], wallflux_top = -o->qw[1];
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int jp = j + 1, jm = j - 1;
      const double coe2 = o->dyfi[j] * 0.5, coe3 = o->dzi * ZND2CL * 0.5;
      const double coe33 = o->dzqi * ZND2CL * o->cthecd, coe22 = o->dyfi[j] * o->cthecd;
      const bool iso_bot = o->isothermal & 1, iso_top = o->isothermal & 2;
      double coe221, coe222;
      if (j == 1) {
        coe221 = o->dyci[jp];
        coe222 = iso_bot ? o->dyci[j] : 1.0;
      } else if (j == ny) {
        coe222 = o->dyci[j];
        coe221 = iso_top ? o->dyci[jp] : 1.0;
      } else {
        coe221 = o->dyci[jp];
        coe222 = o->dyci[j];
      }
      const int kpp = o->kp(k), kmm = o->km(k);
      for (int i = 1; i <= nx; ++i) {
        const int ipp = o->ip(i), imm = o->im(i);
        const double hc = F(hh, i, j, k);
        double dx_rhohu = (F(hh, ipp, j, k) + hc) * (FC(g0, 1, ipp, j, k) + FC(g, 1, ipp, j, k)) -
                          (hc + F(hh, imm, j, k)) * (FC(g0, 1, i, j, k) + FC(g, 1, i, j, k));
        dx_rhohu *= coe1;
        double dy_rhohv = (o->wff[jp] * F(hh, i, jp, k) + o->wfb[jp] * hc) * (FC(g0, 2, i, jp, k) + FC(g, 2, i, jp, k)) -
                          (o->wff[j] * hc + o->wfb[j] * F(hh, i, jm, k)) * (FC(g0, 2, i, j, k) + FC(g, 2, i, j, k));
        dy_rhohv *= coe2;
        double dz_rhohw = (F(hh, i, j, kpp) + hc) * (FC(g0, 3, i, j, kpp) + FC(g, 3, i, j, kpp)) -
                          (hc + F(hh, i, j, kmm)) * (FC(g0, 3, i, j, k) + FC(g, 3, i, j, k));
        dz_rhohw *= coe3;
        const double tc = F(tt, i, j, k), kc = F(kk, i, j, k);
        double dx_kdt = (F(kk, ipp, j, k) + kc) * (F(tt, ipp, j, k) - tc) - (kc + F(kk, imm, j, k)) * (tc - F(tt, imm, j, k));
        dx_kdt *= coe11;
        double kdty1 = (o->wff[jp] * F(kk, i, jp, k) + o->wfb[jp] * kc) * (F(tt, i, jp, k) - tc) * coe221;
        double kdty2 = (o->wff[j] * kc + o->wfb[j] * F(kk, i, jm, k)) * (tc - F(tt, i, jm, k)) * coe222;
        if (j == 1 && !iso_bot)
          kdty2 = -wallflux_bot * coe222;
        else if (j == ny && !iso_top)
          kdty1 = -wallflux_top * coe221;
        const double dy_kdt = (kdty1 - kdty2) * coe22;
        double dz_kdt = (F(kk, i, j, kpp) + kc) * (F(tt, i, j, kpp) - tc) - (F(kk, i, j, kmm) + kc) * (tc - F(tt, i, j, kmm));
        dz_kdt *= coe33;
        F(rhse, i, j, k) = -dx_rhohu - dy_rhohv - dz_rhohw + dx_kdt + dy_kdt + dz_kdt;
      }
    }
}

// ------------------------------------------------------------- staggering
// DENSITY_Staggered (src/MASSFLUX_CALC_IO.f90:242-311).
void density_staggered(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  if (!o->thermal) {
    for (int c = 1; c <= 3; ++c) std::fill(o->rhostg[c].begin(), o->rhostg[c].end(), 1.0);
    return;
  }
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int kmm = o->km(k);
      for (int i = 1; i <= nx; ++i) {
        const int imm = o->im(i);
        FC(rhostg, 1, i, j, k) = (F(dd, i, j, k) + F(dd, imm, j, k) + F(dd0, i, j, k) + F(dd0, imm, j, k)) * XND2CL * 0.5;
        FC(rhostg, 3, i, j, k) = (F(dd, i, j, k) + F(dd, i, j, kmm) + F(dd0, i, j, k) + F(dd0, i, j, kmm)) * ZND2CL * 0.5;
        if (j >= 2)
          FC(rhostg, 2, i, j, k) = (o->wff[j] * (F(dd, i, j, k) + F(dd0, i, j, k)) +
                                    o->wfb[j] * (F(dd, i, j - 1, k) + F(dd0, i, j - 1, k))) * 0.5;
      }
    }
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) {
      FC(rhostg, 2, i, 1, k) = 0.5 * (F(dd0, i, 0, k) + F(dd, i, 0, k));
      FC(rhostg, 2, i, ny + 1, k) = 0.5 * (F(dd0, i, ny + 1, k) + F(dd, i, ny + 1, k));
    }
}

// MU_Staggered (src/MASSFLUX_CALC_IO.f90:147-237).
void mu_staggered(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  if (!o->thermal) {
    for (int c = 1; c <= 3; ++c) std::fill(o->mustg[c].begin(), o->mustg[c].end(), 1.0);
    return;
  }
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int kmm = o->km(k);
      for (int i = 1; i <= nx; ++i) {
        const int imm = o->im(i);
        if (j >= 2) {
          FC(mustg, 1, i, j, k) =
              ((F(mu, i, j, k) + F(mu, imm, j, k) + F(mu0, i, j, k) + F(mu0, imm, j, k)) * o->wff[j] +
               (F(mu, i, j - 1, k) + F(mu, imm, j - 1, k) + F(mu0, i, j - 1, k) + F(mu0, imm, j - 1, k)) * o->wfb[j]) *
              XND2CL * 0.5;
          FC(mustg, 3, i, j, k) =
              ((F(mu, i, j, kmm) + F(mu, i, j, k) + F(mu0, i, j, kmm) + F(mu0, i, j, k)) * o->wff[j] +
               (F(mu, i, j - 1, kmm) + F(mu, i, j - 1, k) + F(mu0, i, j - 1, kmm) + F(mu0, i, j - 1, k)) * o->wfb[j]) *
              ZND2CL * 0.5;
        }
        FC(mustg, 2, i, j, k) = (F(mu, i, j, k) + F(mu, imm, j, k) + F(mu0, i, j, k) + F(mu0, imm, j, k) +
                                 F(mu, i, j, kmm) + F(mu, imm, j, kmm) + F(mu0, i, j, kmm) + F(mu0, imm, j, kmm)) *
                                XND2CL * ZND2CL * 0.5;
      }
    }
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) {
      const double b = 0.5 * (F(mu0, i, 0, k) + F(mu, i, 0, k));
      const double t = 0.5 * (F(mu0, i, ny + 1, k) + F(mu, i, ny + 1, k));
      FC(mustg, 1, i, 1, k) = b;
      FC(mustg, 3, i, 1, k) = b;
      FC(mustg, 1, i, ny + 1, k) = t;
      FC(mustg, 3, i, ny + 1, k) = t;
    }
}

// BC_WALL_Q / BC_WALL_G (src/BC_WALL.f90:185-263, 412-458).
void bc_wall_vec(oracle_io *o, std::vector<double> *f) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) {
      f[1][o->id(i, 0, k)] = 0.0;
      f[3][o->id(i, 0, k)] = 0.0;
      f[2][o->id(i, 1, k)] = 0.0;
      f[2][o->id(i, 0, k)] = 0.0;
      f[1][o->id(i, ny + 1, k)] = 0.0;
      f[3][o->id(i, ny + 1, k)] = 0.0;
      f[2][o->id(i, ny + 1, k)] = 0.0;
    }
}
// BC_WALL_PR / BC_WALL_DPH: zero normal gradient by copy.
void bc_wall_copy(oracle_io *o, std::vector<double> &f) {
  for (int k = 1; k <= o->nz; ++k)
    for (int i = 1; i <= o->nx; ++i) {
      f[o->id(i, 0, k)] = f[o->id(i, 1, k)];
      f[o->id(i, o->ny + 1, k)] = f[o->id(i, o->ny, k)];
    }
}

// VELOCITY_CALC_io (src/MASSFLUX_CALC_IO.f90:82-142).
void velocity_calc(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        FC(q, 1, i, j, k) = FC(g, 1, i, j, k) / FC(rhostg, 1, i, j, k);
        FC(q, 3, i, j, k) = FC(g, 3, i, j, k) / FC(rhostg, 3, i, j, k);
        if (j >= 2) FC(q, 2, i, j, k) = FC(g, 2, i, j, k) / FC(rhostg, 2, i, j, k);
      }
  bc_wall_vec(o, o->q);
}

// DENSITY_TIME_DERIVATION (src/THERM_PROP_UPDATE.f90:225-291), the division by
// (gamma - 2) as written.
void density_time_derivation(oracle_io *o, int ns) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double gp = o->tgam[ns] + o->troh[ns], zr = o->troh[ns], den = o->tgam[ns] - 2.0;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const int ipp = o->ip(i), kpp = o->kp(k);
        const double divx = (FC(g, 1, ipp, j, k) - FC(g, 1, i, j, k)) * o->dxi;
        const double divx0 = (FC(g0, 1, ipp, j, k) - FC(g0, 1, i, j, k)) * o->dxi;
        const double divy = (FC(g, 2, i, j + 1, k) - FC(g, 2, i, j, k)) * o->dyfi[j];
        const double divy0 = (FC(g0, 2, i, j + 1, k) - FC(g0, 2, i, j, k)) * o->dyfi[j];
        const double divz = (FC(g, 3, i, j, kpp) - FC(g, 3, i, j, k)) * o->dzi;
        const double divz0 = (FC(g0, 3, i, j, kpp) - FC(g0, 3, i, j, k)) * o->dzi;
        F(drho, i, j, k) = (gp * (divx + divy + divz) + zr * (divx0 + divy0 + divz0)) / den;
      }
}

// ------------------------------------------------------------- momentum
void convection(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  std::fill(o->qtmp.begin(), o->qtmp.end(), 0.0);
  std::fill(o->dphtmp.begin(), o->dphtmp.end(), 0.0);
  std::fill(o->rhsz.begin(), o->rhsz.end(), 0.0);
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int jp = j + 1, jm = j - 1, kpp = o->kp(k), kmm = o->km(k);
      for (int i = 1; i <= nx; ++i) {
        const int ipp = o->ip(i), imm = o->im(i);
        // CONVECTION_X_io (src/CONVECTION_X.f90:98-140), IC >= NXI
        if (i >= o->nxi()) {
          const double coe1 = o->dxi * XND2CL * XND2CL, coe3 = o->dzi * XND2CL * ZND2CL;
          const double coe2 = o->dyfi[j] * XND2CL, coe32 = coe3;
          double h11f = (FC(g, 1, ipp, j, k) + FC(g, 1, i, j, k)) * (FC(q, 1, ipp, j, k) + FC(q, 1, i, j, k));
          double h11b = (FC(g, 1, i, j, k) + FC(g, 1, imm, j, k)) * (FC(q, 1, i, j, k) + FC(q, 1, imm, j, k));
          double h11 = (h11f - h11b) * coe1;
          double h12f = (FC(g, 2, i, jp, k) + FC(g, 2, imm, jp, k)) *
                        (o->wff[jp] * FC(q, 1, i, jp, k) + o->wfb[jp] * FC(q, 1, i, j, k));
          double h12b = (FC(g, 2, i, j, k) + FC(g, 2, imm, j, k)) *
                        (o->wff[j] * FC(q, 1, i, j, k) + o->wfb[j] * FC(q, 1, i, jm, k));
          double h12 = (h12f - h12b) * coe2;
          double h13f = (FC(g, 3, i, j, kpp) + FC(g, 3, imm, j, kpp)) * (FC(q, 1, i, j, kpp) + FC(q, 1, i, j, k));
          double h13b = (FC(g, 3, i, j, k) + FC(g, 3, imm, j, k)) * (FC(q, 1, i, j, k) + FC(q, 1, i, j, kmm));
          double h13 = (h13f - h13b) * coe32;
          F(qtmp, i, j, k) = -(h11 + h12 + h13);
        }
        // CONVECTION_Y_io (src/CONVECTION_Y.f90:150-200), j >= 2
        if (j >= 2) {
          const double coe1 = o->dxi * XND2CL, coe2 = o->dyci[j] * YND2CL * YND2CL, coe31 = o->dzi * ZND2CL;
          double h21f = (o->wff[j] * FC(g, 1, ipp, j, k) + o->wfb[j] * FC(g, 1, ipp, jm, k)) *
                        (FC(q, 2, ipp, j, k) + FC(q, 2, i, j, k));
          double h21b = (o->wff[j] * FC(g, 1, i, j, k) + o->wfb[j] * FC(g, 1, i, jm, k)) *
                        (FC(q, 2, i, j, k) + FC(q, 2, imm, j, k));
          double h21 = (h21f - h21b) * coe1;
          double h22f = (FC(g, 2, i, jp, k) + FC(g, 2, i, j, k)) * (FC(q, 2, i, jp, k) + FC(q, 2, i, j, k));
          double h22b = (FC(g, 2, i, j, k) + FC(g, 2, i, jm, k)) * (FC(q, 2, i, j, k) + FC(q, 2, i, jm, k));
          double h22 = (h22f - h22b) * coe2;
          double h23f = (o->wff[j] * FC(g, 3, i, j, kpp) + o->wfb[j] * FC(g, 3, i, jm, kpp)) *
                        (FC(q, 2, i, j, kpp) + FC(q, 2, i, j, k));
          double h23b = (o->wff[j] * FC(g, 3, i, j, k) + o->wfb[j] * FC(g, 3, i, jm, k)) *
                        (FC(q, 2, i, j, k) + FC(q, 2, i, j, kmm));
          double h23 = (h23f - h23b) * coe31;
          F(dphtmp, i, j, k) = -(h21 + h22 + h23);
        }
        // CONVECTION_Z_io (src/CONVECTION_Z.f90:133-170)
        {
          const double coe1 = o->dxi * XND2CL * ZND2CL, coe2 = o->dyfi[j] * ZND2CL, coe31 = o->dzi * ZND2CL * ZND2CL;
          double h31f = (FC(g, 1, ipp, j, k) + FC(g, 1, ipp, j, kmm)) * (FC(q, 3, ipp, j, k) + FC(q, 3, i, j, k));
          double h31b = (FC(g, 1, i, j, k) + FC(g, 1, i, j, kmm)) * (FC(q, 3, i, j, k) + FC(q, 3, imm, j, k));
          double h31 = (h31f - h31b) * coe1;
          double h32f = (FC(g, 2, i, jp, k) + FC(g, 2, i, jp, kmm)) *
                        (o->wff[jp] * FC(q, 3, i, jp, k) + o->wfb[jp] * FC(q, 3, i, j, k));
          double h32b = (FC(g, 2, i, j, k) + FC(g, 2, i, j, kmm)) *
                        (o->wff[j] * FC(q, 3, i, j, k) + o->wfb[j] * FC(q, 3, i, jm, k));
          double h32 = (h32f - h32b) * coe2;
          double h33f = (FC(g, 3, i, j, kpp) + FC(g, 3, i, j, k)) * (FC(q, 3, i, j, kpp) + FC(q, 3, i, j, k));
          double h33b = (FC(g, 3, i, j, k) + FC(g, 3, i, j, kmm)) * (FC(q, 3, i, j, k) + FC(q, 3, i, j, kmm));
          double h33 = (h33f - h33b) * coe31;
          F(rhsz, i, j, k) = -(h31 + h32 + h33);
        }
      }
    }
}

// DIVG_U_io (src/DIVG.f90:153-259): div u / 3 at cell centres.
void divg_u(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double divx = (FC(q, 1, o->ip(i), j, k) - FC(q, 1, i, j, k)) * o->dxi;
        const double divy = (FC(q, 2, i, j + 1, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
        const double divz = (FC(q, 3, i, j, o->kp(k)) - FC(q, 3, i, j, k)) * o->dzi;
        F(divu, i, j, k) = (divx + divy + divz) / 3.0;
      }
}

// 0.5 (mu0 + mu) at a cell centre.
inline double muc(const oracle_io *o, int i, int j, int k) { return 0.5 * (F(mu0, i, j, k) + F(mu, i, j, k)); }

// VISCOUS_ALL_EXPLT_X/Y/Z_io, channel branch.
void viscous(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double cv = o->cvisc;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int jp = j + 1, jm = j - 1, kpp = o->kp(k), kmm = o->km(k);
      for (int i = 1; i <= nx; ++i) {
        const int ipp = o->ip(i), imm = o->im(i);
        // X (src/VISCOUS_X_EXPLICIT_io.f90:38-104), IC >= NXI
        if (i >= o->nxi()) {
          const double coe1 = 2.0 * o->dxi * cv, coe3 = o->dzi * cv, coe2 = o->dyfi[j] * cv, coe32 = coe3;
          double dudx = (FC(q, 1, ipp, j, k) - FC(q, 1, i, j, k)) * o->dxi;
          double tau11f = muc(o, i, j, k) * (dudx - F(divu, i, j, k));
          dudx = (FC(q, 1, i, j, k) - FC(q, 1, imm, j, k)) * o->dxi;
          double tau11b = muc(o, imm, j, k) * (dudx - F(divu, imm, j, k));
          double d11 = (tau11f - tau11b) * coe1;
          double vis12p = FC(mustg, 1, i, jp, k);
          double dudy = (FC(q, 1, i, jp, k) - FC(q, 1, i, j, k)) * o->dyci[jp];
          double dvdx = (FC(q, 2, i, jp, k) - FC(q, 2, imm, jp, k)) * o->dxi;
          double tau12f = vis12p * (dudy + dvdx);
          double vis12c = FC(mustg, 1, i, j, k);
          dudy = (FC(q, 1, i, j, k) - FC(q, 1, i, jm, k)) * o->dyci[j];
          dvdx = (FC(q, 2, i, j, k) - FC(q, 2, imm, j, k)) * o->dxi;
          double tau12b = vis12c * (dudy + dvdx);
          double d12 = (tau12f - tau12b) * coe2;
          double vis13p = FC(mustg, 2, i, j, kpp);
          double dudz = (FC(q, 1, i, j, kpp) - FC(q, 1, i, j, k)) * o->dzi;
          double dwdx = (FC(q, 3, i, j, kpp) - FC(q, 3, imm, j, kpp)) * o->dxi;
          double tau13f = vis13p * (dudz + dwdx);
          double vis13c = FC(mustg, 2, i, j, k);
          dudz = (FC(q, 1, i, j, k) - FC(q, 1, i, j, kmm)) * o->dzi;
          dwdx = (FC(q, 3, i, j, k) - FC(q, 3, imm, j, k)) * o->dxi;
          double tau13b = vis13c * (dudz + dwdx);
          double d13 = (tau13f - tau13b) * coe32;
          F(qtmp, i, j, k) = F(qtmp, i, j, k) + d11 + d12 + d13;
        }
        // Y, j >= 2 (src/VISCOUS_Y_EXPLICIT_io.f90, ICHANL branch)
        if (j >= 2) {
          const double coe1 = o->dxi * cv, coe3 = o->dzi * cv, coe2 = 2.0 * o->dyci[j] * cv;
          double dvdy = (FC(q, 2, i, jp, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
          double tau22f = muc(o, i, j, k) * (dvdy - F(divu, i, j, k));
          dvdy = (FC(q, 2, i, j, k) - FC(q, 2, i, jm, k)) * o->dyfi[jm];
          double tau22b = muc(o, i, jm, k) * (dvdy - F(divu, i, jm, k));
          double d22 = (tau22f - tau22b) * coe2;
          double vis21p = FC(mustg, 1, ipp, j, k);
          double dvdx = (FC(q, 2, ipp, j, k) - FC(q, 2, i, j, k)) * o->dxi;
          double dudy = (FC(q, 1, ipp, j, k) - FC(q, 1, ipp, jm, k)) * o->dyci[j];
          double tau21f = vis21p * (dvdx + dudy);
          double vis21c = FC(mustg, 1, i, j, k);
          dvdx = (FC(q, 2, i, j, k) - FC(q, 2, imm, j, k)) * o->dxi;
          dudy = (FC(q, 1, i, j, k) - FC(q, 1, i, jm, k)) * o->dyci[j];
          double tau21b = vis21c * (dvdx + dudy);
          double d21 = (tau21f - tau21b) * coe1;
          double vis23p = FC(mustg, 3, i, j, kpp);
          double dvdz = (FC(q, 2, i, j, kpp) - FC(q, 2, i, j, k)) * o->dzi;
          double dwdy = (FC(q, 3, i, j, kpp) - FC(q, 3, i, jm, kpp)) * o->dyci[j];
          double tau23f = vis23p * (dvdz + dwdy);
          double vis23c = FC(mustg, 3, i, j, k);
          dvdz = (FC(q, 2, i, j, k) - FC(q, 2, i, j, kmm)) * o->dzi;
          dwdy = (FC(q, 3, i, j, k) - FC(q, 3, i, jm, k)) * o->dyci[j];
          double tau23b = vis23c * (dvdz + dwdy);
          double d23 = (tau23f - tau23b) * coe3;
          F(dphtmp, i, j, k) = F(dphtmp, i, j, k) + d21 + d22 + d23;
        }
        // Z (src/VISCOUS_Z_EXPLICIT_io.f90, ICHANL branch)
        {
          const double coe1 = o->dxi * cv, coe3 = 2.0 * o->dzi * cv, coe2 = o->dyfi[j] * cv;
          double dwdz = (FC(q, 3, i, j, kpp) - FC(q, 3, i, j, k)) * o->dzi;
          double tau33f = muc(o, i, j, k) * (dwdz - F(divu, i, j, k));
          dwdz = (FC(q, 3, i, j, k) - FC(q, 3, i, j, kmm)) * o->dzi;
          double tau33b = muc(o, i, j, kmm) * (dwdz - F(divu, i, j, kmm));
          double d33 = (tau33f - tau33b) * coe3;
          double vis31p = FC(mustg, 2, ipp, j, k);
          double dwdx = (FC(q, 3, ipp, j, k) - FC(q, 3, i, j, k)) * o->dxi;
          double dudz = (FC(q, 1, ipp, j, k) - FC(q, 1, ipp, j, kmm)) * o->dzi;
          double tau31f = vis31p * (dwdx + dudz);
          double vis31c = FC(mustg, 2, i, j, k);
          dwdx = (FC(q, 3, i, j, k) - FC(q, 3, imm, j, k)) * o->dxi;
          dudz = (FC(q, 1, i, j, k) - FC(q, 1, i, j, kmm)) * o->dzi;
          double tau31b = vis31c * (dwdx + dudz);
          double d31 = (tau31f - tau31b) * coe1;
          double vis32p = FC(mustg, 3, i, jp, k);
          double dwdy = (FC(q, 3, i, jp, k) - FC(q, 3, i, j, k)) * o->dyci[jp];
          double dvdz = (FC(q, 2, i, jp, k) - FC(q, 2, i, jp, kmm)) * o->dzi;
          double tau32f = vis32p * (dwdy + dvdz);
          double vis32c = FC(mustg, 3, i, j, k);
          dwdy = (FC(q, 3, i, j, k) - FC(q, 3, i, jm, k)) * o->dyci[j];
          dvdz = (FC(q, 2, i, j, k) - FC(q, 2, i, j, kmm)) * o->dzi;
          double tau32b = vis32c * (dwdy + dvdz);
          double d32 = (tau32f - tau32b) * coe2;
          F(rhsz, i, j, k) = F(rhsz, i, j, k) + d31 + d32 + d33;
        }
      }
    }
}

// RHS_MOM_EXPLICIT_io(NS, IDR) (src/RHS_MOM_EXPLICIT_io.f90:1-297) for one
// component; tmp holds EXPLT on entry.  Explicit scheme: tmp holds RHS_io on
// exit.  Semi-implicit scheme (:79-95): rhsio[idr] holds the implicit viscous
// part on entry and RHS_io on exit, with alpha dt times it and alpha dt / 2
// times the density part adv[idr] added.
void rhs_mom(oracle_io *o, int ns, int idr, std::vector<double> &texplt) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const int nyi = idr == 2 ? 2 : 1;
  const double gam = o->tgam[ns], roh = o->troh[ns], alp = o->talp[ns], dt = o->dt;
  const bool imp = o->implicit != 0;
  std::vector<double> &tmp = imp ? o->rhsio[idr] : texplt;
  const double coe2 = alp * dt;
  const int nxi = idr == 1 ? o->nxi() : 1;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = nyi; j <= ny; ++j)
      for (int i = nxi; i <= nx; ++i) {
        const int64_t c = o->id(i, j, k);
        const double rhsc = texplt[c], rhsl = o->explt0[idr][c];
        double r = (gam * rhsc + roh * rhsl) * dt;
        if (imp) r = r + coe2 * o->rhsio[idr][c] + 0.5 * coe2 * o->adv[idr][c];
        o->explt0[idr][c] = rhsc;
        double pgm;
        if (idr == 1)
          pgm = (F(pr, i, j, k) - F(pr, o->im(i), j, k)) * (alp * dt * o->dxi);
        else if (idr == 2)
          pgm = (F(pr, i, j, k) - F(pr, i, j - 1, k)) * (alp * dt * o->dyci[j]);
        else
          pgm = (F(pr, i, j, k) - F(pr, i, j, o->km(k))) * (alp * dt * o->dzi);
        r -= pgm;
        if (o->gravdir == idr) r += o->rhostg[idr][c] * (alp * dt * o->f_a);
        tmp[c] = r;
      }
  if (idr == 1 && !o->coupled) {  // NFLOW = 1 without a TG section (:218)
    double dpgrns = 0.0;
    if (o->flowdrvtp == 1) {
      double s = 0.0;
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          for (int k = 1; k <= nz; ++k) s += tmp[o->id(i, j, k)] / o->dyfi[j];
      dpgrns = s / o->volm;
    } else if (o->flowdrvtp == 2) {
      dpgrns = -0.5 * o->cfgv * alp * dt;
    }
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) tmp[o->id(i, j, k)] -= dpgrns;
  }
}

// FFTPACK RFFTF / RFFTB by their documented definitions, through the complex
// DFT: forward r(1) = sum x, r(2m) = sum x cos, r(2m+1) = -sum x sin,
// r(n) = sum (-1)^i x for even n; backward the unnormalised synthesis.
void rfftf(const oracle_dft *f, int n, double *x, double *w) {
  double *in = w, *out = w + 2 * n, *tmp = w + 4 * n;
  for (int i = 0; i < n; ++i) { in[2 * i] = x[i]; in[2 * i + 1] = 0.0; }
  oracle_dft_run(f, in, out, -1, tmp);
  x[0] = out[0];
  for (int m = 1; 2 * m < n; ++m) { x[2 * m - 1] = out[2 * m]; x[2 * m] = out[2 * m + 1]; }
  if (n % 2 == 0) x[n - 1] = out[n];
}
void rfftb(const oracle_dft *f, int n, double *x, double *w) {
  double *in = w, *out = w + 2 * n, *tmp = w + 4 * n;
  in[0] = x[0]; in[1] = 0.0;
  for (int m = 1; 2 * m < n; ++m) {
    in[2 * m] = x[2 * m - 1]; in[2 * m + 1] = x[2 * m];
    in[2 * (n - m)] = x[2 * m - 1]; in[2 * (n - m) + 1] = -x[2 * m];
  }
  if (n % 2 == 0) { in[n] = x[n - 1]; in[n + 1] = 0.0; }
  oracle_dft_run(f, in, out, +1, tmp);
  for (int i = 0; i < n; ++i) x[i] = out[2 * i];
}
// FFTPACK_ROOT_1D, LP = 1 (src/possion3d_fishpack_reform.f90:98-110).
std::vector<double> roots_periodic(int l, double c) {
  std::vector<double> rt(l + 1, 0.0);  // 1-based
  const double dx = M_PI / (2.0 * (double)l);
  rt[1] = 0.0;
  rt[l] = -4.0 * c;
  for (int i = 3; i <= l; i += 2) {
    const double s = std::sin((double)(i - 1) * dx);
    rt[i - 1] = -4.0 * c * s * s;
    rt[i] = rt[i - 1];
  }
  return rt;
}

// FFTPACK_ROOT_1D for LP = 2..5 (src/possion3d_fishpack_reform.f90:104-163):
// XRT(I) = -4 c sin^2((I - DI) DX), DX = pi / (2 (L + LRDEL)); returns the
// final SCALX that divides the backward transform's result.
std::vector<double> roots_nonperiodic(int lp, int l, double c, double &scalx) {
  const int lrdel = ((lp - 1) * (lp - 3) * (lp - 5)) / 3;
  const double sc = (double)(l + lrdel), dx = M_PI / (2.0 * sc);
  const double di = lp == 2 ? 0.0 : (lp == 4 ? 1.0 : 0.5);
  std::vector<double> rt(l + 1, 0.0);
  for (int i = 1; i <= l; ++i) {
    const double s = std::sin(((double)i - di) * dx);
    rt[i] = -4.0 * c * s * s;
  }
  scalx = (lp == 3 || lp == 5) ? 4.0 * sc : 2.0 * sc;
  return rt;
}

// The real transforms of FFTPACK (libs/fishpack4.1/fftpack.f, the FFTPACK 4
// library FISHPACK 4.1 ships) as direct sums from their documented
// definitions, x 0-based here (x[K - 1] = X(K)): SINT (self-inverse up to
// 2 (N + 1)), SINQF / SINQB and COSQF / COSQB (inverse pairs up to 4 N), COST
// (self-inverse up to 2 (N - 1)).  fwd selects SINQF / COSQF over SINQB /
// COSQB.  O(N^2): test-infrastructure sizes only.
void fftpack_real(int lp, bool fwd, int n, double *x, double *tmp) {
  for (int i = 1; i <= n; ++i) {
    double s = 0.0;
    switch (lp) {
      case 2:  // SINT
        for (int k = 1; k <= n; ++k) s += 2.0 * x[k - 1] * std::sin((double)k * i * M_PI / (n + 1));
        break;
      case 3:
        if (fwd) {  // SINQF
          s = ((i - 1) % 2 ? -1.0 : 1.0) * x[n - 1];
          for (int k = 1; k <= n - 1; ++k) s += 2.0 * x[k - 1] * std::sin((2.0 * i - 1.0) * k * M_PI / (2.0 * n));
        } else {  // SINQB
          for (int k = 1; k <= n; ++k) s += 4.0 * x[k - 1] * std::sin((2.0 * k - 1.0) * i * M_PI / (2.0 * n));
        }
        break;
      case 4:  // COST
        s = x[0] + ((i - 1) % 2 ? -1.0 : 1.0) * x[n - 1];
        for (int k = 2; k <= n - 1; ++k) s += 2.0 * x[k - 1] * std::cos((double)(k - 1) * (i - 1) * M_PI / (n - 1));
        break;
      case 5:
        if (fwd) {  // COSQF
          s = x[0];
          for (int k = 2; k <= n; ++k) s += 2.0 * x[k - 1] * std::cos((2.0 * i - 1.0) * (k - 1) * M_PI / (2.0 * n));
        } else {  // COSQB
          for (int k = 1; k <= n; ++k) s += 4.0 * x[k - 1] * std::cos((2.0 * k - 1.0) * (i - 1) * M_PI / (2.0 * n));
        }
        break;
    }
    tmp[i - 1] = s;
  }
  std::copy(tmp, tmp + n, x);
}

// The quarter-wave pairs (LP 5 COSQF / COSQB, LP 3 SINQF / SINQB) in
// O(N log N) through the N-point complex DFT, by Makhoul's even-odd
// reordering (IEEE Trans. ASSP 28 (1980) 27-34); q_m = exp(-i pi m / (2N)):
//   COSQB(X)_k = 4 Re(q_k V_k), V = DFT(v), v_n = X_{2n}, v_{N-1-n} = X_{2n+1};
//   COSQF(x)_{2n} = Re w_n, COSQF(x)_{2n+1} = Re w_{N-1-n},
//     w = inverse DFT (unnormalised) of conj(q_m) (x_m - i x_{N-m}), x_N = 0;
//   SINQF(x)_k = (-1)^k COSQF(x reversed)_k;  SINQB(X)_k = COSQB((-1)^n X_n)_{N-1-k}.
// w: 6 N doubles of scratch.  N even.
void qwave_fast(int lp, bool fwd, int n, double *x, const oracle_dft *f, double *w) {
  const bool sinq = lp == 3;
  double *in = w, *out = w + 2 * n, *tmp = w + 4 * n;
  auto qc = [&](int m) { return std::cos(M_PI * m / (2.0 * n)); };
  auto qs = [&](int m) { return -std::sin(M_PI * m / (2.0 * n)); };
  if (fwd) {
    for (int m = 0; m < n; ++m) {
      const double a = x[sinq ? n - 1 - m : m], b = m ? x[sinq ? m - 1 : n - m] : 0.0;
      in[2 * m] = qc(m) * a - qs(m) * b;        // conj(q) (a - i b)
      in[2 * m + 1] = -qs(m) * a - qc(m) * b;
    }
    oracle_dft_run(f, in, out, +1, tmp);
    for (int m = 0; m < n; ++m) {
      const int nn = (m & 1) ? n - 1 - (m >> 1) : (m >> 1);
      const double y = out[2 * nn];
      x[m] = (sinq && (m & 1)) ? -y : y;
    }
  } else {
    std::vector<double> xs(x, x + n);
    if (sinq)
      for (int m = 1; m < n; m += 2) xs[m] = -xs[m];
    for (int nn = 0; nn < n; ++nn) {
      const int q = 2 * nn < n ? 2 * nn : 2 * (n - 1 - nn) + 1;
      in[2 * nn] = xs[q];
      in[2 * nn + 1] = 0.0;
    }
    oracle_dft_run(f, in, out, -1, tmp);
    for (int m = 0; m < n; ++m) {
      const int kk = sinq ? n - 1 - m : m;
      x[m] = 4.0 * (qc(kk) * out[2 * kk] - qs(kk) * out[2 * kk + 1]);
    }
  }
}

// Lines longer than this take the quarter-wave pairs through the DFT (the
// GPU parity cases, shorter, keep the direct sums as an independent check).
constexpr int kQwaveFastMin = 64;

// FISHPACK_POIS3D_SIMPLE (src/possion3d_fishpack_reform.f90:431-547) for
// periodic z and the x boundary type lpx: RHSLLPHI -> DPH (interior), ghosts
// by copy.
void fishpack_pois3d(oracle_io *o) {
  const int l = o->nx, m = o->nz, ng = o->ny;
  std::vector<double> fr((size_t)l * m * ng);  // FR(I, K, J): x fastest, then z, then y
  auto FR = [&](int i, int k, int j) -> double & { return fr[(size_t)(i - 1) + (size_t)l * ((k - 1) + (size_t)m * (j - 1))]; };
  for (int j = 1; j <= ng; ++j)
    for (int k = 1; k <= m; ++k)
      for (int i = 1; i <= l; ++i) FR(i, k, j) = F(rhsllphi, i, j, k);
  double scalx = (double)l;
  const std::vector<double> xrt = o->lpx == 1 ? roots_periodic(l, o->dxqi)
                                              : roots_nonperiodic(o->lpx, l, o->dxqi, scalx);
  const std::vector<double> yrt = roots_periodic(m, o->dzqi);
  const int nmax = std::max(l, m);
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<double> w(6 * nmax), t(nmax);
#pragma omp for schedule(static)
    for (int j = 1; j <= ng; ++j) {
      for (int k = 1; k <= m; ++k) {
        for (int i = 1; i <= l; ++i) t[i - 1] = FR(i, k, j);
        if (o->lpx == 1)
          rfftf(o->dftx, l, t.data(), w.data());
        else if ((o->lpx == 3 || o->lpx == 5) && l > kQwaveFastMin)
          qwave_fast(o->lpx, true, l, t.data(), o->dftx, w.data());
        else
          fftpack_real(o->lpx, true, l, t.data(), w.data());
        for (int i = 1; i <= l; ++i) FR(i, k, j) = t[i - 1];
      }
      for (int i = 1; i <= l; ++i) {
        for (int k = 1; k <= m; ++k) t[k - 1] = FR(i, k, j);
        rfftf(o->dftz, m, t.data(), w.data());
        for (int k = 1; k <= m; ++k) FR(i, k, j) = t[k - 1];
      }
    }
  }
  // TRID0 per (x-slot, z-slot) along y (:490-505, :33-63).
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<double> bb(ng + 1), tt(ng + 1), dd(ng + 1);
#pragma omp for collapse(2) schedule(static)
    for (int k = 1; k <= m; ++k)
      for (int i = 1; i <= l; ++i) {
        for (int jy = 1; jy <= ng; ++jy) {
          bb[jy] = o->acph[jy] + xrt[i] + yrt[k];
          tt[jy] = FR(i, k, jy);
        }
        const int nr = ng, mm1 = nr - 1;
        double z = 1.0 / bb[1];
        dd[1] = o->apph[1] * z;
        tt[1] = tt[1] * z;
        for (int jy = 2; jy <= mm1; ++jy) {
          z = 1.0 / (bb[jy] - o->amph[jy] * dd[jy - 1]);
          dd[jy] = o->apph[jy] * z;
          tt[jy] = (tt[jy] - o->amph[jy] * tt[jy - 1]) * z;
        }
        z = bb[nr] - o->amph[nr] * dd[mm1];
        // the zero-shift mode takes TRID0's zero branch: the mean mode of
        // periodic x, the first COST mode
        const bool singular = (xrt[i] == 0.0 && yrt[k] == 0.0);
        if (!singular && std::fabs(z) > 1.0e-14)
          tt[nr] = (tt[nr] - o->amph[nr] * tt[mm1]) / z;
        else
          tt[nr] = 0.0;
        for (int jy = mm1; jy >= 1; --jy) tt[jy] = tt[jy] - dd[jy] * tt[jy + 1];
        for (int jy = 1; jy <= ng; ++jy) FR(i, k, jy) = tt[jy];
      }
  }
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<double> w(6 * nmax), t(nmax);
#pragma omp for schedule(static)
    for (int j = 1; j <= ng; ++j) {
      for (int i = 1; i <= l; ++i) {
        for (int k = 1; k <= m; ++k) t[k - 1] = FR(i, k, j);
        rfftb(o->dftz, m, t.data(), w.data());
        for (int k = 1; k <= m; ++k) FR(i, k, j) = t[k - 1];
      }
      for (int k = 1; k <= m; ++k) {
        for (int i = 1; i <= l; ++i) t[i - 1] = FR(i, k, j);
        if (o->lpx == 1)
          rfftb(o->dftx, l, t.data(), w.data());
        else if ((o->lpx == 3 || o->lpx == 5) && l > kQwaveFastMin)
          qwave_fast(o->lpx, false, l, t.data(), o->dftx, w.data());
        else
          fftpack_real(o->lpx, false, l, t.data(), w.data());
        for (int i = 1; i <= l; ++i) FR(i, k, j) = t[i - 1];
      }
    }
  }
  const double scal = scalx * (double)m;  // SCALX * SCALY
  std::fill(o->dph.begin(), o->dph.end(), 0.0);
  for (int j = 1; j <= ng; ++j)
    for (int k = 1; k <= m; ++k)
      for (int i = 1; i <= l; ++i) F(dph, i, j, k) = FR(i, k, j) / scal;
  bc_wall_copy(o, o->dph);
}


// ------------------------------------------------------------- semi-implicit viscous scheme
// AMVR/APVR of TDMA_COEF (src/TDMA_COEF.f90:77-116), channel: u and w (IDR 1,
// 3) with the wall rows of the half-cell distance (AMVR1, APVRN), v (IDR 2)
// rows 2..ny with row 1 the identity.
void vis_ycoef(oracle_io *o) {
  const int ny = o->ny;
  o->amvr13.assign(ny + 2, 0.0); o->apvr13.assign(ny + 2, 0.0);
  o->amvr2.assign(ny + 2, 0.0); o->apvr2.assign(ny + 2, 0.0);
  for (int j = 2; j <= ny - 1; ++j) {
    o->amvr13[j] = o->dyfi[j] * o->dyci[j];
    o->apvr13[j] = o->dyfi[j] * o->dyci[j + 1];
  }
  double ucaj = 4.0 / (2.0 / o->dyci[2] + 1.0 / o->dyfi[1]);
  o->apvr13[1] = ucaj * o->dyci[2];
  o->amvr1 = ucaj * (2.0 * o->dyfi[1]);
  ucaj = 4.0 / (2.0 / o->dyci[ny] + 1.0 / o->dyfi[ny]);
  o->amvr13[ny] = ucaj * o->dyci[ny];
  o->apvrn = ucaj * (2.0 * o->dyfi[ny]);
  for (int j = 2; j <= ny; ++j) {
    o->amvr2[j] = o->dyfi[j - 1] * o->dyci[j];
    o->apvr2[j] = o->dyfi[j] * o->dyci[j];
  }
}

// DENSITY_implicit_add (src/MASSFLUX_CALC_IO.f90:316-399): DRHOI_STG = 1/rho_stag
// (new and old average) - 1/rho_stag (old density only).
void density_implicit_add(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int c = 1; c <= 3; ++c) std::fill(o->drhoi[c].begin(), o->drhoi[c].end(), 0.0);
  if (!o->thermal) return;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const int imm = o->im(i), kmm = o->km(k);
        double den = (F(dd0, i, j, k) + F(dd0, imm, j, k)) * XND2CL;
        FC(drhoi, 1, i, j, k) = 1.0 / FC(rhostg, 1, i, j, k) - 1.0 / den;
        den = (F(dd0, i, j, k) + F(dd0, i, j, kmm)) * ZND2CL;
        FC(drhoi, 3, i, j, k) = 1.0 / FC(rhostg, 3, i, j, k) - 1.0 / den;
        if (j >= 2) {
          den = o->wff[j] * F(dd0, i, j, k) + o->wfb[j] * F(dd0, i, j - 1, k);
          FC(drhoi, 2, i, j, k) = 1.0 / FC(rhostg, 2, i, j, k) - 1.0 / den;
        }
      }
}

// VISCOUS_PAR_EXPLT_X/Y/Z_io (channel): the viscous terms split into the
// explicit part (added to the convection term in tmp), the part treated
// implicitly by MOMFA_io (rhsio) and the density correction of that part
// (adv, zero unless thermal).  Normal stresses use VISCOUSITY, shear stresses
// MU_STG, as the reference writes them.
void viscous_par(oracle_io *o, int idr, std::vector<double> &tmp) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double cv = o->cvisc, dxi = o->dxi, dzi = o->dzi;
  std::fill(o->rhsio[idr].begin(), o->rhsio[idr].end(), 0.0);  // RHS_io = 0
  const int j0 = idr == 2 ? 2 : 1;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = j0; j <= ny; ++j) {
      const int jp = j + 1, jm = j - 1, kpp = o->kp(k), kmm = o->km(k);
      for (int i = 1; i <= nx; ++i) {
        const int ipp = o->ip(i), imm = o->im(i);
        double ex, im, ad;
        if (idr == 1) {  // src/VISCOUS_X_EXPLICIT_io.f90:150-280
          const double coe1 = -2.0 / 3.0 * dxi * cv, coe2 = o->dyfi[j] * cv, coe32 = dzi * cv;
          double dudx = (FC(q, 1, ipp, j, k) - FC(q, 1, i, j, k)) * dxi;
          double dvdy = (FC(q, 2, i, jp, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
          double dwdz = (FC(q, 3, i, j, kpp) - FC(q, 3, i, j, k)) * dzi;
          const double t11f_ex = F(mu, i, j, k) * (dvdy + dwdz), t11f_im = F(mu, i, j, k) * dudx;
          dudx = (FC(g, 1, ipp, j, k) * FC(drhoi, 1, ipp, j, k) - FC(g, 1, i, j, k) * FC(drhoi, 1, i, j, k)) * dxi;
          const double t11f_ad = F(mu, i, j, k) * dudx;
          dudx = (FC(q, 1, i, j, k) - FC(q, 1, imm, j, k)) * dxi;
          dvdy = (FC(q, 2, imm, jp, k) - FC(q, 2, imm, j, k)) * o->dyfi[j];
          dwdz = (FC(q, 3, imm, j, kpp) - FC(q, 3, imm, j, k)) * dzi;
          const double t11b_ex = F(mu, imm, j, k) * (dvdy + dwdz), t11b_im = F(mu, imm, j, k) * dudx;
          dudx = (FC(g, 1, i, j, k) * FC(drhoi, 1, i, j, k) - FC(g, 1, imm, j, k) * FC(drhoi, 1, imm, j, k)) * dxi;
          const double t11b_ad = F(mu, imm, j, k) * dudx;
          const double d11_ex = (t11f_ex - t11b_ex) * coe1;
          const double d11_im = (t11f_im - t11b_im) * coe1 * (-2.0);
          const double d11_ad = (t11f_ad - t11b_ad) * coe1 * (-2.0);
          const double vis12p = FC(mustg, 1, i, jp, k);
          double dvdx = (FC(q, 2, i, jp, k) - FC(q, 2, imm, jp, k)) * dxi;
          double dudy = (FC(q, 1, i, jp, k) - FC(q, 1, i, j, k)) * o->dyci[jp];
          const double t12f_ex = vis12p * dvdx, t12f_im = vis12p * dudy;
          dudy = (FC(g, 1, i, jp, k) * FC(drhoi, 1, i, jp, k) - FC(g, 1, i, j, k) * FC(drhoi, 1, i, j, k)) * o->dyci[jp];
          const double t12f_ad = vis12p * dudy;
          const double vis12c = FC(mustg, 1, i, j, k);
          dudy = (FC(q, 1, i, j, k) - FC(q, 1, i, jm, k)) * o->dyci[j];
          dvdx = (FC(q, 2, i, j, k) - FC(q, 2, imm, j, k)) * dxi;
          const double t12b_ex = vis12c * dvdx, t12b_im = vis12c * dudy;
          dudy = (FC(g, 1, i, j, k) * FC(drhoi, 1, i, j, k) - FC(g, 1, i, jm, k) * FC(drhoi, 1, i, jm, k)) * o->dyci[j];
          const double t12b_ad = vis12c * dudy;
          const double d12_ex = (t12f_ex - t12b_ex) * coe2, d12_im = (t12f_im - t12b_im) * coe2;
          const double d12_ad = (t12f_ad - t12b_ad) * coe2;
          const double vis13p = FC(mustg, 2, i, j, kpp);
          double dudz = (FC(q, 1, i, j, kpp) - FC(q, 1, i, j, k)) * dzi;
          double dwdx = (FC(q, 3, i, j, kpp) - FC(q, 3, imm, j, kpp)) * dxi;
          const double t13f_ex = vis13p * dwdx, t13f_im = vis13p * dudz;
          // the density part of tau13 differences Q_io (not G_io), as written (:251-252)
          dudz = (FC(q, 1, i, j, kpp) * FC(drhoi, 1, i, j, kpp) - FC(q, 1, i, j, k) * FC(drhoi, 1, i, j, k)) * dzi;
          const double t13f_ad = vis13p * dudz;
          const double vis13c = FC(mustg, 2, i, j, k);
          dudz = (FC(q, 1, i, j, k) - FC(q, 1, i, j, kmm)) * dzi;
          dwdx = (FC(q, 3, i, j, k) - FC(q, 3, imm, j, k)) * dxi;
          const double t13b_ex = vis13c * dwdx, t13b_im = vis13c * dudz;
          dudz = (FC(q, 1, i, j, k) * FC(drhoi, 1, i, j, k) - FC(q, 1, i, j, kmm) * FC(drhoi, 1, i, j, kmm)) * dzi;
          const double t13b_ad = vis13c * dudz;
          const double d13_ex = (t13f_ex - t13b_ex) * coe32, d13_im = (t13f_im - t13b_im) * coe32;
          const double d13_ad = (t13f_ad - t13b_ad) * coe32;
          ex = d11_ex + d12_ex + d13_ex;
          im = d11_im + d12_im + d13_im;
          ad = d11_ad + d12_ad + d13_ad;
        } else if (idr == 2) {  // src/VISCOUS_Y_EXPLICIT_io.f90:296-417
          const double coe1 = dxi * cv, coe3 = dzi * cv, coe2 = -2.0 / 3.0 * o->dyci[j] * cv;
          double dudx = (FC(q, 1, ipp, j, k) - FC(q, 1, i, j, k)) * dxi;
          double dvdy = (FC(q, 2, i, jp, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
          double dwdz = (FC(q, 3, i, j, kpp) - FC(q, 3, i, j, k)) * dzi;
          const double t22f_ex = F(mu, i, j, k) * (dudx + dwdz), t22f_im = F(mu, i, j, k) * dvdy;
          dvdy = (FC(g, 2, i, jp, k) * FC(drhoi, 2, i, jp, k) - FC(g, 2, i, j, k) * FC(drhoi, 2, i, j, k)) * o->dyfi[j];
          const double t22f_ad = F(mu, i, j, k) * dvdy;
          dudx = (FC(q, 1, ipp, jm, k) - FC(q, 1, i, jm, k)) * dxi;
          dvdy = (FC(q, 2, i, j, k) - FC(q, 2, i, jm, k)) * o->dyfi[jm];
          dwdz = (FC(q, 3, i, jm, kpp) - FC(q, 3, i, jm, k)) * dzi;
          const double t22b_ex = F(mu, i, jm, k) * (dudx + dwdz), t22b_im = F(mu, i, jm, k) * dvdy;
          dvdy = (FC(g, 2, i, j, k) * FC(drhoi, 2, i, j, k) - FC(g, 2, i, jm, k) * FC(drhoi, 2, i, jm, k)) * o->dyfi[jm];
          const double t22b_ad = F(mu, i, jm, k) * dvdy;
          const double d22_ex = (t22f_ex - t22b_ex) * coe2;
          const double d22_im = (t22f_im - t22b_im) * coe2 * (-2.0);
          const double d22_ad = (t22f_ad - t22b_ad) * coe2 * (-2.0);
          const double vis21p = FC(mustg, 1, ipp, j, k);
          double dvdx = (FC(q, 2, ipp, j, k) - FC(q, 2, i, j, k)) * dxi;
          double dudy = (FC(q, 1, ipp, j, k) - FC(q, 1, ipp, jm, k)) * o->dyci[j];
          const double t21f_ex = vis21p * dudy, t21f_im = vis21p * dvdx;
          dvdx = (FC(g, 2, ipp, j, k) * FC(drhoi, 2, ipp, j, k) - FC(g, 2, i, j, k) * FC(drhoi, 2, i, j, k)) * dxi;
          const double t21f_ad = vis21p * dvdx;
          const double vis21c = FC(mustg, 1, i, j, k);
          dvdx = (FC(q, 2, i, j, k) - FC(q, 2, imm, j, k)) * dxi;
          dudy = (FC(q, 1, i, j, k) - FC(q, 1, i, jm, k)) * o->dyci[j];
          const double t21b_ex = vis21c * dudy, t21b_im = vis21c * dvdx;
          dvdx = (FC(g, 2, i, j, k) * FC(drhoi, 2, i, j, k) - FC(g, 2, imm, j, k) * FC(drhoi, 2, imm, j, k)) * dxi;
          const double t21b_ad = vis21c * dvdx;
          const double d21_ex = (t21f_ex - t21b_ex) * coe1, d21_im = (t21f_im - t21b_im) * coe1;
          const double d21_ad = (t21f_ad - t21b_ad) * coe1;
          const double vis23p = FC(mustg, 3, i, j, kpp);
          double dvdz = (FC(q, 2, i, j, kpp) - FC(q, 2, i, j, k)) * dzi;
          double dwdy = (FC(q, 3, i, j, kpp) - FC(q, 3, i, jm, kpp)) * o->dyci[j];
          const double t23f_ex = vis23p * dwdy, t23f_im = vis23p * dvdz;
          dvdz = (FC(g, 2, i, j, kpp) * FC(drhoi, 2, i, j, kpp) - FC(g, 2, i, j, k) * FC(drhoi, 2, i, j, k)) * dzi;
          const double t23f_ad = vis23p * dvdz;
          const double vis23c = FC(mustg, 3, i, j, k);
          dvdz = (FC(q, 2, i, j, k) - FC(q, 2, i, j, kmm)) * dzi;
          dwdy = (FC(q, 3, i, j, k) - FC(q, 3, i, jm, k)) * o->dyci[j];
          const double t23b_ex = vis23c * dwdy, t23b_im = vis23c * dvdz;
          dvdz = (FC(g, 2, i, j, k) * FC(drhoi, 2, i, j, k) - FC(g, 2, i, j, kmm) * FC(drhoi, 2, i, j, kmm)) * dzi;
          const double t23b_ad = vis23c * dvdz;
          const double d23_ex = (t23f_ex - t23b_ex) * coe3, d23_im = (t23f_im - t23b_im) * coe3;
          const double d23_ad = (t23f_ad - t23b_ad) * coe3;
          ex = d21_ex + d22_ex + d23_ex;
          im = d21_im + d22_im + d23_im;
          ad = d21_ad + d22_ad + d23_ad;
        } else {  // src/VISCOUS_Z_EXPLICIT_io.f90:324-449
          const double coe1 = dxi * cv, coe3 = -2.0 / 3.0 * dzi * cv, coe2 = o->dyfi[j] * cv;
          double dudx = (FC(q, 1, ipp, j, k) - FC(q, 1, i, j, k)) * dxi;
          double dvdy = (FC(q, 2, i, jp, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
          double dwdz = (FC(q, 3, i, j, kpp) - FC(q, 3, i, j, k)) * dzi;
          const double t33f_ex = F(mu, i, j, k) * (dudx + dvdy), t33f_im = F(mu, i, j, k) * dwdz;
          dwdz = (FC(g, 3, i, j, kpp) * FC(drhoi, 3, i, j, kpp) - FC(g, 3, i, j, k) * FC(drhoi, 3, i, j, k)) * dzi;
          const double t33f_ad = F(mu, i, j, k) * dwdz;
          dudx = (FC(q, 1, ipp, j, kmm) - FC(q, 1, i, j, kmm)) * dxi;
          dvdy = (FC(q, 2, i, jp, kmm) - FC(q, 2, i, j, kmm)) * o->dyfi[j];
          dwdz = (FC(q, 3, i, j, k) - FC(q, 3, i, j, kmm)) * dzi;
          const double t33b_ex = F(mu, i, j, kmm) * (dudx + dvdy), t33b_im = F(mu, i, j, kmm) * dwdz;
          dwdz = (FC(g, 3, i, j, k) * FC(drhoi, 3, i, j, k) - FC(g, 3, i, j, kmm) * FC(drhoi, 3, i, j, kmm)) * dzi;
          const double t33b_ad = F(mu, i, j, kmm) * dwdz;
          const double d33_ex = (t33f_ex - t33b_ex) * coe3;
          const double d33_im = (t33f_im - t33b_im) * coe3 * (-2.0);
          const double d33_ad = (t33f_ad - t33b_ad) * coe3 * (-2.0);
          const double vis31p = FC(mustg, 2, ipp, j, k);
          double dwdx = (FC(q, 3, ipp, j, k) - FC(q, 3, i, j, k)) * dxi;
          double dudz = (FC(q, 1, ipp, j, k) - FC(q, 1, ipp, j, kmm)) * dzi;
          const double t31f_ex = vis31p * dudz, t31f_im = vis31p * dwdx;
          dwdx = (FC(g, 3, ipp, j, k) * FC(drhoi, 3, ipp, j, k) - FC(g, 3, i, j, k) * FC(drhoi, 3, i, j, k)) * dxi;
          const double t31f_ad = vis31p * dwdx;
          const double vis31c = FC(mustg, 2, i, j, k);
          dwdx = (FC(q, 3, i, j, k) - FC(q, 3, imm, j, k)) * dxi;
          dudz = (FC(q, 1, i, j, k) - FC(q, 1, i, j, kmm)) * dzi;
          const double t31b_ex = vis31c * dudz, t31b_im = vis31c * dwdx;
          dwdx = (FC(g, 3, i, j, k) * FC(drhoi, 3, i, j, k) - FC(g, 3, imm, j, k) * FC(drhoi, 3, imm, j, k)) * dxi;
          const double t31b_ad = vis31c * dwdx;
          const double d31_ex = (t31f_ex - t31b_ex) * coe1, d31_im = (t31f_im - t31b_im) * coe1;
          const double d31_ad = (t31f_ad - t31b_ad) * coe1;
          const double vis32p = FC(mustg, 3, i, jp, k);
          double dwdy = (FC(q, 3, i, jp, k) - FC(q, 3, i, j, k)) * o->dyci[jp];
          double dvdz = (FC(q, 2, i, jp, k) - FC(q, 2, i, jp, kmm)) * dzi;
          const double t32f_ex = vis32p * dvdz, t32f_im = vis32p * dwdy;
          dwdy = (FC(g, 3, i, jp, k) * FC(drhoi, 3, i, jp, k) - FC(g, 3, i, j, k) * FC(drhoi, 3, i, j, k)) * o->dyci[jp];
          const double t32f_ad = vis32p * dwdy;
          const double vis32c = FC(mustg, 3, i, j, k);
          dwdy = (FC(q, 3, i, j, k) - FC(q, 3, i, jm, k)) * o->dyci[j];
          dvdz = (FC(q, 2, i, j, k) - FC(q, 2, i, j, kmm)) * dzi;
          const double t32b_ex = vis32c * dvdz, t32b_im = vis32c * dwdy;
          dwdy = (FC(g, 3, i, j, k) * FC(drhoi, 3, i, j, k) - FC(g, 3, i, jm, k) * FC(drhoi, 3, i, jm, k)) * o->dyci[j];
          const double t32b_ad = vis32c * dwdy;
          const double d32_ex = (t32f_ex - t32b_ex) * coe2, d32_im = (t32f_im - t32b_im) * coe2;
          const double d32_ad = (t32f_ad - t32b_ad) * coe2;
          ex = d31_ex + d32_ex + d33_ex;
          im = d31_im + d32_im + d33_im;
          ad = d31_ad + d32_ad + d33_ad;
        }
        const int64_t c = o->id(i, j, k);
        tmp[c] = ex + tmp[c];
        o->rhsio[idr][c] = im;
        o->adv[idr][c] = ad;
      }
    }
}

// TDMAIJI_CYC (src/TDMAIJI_CYC.f90:67-157) for one cyclic line of n >= 3
// unknowns: a x(i-1) + b x(i) + c x(i+1) = r, indices modulo n.  The first
// n-1 unknowns are written as g1 + g2 x(n) (two right-hand sides sharing one
// elimination); the last row then gives x(n).  r is overwritten by x.
void tdma_cyc(int n, const double *a, const double *b, const double *c, double *r, double *h0, double *g1,
              double *g2) {
  h0[0] = c[0] / b[0];
  g1[0] = r[0] / b[0];
  g2[0] = -a[0] / b[0];
  for (int i = 1; i <= n - 3; ++i) {
    const double pp = 1.0 / (b[i] - h0[i - 1] * a[i]);
    const double qq1 = g1[i - 1] * a[i], qq2 = g2[i - 1] * a[i];
    h0[i] = c[i] * pp;
    g1[i] = (r[i] - qq1) * pp;
    g2[i] = -qq2 * pp;
  }
  {
    const int i = n - 2;
    const double pp = 1.0 / (b[i] - h0[i - 1] * a[i]);
    const double qq1 = g1[i - 1] * a[i], qq2 = g2[i - 1] * a[i];
    g1[i] = (r[i] - qq1) * pp;
    g2[i] = (-c[i] - qq2) * pp;
  }
  for (int i = n - 3; i >= 0; --i) {
    g1[i] = -h0[i] * g1[i + 1] + g1[i];
    g2[i] = -h0[i] * g2[i + 1] + g2[i];
  }
  const int l = n - 1;
  const double pp = r[l] - c[l] * g1[0] - a[l] * g1[l - 1];
  const double qq = b[l] + c[l] * g2[0] + a[l] * g2[l - 1];
  r[l] = pp / qq;
  for (int i = l - 1; i >= 0; --i) r[i] = g1[i] + g2[i] * r[l];
}

// TDMAIJJ_nonCYC (src/TDMAIJJ_nonCYC.f90:67-123) with zero boundary values:
// Thomas sweeps; a[0] and c[n-1] are not used.  r is overwritten by x.
void tdma_noncyc(int n, const double *a, const double *b, const double *c, double *r, double *h, double *g) {
  h[0] = c[0] / b[0];
  g[0] = r[0] / b[0];
  for (int j = 1; j <= n - 2; ++j) {
    const double pp = 1.0 / (b[j] - h[j - 1] * a[j]);
    h[j] = c[j] * pp;
    g[j] = (r[j] - a[j] * g[j - 1]) * pp;
  }
  const int l = n - 1;
  const double pp = 1.0 / (b[l] - h[l - 1] * a[l]);
  g[l] = (r[l] - a[l] * g[l - 1]) * pp;
  r[l] = g[l];
  for (int j = l - 1; j >= 0; --j) r[j] = g[j] - h[j] * r[j + 1];
}

// MOMFA_io(NS, IDR) (src/MOMFA_io.f90:17-377): (1 - A_x)(1 - A_z)(1 - A_y) dG
// = RHS_io with variable coefficients from VISCOUSITY, MU_STG and RHO_STG,
// then G += dG from row N2I.
void momfa(oracle_io *o, int ns, int idr) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double facoe = 0.5 * o->talp[ns] * o->dt * o->cvisc;
  const int n2i = idr == 2 ? 2 : 1;
  std::vector<double> &rhs = o->rhsio[idr];
  const std::vector<double> &rs = o->rhostg[idr];
  // MOMFA1_X_io (:48-142), periodic x
  {
    const double coe1 = facoe * 4.0 / 3.0 * o->dxqi, coe2 = facoe * o->dxqi;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
    for (int k = 1; k <= nz; ++k)
      for (int j = n2i; j <= ny; ++j) {
        std::vector<double> a(nx), b(nx), c(nx), r(nx), t0(nx), t1(nx), t2(nx);
        for (int i = 1; i <= nx; ++i) {
          const int imm = o->im(i), ipp = o->ip(i);
          double amu, apu;
          if (idr == 1) {
            amu = -coe1 * F(mu, imm, j, k);
            apu = -coe1 * F(mu, i, j, k);
          } else if (idr == 2) {
            amu = -coe2 * FC(mustg, 1, i, j, k);
            apu = -coe2 * FC(mustg, 1, ipp, j, k);
          } else {
            amu = -coe2 * FC(mustg, 2, i, j, k);
            apu = -coe2 * FC(mustg, 2, ipp, j, k);
          }
          a[i - 1] = amu / rs[o->id(imm, j, k)];
          c[i - 1] = apu / rs[o->id(ipp, j, k)];
          b[i - 1] = 1.0 - (amu + apu) / rs[o->id(i, j, k)];
          r[i - 1] = rhs[o->id(i, j, k)];
        }
        tdma_cyc(nx, a.data(), b.data(), c.data(), r.data(), t0.data(), t1.data(), t2.data());
        for (int i = 1; i <= nx; ++i) rhs[o->id(i, j, k)] = r[i - 1];
      }
  }
  // MOMFA2_Z_io (:145-231), periodic z (RCCI2 = 1 in a channel)
  {
    const double coe1 = facoe * 4.0 / 3.0 * o->dzqi, coe2 = facoe * o->dzqi;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
    for (int i = 1; i <= nx; ++i)
      for (int j = n2i; j <= ny; ++j) {
        std::vector<double> a(nz), b(nz), c(nz), r(nz), t0(nz), t1(nz), t2(nz);
        for (int k = 1; k <= nz; ++k) {
          const int kmm = o->km(k), kpp = o->kp(k);
          double amu, apu;
          if (idr == 1) {
            amu = -coe2 * FC(mustg, 2, i, j, k);
            apu = -coe2 * FC(mustg, 2, i, j, kpp);
          } else if (idr == 2) {
            amu = -coe2 * FC(mustg, 3, i, j, k);
            apu = -coe2 * FC(mustg, 3, i, j, kpp);
          } else {
            amu = -coe1 * F(mu, i, j, kmm);
            apu = -coe1 * F(mu, i, j, k);
          }
          a[k - 1] = amu / rs[o->id(i, j, kmm)];
          c[k - 1] = apu / rs[o->id(i, j, kpp)];
          b[k - 1] = 1.0 - (amu + apu) / rs[o->id(i, j, k)];
          r[k - 1] = rhs[o->id(i, j, k)];
        }
        tdma_cyc(nz, a.data(), b.data(), c.data(), r.data(), t0.data(), t1.data(), t2.data());
        for (int k = 1; k <= nz; ++k) rhs[o->id(i, j, k)] = r[k - 1];
      }
  }
  // MOMFA3_Y_io (:234-377), rows 1..ny for every component
  {
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) {
        std::vector<double> a(ny), b(ny), c(ny), r(ny), t0(ny), t1(ny);
        for (int j = 1; j <= ny; ++j) {
          double amu, apu, am, ap, den;
          if (idr == 1 || idr == 3) {
            const std::vector<double> &fmu = o->mustg[idr];
            const double coe2 = facoe;
            if (j == 1) {
              const double muqt = (F(mu, i, j, k) + F(mu, i, j - 1, k)) * 0.5;
              amu = -coe2 * o->amvr1 * muqt;
              apu = -coe2 * o->apvr13[j] * fmu[o->id(i, j + 1, k)];
              am = 0.0;
              ap = apu / rs[o->id(i, j + 1, k)];
            } else if (j == ny) {
              const double muqt = (F(mu, i, ny, k) + F(mu, i, ny + 1, k)) * 0.5;
              amu = -coe2 * o->amvr13[j] * fmu[o->id(i, j, k)];
              apu = -coe2 * o->apvrn * muqt;
              am = amu / rs[o->id(i, j - 1, k)];
              ap = 0.0;
            } else {
              amu = -coe2 * o->amvr13[j] * fmu[o->id(i, j, k)];
              apu = -coe2 * o->apvr13[j] * fmu[o->id(i, j + 1, k)];
              am = amu / rs[o->id(i, j - 1, k)];
              ap = apu / rs[o->id(i, j + 1, k)];
            }
            den = rs[o->id(i, j, k)];
          } else {
            const double coe1 = facoe * 4.0 / 3.0;
            amu = -coe1 * o->amvr2[j] * F(mu, i, j - 1, k);
            apu = -coe1 * o->apvr2[j] * F(mu, i, j, k);
            if (j == 1) {
              am = amu / rs[o->id(i, 0, k)];
              ap = apu / rs[o->id(i, 2, k)];
            } else {
              am = amu / rs[o->id(i, j - 1, k)];
              ap = apu / rs[o->id(i, j, k)];  // the v face j itself, as written (:349)
            }
            den = rs[o->id(i, j, k)];
          }
          a[j - 1] = am;
          c[j - 1] = ap;
          b[j - 1] = 1.0 - (amu + apu) / den;
          r[j - 1] = rhs[o->id(i, j, k)];
        }
        tdma_noncyc(ny, a.data(), b.data(), c.data(), r.data(), t0.data(), t1.data());
        for (int j = 1; j <= ny; ++j) rhs[o->id(i, j, k)] = r[j - 1];
      }
  }
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = n2i; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) FC(g, idr, i, j, k) = rhs[o->id(i, j, k)] + FC(g, idr, i, j, k);
}

// ------------------------------------------ coupled section: ghost columns
// The boundary operators (oracle_io_bc_*) work on (nz, ny + 2) planes; a
// coupled substep copies the ghost columns they read into the planes and
// writes their results back, so the columns hold the state.
void column_to_plane(oracle_io *o, const std::vector<double> &f, int i, int q) {
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 0; j <= o->ny + 1; ++j) o->bcp[q][o->pj(j, k)] = f[o->id(i, j, k)];
}
void plane_to_column(oracle_io *o, std::vector<double> &f, int i, int q) {
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 0; j <= o->ny + 1; ++j) f[o->id(i, j, k)] = o->bcp[q][o->pj(j, k)];
}

// Coupled momentum boundaries at the start of SOLVERRK3_MOM_IO (:19-24):
// BC_TINLET_FLOW from the TG arrays (ghost column 0 and the first face's u,
// G), then BC_COUTLET_MOM_RK3 on the outlet ghost column NCL1_io + 1.
void coupled_mom_bc(oracle_io *o, int ns) {
  const int nx = o->nx;
  oracle_io_bc_inlet(o, o->tg_nx, o->tg_u, o->tg_v, o->tg_w, o->tg_p);
  for (int c = 1; c <= 3; ++c) {
    plane_to_column(o, o->q[c], 0, ORC_P_IN_U + c - 1);
    plane_to_column(o, o->g[c], 0, ORC_P_IN_GX + c - 1);
  }
  plane_to_column(o, o->pr, 0, ORC_P_IN_P);
  plane_to_column(o, o->dd, 0, ORC_P_IN_RHO);
  for (int c = 1; c <= 3; ++c) {
    column_to_plane(o, o->q[c], nx + 1, ORC_P_OUT_U + c - 1);
    column_to_plane(o, o->g[c], nx + 1, ORC_P_OUT_GX + c - 1);
  }
  column_to_plane(o, o->dd, nx + 1, ORC_P_OUT_RHO);
  oracle_io_bc_outlet_mom(o, ns);
  for (int c = 1; c <= 3; ++c) {
    plane_to_column(o, o->q[c], nx + 1, ORC_P_OUT_U + c - 1);
    plane_to_column(o, o->g[c], nx + 1, ORC_P_OUT_GX + c - 1);
  }
}

// Coupled energy boundaries of SOLVERRK3_ENG_IO (:61-64): BC_TINLET_THERML
// (the reference state on ghost column 0, rows 0..ny+1) and
// BC_COUTLET_ENEG_RK3 on the outlet ghost column.
void coupled_eng_bc(oracle_io *o, int ns) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int k = 1; k <= nz; ++k)
    for (int j = 0; j <= ny + 1; ++j) {
      F(tt, 0, j, k) = 1.0;
      F(kk, 0, j, k) = 1.0;
      F(dd, 0, j, k) = 1.0;
      F(mu, 0, j, k) = 1.0;
      F(rhoh, 0, j, k) = 0.0;
      F(hh, 0, j, k) = 0.0;
    }
  column_to_plane(o, o->q[1], nx + 1, ORC_P_OUT_U);
  std::vector<double> *fs[6] = {&o->dd, &o->rhoh, &o->hh, &o->tt, &o->mu, &o->kk};
  const int qs[6] = {ORC_P_OUT_RHO, ORC_P_OUT_RHOH, ORC_P_OUT_H, ORC_P_OUT_T, ORC_P_OUT_MU, ORC_P_OUT_K};
  for (int a = 0; a < 6; ++a) column_to_plane(o, *fs[a], nx + 1, qs[a]);
  oracle_io_bc_outlet_eng(o, ns);
  for (int a = 0; a < 6; ++a) plane_to_column(o, *fs[a], nx + 1, qs[a]);
}

void mom_io(oracle_io *o, int ns) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int c = 1; c <= 3; ++c) o->g0[c] = o->g[c];  // :15
  if (o->coupled) coupled_mom_bc(o, ns);
  convection(o);
  if (o->implicit) {
    // visthemflg = 1 (:73-87): per component the split viscous terms, the
    // RHS and the factored solve that updates G
    viscous_par(o, 1, o->qtmp);
    rhs_mom(o, ns, 1, o->qtmp);
    momfa(o, ns, 1);
    viscous_par(o, 2, o->dphtmp);
    rhs_mom(o, ns, 2, o->dphtmp);
    momfa(o, ns, 2);
    viscous_par(o, 3, o->rhsz);
    rhs_mom(o, ns, 3, o->rhsz);
    momfa(o, ns, 3);
  } else {
    divg_u(o);
    viscous(o);
    rhs_mom(o, ns, 1, o->qtmp);
    rhs_mom(o, ns, 2, o->dphtmp);
    rhs_mom(o, ns, 3, o->rhsz);
    // MASSFLUX_CALC_IO (src/MASSFLUX_CALC_IO.f90:1-79)
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          if (i >= o->nxi()) FC(g, 1, i, j, k) += F(qtmp, i, j, k);
          FC(g, 3, i, j, k) += F(rhsz, i, j, k);
          if (j >= 2) FC(g, 2, i, j, k) += F(dphtmp, i, j, k);
        }
  }
  bc_wall_vec(o, o->g);
  // DIVG_io (src/DIVG.f90:60-150)
  const double coe0 = 1.0 / o->dt / o->talp[ns];
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double divx = (FC(g, 1, o->ip(i), j, k) - FC(g, 1, i, j, k)) * o->dxi;
        const double divy = (FC(g, 2, i, j + 1, k) - FC(g, 2, i, j, k)) * o->dyfi[j];
        const double divz = (FC(g, 3, i, j, o->kp(k)) - FC(g, 3, i, j, k)) * o->dzi;
        F(rhsllphi, i, j, k) = (divx + divy + divz + F(drho, i, j, k)) * coe0;
      }
  fishpack_pois3d(o);
  // PRCALC_io (src/PRESSURE_CORRECTION.f90:86-122); the semi-implicit branch
  // subtracts BE times the physical Poisson right-hand side (see the header)
  const double be = o->implicit ? 0.5 * o->talp[ns] * o->dt * o->cvisc : 0.0;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        if (o->implicit)
          F(pr, i, j, k) = F(pr, i, j, k) + F(dph, i, j, k) - be * F(rhsllphi, i, j, k);
        else
          F(pr, i, j, k) += F(dph, i, j, k);
      }
  bc_wall_copy(o, o->pr);
  // MASSFLUX_UPDATE_IO (src/VELO_CORRECTION.f90:107-185); coupled: the x
  // flux from NXI = 2 to NXE = NCL1_io + 1, the outlet face against the
  // ghost DPH_io(NCL1_io + 1), which no routine writes (zero)
  const double cx = o->dt * o->talp[ns] * o->dxi, cz = o->dt * o->talp[ns] * o->dzi;
  const int nxe = o->coupled ? nx + 1 : nx;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nxe; ++i) {
        if (i >= o->nxi()) FC(g, 1, i, j, k) -= (F(dph, i, j, k) - F(dph, o->im(i), j, k)) * cx;
        if (i > nx) continue;
        FC(g, 3, i, j, k) -= (F(dph, i, j, k) - F(dph, i, j, o->km(k))) * cz;
        if (j >= 2) FC(g, 2, i, j, k) -= (F(dph, i, j, k) - F(dph, i, j - 1, k)) * (o->dt * o->talp[ns] * o->dyci[j]);
      }
  bc_wall_vec(o, o->g);
}

void eng_io(oracle_io *o, int ns) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  o->mu0 = o->mu;  // :13-16 (DENSITY1 is never read)
  o->dd0 = o->dd;
  rhs_energy(o);
  const double coe1 = o->tgam[ns] * o->dt, coe0 = o->troh[ns] * o->dt;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const int64_t c = o->id(i, j, k);
        double r = o->rhoh[c] + coe1 * o->rhse[c] + coe0 * o->rhse0[c];
        r = std::fmin(o->rhohmax + 1.0e-14, r);  // limiter, thermoStat = table
        o->rhoh[c] = r;
        o->rhse0[c] = o->rhse[c];
      }
  int64_t bad = 0;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads()) reduction(+ : bad)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const int64_t c = o->id(i, j, k);
        // ENTHALPY_UPDATE, DENSITY_UPDATE, ENTHALPY_UPDATE
        double h = o->rhoh[c] / o->dd[c];
        double T, D;
        if (lookup_ht(o, h, T) && lookup_t(o, o->td, T, D))
          o->dd[c] = D;
        else
          ++bad;
        h = o->rhoh[c] / o->dd[c];
        o->hh[c] = h;
        // THERM_PROP_UPDATE (src/THERM_PROP_UPDATE.f90:129-205)
        if (o->shortcuts && std::fabs(h) < 1.0e-10) continue;  // properties kept
        double M, K;
        if (!lookup_ht(o, h, T) || !lookup_t(o, o->tm, T, M) || !lookup_t(o, o->tk, T, K) ||
            !lookup_t(o, o->td, T, D)) {
          ++bad;
          continue;
        }
        o->tt[c] = T;
        o->mu[c] = M;
        o->kk[c] = K;
        o->dd[c] = D;
      }
  o->bad += bad;
  if (o->coupled) coupled_eng_bc(o, ns);
  bc_wall_thermal(o);
}

std::vector<double> *field_ptr(oracle_io *o, int id) {
  switch (id) {
    case ORC_U: return &o->q[1];
    case ORC_V: return &o->q[2];
    case ORC_W: return &o->q[3];
    case ORC_P: return &o->pr;
    case ORC_PHI: return &o->dph;
    case ORC_RHSPHI: return &o->rhsllphi;
    case ORC_IO_GX: return &o->g[1];
    case ORC_IO_GY: return &o->g[2];
    case ORC_IO_GZ: return &o->g[3];
    case ORC_IO_G0X: return &o->g0[1];
    case ORC_IO_G0Y: return &o->g0[2];
    case ORC_IO_G0Z: return &o->g0[3];
    case ORC_IO_H: return &o->hh;
    case ORC_IO_T: return &o->tt;
    case ORC_IO_D: return &o->dd;
    case ORC_IO_MU: return &o->mu;
    case ORC_IO_K: return &o->kk;
    case ORC_IO_RHOH: return &o->rhoh;
    case ORC_IO_D0: return &o->dd0;
    case ORC_IO_MU0: return &o->mu0;
    case ORC_IO_DRHO: return &o->drho;
    case ORC_IO_EX0X: return &o->explt0[1];
    case ORC_IO_EX0Y: return &o->explt0[2];
    case ORC_IO_EX0Z: return &o->explt0[3];
    case ORC_IO_RHSE0: return &o->rhse0;
  }
  return nullptr;
}

double bulk(const oracle_io *o, const std::vector<double> &f) {
  double s = 0.0;
  for (int j = 1; j <= o->ny; ++j)
    for (int i = 1; i <= o->nx; ++i)
      for (int k = 1; k <= o->nz; ++k) s += f[o->id(i, j, k)] / o->dyfi[j];
  s /= o->dzi;
  return s / (o->area_inlet * (double)o->nx);
}

// VELO2MASSFLUX (src/INITIAL_FL_THEML_FLD_io.f90:481-560).
void velo2massflux(oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        FC(g, 1, i, j, k) = FC(q, 1, i, j, k) * FC(rhostg, 1, i, j, k);
        FC(g, 3, i, j, k) = FC(q, 3, i, j, k) * FC(rhostg, 3, i, j, k);
        if (j >= 2) FC(g, 2, i, j, k) = FC(q, 2, i, j, k) * FC(rhostg, 2, i, j, k);
      }
  bc_wall_vec(o, o->g);
}

// ------------------------------------------ coupled inflow/outflow planes
// CONVCTION_OUTLET_U (src/BC_COUTLET_MOM_RK3.f90:101-174, method two):
// U_OUTLET = (max + min) / 2 of the outlet-face mean 0.5 (u(NCL1) + u(NCL1+1)).
double convection_outlet_u(const oracle_io *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  double umax = -1.0e20, umin = 1.0e20;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const double ucc = (FC(q, 1, nx, j, k) + o->bcp[ORC_P_OUT_U][o->pj(j, k)]) * 0.5;
      if (ucc > umax) umax = ucc;
      if (ucc < umin) umin = ucc;
    }
  return 0.5 * (umax + umin);
}

// BC_WALL_G_io / BC_WALL_Q_io (src/BC_WALL.f90:233-256, 412-460) on the outlet
// plane: u, w zero on both ghost rows, v zero on rows 0, 1 and ny + 1.
void outlet_plane_walls(oracle_io *o) {
  const int ny = o->ny, nz = o->nz;
  const int ig[3] = {ORC_P_OUT_GX, ORC_P_OUT_GY, ORC_P_OUT_GZ}, iq[3] = {ORC_P_OUT_U, ORC_P_OUT_V, ORC_P_OUT_W};
  for (int k = 1; k <= nz; ++k)
    for (int s = 0; s < 2; ++s) {
      const int *ids = s ? iq : ig;
      o->bcp[ids[0]][o->pj(0, k)] = 0.0;
      o->bcp[ids[2]][o->pj(0, k)] = 0.0;
      o->bcp[ids[1]][o->pj(1, k)] = 0.0;
      o->bcp[ids[1]][o->pj(0, k)] = 0.0;
      for (int c = 0; c < 3; ++c) o->bcp[ids[c]][o->pj(ny + 1, k)] = 0.0;
    }
}

// The arrays of the current layout, as MEMALLOCT.f90 initialises them
// (src/MEMALLOCT.f90:154-215): zero, properties and the staggered density /
// viscosity 1 (ghost columns keep those values where no routine writes them).
void alloc_fields(oracle_io *o) {
  const int64_t n = o->len();
  for (int c = 1; c <= 3; ++c) {
    o->q[c].assign(n, 0.0); o->g[c].assign(n, 0.0); o->g0[c].assign(n, 0.0); o->explt0[c].assign(n, 0.0);
    o->mustg[c].assign(n, 1.0); o->rhostg[c].assign(n, 1.0);
  }
  for (auto *v : {&o->pr, &o->dph, &o->rhsllphi, &o->qtmp, &o->dphtmp, &o->rhsz, &o->divu, &o->drho, &o->rhoh,
                  &o->hh, &o->rhse, &o->rhse0})
    v->assign(n, 0.0);
  for (auto *v : {&o->tt, &o->dd, &o->dd0, &o->mu, &o->mu0, &o->kk}) v->assign(n, 1.0);
  for (int c = 1; c <= 3; ++c) {
    o->rhsio[c].assign(n, 0.0); o->adv[c].assign(n, 0.0); o->drhoi[c].assign(n, 0.0);
  }
  for (int q = 0; q < ORC_P_COUNT; ++q) o->bcp[q].assign((size_t)(o->ny + 2) * o->nz, 0.0);
  o->bcp[ORC_P_IN_RHO].assign((size_t)(o->ny + 2) * o->nz, 1.0);
}

}  // namespace

extern "C" {

oracle_io *oracle_io_create(int nx, int ny, int nz, double lx, double lz, double str2, int istr2, double ren,
                            double dt, int flowdrvtp, double cfgv, int thermal, double prt, double qw_bot,
                            double qw_top, int gravdir, double f_a) {
  if (nx < 4 || ny < 4 || nz < 4 || (nx % 2) || (nz % 2) || gravdir < 0 || gravdir > 3) return nullptr;
  // the y mesh and Poisson y-coefficients are shared with the TG oracle
  oracle_tg *t = oracle_tg_create(nx, ny, nz, lx, lz, str2, istr2, ren, dt, flowdrvtp, cfgv);
  if (!t) return nullptr;
  oracle_io *o = new oracle_io();
  o->nx = nx; o->ny = ny; o->nz = nz; o->lx = lx; o->lz = lz; o->str2 = str2; o->istr2 = istr2;
  o->ren = ren; o->dt = dt; o->flowdrvtp = flowdrvtp; o->cfgv = cfgv; o->thermal = thermal ? 1 : 0;
  o->prt = prt; o->qw[0] = qw_bot; o->qw[1] = qw_top; o->gravdir = gravdir; o->f_a = f_a;
  std::vector<double> tmp(ny + 2);
  auto coef = [&](int what, std::vector<double> &dst) {
    dst.assign(ny + 2, 0.0);
    int n = oracle_tg_get_coef(t, what, tmp.data());
    for (int j = 1; j <= n; ++j) dst[j] = tmp[j - 1];
  };
  coef(0, o->ynd); coef(1, o->ycc); coef(2, o->dyfi); coef(3, o->dyci); coef(4, o->wff); coef(5, o->wfb);
  coef(6, o->amph); coef(7, o->acph); coef(8, o->apph);
  o->volm = oracle_tg_volm(t);
  oracle_tg_destroy(t);
  o->dxi = nx / lx; o->dzi = nz / lz; o->dxqi = o->dxi * o->dxi; o->dzqi = o->dzi * o->dzi;
  o->cvisc = 1.0 / ren;
  o->cthecd = 1.0 / ren / prt;  // Flow_State.f90:87
  o->area_inlet = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= nz; ++k) o->area_inlet += 1.0 / o->dyfi[j] / o->dzi;
  o->tgam[0] = 1.0; o->tgam[1] = 8.0 / 15.0; o->tgam[2] = 5.0 / 12.0; o->tgam[3] = 3.0 / 4.0;
  o->troh[0] = 0.0; o->troh[1] = 0.0; o->troh[2] = -17.0 / 60.0; o->troh[3] = -5.0 / 12.0;
  for (int n = 0; n < 4; ++n) o->talp[n] = o->tgam[n] + o->troh[n];
  o->sx = nx;
  alloc_fields(o);
  vis_ycoef(o);
  o->dftx = oracle_dft_create(nx);
  o->dftz = oracle_dft_create(nz);
  return o;
}

void oracle_io_destroy(oracle_io *o) {
  if (!o) return;
  oracle_dft_destroy(o->dftx);
  oracle_dft_destroy(o->dftz);
  delete o;
}

int oracle_io_set_table(oracle_io *o, const double *H, const double *T, const double *D, const double *M,
                        const double *K, int n, int shortcuts) {
  if (n < 4) return -1;
  o->ht.build(H, T, n);
  o->td.build(T, D, n);
  o->tm.build(T, M, n);
  o->tk.build(T, K, n);
  o->hd.build(H, D, n);
  o->th.build(T, H, n);
  o->shortcuts = shortcuts ? 1 : 0;
  o->has_table = true;
  // RHOHmax (src/Flow_State.f90:963-990): max of D(h) h over 3n - 1 samples
  double rm = -1e-14;
  for (int i = 2; i <= 3 * n; ++i) {
    const double h = H[0] + (double)(i - 1) * (H[n - 1] - H[0]) / (double)(3 * n);
    double d = 0.0;
    o->hd.eval(h, d);
    if (o->shortcuts && std::fabs(h) < 1.0e-10) d = 1.0;  // Flow_State.f90:1112
    if (d * h > rm) rm = d * h;
  }
  o->rhohmax = rm;
  return 0;
}

double oracle_io_rhohmax(const oracle_io *o) { return o->rhohmax; }

// BCX_io (Dirichlet 1, Neumann 2, periodic 3, src/READINI.f90:117-171) of the
// Poisson solve: FISHPACK's LP (src/possion3d_fishpack_reform.f90:342-346).
int oracle_io_set_bcx(oracle_io *o, int in, int out) {
  int lp = -1;
  if (in == 3 && out == 3) lp = 1;
  if (in == 1 && out == 1) lp = 2;
  if (in == 1 && out == 2) lp = 3;
  if (in == 2 && out == 2) lp = 4;
  if (in == 2 && out == 1) lp = 5;
  if (lp < 0 || o->nx < 4) return -1;
  o->lpx = lp;
  // a non-periodic x is the coupled inflow / outflow section (TGFLOWFLG):
  // the arrays are re-created with the x ghost columns, so this comes before
  // the initial field
  const int coupled = lp != 1 ? 1 : 0;
  if (coupled != o->coupled) {
    o->coupled = coupled;
    o->sx = coupled ? o->nx + 2 : o->nx;
    alloc_fields(o);
  }
  return 0;
}

// FISHPACK_POIS3D_SIMPLE alone: DPH from the current RHSLLPHI.
void oracle_io_pois3d(oracle_io *o) { fishpack_pois3d(o); }

// One real x transform of FISHPACK's LP 2..5 on x (n values): the direct
// documented sums, or (fast, LP 3 / 5 only) the DFT route.
int oracle_fftpack_real(int lp, int fwd, int n, double *x, int fast) {
  if (lp < 2 || lp > 5 || n < 2) return -1;
  std::vector<double> w(6 * (size_t)n);
  if (fast) {
    if ((lp != 3 && lp != 5) || (n & 1)) return -1;
    oracle_dft *f = oracle_dft_create(n);
    qwave_fast(lp, fwd != 0, n, x, f, w.data());
    oracle_dft_destroy(f);
  } else {
    fftpack_real(lp, fwd != 0, n, x, w.data());
  }
  return 0;
}

// BCWALLHEAT = isoThermalWall on the walls of `bits` (bit 0 bottom, bit 1
// top), the wall temperature being qw of that wall; WALL_ISOTHERMAL_GIVEN
// (src/Flow_State.f90:603-645) takes h, rho, mu, k at it from the table's
// T-splines (NIST_SLEVAL_TH/TD/TM/TK).  Call after oracle_io_set_table and
// before the initial field; -1 when a wall temperature is outside the table.
int oracle_io_set_walls(oracle_io *o, int bits) {
  if (bits < 0 || bits > 3 || (bits && (!o->thermal || !o->has_table))) return -1;
  for (int side = 0; side < 2; ++side) {
    if (!(bits & (1 << side))) continue;
    const double tw = o->qw[side];
    double *w = o->wall[side];
    w[0] = tw;
    if (!o->th.eval(tw, w[1]) || !o->td.eval(tw, w[2]) || !o->tm.eval(tw, w[3]) || !o->tk.eval(tw, w[4]))
      return -1;
  }
  o->isothermal = bits;
  return 0;
}

int oracle_io_init_random(oracle_io *o, uint64_t seed, double amp) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  if (o->coupled && !o->tg_u) return -1;
  o->bad = 0;
  // thermal field (INIFIELD_THERMAL_io, src/INITIAL_FL_THEML_FLD_io.f90:352-381)
  std::fill(o->rhoh.begin(), o->rhoh.end(), 0.0);
  std::fill(o->hh.begin(), o->hh.end(), 0.0);
  std::fill(o->rhse0.begin(), o->rhse0.end(), 0.0);
  double T0 = 1.0, D0 = 1.0, M0 = 1.0, K0 = 1.0;
  if (o->thermal && o->has_table && !o->shortcuts) {
    lookup_ht(o, 0.0, T0);
    lookup_t(o, o->td, T0, D0);
    lookup_t(o, o->tm, T0, M0);
    lookup_t(o, o->tk, T0, K0);
  }
  std::fill(o->tt.begin(), o->tt.end(), T0);
  std::fill(o->dd.begin(), o->dd.end(), D0);
  std::fill(o->dd0.begin(), o->dd0.end(), D0);
  std::fill(o->mu.begin(), o->mu.end(), M0);
  std::fill(o->mu0.begin(), o->mu0.end(), M0);
  std::fill(o->kk.begin(), o->kk.end(), K0);
  // velocity: the TG recipe
  for (int c = 1; c <= 3; ++c) {
    std::fill(o->q[c].begin(), o->q[c].end(), 0.0);
    std::fill(o->g[c].begin(), o->g[c].end(), 0.0);
    std::fill(o->g0[c].begin(), o->g0[c].end(), 0.0);
    std::fill(o->explt0[c].begin(), o->explt0[c].end(), 0.0);
  }
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i)
        for (int c = 1; c <= 3; ++c) FC(q, c, i, j, k) = amp * rnd_pm1(seed, c, i, j, k);
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) FC(q, 2, i, 1, k) = 0.0;
  for (int c = 1; c <= 3; ++c)
    for (int j = 1; j <= ny; ++j) {
      double s = 0.0;
      for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= nz; ++k) s += FC(q, c, i, j, k);
      s /= (double)(nx * nz);
      for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= nz; ++k) FC(q, c, i, j, k) -= s;
    }
  for (int j = 1; j <= ny; ++j) {
    const double vini = 1.5 * (1.0 - o->ycc[j] * o->ycc[j]);
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) FC(q, 1, i, j, k) += vini;
  }
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) FC(q, 2, i, 1, k) = 0.0;
  bc_wall_vec(o, o->q);
  const double ub = bulk(o, o->q[1]);
  for (auto &x : o->q[1]) x /= ub;
  // mass flux from the velocity, then unit bulk mass flux (Unified_massflux,
  // src/INITIAL_FL_THEML_FLD_io.f90:653-682)
  density_staggered(o);
  velo2massflux(o);
  const double gm = bulk(o, o->g[1]);
  for (int c = 1; c <= 3; ++c)
    for (auto &x : o->q[c]) x /= gm;
  velo2massflux(o);
  bc_wall_vec(o, o->q);
  if (o->coupled) {
    for (int q = ORC_P_CONV0_X; q <= ORC_P_CONV0_ENG; ++q) std::fill(o->bcp[q].begin(), o->bcp[q].end(), 0.0);
    // outlet ghost column NCL1_io + 1: a copy of the last interior column
    // (the seeded recipe covers the interior; the inlet column comes from
    // the TG section in the projection's BC_TINLET_FLOW)
    for (int c = 1; c <= 3; ++c)
      for (int k = 1; k <= nz; ++k)
        for (int j = 0; j <= ny + 1; ++j) {
          FC(q, c, nx + 1, j, k) = FC(q, c, nx, j, k);
          FC(g, c, nx + 1, j, k) = FC(g, c, nx, j, k);
        }
  }
  std::fill(o->pr.begin(), o->pr.end(), 0.0);
  std::fill(o->dph.begin(), o->dph.end(), 0.0);
  std::fill(o->drho.begin(), o->drho.end(), 0.0);
  mu_staggered(o);
  // CALC_INITIALIZATION_io (src/INITIAL_FL_THEML_FLD_io.f90:133-172)
  if (o->thermal) {
    bc_wall_thermal(o);
    eng_io(o, 0);
    density_staggered(o);
    mu_staggered(o);
  }
  mom_io(o, 0);
  return 0;
}

int oracle_io_set_inlet(oracle_io *o, int nxt, const double *tu, const double *tv, const double *tw,
                        const double *tp) {
  if (!o->coupled || nxt < 1 || !tu || !tv || !tw || !tp) return -1;
  o->tg_nx = nxt;
  o->tg_u = tu; o->tg_v = tv; o->tg_w = tw; o->tg_p = tp;
  return 0;
}

int oracle_io_eng(oracle_io *o, int ns) {
  if (ns < 0 || ns > 3 || !o->thermal || !o->has_table) return -1;
  eng_io(o, ns);
  return 0;
}

int oracle_io_mom(oracle_io *o, int ns) {
  // the coupled section's semi-implicit boundary terms (BC_CBC_TDMA) are
  // unfinished in the reference (src/SOLVERRK3_MOM_IO.f90:22)
  if (ns < 0 || ns > 3 || (o->coupled && (!o->tg_u || o->implicit))) return -1;
  if (ns >= 1) {
    if (o->thermal) {
      density_time_derivation(o, ns);
      density_staggered(o);
      mu_staggered(o);
      if (o->implicit) density_implicit_add(o);  // src/SOLVE.f90:126-128
    }
    velocity_calc(o);
  }
  mom_io(o, ns);
  return 0;
}

int oracle_io_substep(oracle_io *o, int ns) {
  if (ns < 1 || ns > 3 || (o->coupled && !o->tg_u)) return -1;
  if (o->thermal) eng_io(o, ns);
  return oracle_io_mom(o, ns);
}

int oracle_io_step(oracle_io *o) {
  for (int ns = 1; ns <= 3; ++ns)
    if (oracle_io_substep(o, ns)) return -1;
  return 0;
}

int oracle_io_get_field(const oracle_io *o, int id, double *out) {
  auto *f = field_ptr(const_cast<oracle_io *>(o), id);
  if (!f) return -1;
  std::memcpy(out, f->data(), sizeof(double) * f->size());
  return 0;
}
int oracle_io_set_field(oracle_io *o, int id, const double *in) {
  auto *f = field_ptr(o, id);
  if (!f) return -1;
  std::memcpy(f->data(), in, sizeof(double) * f->size());
  return 0;
}

double oracle_io_divmax(const oracle_io *o) {
  double m = 0.0;
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 1; j <= o->ny; ++j)
      for (int i = 1; i <= o->nx; ++i) {
        const double divx = (FC(g, 1, o->ip(i), j, k) - FC(g, 1, i, j, k)) * o->dxi;
        const double divy = (FC(g, 2, i, j + 1, k) - FC(g, 2, i, j, k)) * o->dyfi[j];
        const double divz = (FC(g, 3, i, j, o->kp(k)) - FC(g, 3, i, j, k)) * o->dzi;
        m = std::fmax(m, std::fabs(divx + divy + divz + F(drho, i, j, k)));
      }
  return m;
}

double oracle_io_divmax_q(const oracle_io *o) {
  double m = 0.0;
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 1; j <= o->ny; ++j)
      for (int i = 1; i <= o->nx; ++i) {
        const double divx = (FC(q, 1, o->ip(i), j, k) - FC(q, 1, i, j, k)) * o->dxi;
        const double divy = (FC(q, 2, i, j + 1, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
        const double divz = (FC(q, 3, i, j, o->kp(k)) - FC(q, 3, i, j, k)) * o->dzi;
        m = std::fmax(m, std::fabs(divx + divy + divz));
      }
  return m;
}

double oracle_io_bulk(const oracle_io *o, int what) {
  if (what == 0) return bulk(o, o->q[1]);
  if (what == 1) return bulk(o, o->g[1]);
  return bulk(o, o->hh);
}

int64_t oracle_io_bad_cells(const oracle_io *o) { return o->bad; }

// CFL_io + CFL_VISCOUS (src/CFL.f90:42-133), explicit scheme.
double oracle_io_cfl(const oracle_io *o) {
  double m = 0.0;
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 1; j <= o->ny; ++j) {
      // CFL_VISCOUS is zero for the semi-implicit scheme (src/CFL.f90:121-130)
      const double vis = o->implicit ? 0.0 : 2.0 * o->cvisc * (o->dxqi + o->dzqi + o->dyfi[j] * o->dyfi[j]);
      for (int i = 1; i <= o->nx; ++i) {
        double q = (std::fabs((FC(g, 1, i, j, k) + FC(g, 1, o->ip(i), j, k)) * o->dxi) +
                    std::fabs((FC(g, 2, i, j, k) + FC(g, 2, i, j + 1, k)) * o->dyfi[j]) +
                    std::fabs((FC(g, 3, i, j, k) + FC(g, 3, i, j, o->kp(k))) * o->dzi)) * 0.5;
        q = q + vis;
        m = std::fmax(m, q);
      }
    }
  return m;
}

void oracle_io_set_dt(oracle_io *o, double dt) { o->dt = dt; }

int oracle_io_set_scheme(oracle_io *o, int implicit) {
  if (implicit != 0 && implicit != 1) return -1;
  o->implicit = implicit;
  for (int c = 1; c <= 3; ++c) std::fill(o->drhoi[c].begin(), o->drhoi[c].end(), 0.0);
  return 0;
}


// BC_TINLET_FLOW + BC_TINLET_THERML (src/BC_INLET.f90:2-51, 54-76): the TG
// section's last plane (and its first-face u) feed the IO inlet ghost plane
// i = 0 and the first face i = 1; the inlet ghost properties are the
// reference state (rho = 1).  TG arrays: (nz, ny + 2, nxt).
void oracle_io_bc_inlet(oracle_io *o, int nxt, const double *tu, const double *tv, const double *tw,
                        const double *tp) {
  const int ny = o->ny, nz = o->nz;
  auto T = [&](const double *a, int i, int j, int k) {
    return a[(int64_t)(i - 1) + (int64_t)nxt * ((int64_t)j + (int64_t)(ny + 2) * (k - 1))];
  };
  for (int j = 0; j <= ny + 1; ++j)
    for (int k = 1; k <= nz; ++k) {
      const int64_t pc = o->pj(j, k);
      const double rin = 1.0;  // DENSITY(0, J, K) from BC_TINLET_THERML
      o->bcp[ORC_P_IN_RHO][pc] = rin;
      o->bcp[ORC_P_IN_U][pc] = T(tu, nxt, j, k);
      FC(q, 1, 1, j, k) = T(tu, 1, j, k);
      o->bcp[ORC_P_IN_GX][pc] = o->bcp[ORC_P_IN_U][pc] * rin;
      FC(g, 1, 1, j, k) = FC(q, 1, 1, j, k) * (rin + F(dd, 1, j, k)) * XND2CL;
      o->bcp[ORC_P_IN_V][pc] = T(tv, nxt, j, k);
      o->bcp[ORC_P_IN_GY][pc] = o->bcp[ORC_P_IN_V][pc] * rin;
      o->bcp[ORC_P_IN_W][pc] = T(tw, nxt, j, k);
      o->bcp[ORC_P_IN_GZ][pc] = o->bcp[ORC_P_IN_W][pc] * rin;
      o->bcp[ORC_P_IN_P][pc] = T(tp, nxt, j, k);
    }
}

// BC_COUTLET_MOM_RK3 (src/BC_COUTLET_MOM_RK3.f90:2-97): convective outlet
// dG/dt + U_OUTLET dG/dx = 0 on the ghost plane i = NCL1 + 1 with the RK3
// weights (BC_CONV0 the previous substep's term), then CHK_MassConsv_io
// (src/processing/CHK_conservation.f90:2-71) and the rescaling of the outlet
// x-flux so that inflow - d(rho)/dt = outflow, then the wall conditions.
int oracle_io_bc_outlet_mom(oracle_io *o, int ns) {
  if (ns < 0 || ns > 3) return 1;
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double U = convection_outlet_u(o);
  o->bcs[0] = U;
  const double coe1 = o->dxi * U;
  const int ig[4] = {0, ORC_P_OUT_GX, ORC_P_OUT_GY, ORC_P_OUT_GZ};
  const int iq[4] = {0, ORC_P_OUT_U, ORC_P_OUT_V, ORC_P_OUT_W};
  const int ic[4] = {0, ORC_P_CONV0_X, ORC_P_CONV0_Y, ORC_P_CONV0_Z};
  for (int idr = 1; idr <= 3; ++idr) {
    const int n2i = idr == 2 ? 2 : 1;
    for (int k = 1; k <= nz; ++k)
      for (int j = n2i; j <= ny; ++j) {
        const int64_t pc = o->pj(j, k);
        double &gout = o->bcp[ig[idr]][pc];
        const double conv = -(gout - FC(g, idr, nx, j, k)) * coe1;
        const double rhs = o->tgam[ns] * conv + o->troh[ns] * o->bcp[ic[idr]][pc];
        o->bcp[ic[idr]][pc] = conv;
        gout = gout + o->dt * rhs;
        const double rho = (F(dd, nx, j, k) + o->bcp[ORC_P_OUT_RHO][pc]) * XND2CL;
        o->bcp[iq[idr]][pc] = gout / rho;
      }
  }
  // CHK_MassConsv_io (RCCI1 = 1 in the channel)
  double fin = 0.0, fout = 0.0, mass = 0.0;
  for (int j = 1; j <= ny; ++j) {
    const double coe2 = 1.0 / o->dyfi[j];
    for (int k = 1; k <= nz; ++k) {
      fin += FC(g, 1, 1, j, k) * coe2;
      fout += o->bcp[ORC_P_OUT_GX][o->pj(j, k)] * coe2;
    }
  }
  fin /= o->dzi;
  fout /= o->dzi;
  for (int j = 1; j <= ny; ++j) {
    const double coe2 = 1.0 / o->dyfi[j];
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) mass += F(drho, i, j, k) * coe2;
  }
  mass = mass / o->dzi / o->dxi;
  const double scaling = (fin - mass) / fout;
  o->bcs[1] = scaling;
  o->bcs[2] = fin - mass - fout;
  o->bcs[3] = fin;
  o->bcs[4] = fout;
  o->bcs[5] = mass;
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= nz; ++k) {
      const int64_t pc = o->pj(j, k);
      double &gout = o->bcp[ORC_P_OUT_GX][pc];
      gout = gout * (scaling - 1.0) + gout;
      const double rho = (F(dd, nx, j, k) + o->bcp[ORC_P_OUT_RHO][pc]) * XND2CL;
      o->bcp[ORC_P_OUT_U][pc] = gout / rho;
    }
  outlet_plane_walls(o);
  return 0;
}

// BC_COUTLET_ENEG_RK3 (src/BC_COUTLET_ENEG_RK3.f90:2-41): convective outlet
// for rho h with the RK3 weights, then ENTHALPY_UPDATE, DENSITY_UPDATE,
// ENTHALPY_UPDATE and THERM_PROP_UPDATE on the outlet plane
// (src/THERM_PROP_UPDATE.f90, region IOULET) and BC_WALL_ISOFLUX on its
// ghost rows.
int oracle_io_bc_outlet_eng(oracle_io *o, int ns) {
  if (ns < 0 || ns > 3 || !o->thermal || !o->has_table) return 1;
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double U = convection_outlet_u(o);
  o->bcs[6] = U;
  std::vector<double> &rh = o->bcp[ORC_P_OUT_RHOH], &hh = o->bcp[ORC_P_OUT_H], &tt = o->bcp[ORC_P_OUT_T];
  std::vector<double> &dd = o->bcp[ORC_P_OUT_RHO], &mu = o->bcp[ORC_P_OUT_MU], &kk = o->bcp[ORC_P_OUT_K];
  std::vector<double> &c0 = o->bcp[ORC_P_CONV0_ENG];
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int64_t pc = o->pj(j, k);
      const double conv = -o->dxi * U * (rh[pc] - F(rhoh, nx, j, k));
      const double rhs = o->tgam[ns] * conv + o->troh[ns] * c0[pc];
      c0[pc] = conv;
      rh[pc] = rh[pc] + o->dt * rhs;
    }
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const int64_t pc = o->pj(j, k);
      double h = rh[pc] / dd[pc];
      double T, D;
      if (lookup_ht(o, h, T) && lookup_t(o, o->td, T, D))
        dd[pc] = D;
      else
        ++o->bad;
      h = rh[pc] / dd[pc];
      hh[pc] = h;
      if (o->shortcuts && std::fabs(h) < 1.0e-10) continue;  // properties kept
      double M, K;
      if (!lookup_ht(o, h, T) || !lookup_t(o, o->tm, T, M) || !lookup_t(o, o->tk, T, K) ||
          !lookup_t(o, o->td, T, D)) {
        ++o->bad;
        continue;
      }
      tt[pc] = T;
      mu[pc] = M;
      kk[pc] = K;
      dd[pc] = D;
    }
  for (int k = 1; k <= nz; ++k)
    for (int side = 0; side < 2; ++side) {
      const int j = side == 0 ? 0 : ny + 1;
      double h;
      if (side == 0)
        h = 2.0 * hh[o->pj(1, k)] - o->wff[2] * hh[o->pj(2, k)] - o->wfb[2] * hh[o->pj(1, k)];
      else
        h = 2.0 * hh[o->pj(ny, k)] - o->wff[ny] * hh[o->pj(ny, k)] - o->wfb[ny] * hh[o->pj(ny - 1, k)];
      const int64_t pc = o->pj(j, k);
      hh[pc] = h;
      double T, M, K, D;
      if (!lookup_ht(o, h, T) || !lookup_t(o, o->tm, T, M) || !lookup_t(o, o->tk, T, K) ||
          !lookup_t(o, o->td, T, D)) {
        ++o->bad;
        continue;
      }
      dd[pc] = D;
      tt[pc] = T;
      mu[pc] = M;
      kk[pc] = K;
      rh[pc] = h * D;
    }
  return 0;
}

int oracle_io_get_plane(const oracle_io *o, int which, double *out) {
  if (which < 0 || which >= ORC_P_COUNT) return 1;
  std::copy(o->bcp[which].begin(), o->bcp[which].end(), out);
  return 0;
}

int oracle_io_set_plane(oracle_io *o, int which, const double *in) {
  if (which < 0 || which >= ORC_P_COUNT) return 1;
  std::copy(in, in + o->bcp[which].size(), o->bcp[which].begin());
  return 0;
}

void oracle_io_bc_scalars(const oracle_io *o, double *out) {
  for (int q = 0; q < 7; ++q) out[q] = o->bcs[q];
}

// PP_MEAN_ZX_FLOW_Xperiodic_IO (src/processing/PP_MEAN_ZX.f90:299-872),
// channel branch (RCCI1 = RNDI1 = 1): per y-row j the xz-plane averages of
// the cell-centred velocity U, mass flux G, pressure p, velocity gradient
// D(m,n) = du_m/dx_n and, with the energy equation, of T, rho, h, mu, k and
// the gradients of h and T, each sum scaled by VL1313_io = 1/(nx nz)
// (src/CONSPARA.f90:84).  out holds ny * 360 values; row j-1:
//   U1 (u, v, w, p), G1 (3), UP (3), U2 (6: 11 12 13 22 23 33), UG (6),
//   U3 (10: 111 112 113 122 123 133 222 223 233 333), UGU (10), DVDL1 (3x3),
//   DVDLP (3x3), DVDL2 (9x9: row (m,h), column (n,p)); then T1, D1, H1, M1,
//   T2, D2, H2, DH, PH, DVDL1M (3x3), DVDL1MH (3x3), DVDL1MU (m,n,h),
//   DVDL2M (9x9), UH (3), GH (3), U2DH (6), DhDL1 (3), DhDLP (3), DTDLK (3),
//   DTDLKU (m,n), DTDLKDVDL (m,n,h), DHDLMDVDL (m,n,h) — zero without the
//   energy equation.
void oracle_io_stats(const oracle_io *o, double *out) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double vl = 1.0 / (double)(nx * nz);
  const bool th = o->thermal != 0;
#pragma omp parallel for schedule(static) num_threads(nthreads())
  for (int j = 1; j <= ny; ++j) {
    std::vector<double> acc(360, 0.0);
    const int jp = j + 1, jm = j - 1;
    for (int i = 1; i <= nx; ++i) {
      const int ip = o->ip(i), im = o->im(i);
      for (int k = 1; k <= nz; ++k) {
        const int kp = o->kp(k), km = o->km(k);
        double U[3], G[3], Uip[3], Uim[3], Ujp[3], Ujm[3], Ukp[3], Ukm[3], D[3][3];
        G[0] = (FC(g, 1, i, j, k) + FC(g, 1, ip, j, k)) * 0.5;
        U[0] = (FC(q, 1, i, j, k) + FC(q, 1, ip, j, k)) * 0.5;
        Ujp[0] = (FC(q, 1, i, jp, k) + FC(q, 1, ip, jp, k)) * 0.5;
        Ujm[0] = (FC(q, 1, i, jm, k) + FC(q, 1, ip, jm, k)) * 0.5;
        Ukp[0] = (FC(q, 1, i, j, kp) + FC(q, 1, ip, j, kp)) * 0.5;
        Ukm[0] = (FC(q, 1, i, j, km) + FC(q, 1, ip, j, km)) * 0.5;
        G[2] = (FC(g, 3, i, j, k) + FC(g, 3, i, j, kp)) * 0.5;
        U[2] = (FC(q, 3, i, j, k) + FC(q, 3, i, j, kp)) * 0.5;
        Uip[2] = (FC(q, 3, ip, j, k) + FC(q, 3, ip, j, kp)) * 0.5;
        Uim[2] = (FC(q, 3, im, j, k) + FC(q, 3, im, j, kp)) * 0.5;
        Ujp[2] = (FC(q, 3, i, jp, k) + FC(q, 3, i, jp, kp)) * 0.5;
        Ujm[2] = (FC(q, 3, i, jm, k) + FC(q, 3, i, jm, kp)) * 0.5;
        G[1] = (FC(g, 2, i, j, k) + FC(g, 2, i, jp, k)) * 0.5;
        U[1] = (FC(q, 2, i, j, k) + FC(q, 2, i, jp, k)) * 0.5;
        Uip[1] = (FC(q, 2, ip, j, k) + FC(q, 2, ip, jp, k)) * 0.5;
        Uim[1] = (FC(q, 2, im, j, k) + FC(q, 2, im, jp, k)) * 0.5;
        Ukp[1] = (FC(q, 2, i, j, kp) + FC(q, 2, i, jp, kp)) * 0.5;
        Ukm[1] = (FC(q, 2, i, j, km) + FC(q, 2, i, jp, km)) * 0.5;
        D[0][0] = (FC(q, 1, ip, j, k) - FC(q, 1, i, j, k)) * o->dxi;
        D[0][2] = (Ukp[0] - Ukm[0]) * o->dzi * 0.5;
        D[0][1] = ((Ujp[0] - U[0]) * o->dyci[jp] + (U[0] - Ujm[0]) * o->dyci[j]) * 0.5;
        D[1][0] = (Uip[1] - Uim[1]) * o->dxi * 0.5;
        D[1][2] = (Ukp[1] - Ukm[1]) * o->dzi * 0.5;
        D[1][1] = (FC(q, 2, i, jp, k) - FC(q, 2, i, j, k)) * o->dyfi[j];
        D[2][2] = (FC(q, 3, i, j, kp) - FC(q, 3, i, j, k)) * o->dzi;
        D[2][0] = (Uip[2] - Uim[2]) * o->dxi * 0.5;
        D[2][1] = ((Ujp[2] - U[2]) * o->dyci[jp] + (U[2] - Ujm[2]) * o->dyci[j]) * 0.5;
        const double p = F(pr, i, j, k);
        int a = 0;
        for (int m = 0; m < 3; ++m) acc[a++] += U[m];
        acc[a++] += p;
        for (int m = 0; m < 3; ++m) acc[a++] += G[m];
        for (int m = 0; m < 3; ++m) acc[a++] += U[m] * p;
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n) acc[a++] += U[m] * U[n];
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n) acc[a++] += U[m] * G[n];
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n)
            for (int h = n; h < 3; ++h) acc[a++] += U[m] * U[n] * U[h];
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n)
            for (int h = n; h < 3; ++h) acc[a++] += U[m] * G[n] * U[h];
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) acc[a++] += D[m][n];
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) acc[a++] += D[m][n] * p;
        for (int l1 = 0; l1 < 9; ++l1)
          for (int l2 = 0; l2 < 9; ++l2) acc[a++] += D[l1 / 3][l1 % 3] * D[l2 / 3][l2 % 3];
        if (!th) continue;
        const double T = F(tt, i, j, k), R = F(dd, i, j, k), H = F(hh, i, j, k), MU = F(mu, i, j, k),
                     K = F(kk, i, j, k);
        double dh[3], dT[3];
        dh[0] = (F(hh, ip, j, k) - F(hh, im, j, k)) * o->dxi * 0.5;
        dh[2] = (F(hh, i, j, kp) - F(hh, i, j, km)) * o->dzi * 0.5;
        dh[1] = ((F(hh, i, jp, k) - F(hh, i, j, k)) * o->dyci[jp] + (F(hh, i, j, k) - F(hh, i, jm, k)) * o->dyci[j]) *
                0.5;
        dT[0] = (F(tt, ip, j, k) - F(tt, im, j, k)) * o->dxi * 0.5;
        dT[2] = (F(tt, i, j, kp) - F(tt, i, j, km)) * o->dzi * 0.5;
        dT[1] = ((F(tt, i, jp, k) - F(tt, i, j, k)) * o->dyci[jp] + (F(tt, i, j, k) - F(tt, i, jm, k)) * o->dyci[j]) *
                0.5;
        acc[a++] += T;
        acc[a++] += R;
        acc[a++] += H;
        acc[a++] += MU;
        acc[a++] += T * T;
        acc[a++] += R * R;
        acc[a++] += H * H;
        acc[a++] += H * R;
        acc[a++] += H * p;
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) acc[a++] += D[m][n] * MU;
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) acc[a++] += D[m][n] * MU * H;
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n)
            for (int h = 0; h < 3; ++h) acc[a++] += D[m][n] * MU * U[h];
        for (int l1 = 0; l1 < 9; ++l1)
          for (int l2 = 0; l2 < 9; ++l2) acc[a++] += D[l1 / 3][l1 % 3] * D[l2 / 3][l2 % 3] * MU;
        for (int m = 0; m < 3; ++m) acc[a++] += H * U[m];
        for (int m = 0; m < 3; ++m) acc[a++] += H * G[m];
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n) acc[a++] += R * H * U[m] * U[n];
        for (int m = 0; m < 3; ++m) acc[a++] += dh[m];
        for (int m = 0; m < 3; ++m) acc[a++] += dh[m] * p;
        for (int m = 0; m < 3; ++m) acc[a++] += dT[m] * K;
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) acc[a++] += dT[m] * K * U[n];
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n)
            for (int h = 0; h < 3; ++h) acc[a++] += dT[m] * K * D[n][h];
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n)
            for (int h = 0; h < 3; ++h) acc[a++] += dh[m] * MU * D[n][h];
      }
    }
    double *r = out + (size_t)(j - 1) * 360;
    for (int a = 0; a < 360; ++a) r[a] = acc[a] * vl;
  }
}

}  // extern "C"
