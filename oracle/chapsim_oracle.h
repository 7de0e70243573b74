/*
 * CPU FP64 oracle for the CHAPSim RK3 fractional-step substep.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain restatement of the
 * reference Fortran algorithm used as the checker for the CUDA library.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product path (libchapsim) never links, loads or calls it.
 *
 * Parity pinning: the reference (Fortran 90 + MPI) cannot be compiled in this
 * environment (no Fortran compiler) and ships no golden vectors or tests, so
 * this oracle is "parity unpinned" against reference outputs.  It is pinned
 * instead by the reference's own self-checks restated as asserted tests
 * (Poisson residual, max|div u| after projection, bulk velocity, laminar
 * Poiseuille steadiness) and by an independent numpy restatement that
 * generated the committed fixtures under tests/golden/.
 *
 * Array convention: every 3-D field uses the reference's Fortran layout
 * F(1:nx, 0:ny+1, 1:nz) (x fastest, y with one ghost layer each side, z
 * slowest), i.e. the layout of Q_tg/PR_tg/DPH_tg in MEMALLOCT.f90:99-106.
 * Velocity is stored as three such fields (u, v, w).
 */
#ifndef CHAPSIM_ORACLE_H
#define CHAPSIM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_tg oracle_tg;

/* Field ids for oracle_tg_{get,set}_field. */
enum {
  ORC_U = 0, ORC_V = 1, ORC_W = 2, ORC_P = 3,   /* Q_tg(:,:,:,1..3), PR_tg */
  ORC_PHI = 4,                                  /* DPH_tg  */
  ORC_RHSPHI = 5,                               /* RHSLLPHI_tg */
  ORC_H0U = 6, ORC_H0V = 7, ORC_H0W = 8         /* CONVH0_tg(:,:,:,1..3), no ghosts used */
};

/* Create a TG channel (icase=1, tanh stretching when istr2=1).
 * flowdrvtp: 1 = constant mass flux, 2 = constant pressure gradient (cfgv). */
oracle_tg *oracle_tg_create(int nx, int ny, int nz, double lx, double lz,
                            double str2, int istr2, double ren, double dt,
                            int flowdrvtp, double cfgv);
void oracle_tg_destroy(oracle_tg *o);
int64_t oracle_tg_field_len(const oracle_tg *o); /* nx*(ny+2)*nz */
int oracle_tg_get_field(const oracle_tg *o, int id, double *out);
int oracle_tg_set_field(oracle_tg *o, int id, const double *in);

/* Mesh/coefficient export: what = 0 YND(1:ny+1), 1 YCC(1:ny), 2 DYFI(1:ny),
 * 3 DYCI(1:ny+1), 4 WFF(1:ny+1), 5 WFB(1:ny+1), 6 AMPH, 7 ACPH, 8 APPH (1:ny),
 * 9..11 AMVR/ACVR/APVR(1:ny+1, idr=1), 12..14 idr=2, 15..17 idr=3. */
int oracle_tg_get_coef(const oracle_tg *o, int what, double *out);
double oracle_tg_volm(const oracle_tg *o);

/* Seeded initial field (counter-based splitmix64, see chapsim_init_random). */
void oracle_tg_init_random(oracle_tg *o, uint64_t seed, double amp);
/* Laminar profile only: u = 1.5(1-y^2), v = w = p = 0, ghosts by BC. */
void oracle_tg_init_poiseuille(oracle_tg *o);

/* SOLVERRK3_MOM_tg(NS), NS in 0..3. */
int oracle_tg_substep(oracle_tg *o, int ns);
/* Full step: NS = 1,2,3. */
int oracle_tg_step(oracle_tg *o);

/* Stand-alone pieces, for component tests. */
int oracle_tg_divg(oracle_tg *o, int ns);      /* DIVG_tg: RHSLLPHI from Q */
int oracle_tg_pois3d(oracle_tg *o);            /* FFT99_POIS3D_periodicxz(ITG): PHI from RHSLLPHI */
int oracle_tg_velo_correction(oracle_tg *o, int ns); /* VELOUPDT_tg + BC */
int oracle_tg_prcalc(oracle_tg *o, int ns);    /* PRCALC_tg + BC */

double oracle_tg_divmax(const oracle_tg *o);   /* DIVGCK_tg */
double oracle_tg_bulk(const oracle_tg *o);     /* BULK_VELOCITY_TG */
/* Residual of the discrete Poisson operator: max |L(phi) - rhs| over all
 * cells except the pinned mean-mode row (CHECK_FFT_SOLVER). */
double oracle_tg_pois_residual(const oracle_tg *o);

/* Number of OpenMP threads used (0 = library default). */
/* Complex DFT (interleaved re/im, unnormalised; sign -1 forward, +1
 * inverse); tmp holds n complex values. */
typedef struct oracle_dft oracle_dft;
oracle_dft *oracle_dft_create(int n);
void oracle_dft_destroy(oracle_dft *f);
void oracle_dft_run(const oracle_dft *f, const double *in, double *out, int sign, double *tmp);

/* ------------------------------------------------------------------------
 * IO section: SOLVERRK3_ENG_IO + SOLVERRK3_MOM_IO of an x-periodic channel
 * (BCX_io = 3, no TG section) with the explicit viscous scheme
 * (visthemflg = 0), FISHPACK_POIS3D_SIMPLE Poisson solve, and, when thermal
 * is on, the energy equation with table properties and iso-flux walls.
 * Fields keep the layout F(1:nx, 0:ny+1, 1:nz) (no x ghosts: x is periodic).
 */
typedef struct oracle_io oracle_io;
enum {
  ORC_IO_GX = 20, ORC_IO_GY = 21, ORC_IO_GZ = 22,      /* G_io(:,:,:,1..3) */
  ORC_IO_G0X = 23, ORC_IO_G0Y = 24, ORC_IO_G0Z = 25,   /* G0_io */
  ORC_IO_H = 26, ORC_IO_T = 27, ORC_IO_D = 28,         /* ENTHALPY, TEMPERATURE, DENSITY */
  ORC_IO_MU = 29, ORC_IO_K = 30, ORC_IO_RHOH = 31,     /* VISCOUSITY, THERMCONDT, RHOH */
  ORC_IO_D0 = 32, ORC_IO_MU0 = 33, ORC_IO_DRHO = 34,   /* DENSITY0, VISCOUSITY0, DrhoDtP */
  ORC_IO_EX0X = 35, ORC_IO_EX0Y = 36, ORC_IO_EX0Z = 37,/* EXPLT0_io(:,:,:,1..3) */
  ORC_IO_RHSE0 = 38                                     /* RHS_ENERGY0 */
};
/* qw_bot / qw_top: non-dimensional wall heat flux, positive heats the fluid
 * (WALLFLUX = +qw on the bottom wall, -qw on the top, Flow_State.f90:124-148).
 * gravdir 0 = none, else the buoyancy direction with coefficient f_a. */
oracle_io *oracle_io_create(int nx, int ny, int nz, double lx, double lz, double str2, int istr2, double ren,
                            double dt, int flowdrvtp, double cfgv, int thermal, double prt, double qw_bot,
                            double qw_top, int gravdir, double f_a);
void oracle_io_destroy(oracle_io *o);
/* Table columns H, T, D, M, K (length n, H and T increasing).  shortcuts != 0
 * keeps the reference-state shortcuts (h = 0 -> T = 1, T = 1 -> rho = mu =
 * k = 1, cells with |h| < 1e-10 keep their properties), which assume the
 * reference table normalisation. */
int oracle_io_set_table(oracle_io *o, const double *H, const double *T, const double *D, const double *M,
                        const double *K, int n, int shortcuts);
double oracle_io_rhohmax(const oracle_io *o);
int oracle_io_init_random(oracle_io *o, uint64_t seed, double amp); /* -1: coupled without an inlet source */
int oracle_io_eng(oracle_io *o, int ns);      /* SOLVERRK3_ENG_IO(ns) */
int oracle_io_mom(oracle_io *o, int ns);      /* ns >= 1: DENSITY_TIME_DERIVATION, DENSITY_/MU_Staggered,
                                                 VELOCITY_CALC_io, then SOLVERRK3_MOM_IO(ns); ns = 0: MOM only */
int oracle_io_substep(oracle_io *o, int ns);  /* eng (thermal) + mom */
int oracle_io_step(oracle_io *o);
int oracle_io_get_field(const oracle_io *o, int id, double *out);
int oracle_io_set_field(oracle_io *o, int id, const double *in);
double oracle_io_divmax(const oracle_io *o);   /* DIVGCK_io: max|div G + DrhoDtP| */
double oracle_io_divmax_q(const oracle_io *o); /* max|div u| */
double oracle_io_bulk(const oracle_io *o, int what); /* 0 BULK_VELOCITY_IO, 1 BULK_MASSFLUX_IO, 2 BULK_H_IO */
int64_t oracle_io_bad_cells(const oracle_io *o);     /* table look-ups outside the table so far */
double oracle_io_cfl(const oracle_io *o);            /* CFL_io + CFL_VISCOUS */
void oracle_io_set_dt(oracle_io *o, double dt);
/* visthemflg: 0 explicit viscous terms (default), 1 the semi-implicit scheme
 * (VISCOUS_PAR_EXPLT_*_io + MOMFA_io).  Set before oracle_io_init_random. */
int oracle_io_set_scheme(oracle_io *o, int implicit);
/* Coupled inflow/outflow boundary planes of the IO section (row a16): ghost
 * planes i = 0 and i = NCL1_io + 1, each (nz, ny + 2), ids ORC_P_*. */
#define ORC_P_IN_U 0
#define ORC_P_IN_V 1
#define ORC_P_IN_W 2
#define ORC_P_IN_GX 3
#define ORC_P_IN_GY 4
#define ORC_P_IN_GZ 5
#define ORC_P_IN_P 6
#define ORC_P_IN_RHO 7
#define ORC_P_OUT_U 8
#define ORC_P_OUT_V 9
#define ORC_P_OUT_W 10
#define ORC_P_OUT_GX 11
#define ORC_P_OUT_GY 12
#define ORC_P_OUT_GZ 13
#define ORC_P_OUT_RHO 14
#define ORC_P_OUT_RHOH 15
#define ORC_P_OUT_H 16
#define ORC_P_OUT_T 17
#define ORC_P_OUT_MU 18
#define ORC_P_OUT_K 19
#define ORC_P_CONV0_X 20
#define ORC_P_CONV0_Y 21
#define ORC_P_CONV0_Z 22
#define ORC_P_CONV0_ENG 23
#define ORC_P_COUNT 24
/* BC_TINLET_FLOW + BC_TINLET_THERML from TG arrays (nz, ny + 2, nxt) */
void oracle_io_bc_inlet(oracle_io *o, int nxt, const double *tu, const double *tv, const double *tw,
                        const double *tp);
int oracle_io_bc_outlet_mom(oracle_io *o, int ns); /* BC_COUTLET_MOM_RK3 with CHK_MassConsv_io */
int oracle_io_bc_outlet_eng(oracle_io *o, int ns); /* BC_COUTLET_ENEG_RK3 */
int oracle_io_get_plane(const oracle_io *o, int which, double *out);
int oracle_io_set_plane(oracle_io *o, int which, const double *in);
/* U_OUTLET (momentum), CHK_Mass_CONSV0_SCALING, CHK_MASS_CONSV0, inflow,
 * outflow, mass rate, U_OUTLET (energy) */
void oracle_io_bc_scalars(const oracle_io *o, double *out);
/* x boundary codes of the IO Poisson solve (BCX_io: 1 Dirichlet, 2 Neumann, 3
 * periodic) and the solve alone.  Non-periodic codes make the section the
 * coupled inflow / outflow one (TGFLOWFLG): the arrays are re-created with the
 * x ghost columns i = 0 and nx + 1, (nz, ny + 2, nx + 2), so set them before
 * the initial field. */
int oracle_io_set_bcx(oracle_io *o, int in, int out);
/* Coupled section (non-periodic BCX_io, TGFLOWFLG): the TG arrays (nz, ny + 2,
 * nxt) that BC_TINLET_FLOW reads in the following substeps; kept by pointer. */
int oracle_io_set_inlet(oracle_io *o, int nxt, const double *tu, const double *tv, const double *tw,
                        const double *tp);
void oracle_io_pois3d(oracle_io *o);
/* One x transform of FISHPACK's LP 2..5 (fwd 1: SINT / SINQF / COST / COSQF,
 * 0: the backward ones): direct sums, or with fast = 1 the DFT route of the
 * quarter-wave pairs (LP 3 / 5, even n) that lines longer than 64 take. */
int oracle_fftpack_real(int lp, int fwd, int n, double *x, int fast);
/* iso-thermal walls (bit 0 bottom, bit 1 top; io_oracle.cpp) */
int oracle_io_set_walls(oracle_io *o, int bits);
/* PP_MEAN_ZX_FLOW_Xperiodic_IO: ny * 360 xz-plane averages (io_oracle.cpp) */
void oracle_io_stats(const oracle_io *o, double *out);
double oracle_tg_cfl(const oracle_tg *o);            /* CFL_tg */
void oracle_tg_set_dt(oracle_tg *o, double dt);
void oracle_tg_stats(const oracle_tg *o, double *out); /* PP_MEAN_ZX_FLOW_TG, ny * 122 values */

void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
