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
void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
