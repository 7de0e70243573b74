/*
 * chapsim.h -- C ABI of libchapsim, the B200 (sm_100a) implementation of
 * CHAPSim's RK3 fractional-step substep.
 *
 * The reference (weiwangstfc/CHAPSim1WW, Fortran 90 + MPI) has no plugin or
 * FFI layer: its hot path is a set of Fortran subroutines that take a substep
 * index and work on module-global arrays.  Each entry point below replaces one
 * of those subroutines; the comment names the reference routine (file:line,
 * relative to the CHAPSim1WW project root) it stands in for.  A Fortran host
 * binds them with ISO_C_BINDING interfaces, one bind(C) interface per entry
 * point, passing its module arrays by address.
 *
 * Conventions
 *  - Every function returns an int status: CHAPSIM_OK (0) or a CHAPSIM_ERR_*
 *    code.  chapsim_last_error() gives a one-line message for the last error on
 *    a context.  The reference's equivalent is ERRHDL, which prints and STOPs
 *    (src/WRTHDL.f90:18-30); a Fortran shim calls ERRHDL on a nonzero status.
 *  - The device owns the solution between calls.  Host arrays are uploaded with
 *    chapsim_set_field and read back with chapsim_get_field, in the reference's
 *    own Fortran layout F(1:nx, 0:ny+1, 1:nz) (x fastest, one y ghost layer on
 *    each side, z slowest), the layout of Q_tg/PR_tg/DPH_tg
 *    (src/MEMALLOCT.f90:99-106).  A velocity component of Q_tg(:,:,:,n) is the
 *    contiguous slab starting at Q_tg(1,0,1,n).
 *  - Work is queued on the context's CUDA stream; calls return before the GPU
 *    finishes.  chapsim_sync waits and reports any device-side error.  Calls
 *    that return host data synchronise by themselves.
 *  - One host thread per context; a context is not re-entrant.
 *  - Everything is FP64 at the boundary.
 */
#ifndef CHAPSIM_H
#define CHAPSIM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAPSIM_ABI_VERSION 1

/* status codes */
#define CHAPSIM_OK 0
#define CHAPSIM_ERR_ARG 1         /* invalid argument or size mismatch        */
#define CHAPSIM_ERR_CUDA 2        /* a CUDA runtime call failed               */
#define CHAPSIM_ERR_NOMEM 3       /* device allocation failed                 */
#define CHAPSIM_ERR_STATE 4       /* call not valid in the context's state    */
#define CHAPSIM_ERR_NUMERIC 5     /* NaN/Inf detected by a checked reduction  */
#define CHAPSIM_ERR_UNSUPPORTED 6 /* configuration not supported              */
#define CHAPSIM_ERR_NODEVICE 7    /* no CUDA device visible                   */

/* domain ids: the reference's ITG / IIO parameters (src/modules.f90:46-47) */
#define CHAPSIM_ITG 1
#define CHAPSIM_IIO 2

/* precision forms */
#define CHAPSIM_FP64 0  /* every array and operation in FP64                    */
#define CHAPSIM_MIXED 1 /* FP64 state; FP32 temporaries and spectra (TG), FP32
                           Poisson spectra (IO, explicit viscous scheme); FP64
                           Poisson y-lines, reductions and one FP64-residual
                           refinement sweep of the Poisson solve
                           (chapsim_set_refinement) */

/* field ids for chapsim_set_field / chapsim_get_field (TG domain) */
#define CHAPSIM_F_U 0      /* Q_tg(:,:,:,1)   */
#define CHAPSIM_F_V 1      /* Q_tg(:,:,:,2)   */
#define CHAPSIM_F_W 2      /* Q_tg(:,:,:,3)   */
#define CHAPSIM_F_P 3      /* PR_tg           */
#define CHAPSIM_F_PHI 4    /* DPH_tg          */
#define CHAPSIM_F_RHSPHI 5 /* RHSLLPHI_tg     */
#define CHAPSIM_F_H0U 6    /* CONVH0_tg(:,:,:,1) (y ghosts ignored) */
#define CHAPSIM_F_H0V 7    /* CONVH0_tg(:,:,:,2) */
#define CHAPSIM_F_H0W 8    /* CONVH0_tg(:,:,:,3) */

/* reductions for chapsim_reduce */
#define CHAPSIM_R_DIVMAX 0 /* max |div u|, DIVGCK_tg (src/DIVGCK.f90:16-58)          */
#define CHAPSIM_R_BULK 1   /* bulk velocity, BULK_VELOCITY_TG
                              (src/INITIAL_FL_FLD_TG.f90:122-149)                  */
#define CHAPSIM_R_NANCOUNT 2 /* number of non-finite values in u, v, w, p          */
#define CHAPSIM_R_CFL 7      /* CFLMM: TG CFL_tg (src/CFL.f90:1-40) on u, v, w; IO
                                CFL_io on G plus CFL_VISCOUS (:42-133)            */

/* Per-phase timer slots for chapsim_phase_times (milliseconds, accumulated). */
#define CHAPSIM_PH_RHS 0     /* convection + RHS assembly (+ mass-flux sum)   */
#define CHAPSIM_PH_ADIX 1    /* x Crank-Nicolson factor                       */
#define CHAPSIM_PH_ADIZ 2    /* z Crank-Nicolson factor                       */
#define CHAPSIM_PH_ADIY 3    /* y Crank-Nicolson factor + q += dq + wall BC   */
#define CHAPSIM_PH_FFTX 4    /* divergence + forward real FFT along x         */
#define CHAPSIM_PH_FFTZ 5    /* forward complex FFT along z                   */
#define CHAPSIM_PH_YSOLVE 6  /* Poisson y-tridiagonals (incl. refinement)     */
#define CHAPSIM_PH_IFFTZ 7   /* inverse FFT along z                           */
#define CHAPSIM_PH_IFFTX 8   /* inverse real FFT along x + phi ghosts         */
#define CHAPSIM_PH_CORR 9    /* velocity + pressure correction + wall BC      */
#define CHAPSIM_PH_COUNT 10

/*
 * Run configuration.  Replaces the module globals the reference reads from
 * readdata.ini (src/READINI.f90:43-435) for the TG channel section.
 * Geometry is the plane channel (icase = ICHANL, y in [-1, 1]).
 */
typedef struct chapsim_config {
  int32_t struct_size; /* sizeof(chapsim_config), for ABI checks             */
  int32_t nx;          /* NCL1_tg, even, >= 8                                */
  int32_t ny;          /* NCL2, >= 4                                         */
  int32_t nz;          /* NCL3, even, >= 8                                   */
  double lx;           /* HX_tg, streamwise length                          */
  double lz;           /* HZ, spanwise length                               */
  double str2;         /* STR2, tanh stretching factor                      */
  int32_t istr2;       /* ISTR2: 1 tanh stretching, 0 uniform               */
  int32_t flowdrvtp;   /* FLOWDRVTP: 1 constant mass flux, 2 constant dp/dx */
  double ren;          /* REN, bulk Reynolds number                         */
  double dt;           /* DT, fixed time step                               */
  double cfgv;         /* CFGV, skin-friction coefficient for flowdrvtp=2   */
  int32_t precision;   /* CHAPSIM_FP64 or CHAPSIM_MIXED                     */
  int32_t device;      /* CUDA device ordinal                               */
} chapsim_config;

typedef struct chapsim_ctx chapsim_ctx;
typedef struct chapsim_props chapsim_props; /* property engine (declared below) */

/* Fill *cfg with defaults (64^3, Lx=4pi, Lz=4pi/3, beta=2, Re=2800, dt=1e-3,
 * constant mass flux, FP64, device 0). */
int chapsim_config_default(chapsim_config *cfg);

/* Set-up: MEM_ALLOCAT + COORDJR + TDMA_COEF + CONS_RKCOEF + CONSPARA +
 * FFT99_POIS3D_INIT(ITG) (src/DNS_THERMAL.f90:117-176,
 * src/possion3d_FFT99.f90:54-220).  Allocates all device state. */
int chapsim_create(const chapsim_config *cfg, chapsim_ctx **out);
int chapsim_destroy(chapsim_ctx *ctx);
const char *chapsim_last_error(const chapsim_ctx *ctx);
int chapsim_sync(chapsim_ctx *ctx);

/* Refinement sweeps of the mixed form's Poisson solve: 1 (the default) forms
 * the FP64 residual RHSLLPHI - L phi (the operator of CHECK_FFT_SOLVER,
 * src/PRESSURE_CORRECTION.f90:159-202) and adds its FP32 spectral solve to
 * phi; 0 keeps the single FP32 solve.  No effect on the FP64 form. */
int chapsim_set_refinement(chapsim_ctx *ctx, int sweeps);

/* Fault injection for the bounded device waits (no reference counterpart;
 * the reference's failure path is ERRHDL, print and STOP,
 * src/WRTHDL.f90:18-30).  Queues one kernel on the context's stream that
 * waits, with a spin limit of polls (1 .. 2^20), on an mbarrier nothing
 * completes -- the give-up path of every TMA consumer.  The wait runs out,
 * the kernel records the timeout in the context's device error word and
 * returns; the next chapsim_sync reports CHAPSIM_ERR_CUDA ("device-side wait
 * gave up") and clears the word, after which the context works normally.
 * Neither faults nor hangs the GPU. */
int chapsim_inject_wait_timeout(chapsim_ctx *ctx, int polls);

/* Length in doubles of one Fortran-layout field: nx*(ny+2)*nz. */
int64_t chapsim_field_len(const chapsim_ctx *ctx);

/* Upload / download one field in Fortran layout.  n must equal
 * chapsim_field_len.  host may be pageable or pinned. */
int chapsim_set_field(chapsim_ctx *ctx, int domain, int field, const double *host, int64_t n);
int chapsim_get_field(chapsim_ctx *ctx, int domain, int field, double *host, int64_t n);
/* Device-resident variants: dev is a device pointer on the context's device.
 * The copy is queued on the context's stream and the call returns at once:
 * order other streams' work after it through chapsim_sync or an event on the
 * stream of chapsim_get_stream. */
int chapsim_set_field_device(chapsim_ctx *ctx, int domain, int field, const double *dev, int64_t n);
int chapsim_get_field_device(chapsim_ctx *ctx, int domain, int field, double *dev, int64_t n);
/* Stream-ordered variants of chapsim_set_field / chapsim_get_field: the copy
 * is queued on the context's stream behind earlier work and the call returns
 * at once; it has completed after chapsim_sync (or any call that returns host
 * data).  The host buffer must stay valid until then; with page-locked memory
 * the copy overlaps other contexts' work (two sections, two contexts), with
 * pageable memory it is as synchronous as the plain call.  The reference has
 * no counterpart: its module arrays are host memory
 * (src/MEMALLOCT.f90:99-210); these serve a host that moves the state in and
 * out every step.  FP32 fields of the mixed form are not accepted
 * (CHAPSIM_ERR_UNSUPPORTED). */
int chapsim_set_field_async(chapsim_ctx *ctx, int domain, int field, const double *host, int64_t n);
int chapsim_get_field_async(chapsim_ctx *ctx, int domain, int field, double *host, int64_t n);

/* Mesh and coefficient arrays (host copies), for checks:
 * what = 0 YND(1:ny+1), 1 YCC(1:ny), 2 DYFI(1:ny), 3 DYCI(1:ny+1). */
int chapsim_get_mesh(const chapsim_ctx *ctx, int what, double *out, int64_t n);

/* Seeded initial field: RANDOM_FL_FLD_TG + CALC_INITIALIZATION_tg
 * (src/INITIAL_FL_FLD_TG.f90:2-119).  Uniform perturbations of amplitude amp
 * on u, v, w from a counter-based splitmix64 keyed by (seed, component, i, j,
 * k), xz-mean removal, the laminar profile 1.5(1-y^2) on u, v = 0 at the wall,
 * bulk velocity rescaled to 1.  When project != 0 an NS=0 substep follows
 * (the reference's initial projection).
 * On an IO context: the same velocity recipe, then h = 0 with the table's
 * properties at h = 0 (T = rho = mu = k = 1 when the table keeps the
 * reference shortcuts), G = rho_stag u scaled to unit bulk mass flux
 * (VELO2MASSFLUX, Unified_massflux, src/INITIAL_FL_THEML_FLD_io.f90:481-682),
 * and with project != 0 CALC_INITIALIZATION_io (:133-172): wall ghosts,
 * SOLVERRK3_ENG_IO(0), SOLVERRK3_MOM_IO(0). */
int chapsim_init_random(chapsim_ctx *ctx, uint64_t seed, double amp, int project);

/* SOLVERRK3_MOM_tg(NS) (src/SOLVERRK3_MOM_tg.f90:18-61), NS in 0..3. */
int chapsim_rk3_mom_tg(chapsim_ctx *ctx, int ns);
/* One full time step: NS = 1, 2, 3. */
int chapsim_step_tg(chapsim_ctx *ctx, int nsteps);

/* Stand-alone pieces of the substep (each updates device state only):
 * DIVG_tg(NS) (src/DIVG.f90:21-57): RHSPHI = div(u)/(alpha dt). */
int chapsim_divg(chapsim_ctx *ctx, int domain, int ns);
/* FFT99_POIS3D_periodicxz(IDOMAIN) (src/possion3d_FFT99.f90:254-488):
 * PHI = L^{-1} RHSPHI (plus the ghost copy of BC_WALL_DPH). */
int chapsim_pois3d(chapsim_ctx *ctx, int domain);
/* VELOUPDT_tg(NS) + PRCALC_tg(NS) with their wall BCs
 * (src/VELO_CORRECTION.f90:19-105, src/PRESSURE_CORRECTION.f90:1-24). */
int chapsim_velo_correction(chapsim_ctx *ctx, int domain, int ns);

/* Device reductions (DIVGCK_tg, BULK_VELOCITY_TG, CFL); synchronises. */
int chapsim_reduce(chapsim_ctx *ctx, int domain, int what, double *out);

/* On-device flow statistics.  chapsim_stats computes the xz-plane averages
 * of PP_MEAN_ZX_FLOW_TG (src/processing/PP_MEAN_ZX.f90:1-294) on a TG context
 * or of PP_MEAN_ZX_FLOW_Xperiodic_IO (src/processing/PP_MEAN_ZX.f90:299-872)
 * on an IO context for every y-row and, with accumulate != 0, folds them into
 * the running time average of PP_MEAN_T_TG / PP_MEAN_T_Xperiodic_IO
 * (src/processing/PP_MEAN_T.f90:322-370, 436-520; asymptotic weights 1/N,
 * (N-1)/N).  chapsim_get_stats copies ny * CHAPSIM_STATS_NV (TG) or
 * ny * CHAPSIM_STATS_IO_NV (IO) values (which = 0: xz average, 1: time
 * average) and the sample count.  TG row j-1: U1 (u, v, w, p), UP (3), U2 (11
 * 12 13 22 23 33), U3 (111 112 113 122 123 133 222 223 233 333), DVDL1 (3x3
 * row-major), DVDLP (3x3), DVDL2 (9x9).  IO row j-1: U1 (u, v, w, p), G1
 * (3), UP (3), U2 (6), UG (6, u_m g_n for m <= n), U3 (10), UGU (10,
 * u_m g_n u_h for m <= n <= h), DVDL1 (3x3), DVDLP (3x3), DVDL2 (9x9: row
 * (m,h), column (n,p)); then, with the energy equation (zero otherwise), T1,
 * D1, H1, M1, T2, D2, H2, DH, PH, DVDL1M (3x3), DVDL1MH (3x3), DVDL1MU
 * (m,n,h), DVDL2M (9x9), UH (3), GH (3), U2DH (6), DhDL1 (3), DhDLP (3),
 * DTDLK (3), DTDLKU (m,n), DTDLKDVDL (m,n,h), DHDLMDVDL (m,n,h).
 * chapsim_stats_reset clears the time average (PP_TMEAN_INI_ZERO_TG / _IO). */
#define CHAPSIM_STATS_NV 122
#define CHAPSIM_STATS_IO_NV 360
int chapsim_stats(chapsim_ctx *ctx, int accumulate);
int chapsim_get_stats(chapsim_ctx *ctx, int which, double *out, int64_t n, int64_t *nstatis);
int chapsim_stats_reset(chapsim_ctx *ctx);

/* Instantaneous-field files in the reference's layout (WRT_INSTANT_VARS_TG /
 * READ_3D_VARS, src/processing/WRT_VARS_TG.f90:1-91,
 * src/processing/READ_INTP_3D_VARS.f90:1-84): one file per variable, 4 x
 * int32 (nx, ny, nz, iteration), 3 x float64 (time, Re, dt), then the
 * interior F(1:nx, 1:ny, 1:nz) in Fortran order, native byte order.  Names
 * <dir>DNS_perixz_INSTANT_T<time, Fortran ES15.9>_<var>.D; var U, V, W, P
 * (TG: Q_tg, PR_tg; IO: G_io, PR_io) and, thermal IO, T, D, E.  An IO
 * context created with coupled = 1 (a TG section runs beside it) uses the
 * prefix DNS_perioz, as the reference does in its TG + IO mode
 * (src/processing/WRT_VARS_IO.f90:24-28, RESTART_io.f90:25-29), so the two
 * sections' files never share a name.
 * chapsim_write_instant writes the context's state; chapsim_read_instant
 * restarts from such files (RESTART_INSTANT_VARS_TG / _IO + FLOWSTART's wall
 * conditions; TG: CONVH0 = 0; IO: RHOH = D E, wall ghosts, THERM_PROP_UPDATE,
 * rho0 = rho, mu0 = mu, u = G / rho_stag, G0 = EXPLT0 = RHS_ENERGY0 = 0) and
 * returns the file's iteration and time.  The coupled inflow / outflow
 * section (non-periodic bcx_in / bcx_out) writes DNS_perioz files of
 * I = 1..NCL1E = nx + 1 (its outlet ghost column; NCL1E in the header) and
 * restarts from them with its inlet source set (chapsim_io_set_inlet, the TG
 * context restarted first): BC_TINLET_THERML and BC_TINLET_FLOW fill the
 * inlet ghost column, the outlet column's u, v, w = G / its face density,
 * the BC_CONV0 terms = 0.  A mesh other than the context's is
 * refused (the reference's interpolation, INTP_3D_VARS, is not built).  The
 * *_file_* calls do the same on host arrays in the F(1:nx, 0:ny+1, 1:nz)
 * layout (ghost rows untouched) and need no GPU. */
int chapsim_write_instant(chapsim_ctx *ctx, const char *dir, int iteration, double time);
int chapsim_read_instant(chapsim_ctx *ctx, const char *dir, double time, int *iteration, double *time_out);
/* tg_and_io != 0 gives the DNS_perioz prefix of an IO section that runs
 * beside a TG section. */
int chapsim_instant_file_name(char *buf, int buflen, const char *dir, double time, const char *var, int tg_and_io);
int chapsim_instant_file_write(const char *path, int nx, int ny, int nz, int iteration, double time, double ren,
                               double dt, const double *field);
int chapsim_instant_file_read(const char *path, int nx, int ny, int nz, int *iteration, double *time, double *ren,
                              double *dt, double *field);

/* Change the time step (DT, the variable of the adaptive step-size control
 * SOLVE.f90:156-213 leaves commented out: DT = min(DT0, 5 DT, CFLGV/CFLMM)).
 * Rebuilds every dt-dependent coefficient table; synchronises. */
int chapsim_set_dt(chapsim_ctx *ctx, double dt);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * work against it. */
int chapsim_get_stream(const chapsim_ctx *ctx, void **stream);

/* Phase timers: enable (1) / disable (0) CUDA-event timing between phases of
 * every substep; read accumulated milliseconds per phase and the number of
 * substeps timed; reset clears them. */
int chapsim_phase_timing(chapsim_ctx *ctx, int enable);
int chapsim_phase_times(chapsim_ctx *ctx, double *ms, int n, int64_t *substeps);
int chapsim_phase_reset(chapsim_ctx *ctx);

/* Launch-shape tuning of one context: z planes per block of the RHS kernel
 * (rhs_nzc; on an IO context the momentum RHS) and rows per block of the x
 * transforms (fft_lb, 0 = default).
 * Results do not depend on fft_lb; rhs_nzc changes only the block order of
 * the mass-flux sum (round-off level). */
int chapsim_set_tuning(chapsim_ctx *ctx, int rhs_nzc, int fft_lb);
int chapsim_get_tuning(const chapsim_ctx *ctx, int *rhs_nzc, int *fft_lb);
/* Spectral y-lines per block of the Poisson y-solve (64, 128 = default, or
 * 256).  Results do not depend on it. */
int chapsim_set_line_tuning(chapsim_ctx *ctx, int ysolve_bx);
int chapsim_get_line_tuning(const chapsim_ctx *ctx, int *ysolve_bx);

/* Number of kernel launches the library issued on this context since creation
 * (or the last reset). */
int chapsim_launch_count(const chapsim_ctx *ctx, int64_t *count);
int chapsim_launch_count_reset(chapsim_ctx *ctx);

/* ======================================================================
 * IO domain: the inflow/outflow section run x-periodic (BCX_io = 3, no TG
 * section, src/READINI.f90:121-131), with the explicit viscous scheme
 * (visthemflg = 0, src/readdata.ini:23), the FISHPACK Poisson solver and,
 * when thermal is on, the energy equation with table properties and
 * iso-flux walls.  A context is either a TG or an IO domain; the functions
 * above that take a domain argument accept CHAPSIM_IIO on an IO context.
 *
 * On an IO context: u, v, w = Q_io, p = PR_io, phi = DPH_io, rhsphi =
 * RHSLLPHI_io, H0U/H0V/H0W = EXPLT0_io(:,:,:,1..3), plus the fields below.
 * Precision forms: FP64, and (explicit viscous scheme) CHAPSIM_MIXED, whose
 * fields all stay FP64 and whose Poisson solve runs on FP32 spectra.
 * ====================================================================== */
#define CHAPSIM_F_GX 10     /* G_io(:,:,:,1), mass flux rho u       */
#define CHAPSIM_F_GY 11     /* G_io(:,:,:,2)                        */
#define CHAPSIM_F_GZ 12     /* G_io(:,:,:,3)                        */
#define CHAPSIM_F_G0X 13    /* G0_io: G at the start of the last momentum substep */
#define CHAPSIM_F_G0Y 14
#define CHAPSIM_F_G0Z 15
#define CHAPSIM_F_H 16      /* ENTHALPY    */
#define CHAPSIM_F_T 17      /* TEMPERATURE */
#define CHAPSIM_F_RHO 18    /* DENSITY     */
#define CHAPSIM_F_MU 19     /* VISCOUSITY  */
#define CHAPSIM_F_K 20      /* THERMCONDT  */
#define CHAPSIM_F_RHOH 21   /* RHOH        */
#define CHAPSIM_F_RHO0 22   /* DENSITY0    */
#define CHAPSIM_F_MU0 23    /* VISCOUSITY0 */
#define CHAPSIM_F_DRHO 24   /* DrhoDtP     */
#define CHAPSIM_F_RHSE0 25  /* RHS_ENERGY0 */

/* Coupled inflow/outflow boundary planes of the IO section.  The reference
 * couples the TG section to the IO section's inlet and gives the IO outlet a
 * convective condition (TGFLOWFLG): the IO arrays carry ghost columns i = 0
 * and i = NCL1_io + 1.  An IO context holds those ghost planes, each
 * (nz, ny + 2) doubles at [k * (ny + 2) + j], plus the outlet's RK3 memory
 * terms; the operators below fill and advance them from the context's own
 * fields (its last column i = NCL1_io is the interior next to the outlet).
 * The inlet ghost properties are the reference state (BC_TINLET_THERML:
 * rho = T = mu = k = 1, rho h = h = 0); only rho is stored. */
#define CHAPSIM_P_IN_U 0
#define CHAPSIM_P_IN_V 1
#define CHAPSIM_P_IN_W 2
#define CHAPSIM_P_IN_GX 3
#define CHAPSIM_P_IN_GY 4
#define CHAPSIM_P_IN_GZ 5
#define CHAPSIM_P_IN_P 6
#define CHAPSIM_P_IN_RHO 7
#define CHAPSIM_P_OUT_U 8
#define CHAPSIM_P_OUT_V 9
#define CHAPSIM_P_OUT_W 10
#define CHAPSIM_P_OUT_GX 11
#define CHAPSIM_P_OUT_GY 12
#define CHAPSIM_P_OUT_GZ 13
#define CHAPSIM_P_OUT_RHO 14
#define CHAPSIM_P_OUT_RHOH 15
#define CHAPSIM_P_OUT_H 16
#define CHAPSIM_P_OUT_T 17
#define CHAPSIM_P_OUT_MU 18
#define CHAPSIM_P_OUT_K 19
#define CHAPSIM_P_CONV0_X 20   /* BC_CONV0(:, :, 1..3) */
#define CHAPSIM_P_CONV0_Y 21
#define CHAPSIM_P_CONV0_Z 22
#define CHAPSIM_P_CONV0_ENG 23 /* BC_CONV0_ENG */
#define CHAPSIM_P_COUNT 24

/* BC_TINLET_FLOW + BC_TINLET_THERML (src/BC_INLET.f90:2-76): the TG context's
 * last plane (u, v, w, p at i = NCL1_tg) becomes the inlet ghost plane, the
 * TG first-face u becomes the IO first-face u, and G follows with the inlet
 * density.  Writes the IO context's u and G_io at i = 1 (first face).  Both
 * contexts on one device with equal ny, nz; waits for the TG context's queued
 * work and returns when the planes are written. */
int chapsim_io_bc_inlet(chapsim_ctx *io, chapsim_ctx *tg);
/* BC_COUTLET_MOM_RK3(NS) (src/BC_COUTLET_MOM_RK3.f90:2-97) with
 * CONVCTION_OUTLET_U (:101-174) and CHK_MassConsv_io
 * (src/processing/CHK_conservation.f90:2-71): dG/dt + U_OUTLET dG/dx = 0 on
 * the outlet plane with the RK3 weights of NS, the outlet x-flux rescaled so
 * that inflow - d(rho)/dt = outflow, wall conditions on the plane. */
int chapsim_io_bc_outlet_mom(chapsim_ctx *io, int ns);
/* BC_COUTLET_ENEG_RK3(NS) (src/BC_COUTLET_ENEG_RK3.f90:2-41): the same
 * convective condition for rho h, then the property update of the outlet
 * plane (ENTHALPY_UPDATE, DENSITY_UPDATE, THERM_PROP_UPDATE, region IOULET)
 * and its iso-flux ghost rows.  Needs the energy equation and a table. */
int chapsim_io_bc_outlet_eng(chapsim_ctx *io, int ns);
/* Copy one ghost plane (id CHAPSIM_P_*, n = (ny + 2) * nz) in or out. */
int chapsim_io_set_plane(chapsim_ctx *io, int plane, const double *host, int64_t n);
int chapsim_io_get_plane(chapsim_ctx *io, int plane, double *host, int64_t n);
/* out[0..6]: U_OUTLET of the last momentum call, CHK_Mass_CONSV0_SCALING,
 * CHK_MASS_CONSV0 (inflow - mass rate - outflow before the rescaling),
 * inflow, outflow, mass rate, U_OUTLET of the last energy call; n >= 7. */
int chapsim_io_bc_scalars(chapsim_ctx *io, double *out, int n);

/* IO reductions (chapsim_reduce with domain CHAPSIM_IIO): CHAPSIM_R_DIVMAX is
 * DIVGCK_io's max|div G + DrhoDtP| (src/DIVGCK.f90:60-190), CHAPSIM_R_BULK is
 * BULK_VELOCITY_IO (src/INITIAL_FL_THEML_FLD_io.f90:385-413), and: */
#define CHAPSIM_R_DIVMAX_Q 3 /* max|div u| (DIVGCK_Q_comm_io)              */
#define CHAPSIM_R_BULK_G 4   /* BULK_MASSFLUX_IO                           */
#define CHAPSIM_R_BULK_H 5   /* BULK_H_IO                                  */
#define CHAPSIM_R_BADCELLS 6 /* table look-ups outside the table so far    */
#define CHAPSIM_R_MODEL_AGAIN 8 /* learned properties: 128-cell tiles whose second
                                   enthalpy was evaluated anew rather than by the
                                   first-order expansion, so far              */

typedef struct chapsim_io_config {
  int32_t struct_size; /* sizeof(chapsim_io_config)                               */
  int32_t thermal;     /* thermlflg: 1 energy equation + table properties, 0 off   */
  double prt;          /* PRT0, Prandtl number                                     */
  double qw_bot;       /* iso-flux bottom wall: heat flux, > 0 heats the fluid; an
                          iso-thermal bottom wall: its temperature (WHEAT0_UNDIM) */
  double qw_top;       /* iso-flux top wall (WALLFLUX = -qw_top, Flow_State.f90:124-148);
                          iso-thermal: its temperature                          */
  int32_t gravdir;     /* GRAVDIR: 0 none, 1/2/3 buoyancy along x/y/z             */
  int32_t visc_scheme; /* visthemflg (readdata.ini:23): 0 explicit viscous terms,
                          1 semi-implicit (VISCOUS_PAR_EXPLT_*_io + MOMFA_io,
                          src/SOLVERRK3_MOM_IO.f90:73-87)                       */
  double f_a;          /* F_A, buoyancy coefficient (Flow_State.f90:98-110)         */
  int32_t coupled;     /* TGFLOWFLG beside IOFLOWFLG: a TG section runs with this IO
                          section (src/READINI.f90:121-131); its instantaneous-field
                          files then take the prefix DNS_perioz instead of
                          DNS_perixz (src/processing/WRT_VARS_IO.f90:24-28)      */
  int32_t isothermal;  /* BCWALLHEAT: bit 0 the bottom wall, bit 1 the top wall is
                          iso-thermal (BC_WALL_ISOTHERMAL, src/BC_WALL.f90:462-515:
                          ghost rows hold the wall values of T, h, rho, mu, k,
                          from the table at the wall temperature,
                          WALL_ISOTHERMAL_GIVEN, src/Flow_State.f90:603-645);
                          a clear bit keeps the iso-flux wall (BC_WALL_ISOFLUX)  */
  int32_t bcx_in;      /* BCX_io(1), BCX_io(2) (src/READINI.f90:117-171): 1 Dirichlet, */
  int32_t bcx_out;     /* 2 Neumann, 3 periodic (both 3, the default).  Dirichlet /
                          Neumann ends make the section the coupled inflow /
                          outflow one (TGFLOWFLG, src/READINI.f90:127-131; the
                          reference's example is 2, 1): its fields carry the x
                          ghost columns IC = 0 and NCL1_io + 1, so every field
                          is (nz, ny + 2, nx + 2) (chapsim_field_len), the
                          Poisson solve takes FISHPACK's SINT / SINQ / COST /
                          COSQ x transform, a TG context feeds the inlet
                          (chapsim_io_set_inlet) and the outlet is convective.
                          FP64, explicit viscous terms, iso-flux walls, table
                          properties; statistics, instantaneous-field files and
                          the stand-alone boundary and property entry points
                          are for x-periodic sections                        */
} chapsim_io_config;

/* Defaults: thermal on, Pr = 0.71, qw = 1 on both walls (iso-flux), no
 * buoyancy, explicit viscous terms. */
int chapsim_io_config_default(chapsim_io_config *io);

/* IO domain set-up (MEM_ALLOCAT + COORDJR + FISHPACK_POIS3D_INIT,
 * src/DNS_THERMAL.f90:117-176, src/possion3d_fishpack_reform.f90:337-430):
 * cfg gives the IO grid (nx = NCL1_io, lx = HX_io); precision FP64, or
 * CHAPSIM_MIXED with visc_scheme = 0. */
int chapsim_create_io(const chapsim_config *cfg, const chapsim_io_config *io, chapsim_ctx **out);

/* Property table of an IO context: columns H, T, D, M, K (host, length n >= 4,
 * H and T increasing), splined as NIST_SPLINE_H / NIST_SPLINE_T.  An
 * iso-thermal wall takes its h, rho, mu, k from the table's T-splines at the
 * wall temperature here (CHAPSIM_ERR_ARG when that temperature is outside the
 * table).  shortcuts
 * != 0 keeps the reference-state shortcuts of the look-ups (h = 0 -> T = 1;
 * T = 1 -> rho = mu = k = 1; cells with |h| < 1e-10 keep their properties,
 * src/Flow_State.f90:1068,1470 and src/THERM_PROP_UPDATE.f90:168-173), which
 * assume a table normalised so that h = 0 is the reference state; 0 evaluates
 * the table everywhere.  Also sets RHOHmax (src/Flow_State.f90:963-990). */
int chapsim_set_table(chapsim_ctx *ctx, const double *H, const double *T, const double *D, const double *M,
                      const double *K, int n, int shortcuts);

#define CHAPSIM_PROPS_TABLE 0 /* cubic splines, as THERM_PROP_UPDATE                */
#define CHAPSIM_PROPS_MLP 1   /* learned model on the tensor cores (BF16 operands, FP32
                                 accumulation) where the error gate allows it, table
                                 splines elsewhere                                   */
/* The wall values of an IO context's iso-thermal walls (WALL_ISOTHERMAL_GIVEN,
 * src/Flow_State.f90:603-645: T_WAL_GV, H_WAL_GV, D_WAL_GV, M_WAL_GV, K_WAL_GV):
 * out[5 * side + q], side 0 bottom, 1 top, q = T, h, rho, mu, k; zero for a
 * wall that is not iso-thermal (the reference's zero-initialised arrays). */
int chapsim_io_wall_values(const chapsim_ctx *ctx, double *out, int n);

/* Property evaluation of an IO context (the THERM_PROP_UPDATE of
 * src/THERM_PROP_UPDATE.f90:129-205 with its DENSITY_UPDATE / ENTHALPY_UPDATE
 * companions, as SOLVERRK3_ENG_IO calls them, src/SOLVERRK3_ENG_IO.f90:46-55).
 * mode CHAPSIM_PROPS_TABLE: the table splines (the default, and the state
 * after chapsim_set_table).  mode CHAPSIM_PROPS_MLP: the learned model of the
 * engine pe (trained on the same table and gated by chapsim_props_gate; see
 * the property engine below), copied into the context, so pe may be
 * destroyed afterwards; the energy substep then evaluates the model on the
 * tensor cores and takes the table splines in every h-bin the gate has not
 * cleared for T, rho, mu and k.  The wall ghost rows (BC_WALL_ISOFLUX) keep
 * the table splines.  pe is ignored for the table mode. */
int chapsim_set_props_mode(chapsim_ctx *ctx, int mode, const chapsim_props *pe);
/* THERM_PROP_UPDATE(IREGION) on an IO context: h -> T, mu, k, rho on the
 * interior rows by the table (mode CHAPSIM_PROPS_TABLE) or the context's
 * model (CHAPSIM_PROPS_MLP, after chapsim_set_props_mode); cells with
 * |h| < 1e-10 keep their properties when the table keeps the reference
 * shortcuts; out-of-table cells are counted (CHAPSIM_R_BADCELLS).  Regions:
 * the reference's IMAIND (0) and IALLDM (2), which coincide on an IO
 * context; IOULET (1), the outlet plane, is updated by
 * chapsim_io_bc_outlet_eng. */
#define CHAPSIM_IMAIND 0
#define CHAPSIM_IOULET 1
#define CHAPSIM_IALLDM 2
int chapsim_therm_prop_update(chapsim_ctx *ctx, int iregion, int mode);

/* SOLVERRK3_ENG_IO(NS) (src/SOLVERRK3_ENG_IO.f90:1-77): energy RHS, rho h
 * update with the RHOHmax limiter, ENTHALPY/DENSITY_UPDATE,
 * THERM_PROP_UPDATE and the iso-flux wall ghosts. */
int chapsim_rk3_eng_io(chapsim_ctx *ctx, int ns);
/* SOLVERRK3_MOM_IO(NS) (src/SOLVERRK3_MOM_IO.f90:1-168).  For ns >= 1 it is
 * preceded by what SOLVE runs between the energy and momentum substeps
 * (src/SOLVE.f90:121-132): DENSITY_TIME_DERIVATION, DENSITY_Staggered,
 * MU_Staggered (formed on the fly) and VELOCITY_CALC_io. */
int chapsim_rk3_mom_io(chapsim_ctx *ctx, int ns);
/* nsteps full steps: for NS = 1, 2, 3, eng (thermal) then mom.  A coupled
 * section reads its TG source's fields as they stand (a frozen inflow). */
int chapsim_step_io(chapsim_ctx *ctx, int nsteps);

/* The coupled inflow / outflow section (non-periodic bcx_in / bcx_out).
 * chapsim_io_set_inlet names the TG context (same device, ny, nz) whose
 * fields BC_TINLET_FLOW reads in the section's momentum substeps; from then
 * on the section's kernels run in the TG context's stream order.  tg = NULL
 * detaches (so does destroying either context).  Set it before
 * chapsim_init_random, whose NS = 0 projection applies the inlet.  In a
 * coupled substep (SOLVERRK3_MOM_IO / SOLVERRK3_ENG_IO with TGFLOWFLG,
 * src/SOLVERRK3_MOM_IO.f90:15-168, src/SOLVERRK3_ENG_IO.f90:57-64):
 * BC_TINLET_FLOW and BC_COUTLET_MOM_RK3 with CHK_MassConsv_io on the ghost
 * columns, the x-momentum from the second face (NXI = 2) with no DPGRNS
 * forcing, DIVG_io and FISHPACK_POIS3D_SIMPLE on the IO arrays (the
 * reference's coupled branch passes the TG arrays, :116-121; the IO-only
 * branch's are used here), MASSFLUX_UPDATE_IO up to the outlet face
 * (src/VELO_CORRECTION.f90:124-139), BC_TINLET_THERML and
 * BC_COUTLET_ENEG_RK3.  The inlet face keeps its value, so div G is not
 * projected out of the first column (the cosine basis of the Neumann inlet
 * is even about that column's face); the other columns are divergence-free
 * to round-off. */
int chapsim_io_set_inlet(chapsim_ctx *io, chapsim_ctx *tg);
/* nsteps steps of both sections in SOLVE's order (src/SOLVE.f90:119-134):
 * for NS = 1, 2, 3, SOLVERRK3_MOM_tg(NS), then SOLVERRK3_ENG_IO(NS) and
 * SOLVERRK3_MOM_IO(NS); one captured graph per step. */
int chapsim_step_coupled(chapsim_ctx *tg, chapsim_ctx *io, int nsteps);


/* ======================================================================
 * Thermal properties: table splines (THERM_PROP_UPDATE) and the learned
 * property model.
 *
 * A property engine holds a non-dimensional property table (the columns
 * NIST_H, NIST_T, NIST_D, NIST_M, NIST_K, NIST_CP of the reference's
 * thermal_info module after NIST_TABLE_SCALING, src/Flow_State.f90:394-433),
 * its cubic splines (NIST_SPLINE_H / NIST_SPLINE_T, src/Flow_State.f90:916,
 * 1296, coefficients by CUBIC_SPLINE :1693-1787) and, optionally, a learned
 * model h -> (T, rho, mu, k, cp), which has no counterpart in the reference:
 * per output a least-squares polynomial of degree 5 in x = (h - hmid) / hhalf
 * plus an MLP 1 -> 64 -> 64 -> 5 (tanh) for the standardised residual,
 *   out_o = base_o(x) + mean_o + std_o * MLP(x)_o.
 * ====================================================================== */

/* Build the engine from n >= 4 strictly increasing H (with T increasing too).
 * Columns are host arrays of length n. */
int chapsim_props_create(const double *H, const double *T, const double *D, const double *M, const double *K,
                         const double *CP, int n, int device, chapsim_props **out);
int chapsim_props_destroy(chapsim_props *pe);
const char *chapsim_props_last_error(const chapsim_props *pe);

/* THERM_PROP_UPDATE(IREGION) (src/THERM_PROP_UPDATE.f90:129-205) on n cells
 * of device arrays: h -> T (spline in h), then mu, k, rho (splines in T).
 * Cells with |h| < 1e-10 are left unchanged, as in the reference; cells whose
 * h or T lies outside the table are left unchanged and counted (the
 * reference STOPs there): the call then returns CHAPSIM_ERR_RANGE and
 * *n_out_of_range holds the count.  cp may be NULL; when given it receives
 * cp(h) (spline in h, NIST_HCP).  With mode CHAPSIM_PROPS_MLP each output
 * comes from the learned model where the gate cleared it for the cell's h-bin
 * and from the splines elsewhere.  Work runs on the engine's stream and the
 * call synchronises. */
#define CHAPSIM_ERR_RANGE 8
int chapsim_props_update(chapsim_props *pe, int mode, const double *h, double *T, double *rho, double *mu,
                         double *k, double *cp, int64_t n, int64_t *n_out_of_range);

/* Train the model on the GPU on nsamples table samples drawn uniformly in h
 * from seed: the polynomial base by least squares (host, FP64), then the MLP
 * on the standardised residual by the project's own forward, backward and
 * Adam kernels (FP32): full-batch Adam for `steps` steps, learning rate lr
 * decayed by cosine to lr/100.  *final_loss receives the last mean-squared
 * error of the standardised residuals. */
int chapsim_props_train(chapsim_props *pe, int nsamples, uint64_t seed, int steps, double lr, double *final_loss);

/* Error gate: evaluate the model (the tensor-core inference) and the table
 * splines on 8 points per table interval, split [H_1, H_n] into nbins bins
 * (<= 4096), and clear output o of bin b for the model when its largest
 * error there, relative to the output's largest magnitude over the table, is
 * <= tol; uncleared outputs come from the table.  Returns the number of bins
 * cleared for all of T, rho, mu and k (the outputs THERM_PROP_UPDATE
 * produces) and the worst error of those four.
 * chapsim_props_gate_outputs reports, for the last gate call and each output
 * (T, rho, mu, k, cp), the bins cleared and the worst error (n = 5). */
int chapsim_props_gate(chapsim_props *pe, double tol, int nbins, int *n_mlp_bins, double *max_rel_err);
int chapsim_props_gate_outputs(const chapsim_props *pe, int *bins, double *max_rel_err, int n);

/* Model parameters (float32, 4613 values: W1[64] b1[64] W2[64][64] b2[64]
 * W3[5][64] b3[5]) and its normalisation (42 values: hmid, hhalf, then
 * mean[5], std[5], base[5][6], the polynomial coefficients of each output in
 * powers of x, lowest first). */
int chapsim_props_get_params(const chapsim_props *pe, float *params, int nparams, double *norm, int nnorm);
int chapsim_props_set_params(chapsim_props *pe, const float *params, int nparams, const double *norm, int nnorm);

/* Gradient check: loss and gradient of the MSE over a given batch (host
 * arrays: x = normalised inputs, t = standardised targets [n][5]), computed by
 * the training kernels. */
int chapsim_props_loss_grad(chapsim_props *pe, const float *x, const float *t, int n, double *loss, float *grad,
                            int nparams);

/* ======================================================================
 * Batched channels: many independent TG channels of uneven sizes advanced
 * together.  No reference counterpart (the reference runs one domain per
 * job); each channel is a full chapsim_ctx.  chapsim_batch_step replays ONE
 * captured CUDA graph per time step that holds every channel's three
 * substeps as parallel branches, so small channels fill the GPU together.
 * ====================================================================== */
typedef struct chapsim_batch chapsim_batch;
int chapsim_batch_create(const chapsim_config *cfgs, int n, chapsim_batch **out);
int chapsim_batch_destroy(chapsim_batch *b);
const char *chapsim_batch_last_error(const chapsim_batch *b);
/* The i-th channel's context (for fields and reductions); owned by the batch. */
int chapsim_batch_channel(chapsim_batch *b, int i, chapsim_ctx **ctx);
/* chapsim_init_random on every channel, channel i with seed + i. */
int chapsim_batch_init_random(chapsim_batch *b, uint64_t seed, double amp, int project);
/* Autotuner: for every channel, time each candidate launch shape (z-segment
 * length of the RHS kernel, rows per block of the x transforms, then the
 * y-line block width of the Poisson solve) over `reps` substeps and keep the
 * fastest.  The channel state is saved before and restored after the
 * trials. */
int chapsim_batch_autotune(chapsim_batch *b, int reps);
/* nsteps time steps of every channel (one graph launch per step). */
int chapsim_batch_step(chapsim_batch *b, int nsteps);
int chapsim_batch_sync(chapsim_batch *b);
/* The stream the batch graph is launched on (a cudaStream_t). */
int chapsim_batch_get_stream(const chapsim_batch *b, void **stream);
/* Total kernel launches inside one step's graph. */
int chapsim_batch_kernels_per_step(const chapsim_batch *b, int64_t *count);

/* ======================================================================
 * Allocation-free check.  No counterpart in the reference: it is the
 * DIVGCK_tg maximum (src/DIVGCK.f90:16-58) offered without a context for
 * callers that may not allocate device memory when they need the check --
 * e.g. a host recording its time step into its own CUDA graph (no cudaMalloc
 * while a stream is captured) or a host whose device memory is a fixed pool
 * managed by its own allocator.
 *
 * max |div u| of caller-owned device arrays u, v, w (Fortran layout
 * F(1:nx, 0:ny+1, 1:nz)) with dyfi[j] = DYFI(j) at index j (length >= ny+1),
 * written to *out (a device pointer), on `stream` (a cudaStream_t, NULL for
 * the default stream); the call does not synchronise.  Scratch: one
 * file-scope device array of 65,536 tile maxima (512 KiB, held by every GPU
 * that loads the library until exit), enough for channels of up to 65,536
 * tiles of 32 x 8 (x, y) cells summed over the z planes (for example
 * 256 x 256 x 256); larger channels return CHAPSIM_ERR_TOO_LARGE.  No
 * cudaMalloc, cudaFree or other allocation.  The first call on a device looks
 * up the scratch address with that device current, so make it before any
 * stream capture.  All calls share the scratch (it keeps the last call's
 * tile maxima; every slot a call reads it writes first), so calls that
 * overlap on the GPU race.  The call reports only its own launches: if a CUDA
 * error is already pending on the calling thread it returns CHAPSIM_ERR_CUDA
 * at once, launches nothing and leaves that error for the caller to read. */
#define CHAPSIM_ERR_TOO_LARGE 9
int chapsim_divmax_noalloc(const double *u, const double *v, const double *w, const double *dyfi, int nx, int ny,
                           int nz, double dxi, double dzi, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CHAPSIM_H */
