// Internal definitions shared by the libchapsim translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/chapsim.h"
#include "mlp_tc.cuh"
#include "spline.cuh"

namespace chapsim {

// Device-side parameters of one TG domain, passed by value to every kernel.
// Index convention: field(i, j, k) at i + nx*(j + (ny+2)*k), i in [0,nx),
// j in [0,ny+1] (j = 0 and ny+1 are the wall ghost layers), k in [0,nz).
// Spectral data: S(kx, j, kz) at kx + lp*((j-1) + ny*kz), kx in [0,lh).
struct TGDev {
  int nx, ny, nz, lh;
  int lp;          // pitch of a spectral row: lh rounded up to even (16-byte rows)
  int64_t sy, sz;  // strides of j and k in a field
  // FP64 state
  double *u, *v, *w, *p, *phi, *rhsphi;
  void *h0[3];      // CONVH0 (temporary precision)
  // temporaries (double in the FP64 form, float in the mixed form)
  void *rhs[3];
  void *dq[3];      // x/z-solved increments (banded-inverse path)
  void *spec;       // complex spectral array
  double2 *ypiv;    // Poisson y-line pivots: pp_j then h_j, each in the spectral layout
  double *res;      // FP64 Poisson residual (refinement sweep of the mixed form)
  double *partials; // per-block mass-flux partial sums
  double *scal;     // device scalars: [0] dpgrns, [1..] reduction outputs
  int *err;         // device error word (bounded waits that gave up)
  // mesh coefficients (1-based in j, arrays of length ny+2)
  const double *dyfi, *dyci, *wff, *wfb;
  const double *amvr[3], *acvr[3], *apvr[3];
  const double *amph, *acph, *apph;
  const double *ak1, *ak3;
  double dxi, dzi, dxqi, dzqi, cvisc, dt, volm;
  // IO domain Poisson (FISHPACK_POIS3D_SIMPLE): drho is added to the
  // divergence of the forward x-transform, and pin_last = 1 pins the mean
  // mode at the last y-row instead of decoupling row 1.
  const double *drho;
  int pin_last;
  int skip_rhs;  // 1: the fused forward x-transform does not store RHSLLPHI
  // 1: the coupled inflow / outflow IO section (non-periodic x): the fields
  // carry the ghost columns i = -1 (IC = 0) and i = nx (IC = NCL1_io + 1),
  // sy = nx + 2, and x neighbours do not wrap
  int xnp;
};

// Device-side state of an IO domain (x-periodic channel section), on top of
// the TGDev fields it shares: u, v, w = Q_io, p = PR_io, phi = DPH_io,
// rhsphi = RHSLLPHI_io, h0[0..2] = EXPLT0_io (FP64).  The mass flux G_io and
// its value at the start of the last momentum substep (G0_io) live in the
// two buffers g[0..1]; which one holds G alternates every substep.
struct IODev {
  double *g[2][3];
  double *drho;                               // DrhoDtP
  double *rhoh, *h, *T, *D, *D0, *mu, *mu0, *kap, *rhse0;  // RHOH, ENTHALPY, ..., RHS_ENERGY0
  double *msum;                               // mu0 + mu (derived, kept in step)
  chapsim_spl::Spline ht, td, tm, tk;          // h -> T; T -> rho, mu, k
  double cthecd, qw_bot, qw_top, rhohmax, f_a, cfgv;
  int thermal, shortcuts, gravdir, flowdrvtp;
  // iso-thermal walls: bit 0 bottom, bit 1 top (BCWALLHEAT); wall[side] =
  // T, h, rho, mu, k at the wall temperature (qw_bot / qw_top hold it)
  int isothermal;
  double wall[2][5];
  double *dpg;       // device scalar: DPGRNS of the current substep
  double *part;      // per-block partial sums of the x mass-flux forcing
  unsigned long long *bad;  // table look-ups outside the table
  unsigned long long *model_again;  // learned-property tiles evaluated a second time
  // semi-implicit viscous scheme (visthemflg = 1): DRHOI_STG per component
  // and the wall coefficients AMVR1 / APVRN of TDMA_COEF
  int visc;
  double *drhoi[3];
  double *stg[6];  // MU_STG 1-3, RHO_STG 1-3 of the current substep (energy equation on)
  double amvr1, apvrn;
  // coupled inflow/outflow ghost planes CHAPSIM_P_* ((ny + 2) * nz each, plane
  // q at bcp + q * bps; the coupled substep's own planes P_SAVE_* follow) and
  // their scalars (chapsim_io_bc_scalars)
  double *bcp, *bcs;
  int64_t bps;
};

// Planes after the public CHAPSIM_P_* ones: G0_io of the boundary columns
// kept across a coupled momentum substep (the boundary operators overwrite
// G_io there before the substep's G* is formed): G x, y, z of the inlet ghost
// column, G x of the first face, G x, y, z of the outlet ghost column.
constexpr int P_SAVE_IN = CHAPSIM_P_COUNT;       // + 0..2
constexpr int P_SAVE_FACE1 = CHAPSIM_P_COUNT + 3;
constexpr int P_SAVE_OUT = CHAPSIM_P_COUNT + 4;  // + 0..2
constexpr int P_ALL = CHAPSIM_P_COUNT + 7;

// Per-substep scalars.
constexpr int BAND_ROWS = 13;  // g_0 .. g_12: the widest truncated x / z inverse kept

struct SubParams {
  int ns;
  double gam, roh, alp;
  // y Crank-Nicolson factor rows (length ny+2, j = 1..ny), per component
  const double *ya[3], *ypp[3], *yh[3];
  // cyclic x / z factors: pp, h0, G2 (length n), and scalars
  const double *xpp, *xh0, *xg2;
  double xa, xb, xqq;
  const double *zpp, *zh0, *zg2;
  double za, zb, zqq;
  int flowdrvtp;
  double dp_const;  // flowdrvtp == 2: -0.5*cfgv*alp*dt
  // truncated circulant inverses of the x and z factors (first rows g_0..g_W)
  const double *gx, *gz;
  int wx, wz;
  // the same first rows by value (zero past wx / wz): kernels that index them
  // with compile-time offsets read them from the parameter bank
  double bgx[BAND_ROWS], bgz[BAND_ROWS];
  int band;  // 1: x/z factors applied by k_adixz_band
  // banded inverses of the y factors: yg[c][j*(2*16+1) + 16 + m], m in [-wy, wy]
  const double *yg[3];
  int wy;     // -1: too wide, the Thomas kernel runs
};

struct FFTPlan {
  int n;
  int nrad;
  int rad[16];
  const double2 *tw64;  // exp(-2 pi i m / n), m in [0,n)
  const float2 *tw32;
};

}  // namespace chapsim

struct chapsim_ctx {
  chapsim_config cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;

  chapsim::TGDev d{};
  chapsim::FFTPlan fx{}, fz{};
  // host mesh copies
  std::vector<double> ynd, ycc, dyfi, dyci, wff, wfb;
  double area_inlet = 0.0;
  // host-precomputed substep factor tables and their device copies
  std::vector<double> hcoef;
  double *dcoef = nullptr;
  chapsim::SubParams sp[4]{};
  // allocations owned by the context
  std::vector<void *> allocs;
  int npart = 0;

  // phase timing
  bool timing = false;
  cudaEvent_t ev[CHAPSIM_PH_COUNT + 1]{};  // scratch events for stand-alone use
  static constexpr int kEvSub = 48;       // substeps buffered before a readback
  std::vector<cudaEvent_t> evpool;        // (PH_COUNT + 1) events per buffered substep
  int ev_pending = 0;
  double phase_ms[CHAPSIM_PH_COUNT]{};
  int64_t timed_substeps = 0;

  // TMA descriptors of u, v, w, p for the z-marching RHS kernel
  CUtensorMap rhs_maps[7];
  bool use_tma_rhs = false;
  bool allow_band = true;   // banded x/z inverses when narrow enough
  bool fft_big = false;     // FFT plans with radix 7 or 11
  bool refine = true;       // mixed form: one FP64-residual refinement sweep
  int rhs_nzc = 16;   // z planes per block of k_rhs_tma (autotunable)
  int fft_lb = 0;     // rows per block of the x transforms (0: default)
  int ys_bx = 128;    // spectral y-lines per block of k_ysolve_line (64, 128 or 256; autotunable)
  // IO Poisson with Dirichlet / Neumann x ends (BCX_io): FISHPACK's LP, the
  // spectral descriptor of its nx real x modes and the transposed x-transform
  // matrices (forward with 1 / SCALX)
  int xnp = 0;
  int xoff = 0;  // field pointers start this many values into their allocation (1 with x ghost columns)
  chapsim_ctx *inlet = nullptr;      // coupled section: the TG context feeding BC_TINLET_FLOW
  std::vector<chapsim_ctx *> fed;    // TG context: the coupled sections it feeds
  cudaStream_t own_stream = nullptr;  // the context's stream (a coupled section runs on its TG's)
  cudaGraphExec_t pair_graph[2] = {nullptr, nullptr};  // TG + IO step, by the IO's io_cur at its start
  int64_t pair_kernels = 0;                             // kernels of both contexts in one pair step
  chapsim::TGDev dnp{};
  double *xnp_f = nullptr, *xnp_b = nullptr;
  // LP 3 / 5 (SINQ / COSQ) run through the complex FFT: exp(-i pi m / (2 nx)),
  // m < nx, and 1 / SCALX of the forward transform
  double2 *xnp_qw = nullptr;
  double xnp_rscal = 1.0;
  // CUDA graph of one full step (NS = 1, 2, 3)
  cudaGraphExec_t step_graph = nullptr;
  int64_t kernels_per_step = 0;

  // IO domain (domain == CHAPSIM_IIO)
  int domain = CHAPSIM_ITG;
  chapsim_io_config iocfg{};
  chapsim::IODev io{};
  int io_cur = 0;          // g[io_cur] holds G_io, g[1 - io_cur] holds G0_io
  bool has_table = false;
  int io_npart = 0;
  std::vector<void *> table_allocs;
  std::vector<double> tab[5];  // host copy of the table columns H, T, D, M, K
  cudaGraphExec_t io_graph[2] = {nullptr, nullptr};  // one step starting from io_cur = 0 / 1
  // TMA descriptors of the IO momentum RHS: u, v, w, p, mu0 + mu, g[0][0..2], g[1][0..2], EXPLT0
  CUtensorMap io_maps[14];
  bool use_tma_io = false;
  int io_nzc = 16;  // z planes per block of the TMA momentum RHS
  bool si_smem_set = false;  // semi-implicit solve kernels got their shared-memory limit
  // property evaluation of the energy substep: table splines or the learned
  // model (a copy of a trained engine's model in context-owned buffers)
  int props_mode = CHAPSIM_PROPS_TABLE;
  chapsim_mlp::MlpDev mlp{};
  void *mlp_buf = nullptr;
  bool mlp_smem_set = false;
  // on-device statistics (partials, xz averages, time averages) and the
  // number of samples in the time average
  double *stats_buf = nullptr;
  int64_t nstatis = 0;
};

// Kernel launch wrappers (defined in tg_kernels.cu).
namespace chapsim {
// Phase timer mark: event slot ph of the substep being recorded (timing on).
inline void phase_mark(chapsim_ctx *c, int ph) {
  if (c->timing) cudaEventRecord(c->evpool[(size_t)c->ev_pending * (CHAPSIM_PH_COUNT + 1) + ph], c->stream);
}
int init_kernels(chapsim_ctx *c);
int flush_phase_events(chapsim_ctx *c);
int launch_substep(chapsim_ctx *c, int ns);
int launch_divg(chapsim_ctx *c, int ns);
int launch_pois3d(chapsim_ctx *c);
int xnp_pivots(chapsim_ctx *c);
int xnp_q_setup(chapsim_ctx *c);  // shared-memory limits of the quarter-wave FFT kernels
int xnp_pois3d(chapsim_ctx *c, bool mark = false);  // mark: phase timers 5-8 of a substep
int launch_correction(chapsim_ctx *c, int ns);
int launch_reduce(chapsim_ctx *c, int what, double *host_out);
int launch_bc_q(chapsim_ctx *c);
// fault-injection hook: a bounded mbarrier wait that nothing completes
int launch_wait_probe(chapsim_ctx *c, int polls);
// Poisson solve of an IO domain: DIVG_io of (gx, gy, gz) + drho fused into the
// forward x-transform, then the spectral y-solve with the mean mode pinned at
// the last row, into phi.
int launch_pois_io(chapsim_ctx *c, int ns, double *gx, double *gy, double *gz, const double *drho,
                   bool store_rhs);
// IO domain kernels (io_kernels.cu).
int io_eng(chapsim_ctx *c, int ns);
int io_bc_inlet(chapsim_ctx *c, const chapsim_ctx *tg);
// mass_parts: d.partials already holds the block sums of DrhoDtP / DYFI
int io_bc_outlet_mom(chapsim_ctx *c, int ns, bool mass_parts = false);
int io_bc_outlet_eng(chapsim_ctx *c, int ns);
// coupled section (xnp): DIVG_io of the G buffer buf into RHSLLPHI
int io_np_divg(chapsim_ctx *c, int ns, int buf);
int io_thermal_bc(chapsim_ctx *c);
int io_mom(chapsim_ctx *c, int ns, bool prep);
// semi-implicit scheme: right-hand sides (*npart: the DPGRNS partial count),
// then the x, z, y factor solves writing G* into the other G buffer
int io_mom_si(chapsim_ctx *c, int ns, int *npart);
int io_factor_si(chapsim_ctx *c, int ns);
int io_reduce(chapsim_ctx *c, int what, double *host_out);
int io_correction(chapsim_ctx *c, int ns);
int io_init_maps(chapsim_ctx *c);
int io_refresh_msum(chapsim_ctx *c);
int io_restart_fields(chapsim_ctx *c);
int io_np_restart(chapsim_ctx *c);  // the coupled section's restart sequence
// learned properties (io_kernels.cu): THERM_PROP_UPDATE(IMAIND) by the table
// or the model; kernel attributes; persistent grid size
int io_therm_props(chapsim_ctx *c, int mode);
int mlp_kernel_setup(chapsim_ctx *c);
int mlp_grid(const chapsim_ctx *c, int per_sm);
// the trained model of a property engine and its table (props.cu)
int props_model(const chapsim_props *pe, chapsim_mlp::MlpDev *out, int *device);
bool props_same_table(const chapsim_props *pe, const std::vector<double> *cols5);
// TG statistics (stats.cu)
int stats_run(chapsim_ctx *c, int accumulate);
int stats_get(chapsim_ctx *c, int which, double *host, int64_t n);
int stats_reset(chapsim_ctx *c);
int fill_value(chapsim_ctx *c, double *p, size_t n, double v);
}  // namespace chapsim
