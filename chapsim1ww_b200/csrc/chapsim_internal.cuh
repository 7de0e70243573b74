// Internal definitions shared by the libchapsim translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/chapsim.h"

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
  double2 *ypiv;    // Poisson y-line pivots {pp_j, h_j} per (kx, j, kz)
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
};

// Per-substep scalars.
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
  // CUDA graph of one full step (NS = 1, 2, 3)
  cudaGraphExec_t step_graph = nullptr;
  int64_t kernels_per_step = 0;
};

// Kernel launch wrappers (defined in tg_kernels.cu).
namespace chapsim {
int init_kernels(chapsim_ctx *c);
int flush_phase_events(chapsim_ctx *c);
int launch_substep(chapsim_ctx *c, int ns);
int launch_divg(chapsim_ctx *c, int ns);
int launch_pois3d(chapsim_ctx *c);
int launch_correction(chapsim_ctx *c, int ns);
int launch_reduce(chapsim_ctx *c, int what, double *host_out);
int launch_bc_q(chapsim_ctx *c);
}  // namespace chapsim
