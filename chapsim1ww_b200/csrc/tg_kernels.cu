// sm_100a kernels of the TG channel RK3 substep, SOLVERRK3_MOM_tg
// (src/SOLVERRK3_MOM_tg.f90:18-61 of the CHAPSim1WW reference).
//
// Phase structure (one launch each, all on the context stream):
//   rhs      CONVECTION_X/Y/Z_tg + RHS_CvLpGpS_tg for all three components at
//            once (the three RHS only read the pre-substep velocity), with the
//            constant-mass-flux volume integral reduced per block.
//   dpgrns   fixed-order reduction of the block partials -> uniform dp/dx.
//   adix     MOMFA1_X_tg: cyclic (1 - beta d_xx) lines, staged in shared memory.
//   adiz     MOMFA2_Z_tg: cyclic (1 - beta d_zz) lines, staged in shared memory.
//   adiy     MOMFA3_Y_tg + q += dq + BC_WALL_Q_tg: one thread per (i,k) line.
//   fftx     DIVG_tg + forward real FFT along x (pairs of rows packed as one
//            complex line), scaled 1/nx.
//   fftz     forward complex FFT along z, scaled 1/nz, mean mode zeroed.
//   ysolve   Poisson y-tridiagonal per (kx, kz).
//   ifftz    inverse complex FFT along z.
//   ifftx    inverse real FFT along x -> phi, BC_WALL_DPH ghost copy.
//   corr     VELOUPDT_tg + PRCALC_tg + BC_WALL_Q_tg/BC_WALL_PR_tg.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdio.h>
#include <string.h>

#include "chapsim_internal.cuh"
#include "fft_smem.cuh"
#include "tma.cuh"

namespace chapsim {

#define CK(call)                                                          \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      return CHAPSIM_ERR_CUDA;                                            \
    }                                                                     \
  } while (0)

#define LAUNCHED()                                   \
  do {                                               \
    ++c->launches;                                   \
    cudaError_t e_ = cudaGetLastError();             \
    if (e_ != cudaSuccess) {                         \
      c->err = std::string("kernel launch: ") + cudaGetErrorString(e_); \
      return CHAPSIM_ERR_CUDA;                       \
    }                                                \
  } while (0)

template <typename T> struct Cplx;
template <> struct Cplx<double> { typedef double2 type; };
template <> struct Cplx<float> { typedef float2 type; };

// ----------------------------------------------------------------- helpers
__device__ __forceinline__ int wrapp(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int wrapm(int i, int n) { return i == 0 ? n - 1 : i - 1; }

// Deterministic block sum (fixed shuffle tree, then warps in index order).
__device__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5, nw = (nt + 31) >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (tid == 0)
    for (int i = 0; i < nw; ++i) s += sh[i];
  __syncthreads();
  return s;  // valid in thread 0
}
__device__ double block_max(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5, nw = (nt + 31) >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (tid == 0)
    for (int i = 0; i < nw; ++i) s = fmax(s, sh[i]);
  __syncthreads();
  return s;
}

// ============================================================ rhs kernel
// CONVECTION_X_tg (src/CONVECTION_X.f90:23-74), CONVECTION_Y_tg
// (src/CONVECTION_Y.f90:22-91, channel branch; the bottom wall face j = 1 is
// skipped), CONVECTION_Z_tg (src/CONVECTION_Z.f90:22-75) and RHS_CvLpGpS_tg
// (src/RHS_CvLpGpS_tg.f90:61-176): rhs = dt[gam H + roh H0 + alp/Re L(q)]
// - alp dt grad(p); H0 <- H.  Partial volume integrals of rhs_u/DYFI feed the
// constant-mass-flux correction (:183-198).
constexpr int RHS_BX = 32, RHS_BY = 8;

template <typename T>
__global__ void __launch_bounds__(RHS_BX *RHS_BY)
k_rhs(TGDev d, SubParams sp) {
  __shared__ double sh[32];
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * RHS_BX + threadIdx.x;
  const int j = blockIdx.y * RHS_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  double part = 0.0;
  if (i < nx && j <= ny) {
    const int nz = d.nz;
    const int ip = wrapp(i, nx), im = wrapm(i, nx);
    const int kp = wrapp(k, nz), km = wrapm(k, nz);
    const int64_t sy = d.sy, sz = d.sz;
    const int64_t c0 = i + sy * j + sz * k;
    const int64_t cip = c0 + (ip - i), cim = c0 + (im - i);
    const int64_t ckp = c0 + sz * (kp - k), ckm = c0 + sz * (km - k);
    const double *__restrict__ U = d.u;
    const double *__restrict__ V = d.v;
    const double *__restrict__ W = d.w;
    const double *__restrict__ P = d.p;
    const double u0 = U[c0], uip = U[cip], uim = U[cim], ujp = U[c0 + sy], ujm = U[c0 - sy];
    const double ukp = U[ckp], ukm = U[ckm], uipjm = U[cip - sy], uipkm = U[cip + (ckm - c0)];
    const double v0 = V[c0], vim = V[cim], vip = V[cip], vjp = V[c0 + sy], vimjp = V[cim + sy];
    const double vjm = V[c0 - sy], vkp = V[ckp], vkm = V[ckm], vjpkm = V[ckm + sy];
    const double w0 = W[c0], wim = W[cim], wip = W[cip], wkp = W[ckp], wimkp = W[cim + (ckp - c0)];
    const double wkm = W[ckm], wjm = W[c0 - sy], wjp = W[c0 + sy], wjmkp = W[ckp - sy];
    const double wffj = d.wff[j], wfbj = d.wfb[j], wffp = d.wff[j + 1], wfbp = d.wfb[j + 1];
    const double dyfi = d.dyfi[j];
    const double dxi = d.dxi, dzi = d.dzi;
    const double coe1 = sp.alp * d.cvisc;
    const double coe2 = sp.alp * d.dt;
    // ---- x momentum
    {
      const double h11 = ((uip + u0) * (uip + u0) - (uim + u0) * (uim + u0)) * (0.25 * dxi);
      const double h12 = ((vjp + vimjp) * (wffp * ujp + wfbp * u0) - (v0 + vim) * (wffj * u0 + wfbj * ujm)) *
                         (dyfi * 0.5);
      const double h13 = ((wkp + wimkp) * (ukp + u0) - (w0 + wim) * (u0 + ukm)) * (0.25 * dzi);
      const double H = -(h11 + h12 + h13);
      T *h0 = reinterpret_cast<T *>(d.h0[0]);
      const double rhsc = sp.gam * H + sp.roh * (double)h0[c0];
      const double lap = (uip - 2.0 * u0 + uim) * d.dxqi + (ukp - 2.0 * u0 + ukm) * d.dzqi +
                         (ujp * d.apvr[0][j] + u0 * d.acvr[0][j] + ujm * d.amvr[0][j]);
      h0[c0] = (T)H;
      const double pgm = (P[c0] - P[cim]) * dxi * coe2;
      const double r = (rhsc + coe1 * lap) * d.dt - pgm;
      reinterpret_cast<T *>(d.rhs[0])[c0] = (T)r;
      part = r / dyfi;
    }
    // ---- y momentum (faces j >= 2)
    if (j >= 2) {
      const double h21 = ((wffj * uip + wfbj * uipjm) * (vip + v0) - (wffj * u0 + wfbj * ujm) * (v0 + vim)) *
                         (dxi * 0.5);
      const double h22 = ((vjp + v0) * (vjp + v0) - (v0 + vjm) * (v0 + vjm)) * (d.dyci[j] * 0.25);
      const double h23 = ((wffj * wkp + wfbj * wjmkp) * (vkp + v0) - (wffj * w0 + wfbj * wjm) * (v0 + vkm)) *
                         (dzi * 0.5);
      const double H = -(h21 + h22 + h23);
      T *h0 = reinterpret_cast<T *>(d.h0[1]);
      const double rhsc = sp.gam * H + sp.roh * (double)h0[c0];
      const double lap = (vip - 2.0 * v0 + vim) * d.dxqi + (vkp - 2.0 * v0 + vkm) * d.dzqi +
                         (vjp * d.apvr[1][j] + v0 * d.acvr[1][j] + vjm * d.amvr[1][j]);
      h0[c0] = (T)H;
      const double pgm = (P[c0] - P[c0 - sy]) * d.dyci[j] * coe2;
      reinterpret_cast<T *>(d.rhs[1])[c0] = (T)((rhsc + coe1 * lap) * d.dt - pgm);
    }
    // ---- z momentum
    {
      const double h31 = ((uip + uipkm) * (wip + w0) - (u0 + ukm) * (w0 + wim)) * (0.25 * dxi);
      const double h32 = ((vjp + vjpkm) * (wffp * wjp + wfbp * w0) - (v0 + vkm) * (wffj * w0 + wfbj * wjm)) *
                         (dyfi * 0.5);
      const double h33 = ((wkp + w0) * (wkp + w0) - (w0 + wkm) * (w0 + wkm)) * (0.25 * dzi);
      const double H = -(h31 + h32 + h33);
      T *h0 = reinterpret_cast<T *>(d.h0[2]);
      const double rhsc = sp.gam * H + sp.roh * (double)h0[c0];
      const double lap = (wip - 2.0 * w0 + wim) * d.dxqi + (wkp - 2.0 * w0 + wkm) * d.dzqi +
                         (wjp * d.apvr[2][j] + w0 * d.acvr[2][j] + wjm * d.amvr[2][j]);
      h0[c0] = (T)H;
      const double pgm = (P[c0] - P[ckm]) * dzi * coe2;
      reinterpret_cast<T *>(d.rhs[2])[c0] = (T)((rhsc + coe1 * lap) * d.dt - pgm);
    }
  }
  const double s = block_sum(part, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    d.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
}

// Same arithmetic as k_rhs, organised as a 2.5-D stencil: a block owns a
// 32 x 8 (x, y) tile and marches along z over nzc planes.  Each plane of u,
// v, w, p arrives in shared memory as one TMA box of 36 x 10 doubles
// (x0-2 .. x0+33, j0-1 .. j0+8; the x start is 16-byte aligned), in a ring of
// four plane slots, so plane k+2 is in flight while plane k is computed.
// Periodic x neighbours outside the box are patched in from global memory on
// the first and last x tiles; z wraps by plane index.
constexpr int RT_BXW = 36, RT_BYW = 10, RT_PLANE = RT_BXW * RT_BYW;
// field planes are padded to 368 doubles (2944 B) so every TMA destination is
// 128-byte aligned; a slot holds u, v, w, p of one plane (36 x 10 boxes) and
// the three H0 components of that plane (32 x 8 boxes of T).
constexpr int RT_PST = 368;
constexpr int RT_HBOX = RHS_BX * RHS_BY;  // 256 values
static_assert((RT_PST * 8) % 128 == 0 && RT_PST >= RT_PLANE, "TMA destinations must stay 128-byte aligned");
template <typename T> struct RtLayout {
  static constexpr size_t field_bytes = (size_t)4 * RT_PST * sizeof(double);
  static constexpr size_t h0_bytes = (size_t)RT_HBOX * sizeof(T);  // 2048 or 1024: multiples of 128
  static constexpr size_t slot_bytes = field_bytes + 3 * h0_bytes;
  static constexpr size_t smem_bytes = 4 * slot_bytes + 4 * sizeof(uint64_t);
  static constexpr uint32_t tx_bytes = (uint32_t)(4 * RT_PLANE * sizeof(double) + 3 * RT_HBOX * sizeof(T));
};
struct RhsMaps {
  CUtensorMap m[7];  // u, v, w, p, H0u, H0v, H0w
};

template <typename T>
__global__ void __launch_bounds__(RHS_BX *RHS_BY, 3)
k_rhs_tma(const __grid_constant__ RhsMaps maps, TGDev d, SubParams sp, int nzc) {
  typedef RtLayout<T> L;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto slot_f = [&](int sl) { return reinterpret_cast<double *>(smem_raw + (size_t)sl * L::slot_bytes); };
  auto slot_h = [&](int sl, int c) {
    return reinterpret_cast<T *>(smem_raw + (size_t)sl * L::slot_bytes + L::field_bytes + (size_t)c * L::h0_bytes);
  };
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + 4 * L::slot_bytes);
  __shared__ double red[32];
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + RHS_BX * ty;
  const int x0 = blockIdx.x * RHS_BX, j0 = 1 + blockIdx.y * RHS_BY;
  const int kbeg = blockIdx.z * nzc;
  const int kend = min(kbeg + nzc, nz);
  const int i = x0 + tx, j = j0 + ty;
  const bool active = (i < nx) && (j <= ny);
  const bool left_edge = (x0 == 0), right_edge = (x0 + RHS_BX >= nx);
  const int right_col = nx - x0 + 2;  // smem column of x = nx (wraps to 0)
  if (tid == 0) {
    for (int s = 0; s < 4; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto slot_of = [&](int k) { return (k - kbeg + 1) & 3; };
  auto issue = [&](int k) {
    const int sl = slot_of(k);
    const int kz = k < 0 ? k + nz : (k >= nz ? k - nz : k);
    mbar_expect_tx(&bar[sl], L::tx_bytes);
    for (int f = 0; f < 4; ++f) tma_load_3d(slot_f(sl) + f * RT_PST, &maps.m[f], x0 - 2, j0 - 1, kz, &bar[sl]);
    for (int c3 = 0; c3 < 3; ++c3) tma_load_3d(slot_h(sl, c3), &maps.m[4 + c3], x0, j0, kz, &bar[sl]);
  };
  uint32_t par = 0;  // parity bit per slot, packed
  auto wait_plane = [&](int k) -> bool {
    const int sl = slot_of(k);
    const bool ok = mbar_wait(&bar[sl], (par >> sl) & 1u, d.err);
    par ^= 1u << sl;
    // periodic x patches (generic-proxy writes, fenced before the slot is reused)
    const int kz = k < 0 ? k + nz : (k >= nz ? k - nz : k);
    if (left_edge && tid < 40) {
      const int f = tid / 10, r = tid - f * 10, jr = j0 - 1 + r;
      if (jr <= ny + 1) {
        const double *src = f == 0 ? d.u : (f == 1 ? d.v : (f == 2 ? d.w : d.p));
        slot_f(sl)[f * RT_PST + r * RT_BXW + 1] = src[(nx - 1) + d.sy * jr + d.sz * kz];
      }
    }
    if (right_edge && tid >= 64 && tid < 104) {
      const int q = tid - 64, f = q / 10, r = q - f * 10, jr = j0 - 1 + r;
      if (jr <= ny + 1) {
        const double *src = f == 0 ? d.u : (f == 1 ? d.v : (f == 2 ? d.w : d.p));
        slot_f(sl)[f * RT_PST + r * RT_BXW + right_col] = src[d.sy * jr + d.sz * kz];
      }
    }
    return ok;
  };
  if (tid == 0) {
    issue(kbeg - 1);
    issue(kbeg);
    issue(kbeg + 1);
  }
  bool ok = wait_plane(kbeg - 1);
  ok = wait_plane(kbeg) && ok;
  double part = 0.0;
  const double dxi = d.dxi, dzi = d.dzi, dt = d.dt;
  const double coe1 = sp.alp * d.cvisc, coe2 = sp.alp * dt;
  const int xx = tx + 2, yy = ty + 1;
  // per-row metric and viscous y-operator coefficients, staged once per block
  __shared__ double ycoef[RHS_BY][16];
  if (tid < RHS_BY * 16) {
    const int r = tid >> 4, q = tid & 15, jr = j0 + r;
    double v = 0.0;
    if (jr <= ny) {
      switch (q) {
        case 0: v = d.wff[jr]; break;
        case 1: v = d.wfb[jr]; break;
        case 2: v = d.wff[jr + 1]; break;
        case 3: v = d.wfb[jr + 1]; break;
        case 4: v = d.dyfi[jr]; break;
        case 5: v = d.dyci[jr]; break;
        default:
          if (q < 15) {
            const int cc = (q - 6) / 3, t3 = (q - 6) % 3;
            v = t3 == 0 ? d.apvr[cc][jr] : (t3 == 1 ? d.acvr[cc][jr] : d.amvr[cc][jr]);
          }
      }
    }
    ycoef[r][q] = v;
  }
  const double *yc = ycoef[ty];
  for (int k = kbeg; k < kend; ++k) {
    if (tid == 0 && k + 2 <= kend) {
      fence_proxy_async();
      issue(k + 2);
    }
    ok = wait_plane(k + 1) && ok;
    __syncthreads();
    if (active && ok) {
      const double *Sm = slot_f(slot_of(k - 1));
      const double *Sc = slot_f(slot_of(k));
      const double *Sp = slot_f(slot_of(k + 1));
      const int hc = tid;  // this cell in the 32 x 8 H0 boxes
#define AT(base, f, dx, dy) base[(f) * RT_PST + (yy + (dy)) * RT_BXW + xx + (dx)]
      const double u0 = AT(Sc, 0, 0, 0), uip = AT(Sc, 0, 1, 0), uim = AT(Sc, 0, -1, 0);
      const double ujp = AT(Sc, 0, 0, 1), ujm = AT(Sc, 0, 0, -1), ukp = AT(Sp, 0, 0, 0), ukm = AT(Sm, 0, 0, 0);
      const double uipjm = AT(Sc, 0, 1, -1), uipkm = AT(Sm, 0, 1, 0);
      const double v0 = AT(Sc, 1, 0, 0), vim = AT(Sc, 1, -1, 0), vip = AT(Sc, 1, 1, 0), vjp = AT(Sc, 1, 0, 1);
      const double vimjp = AT(Sc, 1, -1, 1), vjm = AT(Sc, 1, 0, -1), vkp = AT(Sp, 1, 0, 0), vkm = AT(Sm, 1, 0, 0);
      const double vjpkm = AT(Sm, 1, 0, 1);
      const double w0 = AT(Sc, 2, 0, 0), wim = AT(Sc, 2, -1, 0), wip = AT(Sc, 2, 1, 0), wkp = AT(Sp, 2, 0, 0);
      const double wimkp = AT(Sp, 2, -1, 0), wkm = AT(Sm, 2, 0, 0), wjm = AT(Sc, 2, 0, -1), wjp = AT(Sc, 2, 0, 1);
      const double wjmkp = AT(Sp, 2, 0, -1);
      const double p0 = AT(Sc, 3, 0, 0), pim = AT(Sc, 3, -1, 0), pjm = AT(Sc, 3, 0, -1), pkm = AT(Sm, 3, 0, 0);
#undef AT
      const int64_t c0 = i + d.sy * j + d.sz * k;
      {
        const double h11 = ((uip + u0) * (uip + u0) - (uim + u0) * (uim + u0)) * (0.25 * dxi);
        const double h12 = ((vjp + vimjp) * (yc[2] * ujp + yc[3] * u0) - (v0 + vim) * (yc[0] * u0 + yc[1] * ujm)) *
                           (yc[4] * 0.5);
        const double h13 = ((wkp + wimkp) * (ukp + u0) - (w0 + wim) * (u0 + ukm)) * (0.25 * dzi);
        const double H = -(h11 + h12 + h13);
        T *h0 = reinterpret_cast<T *>(d.h0[0]);
        const double rhsc = sp.gam * H + sp.roh * (double)slot_h(slot_of(k), 0)[hc];
        const double lap = (uip - 2.0 * u0 + uim) * d.dxqi + (ukp - 2.0 * u0 + ukm) * d.dzqi +
                           (ujp * yc[6] + u0 * yc[7] + ujm * yc[8]);
        h0[c0] = (T)H;
        const double pgm = (p0 - pim) * dxi * coe2;
        const double r = (rhsc + coe1 * lap) * dt - pgm;
        reinterpret_cast<T *>(d.rhs[0])[c0] = (T)r;
        part += r / yc[4];
      }
      if (j >= 2) {
        const double h21 = ((yc[0] * uip + yc[1] * uipjm) * (vip + v0) - (yc[0] * u0 + yc[1] * ujm) * (v0 + vim)) *
                           (dxi * 0.5);
        const double h22 = ((vjp + v0) * (vjp + v0) - (v0 + vjm) * (v0 + vjm)) * (yc[5] * 0.25);
        const double h23 = ((yc[0] * wkp + yc[1] * wjmkp) * (vkp + v0) - (yc[0] * w0 + yc[1] * wjm) * (v0 + vkm)) *
                           (dzi * 0.5);
        const double H = -(h21 + h22 + h23);
        T *h0 = reinterpret_cast<T *>(d.h0[1]);
        const double rhsc = sp.gam * H + sp.roh * (double)slot_h(slot_of(k), 1)[hc];
        const double lap = (vip - 2.0 * v0 + vim) * d.dxqi + (vkp - 2.0 * v0 + vkm) * d.dzqi +
                           (vjp * yc[9] + v0 * yc[10] + vjm * yc[11]);
        h0[c0] = (T)H;
        const double pgm = (p0 - pjm) * yc[5] * coe2;
        reinterpret_cast<T *>(d.rhs[1])[c0] = (T)((rhsc + coe1 * lap) * dt - pgm);
      }
      {
        const double h31 = ((uip + uipkm) * (wip + w0) - (u0 + ukm) * (w0 + wim)) * (0.25 * dxi);
        const double h32 = ((vjp + vjpkm) * (yc[2] * wjp + yc[3] * w0) - (v0 + vkm) * (yc[0] * w0 + yc[1] * wjm)) *
                           (yc[4] * 0.5);
        const double h33 = ((wkp + w0) * (wkp + w0) - (w0 + wkm) * (w0 + wkm)) * (0.25 * dzi);
        const double H = -(h31 + h32 + h33);
        T *h0 = reinterpret_cast<T *>(d.h0[2]);
        const double rhsc = sp.gam * H + sp.roh * (double)slot_h(slot_of(k), 2)[hc];
        const double lap = (wip - 2.0 * w0 + wim) * d.dxqi + (wkp - 2.0 * w0 + wkm) * d.dzqi +
                           (wjp * yc[12] + w0 * yc[13] + wjm * yc[14]);
        h0[c0] = (T)H;
        const double pgm = (p0 - pkm) * dzi * coe2;
        reinterpret_cast<T *>(d.rhs[2])[c0] = (T)((rhsc + coe1 * lap) * dt - pgm);
      }
    }
    __syncthreads();
  }
  // every issued plane has been waited for (kbeg-1 .. kend), so no bulk copy
  // is in flight when the block exits
  const double s = block_sum(part, red);
  if (tid == 0) d.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
}

// Fixed-order reduction of the mass-flux partials; scal[0] = DPGRNS.
__global__ void __launch_bounds__(1024) k_dpgrns(TGDev d, SubParams sp, int npart) {
  __shared__ double sh[32];
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int stride = blockDim.x * 8;
  for (int t0 = threadIdx.x; t0 < npart; t0 += stride) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int t = t0 + q * blockDim.x;
      if (t < npart) a[q] += d.partials[t];
    }
  }
  double s = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
  s = block_sum(s, sh);
  if (threadIdx.x == 0) d.scal[0] = sp.flowdrvtp == 1 ? s / d.volm : (sp.flowdrvtp == 2 ? sp.dp_const : 0.0);
}

// ============================================================ cyclic lines
// TDMAIJI_CYC (src/TDMAIJI_CYC.f90:67-154) with the coefficient-only parts
// (pivots pp, h0 and the second right-hand side G2 after back substitution,
// plus the corner denominator qq) precomputed on the host, because every line
// of the x and z factors has the same constant coefficients.  s points to the
// line in shared memory, element m at s[m*st].
template <typename T>
__device__ __forceinline__ void cyc_line(T *s, int st, int n, const double *__restrict__ pp,
                                         const double *__restrict__ h0, const double *__restrict__ g2,
                                         double a, double c, double b, double qq) {
  double g = (double)s[0] / b;
  s[0] = (T)g;
  for (int m = 1; m <= n - 2; ++m) {
    g = ((double)s[m * st] - g * a) * pp[m];
    s[m * st] = (T)g;
  }
  // back substitution of g1 (g2 is precomputed)
  double gn = g;  // g1[n-2]
  for (int m = n - 3; m >= 0; --m) {
    gn = (double)s[m * st] - h0[m] * gn;
    s[m * st] = (T)gn;
  }
  const double g10 = gn;
  const double g1n2 = (double)s[(n - 2) * st];
  const double xn = ((double)s[(n - 1) * st] - c * g10 - a * g1n2) / qq;
  s[(n - 1) * st] = (T)xn;
  for (int m = n - 2; m >= 0; --m) s[m * st] = (T)((double)s[m * st] + g2[m] * xn);
}

// MOMFA1_X_tg (src/MOMFA_tg.f90:52-107): rows j0.. of plane k, all three
// components (grid.z), rows contiguous in memory.  The u rows first take off
// the mass-flux correction DPGRNS (src/RHS_CvLpGpS_tg.f90:205-211).
template <typename T>
__global__ void __launch_bounds__(128) k_adix(TGDev d, SubParams sp, int lb) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw);
  const int nx = d.nx, ny = d.ny;
  const int comp = blockIdx.z;
  const int k = blockIdx.y;
  const int jbeg = (comp == 1 ? 2 : 1) + blockIdx.x * lb;
  if (jbeg > ny) return;
  const int nrow = min(lb, ny - jbeg + 1);
  T *g = reinterpret_cast<T *>(d.rhs[comp]) + d.sy * jbeg + d.sz * k;
  const int ld = nx + 1;
  const double sub = comp == 0 ? d.scal[0] : 0.0;
  const int tot = nrow * nx;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int r = t / nx, i = t - r * nx;
    s[r * ld + i] = (T)((double)g[t] - sub);
  }
  // double-precision coefficient tables into shared memory
  double *cf = reinterpret_cast<double *>(smem_raw + (((size_t)lb * ld * sizeof(T) + 15) & ~(size_t)15));
  for (int t = threadIdx.x; t < nx; t += blockDim.x) {
    cf[t] = sp.xpp[t];
    cf[nx + t] = sp.xh0[t];
    cf[2 * nx + t] = sp.xg2[t];
  }
  __syncthreads();
  if (threadIdx.x < nrow)
    cyc_line<T>(s + threadIdx.x * ld, 1, nx, cf, cf + nx, cf + 2 * nx, sp.xa, sp.xa, sp.xb, sp.xqq);
  __syncthreads();
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int r = t / nx, i = t - r * nx;
    g[t] = s[r * ld + i];
  }
}

// MOMFA2_Z_tg (src/MOMFA_tg.f90:111-170): lines along z for consecutive i at
// row j; tile [nz][LZ] in shared memory.
constexpr int LZ = 32;
template <typename T>
__global__ void __launch_bounds__(128) k_adiz(TGDev d, SubParams sp) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw);
  const int nx = d.nx, nz = d.nz;
  const int comp = blockIdx.z;
  const int j = blockIdx.y + 1;
  if (comp == 1 && j == 1) return;
  const int i0 = blockIdx.x * LZ;
  const int nl = min(LZ, nx - i0);
  T *g = reinterpret_cast<T *>(d.rhs[comp]) + i0 + d.sy * j;
  const int tot = nz * LZ;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int kk = t / LZ, l = t - kk * LZ;
    if (l < nl) s[kk * LZ + l] = g[d.sz * kk + l];
  }
  double *cf = reinterpret_cast<double *>(smem_raw + (((size_t)nz * LZ * sizeof(T) + 15) & ~(size_t)15));
  for (int t = threadIdx.x; t < nz; t += blockDim.x) {
    cf[t] = sp.zpp[t];
    cf[nz + t] = sp.zh0[t];
    cf[2 * nz + t] = sp.zg2[t];
  }
  __syncthreads();
  if (threadIdx.x < nl) cyc_line<T>(s + threadIdx.x, LZ, nz, cf, cf + nz, cf + 2 * nz, sp.za, sp.za, sp.zb, sp.zqq);
  __syncthreads();
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int kk = t / LZ, l = t - kk * LZ;
    if (l < nl) g[d.sz * kk + l] = s[kk * LZ + l];
  }
}

// ============================================================ x/z factors
// MOMFA1_X_tg + MOMFA2_Z_tg (src/MOMFA_tg.f90:52-170) applied as the exact
// inverses of their constant-coefficient cyclic tridiagonal matrices.  The
// inverse of (1 - beta delta) on a periodic line is a symmetric circulant whose
// first row g_m (computed on the host by solving A g = e_0 with the same
// two-sweep algorithm) decays geometrically; it is kept up to the width W past
// which the neglected entries sum to < 2^-60 g_0, i.e. below FP64 round-off of
// the solution.  (Wider inverses fall back to k_adix/k_adiz.)  One pass reads
// rhs with an (x, z) halo, applies the x then the z inverse, writes dq.
constexpr int BAND_WMAX = 12;
// z-marching form: a block owns a 32 (x) by 8 (j) tile and a segment of z
// planes.  Each rhs plane of the tile (with its periodic x halo) is loaded
// once, BM_PF planes ahead of its use (a register queue, so that enough loads
// are in flight to cover HBM latency), into a double-buffered shared row; the
// x inverse is applied from it, and each thread keeps the last 2*WZ+1
// x-solved values of its own column in registers: the z inverse over that
// window gives the output plane k - WZ.  WX, WZ are compile-time widths at
// least the inverses' widths (the extra weights are zero), so both stencils
// unroll with their weights read from the parameter bank; the plane loop is
// unrolled by the window length so that the window rotates through static
// register indices.
constexpr int BM_TX = 32, BM_TY = 8, BM_SEG = 64, BM_PF = 1;  // deeper queues measured slower (registers)
constexpr int BAND_TW[5] = {2, 4, 6, 8, 12};  // compiled widths
static_assert(BAND_TW[4] == BAND_WMAX && BAND_WMAX + 1 == BAND_ROWS, "the widest compiled band is the host's limit");
template <typename T, int WX, int WZ>
__global__ void __launch_bounds__(BM_TX *BM_TY) k_adixz_band(TGDev d, SubParams sp) {
  constexpr int RS = 2 * WZ + 1, XW = BM_TX + 2 * WX;
  __shared__ double tin[2][BM_TY][XW];
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int comp = blockIdx.z % 3, seg = blockIdx.z / 3;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * BM_TX, j = 1 + blockIdx.y * BM_TY + ty;
  const int kb = seg * BM_SEG, ke = min(kb + BM_SEG, nz);
  const bool row_ok = (j <= ny) && !(comp == 1 && j == 1);
  const double sub = comp == 0 ? d.scal[0] : 0.0;
  const T *src = reinterpret_cast<const T *>(d.rhs[comp]) + d.sy * (row_ok ? j : 1);
  // this thread's input columns: x0 - WX + tx and x0 - WX + tx + 32 (if < XW)
  int xa = (x0 - WX + tx) % nx;
  xa = xa < 0 ? xa + nx : xa;
  const bool has_b = tx + BM_TX < XW;
  int xb = (x0 - WX + tx + BM_TX) % nx;
  xb = xb < 0 ? xb + nx : xb;
  // planes [pbeg, pend); the host keeps 2 w + 1 <= nz and WZ <= 2 w, so
  // -nz < pbeg and one wrap per step suffices
  const int pbeg = kb - WZ, pend = ke + WZ;
  const int64_t wrap = d.sz * (int64_t)nz;
  int lk = pbeg < 0 ? pbeg + nz : pbeg;  // next plane to load
  const T *lplane = src + d.sz * (int64_t)lk;
  double na[BM_PF], nb[BM_PF];
#pragma unroll
  for (int q = 0; q < BM_PF; ++q) {
    na[q] = 0.0;
    nb[q] = 0.0;
    if (row_ok && pbeg + q < pend) {
      na[q] = (double)lplane[xa] - sub;
      if (has_b) nb[q] = (double)lplane[xb] - sub;
    }
    lplane += d.sz;
    if (++lk == nz) { lk = 0; lplane -= wrap; }
  }
  const int i = x0 + tx;
  T *dst = reinterpret_cast<T *>(d.dq[comp]) + d.sy * j + i;
  double win[RS];  // slot s: plane p0 + s once written in this chunk
#pragma unroll
  for (int q = 0; q < RS; ++q) win[q] = 0.0;
  int buf = 0;
  for (int p0 = pbeg; p0 < pend; p0 += RS) {
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      const int p = p0 + u;
      if (p >= pend) break;  // uniform over the block
      // publish plane p, queue plane p + BM_PF.  One barrier per plane: a
      // buffer is rewritten two planes later, after every thread has passed
      // the barrier of the plane between.
      double *row = tin[buf][ty];
      buf ^= 1;
      row[tx] = na[0];
      if (has_b) row[tx + BM_TX] = nb[0];
#pragma unroll
      for (int q = 0; q + 1 < BM_PF; ++q) {
        na[q] = na[q + 1];
        nb[q] = nb[q + 1];
      }
      if (row_ok && p + BM_PF < pend) {
        na[BM_PF - 1] = (double)lplane[xa] - sub;
        if (has_b) nb[BM_PF - 1] = (double)lplane[xb] - sub;
      }
      lplane += d.sz;
      if (++lk == nz) { lk = 0; lplane -= wrap; }
      __syncthreads();
      const double *rr = row + tx + WX;
      double xs = sp.bgx[0] * rr[0];
#pragma unroll
      for (int m = 1; m <= WX; ++m) xs += sp.bgx[m] * (rr[-m] + rr[m]);
      win[u] = xs;
      if (p - WZ >= kb) {
        // window planes p - 2 WZ .. p; plane p - t sits in slot (u - t) mod RS
        double acc = sp.bgz[0] * win[(u + WZ + 1) % RS];
#pragma unroll
        for (int m = 1; m <= WZ; ++m) acc += sp.bgz[m] * (win[(u + WZ + 1 - m) % RS] + win[(u + WZ + 1 + m) % RS]);
        if (row_ok && i < nx) dst[d.sz * (int64_t)(p - WZ)] = (T)acc;
      }
    }
  }
}

// Row form of the same factors, used when a block can own whole x rows
// (nx = CPT * blockDim.x with blockDim.x <= 256): each plane of the block's
// rows arrives as contiguous rows (no x halo is loaded: the periodic halo is
// written into shared memory from the row itself), thread tx owns columns
// tx + c * blockDim.x, c < CPT, and keeps their z windows in registers.
// Segments of seglen planes per block.
template <typename T, int WX, int WZ, int CPT>
__global__ void __launch_bounds__(256) k_adixz_row(TGDev d, SubParams sp, int seglen) {
  constexpr int RS = 2 * WZ + 1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double *rows = reinterpret_cast<double *>(smem_raw);  // [2][blockDim.y][nx + 2 WX]
  const int nx = d.nx, ny = d.ny, nz = d.nz, RW = nx + 2 * WX;
  const int btx = blockDim.x, tx = threadIdx.x, ty = threadIdx.y;
  const int j = 1 + blockIdx.x * blockDim.y + ty;
  const int comp = blockIdx.y % 3, seg = blockIdx.y / 3;
  const int kb = seg * seglen, ke = min(kb + seglen, nz);
  const bool row_ok = (j <= ny) && !(comp == 1 && j == 1);
  const double sub = comp == 0 ? d.scal[0] : 0.0;
  const T *src = reinterpret_cast<const T *>(d.rhs[comp]) + d.sy * (row_ok ? j : 1) + tx;
  // planes [pbeg, pend); the host keeps 2 w + 1 <= nz and WZ <= 2 w, so
  // -nz < pbeg and one wrap per step suffices
  const int pbeg = kb - WZ, pend = ke + WZ;
  const int64_t wrap = d.sz * (int64_t)nz;
  int lk = pbeg < 0 ? pbeg + nz : pbeg;  // next plane to load
  const T *lplane = src + d.sz * (int64_t)lk;
  double na[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) na[c] = row_ok ? (double)lplane[c * btx] - sub : 0.0;
  lplane += d.sz;
  if (++lk == nz) { lk = 0; lplane -= wrap; }
  T *dst = reinterpret_cast<T *>(d.dq[comp]) + d.sy * j + tx;
  double win[CPT][RS];
#pragma unroll
  for (int c = 0; c < CPT; ++c)
#pragma unroll
    for (int q = 0; q < RS; ++q) win[c][q] = 0.0;
  int buf = 0;
  for (int p0 = pbeg; p0 < pend; p0 += RS) {
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      const int p = p0 + u;
      if (p >= pend) break;  // uniform over the block
      // publish plane p with its periodic halo (every position of the row
      // is written for every plane), load plane p + 1.  One barrier per
      // plane: a buffer is rewritten two planes later.
      double *row = rows + (size_t)(buf * blockDim.y + ty) * RW;
      buf ^= 1;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int col = tx + c * btx;
        row[col + WX] = na[c];
        if (col < WX) row[col + nx + WX] = na[c];
        if (col >= nx - WX) row[col - nx + WX] = na[c];
      }
      if (row_ok && p + 1 < pend) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) na[c] = (double)lplane[c * btx] - sub;
      }
      lplane += d.sz;
      if (++lk == nz) { lk = 0; lplane -= wrap; }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const double *rr = row + tx + c * btx + WX;
        double xs = sp.bgx[0] * rr[0];
#pragma unroll
        for (int m = 1; m <= WX; ++m) xs += sp.bgx[m] * (rr[-m] + rr[m]);
        win[c][u] = xs;
      }
      if (p - WZ >= kb) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          // window planes p - 2 WZ .. p; plane p - t sits in slot (u - t) mod RS
          double acc = sp.bgz[0] * win[c][(u + WZ + 1) % RS];
#pragma unroll
          for (int m = 1; m <= WZ; ++m)
            acc += sp.bgz[m] * (win[c][(u + WZ + 1 - m) % RS] + win[c][(u + WZ + 1 + m) % RS]);
          if (row_ok) dst[c * btx + d.sz * (int64_t)(p - WZ)] = (T)acc;
        }
      }
    }
  }
}

template <typename T, int WX, int WZ>
static void launch_adixz_w(dim3 grid, cudaStream_t st, const TGDev &d, const SubParams &sp) {
  k_adixz_band<T, WX, WZ><<<grid, dim3(BM_TX, BM_TY), 0, st>>>(d, sp);
}
static int band_tw_index(int w) {
  for (int q = 0; q < 5; ++q)
    if (w <= BAND_TW[q]) return q;
  return -1;
}
#define CHAPSIM_ADIXZ_ROW(T, WX)                                                                          \
  { launch_adixz_w<T, WX, 2>, launch_adixz_w<T, WX, 4>, launch_adixz_w<T, WX, 6>, launch_adixz_w<T, WX, 8>, \
    launch_adixz_w<T, WX, 12> }
template <typename T>
static void launch_adixz(dim3 grid, cudaStream_t st, const TGDev &d, const SubParams &sp) {
  typedef void (*Fn)(dim3, cudaStream_t, const TGDev &, const SubParams &);
  static const Fn fns[5][5] = {CHAPSIM_ADIXZ_ROW(T, 2), CHAPSIM_ADIXZ_ROW(T, 4), CHAPSIM_ADIXZ_ROW(T, 6),
                               CHAPSIM_ADIXZ_ROW(T, 8), CHAPSIM_ADIXZ_ROW(T, 12)};
  // the band form is on only when 0 <= wx, wz <= BAND_WMAX
  fns[band_tw_index(sp.wx)][band_tw_index(sp.wz)](grid, st, d, sp);
}
#undef CHAPSIM_ADIXZ_ROW

constexpr int AR_SEG = 64;  // planes per block of the row form
// columns per thread of the row form for this nx (0: the tile form runs)
static int adixz_row_cpt(int nx) {
  if (nx <= 256) return 1;
  if (nx <= 512 && nx % 2 == 0) return 2;
  return 0;
}
template <typename T, int WX, int WZ, int CPT>
static void launch_adixz_row_w(dim3 grid, dim3 blk, size_t smem, cudaStream_t st, const TGDev &d,
                               const SubParams &sp) {
  k_adixz_row<T, WX, WZ, CPT><<<grid, blk, smem, st>>>(d, sp, AR_SEG);
}
#define CHAPSIM_ADIXZ_RROW(T, WX, CPT)                                                            \
  { launch_adixz_row_w<T, WX, 2, CPT>, launch_adixz_row_w<T, WX, 4, CPT>, launch_adixz_row_w<T, WX, 6, CPT>, \
    launch_adixz_row_w<T, WX, 8, CPT>, launch_adixz_row_w<T, WX, 12, CPT> }
// the row form of the x / z factors; false when this nx needs the tile form
template <typename T>
static bool launch_adixz_rows(cudaStream_t st, const TGDev &d, const SubParams &sp) {
  const int cpt = adixz_row_cpt(d.nx);
  if (!cpt) return false;
  typedef void (*Fn)(dim3, dim3, size_t, cudaStream_t, const TGDev &, const SubParams &);
  static const Fn f1[5][5] = {CHAPSIM_ADIXZ_RROW(T, 2, 1), CHAPSIM_ADIXZ_RROW(T, 4, 1), CHAPSIM_ADIXZ_RROW(T, 6, 1),
                              CHAPSIM_ADIXZ_RROW(T, 8, 1), CHAPSIM_ADIXZ_RROW(T, 12, 1)};
  static const Fn f2[5][5] = {CHAPSIM_ADIXZ_RROW(T, 2, 2), CHAPSIM_ADIXZ_RROW(T, 4, 2), CHAPSIM_ADIXZ_RROW(T, 6, 2),
                              CHAPSIM_ADIXZ_RROW(T, 8, 2), CHAPSIM_ADIXZ_RROW(T, 12, 2)};
  const int iw = band_tw_index(sp.wx), iz = band_tw_index(sp.wz);
  const int btx = d.nx / cpt, bty = btx >= 256 ? 1 : 256 / btx;
  dim3 blk(btx, bty), grid((d.ny + bty - 1) / bty, 3 * ((d.nz + AR_SEG - 1) / AR_SEG));
  const size_t smem = (size_t)2 * bty * (d.nx + 2 * BAND_TW[iw]) * sizeof(double);
  (cpt == 1 ? f1 : f2)[iw][iz](grid, blk, smem, st, d, sp);
  return true;
}
#undef CHAPSIM_ADIXZ_RROW

// MOMFA3_Y_tg (src/MOMFA_tg.f90:173-240) applied as the banded part of the
// exact inverse of each component's y tridiagonal matrix (rows j = 1..ny),
// G[j][m] = (A^{-1})_{j, j+m} for |m| <= WY, precomputed on the host from
// the Thomas sweeps and truncated where the dropped entries of every row sum
// to < 2^-60 of its largest entry.  Then q += dq and BC_WALL_Q_tg.  A block
// owns 32 x-columns, AY_JT rows and one z plane; rows outside [1, ny] carry
// zero weight.  Per component the block stages its tile of dq (with the y
// halo) and its AY_JT band rows of G (zero past WY, one zero pad) in shared
// memory; each thread then computes AY_R consecutive rows of its column,
// reading each tile value once and the band coefficients as 16-byte
// broadcast pairs.  W is a compile-time width at least WY.  The v line's
// row-1 right-hand side is the final u increment at j = 1 (the reference
// quirk described at k_adiy_smem), computed here from the u data.
constexpr int AY_JT = 32, AY_TX = 32, AY_TY = 8, AYB_WMAX = 16, AY_R = AY_JT / AY_TY;
constexpr int AY_TW[6] = {2, 4, 6, 8, 12, 16};  // compiled widths
static_assert(AY_TW[5] == AYB_WMAX, "the widest compiled band is the host's limit");
template <typename T, int W>
__global__ void __launch_bounds__(AY_TX *AY_TY) k_adiy_band(TGDev d, SubParams sp) {
  constexpr int NT = AY_R + 2 * W + 1;  // tile values per thread; the last one meets a zero weight
  constexpr int GS = 2 * W + 2;         // band row stride in shared memory (even: pairs stay 16-byte aligned)
  __shared__ double tile[(AY_JT + 2 * W + 1) * AY_TX];
  __shared__ __align__(16) double gsh[AY_JT * GS];
  __shared__ double du1[AY_TX];
  const int nx = d.nx, ny = d.ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + AY_TX * ty;
  const int x0 = blockIdx.x * AY_TX, j0 = 1 + blockIdx.y * AY_JT, k = blockIdx.z;
  const int i = x0 + tx;
  const bool col_ok = i < nx;
  const int64_t base = (int64_t)i + d.sz * k;
  const int nrow = AY_JT + 2 * W;  // tile rows j0-W .. j0+AY_JT-1+W, then one zero row
  const int jr0 = ty * AY_R;
  for (int comp = 0; comp < 3; ++comp) {
    const T *src = reinterpret_cast<const T *>(d.dq[comp]);
    for (int r = ty; r <= nrow; r += AY_TY) {
      const int j = j0 - W + r;
      double v = 0.0;
      if (col_ok && r < nrow && j >= 1 && j <= ny) v = (double)src[base + d.sy * j];
      tile[r * AY_TX + tx] = v;
    }
    // the block's band rows G[j][m], m = -W .. W + 1 (the last zero); rows
    // past ny repeat row ny and are discarded
    const double *G = sp.yg[comp];
    for (int t = tid; t < AY_JT * GS; t += AY_TX * AY_TY) {
      const int r = t / GS, m = t - r * GS - W, j = min(j0 + r, ny);
      gsh[t] = m <= W ? G[(size_t)j * (2 * AYB_WMAX + 1) + AYB_WMAX + m] : 0.0;
    }
    if (comp == 1 && j0 == 1) {
      __syncthreads();
      if (ty == 0) tile[(1 - j0 + W) * AY_TX + tx] = du1[tx];  // row j = 1 of v <- u increment
    }
    __syncthreads();
    double *q = comp == 0 ? d.u : (comp == 1 ? d.v : d.w);
    const int jlo = comp == 1 ? 2 : 1;
    double acc[AY_R];
    double2 cp[AY_R];
#pragma unroll
    for (int r = 0; r < AY_R; ++r) {
      acc[r] = 0.0;
      cp[r] = make_double2(0.0, 0.0);
    }
    // tile row jr0 + qq feeds row r with the weight G[j0 + jr0 + r][qq - r - W]
#pragma unroll
    for (int qq = 0; qq < NT; ++qq) {
      const double v = tile[(jr0 + qq) * AY_TX + tx];
#pragma unroll
      for (int r = 0; r < AY_R; ++r) {
        const int m2 = qq - r;  // m + W
        if (m2 < 0 || m2 > 2 * W + 1) continue;
        if ((m2 & 1) == 0) cp[r] = *reinterpret_cast<const double2 *>(gsh + (jr0 + r) * GS + m2);
        acc[r] += ((m2 & 1) ? cp[r].y : cp[r].x) * v;
      }
    }
#pragma unroll
    for (int r = 0; r < AY_R; ++r) {
      const int j = j0 + jr0 + r;
      if (j > ny) break;  // uniform over the warp (one warp per ty)
      if (comp == 0 && j == 1) du1[tx] = acc[r];
      if (col_ok && j >= jlo) q[base + d.sy * j] += acc[r];
    }
    if (col_ok && ty == 0) {
      if (j0 == 1) {
        q[base] = 0.0;
        if (comp == 1) q[base + d.sy] = 0.0;
      }
      if (j0 + AY_JT > ny) q[base + d.sy * (ny + 1)] = 0.0;
    }
    __syncthreads();
  }
}
template <typename T, int W>
static void launch_adiy_w(dim3 grid, cudaStream_t st, const TGDev &d, const SubParams &sp) {
  k_adiy_band<T, W><<<grid, dim3(AY_TX, AY_TY), 0, st>>>(d, sp);
}
// the band form of the y factors (the host keeps 0 <= wy <= AYB_WMAX when it is on)
template <typename T>
static void launch_adiy(dim3 grid, cudaStream_t st, const TGDev &d, const SubParams &sp) {
  typedef void (*Fn)(dim3, cudaStream_t, const TGDev &, const SubParams &);
  static const Fn fns[6] = {launch_adiy_w<T, 2>, launch_adiy_w<T, 4>, launch_adiy_w<T, 6>,
                            launch_adiy_w<T, 8>, launch_adiy_w<T, 12>, launch_adiy_w<T, 16>};
  int q = 0;
  while (q < 5 && sp.wy > AY_TW[q]) ++q;
  fns[q](grid, st, d, sp);
}

// ============================================================ y lines
// MOMFA3_Y_tg with the lines staged in shared memory: a block owns 32
// consecutive i at one k; all 128 threads load the [ny][32] tile (coalesced,
// many loads in flight), warp 0 runs the Thomas sweeps from shared memory with
// the precomputed pivots, all threads add the increment to q.  The v line's
// row 1 takes the u increment at j = 1, as in the reference (RHS_tg row 1 is
// not rebuilt for IDR = 2, src/RHS_CvLpGpS_tg.f90:61-62, while MOMFA3_Y_tg
// solves rows 1..ny, src/MOMFA_tg.f90:209-234).
constexpr int AY_TL = 32;
template <typename T>
__global__ void __launch_bounds__(128) k_adiy_smem(TGDev d, SubParams sp, int from_dq) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *tile = reinterpret_cast<T *>(smem_raw);
  const int nx = d.nx, ny = d.ny;
  const int i0 = blockIdx.x * AY_TL, k = blockIdx.y;
  const int tid = threadIdx.x;
  const int nl = min(AY_TL, nx - i0);
  const int64_t sy = d.sy;
  const int64_t base = i0 + d.sz * k;
  double du1 = 0.0;
  for (int comp = 0; comp < 3; ++comp) {
    const T *src = reinterpret_cast<const T *>(from_dq ? d.dq[comp] : d.rhs[comp]) + base;
    for (int t = tid; t < ny * AY_TL; t += blockDim.x) {
      const int r = t / AY_TL, l = t - r * AY_TL;
      if (l < nl) tile[t] = src[l + sy * (r + 1)];
    }
    __syncthreads();
    if (tid < nl) {
      const double *__restrict__ a = sp.ya[comp];
      const double *__restrict__ pp = sp.ypp[comp];
      const double *__restrict__ h = sp.yh[comp];
      T *col = tile + tid;
      double g = (comp == 1 ? du1 : (double)col[0]) * pp[1];
      col[0] = (T)g;
      for (int jj = 2; jj <= ny; ++jj) {
        g = ((double)col[(jj - 1) * AY_TL] - a[jj] * g) * pp[jj];
        col[(jj - 1) * AY_TL] = (T)g;
      }
      double x = g;
      for (int jj = ny - 1; jj >= 1; --jj) {
        x = (double)col[(jj - 1) * AY_TL] - h[jj] * x;
        col[(jj - 1) * AY_TL] = (T)x;
      }
      if (comp == 0) du1 = x;
    }
    __syncthreads();
    double *q = (comp == 0 ? d.u : (comp == 1 ? d.v : d.w)) + base;
    const int jlo = comp == 1 ? 2 : 1;
    for (int t = tid; t < ny * AY_TL; t += blockDim.x) {
      const int r = t / AY_TL, l = t - r * AY_TL;
      if (l < nl && r + 1 >= jlo) q[l + sy * (r + 1)] += (double)tile[t];
    }
    if (tid < nl) {
      q[tid] = 0.0;
      q[tid + sy * (ny + 1)] = 0.0;
      if (comp == 1) q[tid + sy] = 0.0;
    }
    __syncthreads();
  }
}

// ============================================================ Poisson
// DIVG_tg (src/DIVG.f90:21-57) fused with the forward real transform along x
// of FFT99_POIS3D_periodicxz (src/possion3d_FFT99.f90:265-318).  A block owns
// lb consecutive rows j of plane k.  Its inputs arrive by bulk copies
// (cp.async.bulk, one per array: u rows, v rows plus one, w rows of planes k
// and k+1, all contiguous in memory) completed on one mbarrier; the
// divergence is formed in shared memory, rows are packed in pairs as complex
// lines, transformed, separated and scaled by 1/nx.  mode 0 computes the
// divergence (and stores RHSLLPHI); mode 1 transforms the stored RHSLLPHI;
// mode 2 the Poisson residual.
__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) & ~(size_t)127; }
// dr != 0 reserves lb rows for DrhoDtP (IO contexts)
template <typename C> __host__ __device__ constexpr size_t fftx_smem_bytes(int nx, int lb, int dr = 0) {
  return align128((size_t)(lb / 2) * nx * sizeof(C)) + (size_t)((4 + dr) * lb + 1) * nx * sizeof(double);
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <typename T, bool BIG>
__global__ void __launch_bounds__(256, BIG ? 2 : 3) k_fftx(TGDev d, SubParams sp, FFTPlan pl, int lb, int mode) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  __shared__ int rad[16];
  const int nx = d.nx, ny = d.ny, lh = d.lh;
  const int k = blockIdx.y;
  const int jbeg = 1 + blockIdx.x * lb;
  const int nrow = min(lb, ny - jbeg + 1);
  const int nl = lb / 2;
  const int tid = threadIdx.x;
  C *A = reinterpret_cast<C *>(smem_raw);
  double *in = reinterpret_cast<double *>(smem_raw + align128((size_t)nl * nx * sizeof(C)));
  C *B = reinterpret_cast<C *>(in);  // FFT scratch, reuses the input area once A is filled
  double *U = in, *V = in + (size_t)lb * nx, *W0 = V + (size_t)(lb + 1) * nx, *W1 = W0 + (size_t)lb * nx;
  double *DR = W1 + (size_t)lb * nx;  // DrhoDtP rows (IO, mode 0)
  const bool dr = mode == 0 && d.drho != nullptr;
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (tid < 16) rad[tid] = pl.rad[tid];
  __syncthreads();
  const int kp = wrapp(k, d.nz);
  const uint32_t rowb = (uint32_t)nx * sizeof(double);
  const int64_t row0 = d.sy * jbeg;
  if (tid == 0) {
    if (mode == 0) {
      mbar_expect_tx(&bar, ((dr ? 5 : 4) * nrow + 1) * rowb);
      bulk_g2s(U, d.u + row0 + d.sz * k, nrow * rowb, &bar);
      bulk_g2s(V, d.v + row0 + d.sz * k, (nrow + 1) * rowb, &bar);
      bulk_g2s(W0, d.w + row0 + d.sz * k, nrow * rowb, &bar);
      bulk_g2s(W1, d.w + row0 + d.sz * kp, nrow * rowb, &bar);
      if (dr) bulk_g2s(DR, d.drho + row0 + d.sz * k, nrow * rowb, &bar);
    } else {
      mbar_expect_tx(&bar, nrow * rowb);
      bulk_g2s(U, (mode == 1 ? d.rhsphi : d.res) + row0 + d.sz * k, nrow * rowb, &bar);
    }
  }
  if (!mbar_wait(&bar, 0, d.err)) {
    mbar_wait(&bar, 0, d.err);  // let copies in flight land before the block exits
    return;
  }
  const double coe0 = 1.0 / (d.dt * sp.alp);
  for (int t = tid; t < lb * nx; t += blockDim.x) {
    const int r = t / nx, i = t - r * nx;
    double val = 0.0;
    if (r < nrow) {
      if (mode == 0) {
        const int ip = wrapp(i, nx);
        const int j = jbeg + r;
        double dv = (U[r * nx + ip] - U[r * nx + i]) * d.dxi + (V[(r + 1) * nx + i] - V[r * nx + i]) * d.dyfi[j] +
                    (W1[r * nx + i] - W0[r * nx + i]) * d.dzi;
        if (dr) dv += DR[r * nx + i];  // DIVG_io: + DrhoDtP
        val = dv * coe0;
        if (!d.skip_rhs) d.rhsphi[row0 + d.sz * k + (int64_t)r * nx + i] = val;
      } else {
        val = U[r * nx + i];
      }
    }
    C *z = A + swz((r >> 1) * nx + i);
    if (r & 1) z->y = (T)val; else z->x = (T)val;
  }
  __syncthreads();
  C *res = fft_lines<C, BIG>(A, B, nl, nx, nx, rad, pl.nrad, (const C *)(sizeof(T) == 8 ? (const void *)pl.tw64 : (const void *)pl.tw32), -1);
  const T scale = (T)(1.0 / nx);
  C *S = reinterpret_cast<C *>(d.spec);
  for (int t = tid; t < nl * lh; t += blockDim.x) {
    const int p = t / lh, kx = t - p * lh;
    const C z = res[swz(p * nx + kx)];
    const C zc = cconj(res[swz(p * nx + (kx == 0 ? 0 : nx - kx))]);
    C x0, x1;
    x0.x = (T)0.5 * (z.x + zc.x) * scale;
    x0.y = (T)0.5 * (z.y + zc.y) * scale;
    // x1 = -i (z - zc) / 2
    x1.x = (T)0.5 * (z.y - zc.y) * scale;
    x1.y = (T)-0.5 * (z.x - zc.x) * scale;
    const int r0 = 2 * p;
    if (r0 < nrow) S[kx + (int64_t)d.lp * ((jbeg + r0 - 1) + (int64_t)ny * k)] = x0;
    if (r0 + 1 < nrow) S[kx + (int64_t)d.lp * ((jbeg + r0) + (int64_t)ny * k)] = x1;
  }
}

// Complex transform along z for lz consecutive kx at row j
// (src/possion3d_FFT99.f90:301-317 forward with 1/nz and the (1,1,1) mode
// zeroed (:324-327); :448-458 inverse).  The block's nz rows of lz spectral
// values (contiguous in memory) arrive by one bulk copy each, all completing
// on one mbarrier, into a line-interleaved buffer A[kz * lz + l]; the
// Stockham stages then run on the interleaved layout.
template <typename T, bool BIG>
__global__ void __launch_bounds__(256, BIG ? 2 : 3) k_fftz(TGDev d, FFTPlan pl, int lz, int sign) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  __shared__ int rad[16];
  const int nz = d.nz, ny = d.ny, lh = d.lh;
  const int j = blockIdx.y + 1;
  const int kx0 = blockIdx.x * lz;
  const int nl = min(lz, lh - kx0);
  // copies move whole 16-byte units: a float2 row is rounded up to an even
  // count (the pitch lp is even, so the extra value is the row's padding)
  const int nc = sizeof(C) == 8 ? ((nl + 1) & ~1) : nl;
  const int tid = threadIdx.x;
  C *A = reinterpret_cast<C *>(smem_raw);
  C *B = A + (size_t)lz * nz;
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (tid < 16) rad[tid] = pl.rad[tid];
  __syncthreads();
  C *S = reinterpret_cast<C *>(d.spec) + kx0 + (int64_t)d.lp * (j - 1);
  const int64_t skz = (int64_t)d.lp * ny;
  const uint32_t rowb = (uint32_t)(nc * sizeof(C));
  if (tid == 0) mbar_expect_tx(&bar, rowb * (uint32_t)nz);
  __syncthreads();
  for (int kz = tid; kz < nz; kz += blockDim.x) bulk_g2s(A + (size_t)kz * lz, S + skz * kz, rowb, &bar);
  if (nc < lz) {  // columns past the end of the spectrum: zeros
    const int w = lz - nc;
    for (int t = tid; t < nz * w; t += blockDim.x) {
      const int kz = t / w;
      C z; z.x = 0; z.y = 0;
      A[(size_t)kz * lz + nc + (t - kz * w)] = z;
    }
  }
  if (!mbar_wait(&bar, 0, d.err)) {
    mbar_wait(&bar, 0, d.err);  // let copies in flight land before the block exits
    return;
  }
  __syncthreads();
  C *res = fft_lines_il<C, BIG>(A, B, lz, nz, rad, pl.nrad,
                                (const C *)(sizeof(T) == 8 ? (const void *)pl.tw64 : (const void *)pl.tw32), sign);
  const T scale = sign < 0 ? (T)(1.0 / nz) : (T)1;
  const int llz = __ffs(lz) - 1;  // lz is a power of two
  for (int t = tid; t < nz * lz; t += blockDim.x) {
    const int kz = t >> llz, l = t & (lz - 1);
    if (l < nl) {
      C v = res[t];
      v.x *= scale;
      v.y *= scale;
      if (sign < 0 && j == 1 && kz == 0 && kx0 + l == 0 && !d.pin_last) { v.x = 0; v.y = 0; }
      S[skz * kz + l] = v;
    }
  }
}

// Pivots of the Poisson y-tridiagonals, computed once per context: for every
// (kx, kz) the forward-elimination factors pp_j = 1/(B_j - h_{j-1} A_j) and
// h_j = C_j pp_j of the matrix of src/possion3d_FFT99.f90:334-443 with the
// coefficients of TDMA_PHI_COEF (:185-220): A = AMPH, B = ACPH - AK1 - AK3,
// C = APPH, and for the mean mode (kx = kz = 0) row 1 decoupled.  Stored in
// the spectral layout as two arrays, pp then h (each lp * ny * nz values):
// the forward sweep reads only pp, the back substitution only h.
__global__ void k_ypivots(TGDev d) {
  const int lh = d.lh, ny = d.ny;
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int kz = blockIdx.y;
  if (kx >= lh) return;
  const int64_t base = kx + (int64_t)d.lp * ny * kz;
  double *PP = reinterpret_cast<double *>(d.ypiv) + base;
  double *HH = reinterpret_cast<double *>(d.ypiv) + (int64_t)d.lp * ny * d.nz + base;
  const double shift = d.ak1[kx] + d.ak3[kz];
  // the zero-shift line: the mean mode (kx = kz = 0) of periodic x, the first
  // COST mode of Neumann x ends
  const bool mean = (d.ak1[kx] == 0.0 && d.ak3[kz] == 0.0);
  const bool pin1 = mean && !d.pin_last, pinn = mean && d.pin_last;
  double b = d.acph[1] - shift;
  double pp = 1.0 / b;
  double h = (pin1 ? 0.0 : d.apph[1]) * pp;
  PP[0] = pin1 ? 0.0 : pp;  // pp = 0 zeroes the pinned row
  HH[0] = h;
  for (int j = 2; j <= ny; ++j) {
    b = d.acph[j] - shift;
    // TRID0's zero branch for the singular last pivot of the mean mode
    // (src/possion3d_fishpack_reform.f90:53-58): phi(ny) = 0
    pp = (pinn && j == ny) ? 0.0 : 1.0 / (b - h * d.amph[j]);
    h = j < ny ? d.apph[j] * pp : 0.0;
    PP[(int64_t)d.lp * (j - 1)] = pp;
    HH[(int64_t)d.lp * (j - 1)] = h;
  }
}

// Poisson y-tridiagonal solves, one thread per (kx, kz) line straight from
// global memory: consecutive threads own consecutive kx, so every row access
// is coalesced.  The forward-swept g is written over the spectral data in
// place and read back by the back substitution.  Each sweep loads the next
// YB rows (values and pivots) into registers before it computes and stores
// them, so YB loads per thread are in flight instead of one.
constexpr int YB = 8;
template <typename T>
__global__ void __launch_bounds__(256) k_ysolve_line(TGDev d) {
  typedef typename Cplx<T>::type C;
  const int lh = d.lh, ny = d.ny;
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kz = blockIdx.y;
  if (kx >= lh) return;
  const int64_t base = kx + (int64_t)d.lp * ny * kz, st = d.lp;
  C *__restrict__ S = reinterpret_cast<C *>(d.spec) + base;
  const double *__restrict__ PP = reinterpret_cast<const double *>(d.ypiv) + base;
  const double *__restrict__ HH = reinterpret_cast<const double *>(d.ypiv) + (int64_t)d.lp * ny * d.nz + base;
  double gr = 0.0, gi = 0.0;
  for (int j0 = 1; j0 <= ny; j0 += YB) {
    C r[YB];
    double p[YB], a[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j <= ny) {
        r[u] = S[st * (j - 1)];
        p[u] = __ldg(PP + st * (j - 1));
        a[u] = d.amph[j];
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j <= ny) {
        if (j == 1) {
          gr = (double)r[u].x * p[u];
          gi = (double)r[u].y * p[u];
        } else {
          gr = ((double)r[u].x - a[u] * gr) * p[u];
          gi = ((double)r[u].y - a[u] * gi) * p[u];
        }
        C o; o.x = (T)gr; o.y = (T)gi;
        S[st * (j - 1)] = o;
      }
    }
  }
  double xr = gr, xi = gi;  // x_ny = g_ny
  for (int j0 = ny - 1; j0 >= 1; j0 -= YB) {
    C r[YB];
    double h[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 - u;
      if (j >= 1) {
        r[u] = S[st * (j - 1)];
        h[u] = __ldg(HH + st * (j - 1));
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 - u;
      if (j >= 1) {
        xr = (double)r[u].x - h[u] * xr;
        xi = (double)r[u].y - h[u] * xi;
        C o; o.x = (T)xr; o.y = (T)xi;
        S[st * (j - 1)] = o;
      }
    }
  }
}

// Poisson y-lines of the quarter-wave x transforms (LP 3 and 5), whose nx
// real x modes sit two to a complex line: line p holds mode 2p in its real
// and mode 2p + 1 in its imaginary part, so after the complex z transform
// Z(kz) = A(kz) + i B(kz), with A and B the z transforms of the two real mode
// planes (A(nz - kz) = conj A(kz), B likewise).  One thread takes rows kz and
// nz - kz of line p: A = (Z(kz) + conj Z(nz - kz)) / 2 and B = (Z(kz) -
// conj Z(nz - kz)) / 2i are solved with the pivots of modes 2p and 2p + 1
// (q: the packed descriptor; s: the descriptor of nx single lines that holds
// the pivots, whose shifts at kz and nz - kz are equal) and packed back into
// both rows.  The forward sweep keeps g_A in row kz and g_B in row nz - kz;
// rows 0 and nz / 2 are their own partners, where A and B are real and share
// the row's one complex value.  These transforms have no zero shift, so no
// mode is pinned.  Half the lines of the unpacked form go through the z
// transforms and the y-lines.
constexpr int YP = 8;
__global__ void __launch_bounds__(128) k_ysolve_pair(TGDev q, TGDev s) {
  const int ny = q.ny, nz = q.nz;
  const int p = blockIdx.x * blockDim.x + threadIdx.x, kz = blockIdx.y;
  if (p >= q.lh) return;
  const int kc = kz ? nz - kz : 0;
  const bool self = kc == kz;
  const int64_t st = q.lp, sp = s.lp;
  double2 *__restrict__ Z1 = reinterpret_cast<double2 *>(q.spec) + p + st * ny * kz;
  double2 *__restrict__ Z2 = reinterpret_cast<double2 *>(q.spec) + p + st * ny * kc;
  // pivots of modes 2p and 2p + 1 side by side (16-byte aligned: sp even)
  const double *__restrict__ PP = reinterpret_cast<const double *>(s.ypiv) + 2 * p + sp * ny * kz;
  const double *__restrict__ HH = PP + sp * ny * s.nz;
  double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
  for (int j0 = 1; j0 <= ny; j0 += YP) {
    double2 z1[YP], z2[YP], pv[YP];
    double a[YP];
#pragma unroll
    for (int u = 0; u < YP; ++u) {
      const int j = j0 + u;
      if (j <= ny) {
        z1[u] = Z1[st * (j - 1)];
        z2[u] = Z2[st * (j - 1)];
        pv[u] = __ldg(reinterpret_cast<const double2 *>(PP + sp * (j - 1)));
        a[u] = q.amph[j];
      }
    }
#pragma unroll
    for (int u = 0; u < YP; ++u) {
      const int j = j0 + u;
      if (j <= ny) {
        const double Ar = 0.5 * (z1[u].x + z2[u].x), Ai = 0.5 * (z1[u].y - z2[u].y);
        const double Br = 0.5 * (z1[u].y + z2[u].y), Bi = -0.5 * (z1[u].x - z2[u].x);
        if (j == 1) {
          ar = Ar * pv[u].x; ai = Ai * pv[u].x;
          br = Br * pv[u].y; bi = Bi * pv[u].y;
        } else {
          ar = (Ar - a[u] * ar) * pv[u].x; ai = (Ai - a[u] * ai) * pv[u].x;
          br = (Br - a[u] * br) * pv[u].y; bi = (Bi - a[u] * bi) * pv[u].y;
        }
        if (self) {
          Z1[st * (j - 1)] = make_double2(ar, br);  // ai = bi = 0 here
        } else {
          Z1[st * (j - 1)] = make_double2(ar, ai);
          Z2[st * (j - 1)] = make_double2(br, bi);
        }
      }
    }
  }
  // x_ny = g_ny; each row packed back: Z(kz) = A + i B, Z(nz - kz) = conj A + i conj B
  Z1[st * (ny - 1)] = make_double2(ar - bi, ai + br);
  if (!self) Z2[st * (ny - 1)] = make_double2(ar + bi, br - ai);
  for (int j0 = ny - 1; j0 >= 1; j0 -= YP) {
    double2 g1[YP], g2[YP], hv[YP];
#pragma unroll
    for (int u = 0; u < YP; ++u) {
      const int j = j0 - u;
      if (j >= 1) {
        g1[u] = Z1[st * (j - 1)];
        g2[u] = Z2[st * (j - 1)];
        hv[u] = __ldg(reinterpret_cast<const double2 *>(HH + sp * (j - 1)));
      }
    }
#pragma unroll
    for (int u = 0; u < YP; ++u) {
      const int j = j0 - u;
      if (j >= 1) {
        const double gar = g1[u].x, gai = self ? 0.0 : g1[u].y;
        const double gbr = self ? g1[u].y : g2[u].x, gbi = self ? 0.0 : g2[u].y;
        ar = gar - hv[u].x * ar; ai = gai - hv[u].x * ai;
        br = gbr - hv[u].y * br; bi = gbi - hv[u].y * bi;
        Z1[st * (j - 1)] = make_double2(ar - bi, ai + br);
        if (!self) Z2[st * (j - 1)] = make_double2(ar + bi, br - ai);
      }
    }
  }
}

// Inverse real transform along x (src/possion3d_FFT99.f90:461-485): the
// block's lb spectral rows (contiguous, pitch lp) arrive by one bulk copy;
// pairs of rows are rebuilt as one complex Hermitian-extended line and
// transformed; phi ghosts copied (BC_WALL_DPH, src/BC_WALL.f90:342-364).
// accumulate != 0 adds the result to phi (refinement sweep).  The FFT
// scratch reuses the staging area of the spectral rows once the lines are
// packed (lb * lp >= lb / 2 * nx, since lp > nx / 2).
template <typename C> __host__ __device__ constexpr size_t ifftx_smem_bytes(int nx, int lp, int lb) {
  return align128((size_t)lb * lp * sizeof(C)) + align128((size_t)(lb / 2) * nx * sizeof(C));
}

template <typename T, bool BIG>
__global__ void __launch_bounds__(256, BIG ? 2 : 3) k_ifftx(TGDev d, FFTPlan pl, int lb, int accumulate) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  __shared__ int rad[16];
  const int nx = d.nx, ny = d.ny, lh = d.lh, lp = d.lp;
  const int k = blockIdx.y;
  const int jbeg = 1 + blockIdx.x * lb;
  const int nrow = min(lb, ny - jbeg + 1);
  const int nl = lb / 2;
  const int tid = threadIdx.x;
  C *SP = reinterpret_cast<C *>(smem_raw);
  C *A = reinterpret_cast<C *>(smem_raw + align128((size_t)lb * lp * sizeof(C)));
  C *B = SP;  // FFT scratch: the spectral rows are dead once packed into A
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (tid < 16) rad[tid] = pl.rad[tid];
  __syncthreads();
  if (tid == 0) {
    const uint32_t bytes = (uint32_t)(nrow * lp * sizeof(C));
    mbar_expect_tx(&bar, bytes);
    bulk_g2s(SP, reinterpret_cast<const C *>(d.spec) + (int64_t)lp * ((jbeg - 1) + (int64_t)ny * k), bytes, &bar);
  }
  if (!mbar_wait(&bar, 0, d.err)) {
    mbar_wait(&bar, 0, d.err);
    return;
  }
  for (int t = tid; t < nl * lh; t += blockDim.x) {
    const int p = t / lh, kx = t - p * lh;
    const int r0 = 2 * p;
    C x0, x1;
    x0.x = 0; x0.y = 0; x1.x = 0; x1.y = 0;
    if (r0 < nrow) x0 = SP[r0 * lp + kx];
    if (r0 + 1 < nrow) x1 = SP[(r0 + 1) * lp + kx];
    if (kx == 0 || 2 * kx == nx) { x0.y = 0; x1.y = 0; }
    // Z(k) = X0 + i X1 ; Z(n-k) = conj(X0) + i conj(X1)
    C z; z.x = x0.x - x1.y; z.y = x0.y + x1.x;
    A[swz(p * nx + kx)] = z;
    if (kx != 0 && 2 * kx != nx) {
      C zc; zc.x = x0.x + x1.y; zc.y = -x0.y + x1.x;
      A[swz(p * nx + (nx - kx))] = zc;
    }
  }
  __syncthreads();
  C *res = fft_lines<C, BIG>(A, B, nl, nx, nx, rad, pl.nrad, (const C *)(sizeof(T) == 8 ? (const void *)pl.tw64 : (const void *)pl.tw32), +1);
  for (int t = tid; t < nrow * nx; t += blockDim.x) {
    const int r = t / nx, i = t - r * nx;
    const int j = jbeg + r;
    const C z = res[swz((r >> 1) * nx + i)];
    const double val = (r & 1) ? (double)z.y : (double)z.x;
    const int64_t c0 = i + d.sy * j + d.sz * k;
    const double out = accumulate ? d.phi[c0] + val : val;
    d.phi[c0] = out;
    if (j == 1) d.phi[c0 - d.sy] = out;
    if (j == ny) d.phi[c0 + d.sy] = out;
  }
}

// FP64 residual of the discrete Poisson operator the spectral solver inverts
// (the operator of CHECK_FFT_SOLVER, src/PRESSURE_CORRECTION.f90:159-202):
// res = RHSLLPHI - [d_xx + d_zz + L_y] phi, with L_y the folded Neumann
// y-operator AMPH/ACPH/APPH.  Feeds the refinement sweep of the mixed form.
__global__ void __launch_bounds__(RHS_BX *RHS_BY) k_pois_residual(TGDev d) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * RHS_BX + threadIdx.x;
  const int j = blockIdx.y * RHS_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy;
  const int64_t c0 = i + sy * j + d.sz * k;
  const int ip = wrapp(i, nx), im = wrapm(i, nx), kp = wrapp(k, d.nz), km = wrapm(k, d.nz);
  const double f = d.phi[c0];
  double l = (d.phi[c0 + (ip - i)] - 2.0 * f + d.phi[c0 + (im - i)]) * d.dxqi +
             (d.phi[c0 + d.sz * (kp - k)] - 2.0 * f + d.phi[c0 + d.sz * (km - k)]) * d.dzqi + d.acph[j] * f;
  if (j > 1) l += d.amph[j] * d.phi[c0 - sy];
  if (j < ny) l += d.apph[j] * d.phi[c0 + sy];
  d.res[c0] = d.rhsphi[c0] - l;
}

// VELOUPDT_tg (src/VELO_CORRECTION.f90:19-105), PRCALC_tg
// (src/PRESSURE_CORRECTION.f90:1-24) and the wall BCs of u, v, w, p.
__global__ void __launch_bounds__(RHS_BX *RHS_BY) k_corr(TGDev d, SubParams sp) {
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * RHS_BX + threadIdx.x;
  const int j = blockIdx.y * RHS_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  if (i >= nx || j > ny) return;
  const int64_t sy = d.sy;
  const int64_t c0 = i + sy * j + d.sz * k;
  const int im = wrapm(i, nx), km = wrapm(k, d.nz);
  const double phi = d.phi[c0];
  const double cx = d.dt * sp.alp * d.dxi, cz = d.dt * sp.alp * d.dzi;
  d.u[c0] -= (phi - d.phi[c0 + (im - i)]) * cx;
  d.w[c0] -= (phi - d.phi[c0 + d.sz * (km - k)]) * cz;
  if (j >= 2) d.v[c0] -= (phi - d.phi[c0 - sy]) * (d.dt * sp.alp * d.dyci[j]);
  const double be = 0.5 * sp.alp * d.dt * d.cvisc;
  const double pn = d.p[c0] + phi - be * d.rhsphi[c0];
  d.p[c0] = pn;
  if (j == 1) {
    d.u[c0 - sy] = 0.0; d.w[c0 - sy] = 0.0; d.v[c0 - sy] = 0.0; d.v[c0] = 0.0;
    d.p[c0 - sy] = pn;
  }
  if (j == ny) {
    d.u[c0 + sy] = 0.0; d.w[c0 + sy] = 0.0; d.v[c0 + sy] = 0.0;
    d.p[c0 + sy] = pn;
  }
}

// Stand-alone BC_WALL_Q_tg on all ghost cells.
__global__ void k_bc_q(TGDev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (i >= d.nx) return;
  const int64_t c1 = i + d.sy + d.sz * k;
  d.u[c1 - d.sy] = 0.0; d.w[c1 - d.sy] = 0.0; d.v[c1 - d.sy] = 0.0; d.v[c1] = 0.0;
  const int64_t cn = i + d.sy * (d.ny + 1) + d.sz * k;
  d.u[cn] = 0.0; d.w[cn] = 0.0; d.v[cn] = 0.0;
}

// ============================================================ reductions
// what 0: max |div u| (DIVGCK_tg, src/DIVGCK.f90:16-58) -> block maxima
// what 1: sum u/DYFI (BULK_VELOCITY_TG) -> block sums
// what 2: count of non-finite u, v, w, p -> block sums
__global__ void __launch_bounds__(RHS_BX *RHS_BY) k_reduce_part(TGDev d, int what) {
  __shared__ double sh[32];
  const int nx = d.nx, ny = d.ny;
  const int i = blockIdx.x * RHS_BX + threadIdx.x;
  const int j = blockIdx.y * RHS_BY + threadIdx.y + 1;
  const int k = blockIdx.z;
  double v = 0.0;
  if (i < nx && j <= ny) {
    const int64_t c0 = i + d.sy * j + d.sz * k;
    if (what == 0) {
      const int ip = wrapp(i, nx), kp = wrapp(k, d.nz);
      const double dv = (d.u[c0 + (ip - i)] - d.u[c0]) * d.dxi + (d.v[c0 + d.sy] - d.v[c0]) * d.dyfi[j] +
                        (d.w[c0 + d.sz * (kp - k)] - d.w[c0]) * d.dzi;
      v = fabs(dv);
      if (dv != dv) v = __longlong_as_double(0x7ff0000000000000ll);  // NaN -> +inf
    } else if (what == 1) {
      v = d.u[c0] / d.dyfi[j];
    } else if (what == 3) {
      // CFL_tg (src/CFL.f90:1-40): 0.5 (|u+u_ip| dxi + |v+v_jp| dyfi + |w+w_kp| dzi)
      const int ip = wrapp(i, nx), kp = wrapp(k, d.nz);
      v = (fabs((d.u[c0] + d.u[c0 + (ip - i)]) * d.dxi) + fabs((d.v[c0] + d.v[c0 + d.sy]) * d.dyfi[j]) +
           fabs((d.w[c0] + d.w[c0 + d.sz * (kp - k)]) * d.dzi)) * 0.5;
    } else {
      v = (double)(!isfinite(d.u[c0])) + (double)(!isfinite(d.v[c0])) + (double)(!isfinite(d.w[c0])) +
          (double)(!isfinite(d.p[c0]));
    }
  }
  const bool mx = what == 0 || what == 3;
  const double s = mx ? block_max(v, sh) : block_sum(v, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    d.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
}

__global__ void __launch_bounds__(1024) k_reduce_final(TGDev d, int what, int npart) {
  __shared__ double sh[32];
  double s = 0.0;
  const bool mx = what == 0 || what == 3;
  for (int t = threadIdx.x; t < npart; t += blockDim.x) s = mx ? fmax(s, d.partials[t]) : s + d.partials[t];
  s = mx ? block_max(s, sh) : block_sum(s, sh);
  if (threadIdx.x == 0) d.scal[1] = s;
}

// ============================================================ launchers


// Read back every buffered substep's phase events and accumulate them.
int flush_phase_events(chapsim_ctx *c) {
  if (c->ev_pending == 0) return CHAPSIM_OK;
  const size_t last = (size_t)(c->ev_pending - 1) * (CHAPSIM_PH_COUNT + 1) + CHAPSIM_PH_COUNT;
  CK(cudaEventSynchronize(c->evpool[last]));
  for (int s = 0; s < c->ev_pending; ++s) {
    cudaEvent_t *e = &c->evpool[(size_t)s * (CHAPSIM_PH_COUNT + 1)];
    for (int ph = 0; ph < CHAPSIM_PH_COUNT; ++ph) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e[ph], e[ph + 1]));
      c->phase_ms[ph] += ms;
    }
  }
  c->timed_substeps += c->ev_pending;
  c->ev_pending = 0;
  return CHAPSIM_OK;
}

template <typename T> struct Prec {
  typedef typename Cplx<T>::type C;
  static int max_fftx_lb(int nx, int dr) {
    int lb = 2;
    while (lb < 32 && fftx_smem_bytes<C>(nx, lb + 2, dr) <= 110 * 1024) lb += 2;
    return lb;
  }
  static int dr_rows(const chapsim_ctx *c) { return c->domain == CHAPSIM_IIO ? 1 : 0; }
  static int fftx_lb(const chapsim_ctx *c) {
    const int dr = dr_rows(c);
    if (c->fft_lb >= 2 && c->fft_lb <= max_fftx_lb(c->d.nx, dr)) return c->fft_lb & ~1;
    // rows per block of the forward x transform: the most rows whose inputs
    // fit in 74 KB (three blocks per SM) when that is at least four rows,
    // else the most that fit in 110 KB (measured on the 256x192x256 and
    // 512x192x256 channels)
    int lb = 2;
    while (lb < 32 && fftx_smem_bytes<C>(c->d.nx, lb + 2, dr) <= 74 * 1024) lb += 2;
    return lb >= 4 ? lb : max_fftx_lb(c->d.nx, dr);
  }
  // rows per block of the inverse x transform: the most rows whose buffers
  // fit in 74 KB, so that three blocks share an SM, as a power of two (at
  // power-of-two nx the lines' butterflies then fill whole passes of the
  // block's 256 threads)
  static int ifftx_lb(const chapsim_ctx *c) {
    int lb = 2;
    while (lb < 32 && ifftx_smem_bytes<C>(c->d.nx, c->d.lp, 2 * lb) <= 74 * 1024) lb *= 2;
    return lb;
  }
  static size_t fftx_smem(const chapsim_ctx *c, int lb) { return fftx_smem_bytes<C>(c->d.nx, lb, dr_rows(c)); }
  static size_t ifftx_smem(int nx, int lp, int lb) { return ifftx_smem_bytes<C>(nx, lp, lb); }
  static int fftz_lz(int nz) {
    // lines per block of the z transforms: a power of two up to 16 whose two
    // buffers fit in 72 KB, so that three blocks share an SM
    int lz = 16;
    while (lz > 2 && (size_t)2 * lz * nz * sizeof(C) > 72 * 1024) lz >>= 1;
    return lz;
  }
  static size_t fftz_smem(int nz, int lz) { return (size_t)2 * lz * nz * sizeof(C); }
  static size_t adiy_smem(int ny) { return (size_t)ny * AY_TL * sizeof(T); }
  static int adix_lb(int nx) {
    int lb = (int)(96 * 1024 / ((size_t)(nx + 1) * sizeof(T)));
    if (lb > 64) lb = 64;
    if (lb < 1) lb = 1;
    return lb;
  }
  static size_t adix_smem(int nx, int lb) {
    return (((size_t)lb * (nx + 1) * sizeof(T) + 15) & ~(size_t)15) + 3 * (size_t)nx * sizeof(double);
  }
  static size_t adiz_smem(int nz) {
    return (((size_t)nz * LZ * sizeof(T) + 15) & ~(size_t)15) + 3 * (size_t)nz * sizeof(double);
  }
  static size_t rhs_tma_smem() { return RtLayout<T>::smem_bytes; }

  // Dynamic shared-memory limits are per kernel and process wide, so they are
  // raised once to the device's opt-in maximum rather than to one context's
  // sizes (a later, smaller context must not lower them for earlier ones).
  static int init(chapsim_ctx *c) {
    const int ny = c->d.ny;
    if (adiy_smem(ny) > 200 * 1024) {
      c->err = "ny too large for the shared-memory y-line kernels";
      return CHAPSIM_ERR_UNSUPPORTED;
    }
    int maxs = 0;
    CK(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    const void *dyn[] = {(const void *)k_rhs_tma<T>,      (const void *)k_adix<T>,           (const void *)k_adiz<T>,
                         (const void *)k_fftx<T, false>,  (const void *)k_ifftx<T, false>,   (const void *)k_fftz<T, false>,
                         (const void *)k_fftx<T, true>,   (const void *)k_ifftx<T, true>,    (const void *)k_fftz<T, true>,
                         (const void *)k_adiy_smem<T>};
    for (const void *f : dyn) {
      cudaFuncAttributes fa;
      CK(cudaFuncGetAttributes(&fa, f));
      CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs - (int)fa.sharedSizeBytes));
      CK(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    }
    return CHAPSIM_OK;
  }

  // mode 0: divergence of q; 1: stored RHSLLPHI; 2: residual buffer
  static int fftx(chapsim_ctx *c, int ns, int mode) {
    TGDev &d = c->d;
    const int lb = fftx_lb(c);
    dim3 grid((d.ny + lb - 1) / lb, d.nz);
    if (c->fft_big)
      k_fftx<T, true><<<grid, 256, fftx_smem(c, lb), c->stream>>>(d, c->sp[ns], c->fx, lb, mode);
    else
      k_fftx<T, false><<<grid, 256, fftx_smem(c, lb), c->stream>>>(d, c->sp[ns], c->fx, lb, mode);
    LAUNCHED();
    return CHAPSIM_OK;
  }

  static int spectral_solve(chapsim_ctx *c, int accumulate, bool mark) {
    TGDev &d = c->d;
    const int lz = fftz_lz(d.nz), lb = ifftx_lb(c);
    if (mark) phase_mark(c, CHAPSIM_PH_FFTZ);
    {
      dim3 grid((d.lh + lz - 1) / lz, d.ny);
      if (c->fft_big)
        k_fftz<T, true><<<grid, 256, fftz_smem(d.nz, lz), c->stream>>>(d, c->fz, lz, -1);
      else
        k_fftz<T, false><<<grid, 256, fftz_smem(d.nz, lz), c->stream>>>(d, c->fz, lz, -1);
      LAUNCHED();
    }
    if (mark) phase_mark(c, CHAPSIM_PH_YSOLVE);
    {
      const int bx = c->ys_bx;
      dim3 grid((d.lh + bx - 1) / bx, d.nz);
      k_ysolve_line<T><<<grid, bx, 0, c->stream>>>(d);
      LAUNCHED();
    }
    if (mark) phase_mark(c, CHAPSIM_PH_IFFTZ);
    {
      dim3 grid((d.lh + lz - 1) / lz, d.ny);
      if (c->fft_big)
        k_fftz<T, true><<<grid, 256, fftz_smem(d.nz, lz), c->stream>>>(d, c->fz, lz, +1);
      else
        k_fftz<T, false><<<grid, 256, fftz_smem(d.nz, lz), c->stream>>>(d, c->fz, lz, +1);
      LAUNCHED();
    }
    if (mark) phase_mark(c, CHAPSIM_PH_IFFTX);
    {
      dim3 grid((d.ny + lb - 1) / lb, d.nz);
      if (c->fft_big)
        k_ifftx<T, true><<<grid, 256, ifftx_smem(d.nx, d.lp, lb), c->stream>>>(d, c->fx, lb, accumulate);
      else
        k_ifftx<T, false><<<grid, 256, ifftx_smem(d.nx, d.lp, lb), c->stream>>>(d, c->fx, lb, accumulate);
      LAUNCHED();
    }
    return CHAPSIM_OK;
  }

  // Poisson solve of RHSLLPHI (computed from q when mode == 0).  The mixed
  // form adds one refinement sweep: residual in FP64, second FP32 solve,
  // correction accumulated into phi.
  static int poisson(chapsim_ctx *c, int ns, int mode) {
    TGDev &d = c->d;
    phase_mark(c, CHAPSIM_PH_FFTX);
    int rc = fftx(c, ns, mode);
    if (rc) return rc;
    rc = spectral_solve(c, 0, true);
    if (rc) return rc;
    if (sizeof(T) == 4 && c->refine) {
      dim3 grid((d.nx + RHS_BX - 1) / RHS_BX, (d.ny + RHS_BY - 1) / RHS_BY, d.nz);
      k_pois_residual<<<grid, dim3(RHS_BX, RHS_BY), 0, c->stream>>>(d);
      LAUNCHED();
      rc = fftx(c, ns, 2);
      if (rc) return rc;
      rc = spectral_solve(c, 1, false);
      if (rc) return rc;
    }
    return CHAPSIM_OK;
  }

  static int substep(chapsim_ctx *c, int ns) {
    TGDev &d = c->d;
    const SubParams &sp = c->sp[ns];
    phase_mark(c, CHAPSIM_PH_RHS);
    {
      dim3 grid((d.nx + RHS_BX - 1) / RHS_BX, (d.ny + RHS_BY - 1) / RHS_BY, d.nz);
      if (c->use_tma_rhs) {
        const int nzc = c->rhs_nzc;
        grid.z = (d.nz + nzc - 1) / nzc;
        RhsMaps maps;
        memcpy(maps.m, c->rhs_maps, sizeof(maps.m));
        k_rhs_tma<T><<<grid, dim3(RHS_BX, RHS_BY), rhs_tma_smem(), c->stream>>>(maps, d, sp, nzc);
      } else {
        k_rhs<T><<<grid, dim3(RHS_BX, RHS_BY), 0, c->stream>>>(d, sp);
      }
      LAUNCHED();
      const int npart = grid.x * grid.y * grid.z;
      k_dpgrns<<<1, 1024, 0, c->stream>>>(d, sp, npart);
      LAUNCHED();
    }
    phase_mark(c, CHAPSIM_PH_ADIX);
    if (sp.band) {
      dim3 grid((d.nx + BM_TX - 1) / BM_TX, (d.ny + BM_TY - 1) / BM_TY, 3 * ((d.nz + BM_SEG - 1) / BM_SEG));
      if (!launch_adixz_rows<T>(c->stream, d, sp)) launch_adixz<T>(grid, c->stream, d, sp);
      LAUNCHED();
      phase_mark(c, CHAPSIM_PH_ADIZ);
    } else {
      const int lb = adix_lb(d.nx);
      dim3 grid((d.ny + lb - 1) / lb, d.nz, 3);
      k_adix<T><<<grid, 128, adix_smem(d.nx, lb), c->stream>>>(d, sp, lb);
      LAUNCHED();
      phase_mark(c, CHAPSIM_PH_ADIZ);
      dim3 grid2((d.nx + LZ - 1) / LZ, d.ny, 3);
      k_adiz<T><<<grid2, 128, adiz_smem(d.nz), c->stream>>>(d, sp);
      LAUNCHED();
    }
    phase_mark(c, CHAPSIM_PH_ADIY);
    if (sp.band && sp.wy >= 0) {
      dim3 grid((d.nx + AY_TX - 1) / AY_TX, (d.ny + AY_JT - 1) / AY_JT, d.nz);
      launch_adiy<T>(grid, c->stream, d, sp);
      LAUNCHED();
    } else {
      dim3 grid((d.nx + AY_TL - 1) / AY_TL, d.nz);
      k_adiy_smem<T><<<grid, 128, adiy_smem(d.ny), c->stream>>>(d, sp, sp.band);
      LAUNCHED();
    }
    int rc = poisson(c, ns, 0);
    if (rc) return rc;
    phase_mark(c, CHAPSIM_PH_CORR);
    rc = launch_correction(c, ns);
    if (rc) return rc;
    if (c->timing) {
      phase_mark(c, CHAPSIM_PH_COUNT);
      if (++c->ev_pending == chapsim_ctx::kEvSub) return flush_phase_events(c);
    }
    return CHAPSIM_OK;
  }
};

// TMA descriptors of u, v, w, p (FP64, box 36 x 10 x 1) and of the three H0
// components (temporary precision, box 32 x 8 x 1); no swizzle, out-of-bounds
// boxes zero filled.
static int make_rhs_maps(chapsim_ctx *c) {
  TGDev &d = c->d;
  c->use_tma_rhs = false;
  // small grids use k_rhs; the coupled IO section (fields offset by its ghost
  // column) never runs the TG momentum RHS
  if (d.nx < RT_BXW || d.ny < 8 || d.xnp) return CHAPSIM_OK;
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&encode, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !encode) {
    cudaGetLastError();
    return CHAPSIM_OK;
  }
  const bool mixed = c->cfg.precision == CHAPSIM_MIXED;
  const size_t hsz = mixed ? sizeof(float) : sizeof(double);
  void *f[7] = {d.u, d.v, d.w, d.p, d.h0[0], d.h0[1], d.h0[2]};
  cuuint64_t dims[3] = {(cuuint64_t)d.nx, (cuuint64_t)(d.ny + 2), (cuuint64_t)d.nz};
  cuuint64_t strides[2] = {(cuuint64_t)d.sy * sizeof(double), (cuuint64_t)d.sz * sizeof(double)};
  cuuint64_t hstrides[2] = {(cuuint64_t)d.sy * hsz, (cuuint64_t)d.sz * hsz};
  cuuint32_t box[3] = {RT_BXW, RT_BYW, 1};
  cuuint32_t hbox[3] = {RHS_BX, RHS_BY, 1};
  cuuint32_t es[3] = {1, 1, 1};
  if ((d.sy * hsz) % 16 != 0) return CHAPSIM_OK;  // TMA strides must be multiples of 16 bytes
  for (int m = 0; m < 7; ++m) {
    const bool h = m >= 4;
    CUresult r = encode(&c->rhs_maps[m], (h && mixed) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                        3, f[m], dims, h ? hstrides : strides, h ? hbox : box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      c->err = "cuTensorMapEncodeTiled failed";
      return CHAPSIM_ERR_CUDA;
    }
  }
  c->use_tma_rhs = true;
  return CHAPSIM_OK;
}

int init_kernels(chapsim_ctx *c) {
  int rc = make_rhs_maps(c);
  if (rc) return rc;
  {
    TGDev &d = c->d;
    dim3 grid((d.lh + 127) / 128, d.nz);
    k_ypivots<<<grid, 128, 0, c->stream>>>(d);
    LAUNCHED();
  }
  c->fft_big = false;
  for (int s2 = 0; s2 < 16; ++s2)
    if (c->fx.rad[s2] == 7 || c->fx.rad[s2] == 11 || c->fz.rad[s2] == 7 || c->fz.rad[s2] == 11) c->fft_big = true;
  return c->cfg.precision == CHAPSIM_MIXED ? Prec<float>::init(c) : Prec<double>::init(c);
}

int launch_divg(chapsim_ctx *c, int ns) {
  // DIVG_tg alone: the fused divergence + x-transform kernel in mode 0 stores
  // RHSLLPHI (its spectral output is scratch).
  return c->cfg.precision == CHAPSIM_MIXED ? Prec<float>::fftx(c, ns, 0) : Prec<double>::fftx(c, ns, 0);
}

int launch_pois_io(chapsim_ctx *c, int ns, double *gx, double *gy, double *gz, const double *drho,
                   bool store_rhs) {
  // the fused divergence of the forward x-transform reads u, v, w: point them
  // at the provisional mass flux for these launches only
  const TGDev saved = c->d;
  c->d.u = gx; c->d.v = gy; c->d.w = gz; c->d.drho = drho;
  const bool mixed = c->cfg.precision == CHAPSIM_MIXED;
  // the mixed form's refinement sweep forms its residual from RHSLLPHI
  c->d.skip_rhs = (store_rhs || (mixed && c->refine)) ? 0 : 1;
  const int rc = mixed ? Prec<float>::poisson(c, ns, 0) : Prec<double>::poisson(c, ns, 0);
  c->d = saved;
  return rc;
}

// ---------------------------------------------- non-periodic x (IO Poisson)
// FISHPACK_POIS3D_SIMPLE with Dirichlet / Neumann x ends
// (src/possion3d_fishpack_reform.f90:104-163, 431-547): the x transform is
// FFTPACK's SINT, SINQF / SINQB, COST or COSQF / COSQB, applied as a dense
// nx x nx matrix (stored transposed: threads computing consecutive outputs
// read consecutive entries) to every (j, k) row.  The real x modes occupy
// the real parts of a complex spectral array of nx lines, on which the z
// transforms and the y-line solves of the periodic path run unchanged (line
// I shifted by -XRT(I)).  The forward matrix carries 1 / SCALX; the z
// transforms carry 1 / nz, as in the periodic path.
__global__ void __launch_bounds__(128) k_xnp_fwd(TGDev d, TGDev s, const double *__restrict__ ft) {
  extern __shared__ double xrow[];
  const int j = blockIdx.x + 1, k = blockIdx.y, nx = d.nx;
  const double *src = d.rhsphi + d.sy * j + d.sz * k;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) xrow[i] = src[i];
  __syncthreads();
  double2 *dst = reinterpret_cast<double2 *>(s.spec) + (int64_t)s.lp * (j - 1) + (int64_t)s.lp * s.ny * k;
  for (int m = threadIdx.x; m < s.lp; m += blockDim.x) {
    double acc = 0.0;
    if (m < nx)
      for (int q = 0; q < nx; ++q) acc = fma(ft[(size_t)q * nx + m], xrow[q], acc);
    dst[m] = make_double2(acc, 0.0);
  }
}

__global__ void __launch_bounds__(128) k_xnp_bwd(TGDev d, TGDev s, const double *__restrict__ bt) {
  extern __shared__ double xrow[];
  const int j = blockIdx.x + 1, k = blockIdx.y, nx = d.nx, ny = d.ny;
  const double2 *src = reinterpret_cast<const double2 *>(s.spec) + (int64_t)s.lp * (j - 1) + (int64_t)s.lp * s.ny * k;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) xrow[i] = src[i].x;
  __syncthreads();
  double *dst = d.phi + d.sy * j + d.sz * k;
  for (int m = threadIdx.x; m < nx; m += blockDim.x) {
    double acc = 0.0;
    for (int q = 0; q < nx; ++q) acc = fma(bt[(size_t)q * nx + m], xrow[q], acc);
    dst[m] = acc;
    if (j == 1) dst[m - d.sy] = acc;   // BC_WALL_DPH: ghost rows by copy
    if (j == ny) dst[m + d.sy] = acc;
  }
}


// The quarter-wave pairs (LP 5: COSQF / COSQB, LP 3: SINQF / SINQB) through
// the N-point complex FFT of the periodic path (Makhoul's even-odd reordering,
// IEEE Trans. ASSP 28 (1980) 27-34), two real rows per complex line:
//   COSQB(X)_k = 4 Re(q_k V_k),  V = FFT(v), v_n = X_{2n}, v_{N-1-n} = X_{2n+1};
//   COSQF(x)_{2n} = w_n, COSQF(x)_{2n+1} = w_{N-1-n},
//     w = sum_m conj(q_m) (x_m - i x_{N-m}) e^{+2 pi i m n / N}  (x_N = 0);
//   SINQF(x)_k = (-1)^k COSQF(x reversed)_k,
//   SINQB(X)_k = COSQB((-1)^n X_n)_{N-1-k},
// with q_m = exp(-i pi m / (2N)) (table qw).  They equal FFTPACK's documented
// sums (the dense-matrix kernels above) to round-off.  Rows of lb per block;
// the rows sit at an 8-byte offset in the coupled layout, so they are read
// with plain loads.
__host__ __device__ constexpr size_t xq_cplx(int nx, int lb) { return (((size_t)(lb / 2) * nx + 7) / 8) * 8; }
// the second buffer holds lb input rows of nx + 2 values (ghost columns
// included) first, the FFT scratch afterwards
__host__ __device__ constexpr size_t xq_in_bytes(int nx, int lb) {
  return align128(xq_cplx(nx, lb) * sizeof(double2)) > align128((size_t)lb * (nx + 2) * sizeof(double))
             ? align128(xq_cplx(nx, lb) * sizeof(double2))
             : align128((size_t)lb * (nx + 2) * sizeof(double));
}
__host__ __device__ constexpr size_t xq_smem_bytes(int nx, int lb) {
  return align128(xq_cplx(nx, lb) * sizeof(double2)) + xq_in_bytes(nx, lb);
}

template <bool BIG>
__global__ void __launch_bounds__(256) k_xnp_qfwd(TGDev d, TGDev s, FFTPlan pl, const double2 *__restrict__ qw, int lb,
                                                  int sinq, double rscal) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int rad[16];
  __shared__ uint64_t bar;
  const int nx = d.nx, ny = d.ny, k = blockIdx.y, jbeg = 1 + blockIdx.x * lb;
  const int nrow = min(lb, ny - jbeg + 1), nl = lb / 2, tid = threadIdx.x;
  const int sy = d.sy;  // nx + 2: rows from the inlet ghost column, one value before the field pointer
  double2 *A = reinterpret_cast<double2 *>(smem_raw);
  double *in = reinterpret_cast<double *>(smem_raw + align128(xq_cplx(nx, lb) * sizeof(double2)));
  double2 *B = reinterpret_cast<double2 *>(in);  // FFT scratch once A is filled
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (tid < 16) rad[tid] = pl.rad[tid];
  __syncthreads();
  // the block's rows of RHSLLPHI by one bulk copy each ((nx + 2) * 8 bytes,
  // 16-byte aligned: nx is even and the allocation starts at the ghost column)
  const uint32_t rowb = (uint32_t)(sy * sizeof(double));
  if (tid == 0) mbar_expect_tx(&bar, rowb * (uint32_t)nrow);
  __syncthreads();
  const double *src = d.rhsphi - 1 + (int64_t)d.sz * k + (int64_t)sy * jbeg;
  for (int r = tid; r < nrow; r += blockDim.x) bulk_g2s(in + (size_t)r * sy, src + (int64_t)sy * r, rowb, &bar);
  for (int t = tid; t < (lb - nrow) * sy; t += blockDim.x) in[(size_t)nrow * sy + t] = 0.0;
  if (!mbar_wait(&bar, 0, d.err)) {
    mbar_wait(&bar, 0, d.err);  // let copies in flight land before the block exits
    return;
  }
  __syncthreads();
  for (int t = tid; t < nl * nx; t += blockDim.x) {
    const int p = t / nx, m = t - p * nx;
    const double *r0 = in + (size_t)2 * p * sy + 1, *r1 = r0 + sy;
    const int im = sinq ? nx - 1 - m : m, ic = sinq ? m - 1 : nx - m;  // x_m, x_{N-m} (SINQF: reversed row)
    const double a0 = r0[im], a1 = r1[im];
    const double b0 = m ? r0[ic] : 0.0, b1 = m ? r1[ic] : 0.0;
    const double2 q = qw[m];  // conj(q) (a - i b) = (qx a - qy b) + i (-qy a - qx b)
    const double v1x = q.x * a0 - q.y * b0, v1y = -q.y * a0 - q.x * b0;
    const double v2x = q.x * a1 - q.y * b1, v2y = -q.y * a1 - q.x * b1;
    A[swz(p * nx + m)] = make_double2(v1x - v2y, v1y + v2x);  // V1 + i V2
  }
  __syncthreads();
  const double2 *res = fft_lines<double2, BIG>(A, B, nl, nx, nx, rad, pl.nrad, pl.tw64, +1);
  double *S = reinterpret_cast<double *>(s.spec);
  for (int t = tid; t < nrow * nx; t += blockDim.x) {
    const int r = t / nx, m = t - r * nx;
    const int n = (m & 1) ? nx - 1 - (m >> 1) : (m >> 1);
    const double2 z = res[swz((r >> 1) * nx + n)];
    double y = (r & 1) ? z.y : z.x;
    if (sinq && (m & 1)) y = -y;
    S[m + 2 * (int64_t)s.lp * ((jbeg + r - 1) + (int64_t)ny * k)] = y * rscal;  // mode m: line m / 2, part m % 2
  }
}

template <bool BIG>
__global__ void __launch_bounds__(256) k_xnp_qbwd(TGDev d, TGDev s, FFTPlan pl, const double2 *__restrict__ qw, int lb,
                                                  int sinq) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int rad[16];
  __shared__ uint64_t bar;
  const int nx = d.nx, ny = d.ny, k = blockIdx.y, jbeg = 1 + blockIdx.x * lb;
  const int nrow = min(lb, ny - jbeg + 1), nl = lb / 2, tid = threadIdx.x;
  double2 *A = reinterpret_cast<double2 *>(smem_raw);
  double *in = reinterpret_cast<double *>(smem_raw + align128(xq_cplx(nx, lb) * sizeof(double2)));
  double2 *B = reinterpret_cast<double2 *>(in);
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (tid < 16) rad[tid] = pl.rad[tid];
  __syncthreads();
  // the block's packed spectral rows (nx values each, 16-byte aligned: the
  // pitch 2 lp is a multiple of 4) by one bulk copy each
  const uint32_t rowb = (uint32_t)(nx * sizeof(double));
  if (tid == 0) mbar_expect_tx(&bar, rowb * (uint32_t)nrow);
  __syncthreads();
  const double *S = reinterpret_cast<const double *>(s.spec) + 2 * (int64_t)s.lp * ((jbeg - 1) + (int64_t)ny * k);
  for (int r = tid; r < nrow; r += blockDim.x)
    bulk_g2s(in + (size_t)r * nx, S + 2 * (int64_t)s.lp * r, rowb, &bar);
  for (int t = tid; t < (lb - nrow) * nx; t += blockDim.x) in[(size_t)nrow * nx + t] = 0.0;
  if (!mbar_wait(&bar, 0, d.err)) {
    mbar_wait(&bar, 0, d.err);  // let copies in flight land before the block exits
    return;
  }
  __syncthreads();
  for (int t = tid; t < nl * nx; t += blockDim.x) {
    const int p = t / nx, n = t - p * nx;
    const int q = 2 * n < nx ? 2 * n : 2 * (nx - 1 - n) + 1;  // v_n = X_{2n}, v_{N-1-n} = X_{2n+1}
    const double sg = (sinq && (q & 1)) ? -1.0 : 1.0;          // SINQB: (-1)^n X_n
    A[swz(p * nx + n)] = make_double2(sg * in[(size_t)2 * p * nx + q], sg * in[(size_t)(2 * p + 1) * nx + q]);
  }
  __syncthreads();
  const double2 *res = fft_lines<double2, BIG>(A, B, nl, nx, nx, rad, pl.nrad, pl.tw64, -1);
  for (int t = tid; t < nrow * nx; t += blockDim.x) {
    const int r = t / nx, m = t - r * nx;
    const int kk = sinq ? nx - 1 - m : m;
    const double2 z = res[swz((r >> 1) * nx + kk)], zc = res[swz((r >> 1) * nx + (kk ? nx - kk : 0))];
    // V1 = (Z_k + conj Z_{N-k}) / 2, V2 = (Z_k - conj Z_{N-k}) / (2i)
    double vx, vy;
    if (r & 1) {
      vx = 0.5 * (z.y + zc.y);
      vy = -0.5 * (z.x - zc.x);
    } else {
      vx = 0.5 * (z.x + zc.x);
      vy = 0.5 * (z.y - zc.y);
    }
    const double2 q = qw[kk];
    const double y = 4.0 * (q.x * vx - q.y * vy);
    const int j = jbeg + r;
    double *dst = d.phi + d.sy * j + d.sz * k;
    dst[m] = y;
    if (j == 1) dst[m - d.sy] = y;  // BC_WALL_DPH: ghost rows by copy
    if (j == ny) dst[m + d.sy] = y;
  }
}

int xnp_pivots(chapsim_ctx *c) {
  TGDev &s = c->dnp;
  dim3 grid((s.lh + 127) / 128, s.nz);
  k_ypivots<<<grid, 128, 0, c->stream>>>(s);
  LAUNCHED();
  return CHAPSIM_OK;
}

// rows per block of the quarter-wave transforms: the most, as a power of two
// up to 32, whose two buffers fit in 74 KB (three blocks per SM)
int xnp_q_lb(int nx) {
  int lb = 2;
  while (lb < 32 && xq_smem_bytes(nx, 2 * lb) <= 74 * 1024) lb *= 2;
  return lb;
}

int xnp_q_setup(chapsim_ctx *c) {
  const size_t sm = xq_smem_bytes(c->d.nx, xnp_q_lb(c->d.nx));
  for (const void *f : {(const void *)k_xnp_qfwd<false>, (const void *)k_xnp_qfwd<true>,
                        (const void *)k_xnp_qbwd<false>, (const void *)k_xnp_qbwd<true>})
    CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  return CHAPSIM_OK;
}

int xnp_pois3d(chapsim_ctx *c, bool mark) {
  TGDev &d = c->d, &s = c->dnp;
  const size_t sm = (size_t)d.nx * sizeof(double);
  const dim3 rows(d.ny, d.nz);
  const bool q = c->xnp_qw != nullptr;  // LP 3 / 5 through the FFT
  const int lb = xnp_q_lb(d.nx);
  const size_t smq = xq_smem_bytes(d.nx, lb);
  const dim3 qgrid((d.ny + lb - 1) / lb, d.nz);
  const int sinq = c->xnp == 3;
  // the quarter-wave transforms' modes two to a complex line (nx even): nx / 2
  // lines in the spectral array of s
  TGDev qs = s;
  qs.lh = d.nx / 2;
  qs.lp = (qs.lh + 1) & ~1;
  const TGDev &z = q ? qs : s;
  if (q && c->fft_big)
    k_xnp_qfwd<true><<<qgrid, 256, smq, c->stream>>>(d, qs, c->fx, c->xnp_qw, lb, sinq, c->xnp_rscal);
  else if (q)
    k_xnp_qfwd<false><<<qgrid, 256, smq, c->stream>>>(d, qs, c->fx, c->xnp_qw, lb, sinq, c->xnp_rscal);
  else
    k_xnp_fwd<<<rows, 128, sm, c->stream>>>(d, s, c->xnp_f);
  LAUNCHED();
  typedef Prec<double> P;
  const int lz = P::fftz_lz(d.nz);
  const dim3 gz((z.lh + lz - 1) / lz, d.ny);
  if (mark) phase_mark(c, CHAPSIM_PH_FFTZ);
  if (c->fft_big)
    k_fftz<double, true><<<gz, 256, P::fftz_smem(d.nz, lz), c->stream>>>(z, c->fz, lz, -1);
  else
    k_fftz<double, false><<<gz, 256, P::fftz_smem(d.nz, lz), c->stream>>>(z, c->fz, lz, -1);
  LAUNCHED();
  if (mark) phase_mark(c, CHAPSIM_PH_YSOLVE);
  if (q) {
    dim3 grid((qs.lh + 127) / 128, d.nz / 2 + 1);
    k_ysolve_pair<<<grid, 128, 0, c->stream>>>(qs, s);
  } else {
    const int bx = c->ys_bx;
    dim3 grid((s.lh + bx - 1) / bx, d.nz);
    k_ysolve_line<double><<<grid, bx, 0, c->stream>>>(s);
  }
  LAUNCHED();
  if (mark) phase_mark(c, CHAPSIM_PH_IFFTZ);
  if (c->fft_big)
    k_fftz<double, true><<<gz, 256, P::fftz_smem(d.nz, lz), c->stream>>>(z, c->fz, lz, +1);
  else
    k_fftz<double, false><<<gz, 256, P::fftz_smem(d.nz, lz), c->stream>>>(z, c->fz, lz, +1);
  LAUNCHED();
  if (mark) phase_mark(c, CHAPSIM_PH_IFFTX);
  if (q && c->fft_big)
    k_xnp_qbwd<true><<<qgrid, 256, smq, c->stream>>>(d, qs, c->fx, c->xnp_qw, lb, sinq);
  else if (q)
    k_xnp_qbwd<false><<<qgrid, 256, smq, c->stream>>>(d, qs, c->fx, c->xnp_qw, lb, sinq);
  else
    k_xnp_bwd<<<rows, 128, sm, c->stream>>>(d, s, c->xnp_b);
  LAUNCHED();
  return CHAPSIM_OK;
}

int launch_pois3d(chapsim_ctx *c) {
  return c->cfg.precision == CHAPSIM_MIXED ? Prec<float>::poisson(c, 1, 1) : Prec<double>::poisson(c, 1, 1);
}

int launch_substep(chapsim_ctx *c, int ns) {
  return c->cfg.precision == CHAPSIM_MIXED ? Prec<float>::substep(c, ns) : Prec<double>::substep(c, ns);
}

int launch_correction(chapsim_ctx *c, int ns) {
  TGDev &d = c->d;
  dim3 grid((d.nx + RHS_BX - 1) / RHS_BX, (d.ny + RHS_BY - 1) / RHS_BY, d.nz);
  k_corr<<<grid, dim3(RHS_BX, RHS_BY), 0, c->stream>>>(d, c->sp[ns]);
  LAUNCHED();
  return CHAPSIM_OK;
}

int launch_bc_q(chapsim_ctx *c) {
  TGDev &d = c->d;
  dim3 grid((d.nx + 127) / 128, d.nz);
  k_bc_q<<<grid, 128, 0, c->stream>>>(d);
  LAUNCHED();
  return CHAPSIM_OK;
}

int launch_reduce(chapsim_ctx *c, int what, double *host_out) {
  TGDev &d = c->d;
  dim3 grid((d.nx + RHS_BX - 1) / RHS_BX, (d.ny + RHS_BY - 1) / RHS_BY, d.nz);
  k_reduce_part<<<grid, dim3(RHS_BX, RHS_BY), 0, c->stream>>>(d, what);
  LAUNCHED();
  k_reduce_final<<<1, 1024, 0, c->stream>>>(d, what, (int)(grid.x * grid.y * grid.z));
  LAUNCHED();
  double v = 0.0;
  CK(cudaMemcpyAsync(&v, d.scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *host_out = v;
  return CHAPSIM_OK;
}

// Fault-injection hook for the bounded waits: one warp initialises an
// mbarrier that expects one arrival, never arrives on it, and waits with a
// spin limit of `polls`.  The wait gives up, records kErrTmaTimeout in the
// context's error word and the kernel returns; no copy is in flight, so
// nothing else needs draining.  It exercises the same give-up path every TMA
// consumer uses, with a limit small enough to end in microseconds.
__global__ void k_wait_probe(int *err, uint32_t polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
  mbar_wait(&bar, 0, err, polls);
  __syncwarp();
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar)) : "memory");
}

int launch_wait_probe(chapsim_ctx *c, int polls) {
  k_wait_probe<<<1, 32, 0, c->stream>>>(c->d.err, (uint32_t)polls);
  LAUNCHED();
  return CHAPSIM_OK;
}

}  // namespace chapsim
