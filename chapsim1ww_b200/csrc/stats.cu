// On-device flow statistics of the TG channel: the xz-plane averages of
// PP_MEAN_ZX_FLOW_TG (src/processing/PP_MEAN_ZX.f90:1-294) and their running
// time average PP_MEAN_T_TG (src/processing/PP_MEAN_T.f90:322-370), so that a
// host needs no per-step download of the field to keep its statistics.
//
// Per y-row j the 122 values are, in this order:
//   U1 (4)     mean of the cell-centred u, v, w (x 0.5 x 2) and p
//   UP (3)     u_i p
//   U2 (6)     u_i u_j, upper triangle (11 12 13 22 23 33)
//   U3 (10)    u_i u_j u_k, upper tetrahedron (111 112 113 122 123 133 222 223 233 333)
//   DVDL1 (9)  du_m/dx_n, row-major (m, n)
//   DVDLP (9)  du_m/dx_n p
//   DVDL2 (81) (du_m/dx_h)(du_n/dx_p), row (m,h), column (n,p)
// with the reference's scaling (VL1313 = 1/(nx nz) and the 0.5 factors of the
// cell-centred sums).
//
// Reduction: grid (ny, NBK k-chunks, 2 groups); every block sums its cells in
// a fixed order and writes one partial per accumulator; a second kernel adds
// the NBK partials of each row in order and applies the scaling, so the
// result is bit-reproducible.  Group 0 holds U1, UP, U2, U3, DVDL1, DVDLP
// (41 values), group 1 the upper triangle of the symmetric DVDL2 (45).
#include <cuda_runtime.h>

#include <string>

#include "chapsim_internal.cuh"

namespace chapsim {
namespace {

constexpr int ST_NV = 122, ST_G0 = 41, ST_G1 = 45, ST_NBK = 4, ST_TPB = 128;

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

// The 13 per-cell quantities: U_cct(1..3), p, and DVDL_cct(3x3) (unscaled).
struct CellQ {
  double U[3], p, D[9];
};

__device__ __forceinline__ CellQ cell_quantities(const TGDev &d, int i, int j, int k) {
  const int nx = d.nx, nz = d.nz;
  const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
  const int kp = k + 1 == nz ? 0 : k + 1, km = k == 0 ? nz - 1 : k - 1;
  const int64_t sy = d.sy, sz = d.sz;
  const int64_t c = i + sy * j + sz * k;
  const int64_t oxp = ip - i, oxm = im - i, ozp = sz * (kp - k), ozm = sz * (km - k);
  const double *u = d.u, *v = d.v, *w = d.w;
  CellQ q;
  // U_cct and its neighbours (src/processing/PP_MEAN_ZX.f90:79-121, channel branch)
  const double u0 = u[c] + u[c + oxp];
  const double ujp = u[c + sy] + u[c + sy + oxp], ujm = u[c - sy] + u[c - sy + oxp];
  const double ukp = u[c + ozp] + u[c + ozp + oxp], ukm = u[c + ozm] + u[c + ozm + oxp];
  const double w0 = w[c] + w[c + ozp];
  const double wip = w[c + oxp] + w[c + oxp + ozp], wim = w[c + oxm] + w[c + oxm + ozp];
  const double wjp = w[c + sy] + w[c + sy + ozp], wjm = w[c - sy] + w[c - sy + ozp];
  const double v0 = v[c] + v[c + sy];
  const double vip = v[c + oxp] + v[c + oxp + sy], vim = v[c + oxm] + v[c + oxm + sy];
  const double vkp = v[c + ozp] + v[c + ozp + sy], vkm = v[c + ozm] + v[c + ozm + sy];
  q.U[0] = u0; q.U[1] = v0; q.U[2] = w0;
  q.p = d.p[c];
  const double dycp = d.dyci[j + 1], dycj = d.dyci[j];
  q.D[0] = u[c + oxp] - u[c];
  q.D[1] = (ujp - u0) * dycp + (u0 - ujm) * dycj;
  q.D[2] = ukp - ukm;
  q.D[3] = vip - vim;
  q.D[4] = (v[c + sy] - v[c]) * d.dyfi[j];
  q.D[5] = vkp - vkm;
  q.D[6] = wip - wim;
  q.D[7] = (wjp - w0) * dycp + (w0 - wjm) * dycj;
  q.D[8] = w[c + ozp] - w[c];
  return q;
}

template <int G>
__global__ void __launch_bounds__(ST_TPB) k_stats_part(TGDev d, double *part) {
  constexpr int NA = G == 0 ? ST_G0 : ST_G1;
  __shared__ double red[ST_TPB / 32][NA];
  const int j = blockIdx.x + 1;
  const int nx = d.nx, nz = d.nz;
  const int k0 = (int)((int64_t)nz * blockIdx.y / ST_NBK), k1 = (int)((int64_t)nz * (blockIdx.y + 1) / ST_NBK);
  double acc[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) acc[a] = 0.0;
  const int ncell = nx * (k1 - k0);
  for (int t = threadIdx.x; t < ncell; t += ST_TPB) {
    const int kk = k0 + t / nx, i = t % nx;
    const CellQ q = cell_quantities(d, i, j, kk);
    if (G == 0) {
      int a = 0;
#pragma unroll
      for (int m = 0; m < 3; ++m) acc[a++] += q.U[m];
      acc[a++] += q.p;
#pragma unroll
      for (int m = 0; m < 3; ++m) acc[a++] += q.U[m] * q.p;
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = m; n < 3; ++n) acc[a++] += q.U[m] * q.U[n];
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = m; n < 3; ++n)
#pragma unroll
          for (int h = n; h < 3; ++h) acc[a++] += q.U[m] * q.U[n] * q.U[h];
#pragma unroll
      for (int m = 0; m < 9; ++m) acc[a++] += q.D[m];
#pragma unroll
      for (int m = 0; m < 9; ++m) acc[a++] += q.D[m] * q.p;
    } else {
      int a = 0;
#pragma unroll
      for (int l1 = 0; l1 < 9; ++l1)
#pragma unroll
        for (int l2 = l1; l2 < 9; ++l2) acc[a++] += q.D[l1] * q.D[l2];
    }
  }
  // fixed-order block reduction: warp tree, then the warps in order
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    double v = acc[a];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][a] = v;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < NA; a += ST_TPB) {
    double s = 0.0;
    for (int q = 0; q < ST_TPB / 32; ++q) s += red[q][a];
    part[((size_t)(j - 1) * ST_NBK + blockIdx.y) * (ST_G0 + ST_G1) + (G == 0 ? 0 : ST_G0) + a] = s;
  }
}

// Sum the k-chunk partials of each row in order, scale as the reference does,
// expand the DVDL2 triangle, and (accumulate != 0) fold into the time average.
__global__ void k_stats_final(TGDev d, const double *part, double *xz, double *xzt, double coe2, double coe3,
                              int accumulate) {
  const int j = blockIdx.x + 1;
  const double vl = 1.0 / ((double)d.nx * (double)d.nz);
  const double cog1[9] = {vl * d.dxi, vl * 0.25, vl * 0.25 * d.dzi, vl * 0.25 * d.dxi, vl,
                          vl * 0.25 * d.dzi, vl * 0.25 * d.dxi, vl * 0.25, vl * d.dzi};
  double *out = xz + (size_t)(j - 1) * ST_NV;
  for (int a = threadIdx.x; a < ST_G0 + 81; a += blockDim.x) {
    // source accumulator index and scale of output value a (group-0 part and
    // the 81 DVDL2 entries from the upper triangle)
    int src;
    double sc;
    int o;
    if (a < ST_G0) {
      src = a;
      o = a;
      if (a < 3) sc = vl * 0.5;                   // U1 u, v, w
      else if (a == 3) sc = vl;                   // U1 p
      else if (a < 7) sc = vl * 0.5;              // UP
      else if (a < 13) sc = vl * (0.5 * 0.5);     // U2
      else if (a < 23) sc = vl * (0.5 * 0.5 * 0.5);  // U3
      else if (a < 32) sc = cog1[a - 23];         // DVDL1
      else sc = cog1[a - 32];                     // DVDLP
    } else {
      const int e = a - ST_G0, l1 = e / 9, l2 = e % 9;
      const int lo = l1 < l2 ? l1 : l2, hi = l1 < l2 ? l2 : l1;
      src = ST_G0 + lo * 9 - lo * (lo - 1) / 2 + (hi - lo);
      o = ST_G0 + e;
      sc = cog1[l1] * cog1[l2];
    }
    double s = 0.0;
    for (int b = 0; b < ST_NBK; ++b) s += part[((size_t)(j - 1) * ST_NBK + b) * (ST_G0 + ST_G1) + src];
    const double val = s * sc;
    out[o] = val;
    if (accumulate) {
      double *t = xzt + (size_t)(j - 1) * ST_NV + o;
      *t = coe3 * *t + coe2 * val;
    }
  }
}

}  // namespace

int stats_run(chapsim_ctx *c, int accumulate) {
  TGDev &d = c->d;
  if (!c->stats_buf) {
    const size_t np = (size_t)d.ny * ST_NBK * (ST_G0 + ST_G1), nv = (size_t)d.ny * ST_NV;
    void *p = nullptr;
    CK(cudaMalloc(&p, (np + 2 * nv) * sizeof(double)));
    c->allocs.push_back(p);
    c->stats_buf = (double *)p;
    CK(cudaMemsetAsync(p, 0, (np + 2 * nv) * sizeof(double), c->stream));
  }
  double *part = c->stats_buf, *xz = part + (size_t)d.ny * ST_NBK * (ST_G0 + ST_G1), *xzt = xz + (size_t)d.ny * ST_NV;
  k_stats_part<0><<<dim3(d.ny, ST_NBK), ST_TPB, 0, c->stream>>>(d, part);
  LAUNCHED();
  k_stats_part<1><<<dim3(d.ny, ST_NBK), ST_TPB, 0, c->stream>>>(d, part);
  LAUNCHED();
  double coe2 = 0.0, coe3 = 0.0;
  if (accumulate) {  // T_Asymptotic_Average
    c->nstatis += 1;
    coe2 = 1.0 / (double)c->nstatis;
    coe3 = (double)(c->nstatis - 1) / (double)c->nstatis;
  }
  k_stats_final<<<d.ny, 128, 0, c->stream>>>(d, part, xz, xzt, coe2, coe3, accumulate);
  LAUNCHED();
  return CHAPSIM_OK;
}

int stats_reset(chapsim_ctx *c) {
  c->nstatis = 0;
  if (!c->stats_buf) return CHAPSIM_OK;
  const size_t nv = (size_t)c->d.ny * ST_NV;
  double *xzt = c->stats_buf + (size_t)c->d.ny * ST_NBK * (ST_G0 + ST_G1) + nv;
  CK(cudaMemsetAsync(xzt, 0, nv * sizeof(double), c->stream));
  return CHAPSIM_OK;
}

int stats_get(chapsim_ctx *c, int which, double *host, int64_t n) {
  TGDev &d = c->d;
  if (!c->stats_buf || n != (int64_t)d.ny * ST_NV) return CHAPSIM_ERR_ARG;
  const double *xz = c->stats_buf + (size_t)d.ny * ST_NBK * (ST_G0 + ST_G1);
  const double *src = which == 0 ? xz : xz + (size_t)d.ny * ST_NV;
  CK(cudaMemcpyAsync(host, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAPSIM_OK;
}

}  // namespace chapsim
