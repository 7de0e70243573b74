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
//
// IO section (x-periodic): PP_MEAN_ZX_FLOW_Xperiodic_IO
// (src/processing/PP_MEAN_ZX.f90:299-872) and PP_MEAN_T_Xperiodic_IO
// (src/processing/PP_MEAN_T.f90:436-520, the xz fields): 360 values per row
// (141 flow, 219 with the energy equation; the order is stated at
// io_terms).  Every value is the xz-mean of a product of at most four of 28
// per-cell quantities (1, U, p, G, the velocity gradient D, T, rho, h, mu, k
// and the gradients of h and T); a table of factor indices drives one
// generic kernel.  Grid (ny, ST_NBK k-chunks, 8 groups of 45 values).
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

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

// ------------------------------------------------------------- IO section
constexpr int SI_NV = 360, SI_NB = 28, SI_GS = 45, SI_NG = SI_NV / SI_GS;
// per-cell quantity slots
enum { B_1 = 0, B_U = 1, B_P = 4, B_G = 5, B_D = 8, B_T = 17, B_R = 18, B_H = 19, B_M = 20, B_K = 21, B_DH = 22,
       B_DT = 25 };

// Factor table of the 360 IO statistics, in output order; each entry packs
// four slot indices (unused factors are slot B_1 = 1.0, placed last, so the
// product of the used ones is evaluated left to right as written).
std::vector<uint32_t> io_terms() {
  std::vector<uint32_t> t;
  auto add = [&](int a, int b = B_1, int c = B_1, int d = B_1) {
    t.push_back((uint32_t)a | ((uint32_t)b << 8) | ((uint32_t)c << 16) | ((uint32_t)d << 24));
  };
  auto D = [](int m, int n) { return B_D + 3 * m + n; };
  for (int m = 0; m < 3; ++m) add(B_U + m);                     // U1: u, v, w
  add(B_P);                                                      //     p
  for (int m = 0; m < 3; ++m) add(B_G + m);                     // G1
  for (int m = 0; m < 3; ++m) add(B_U + m, B_P);                // UP
  for (int m = 0; m < 3; ++m)
    for (int n = m; n < 3; ++n) add(B_U + m, B_U + n);          // U2
  for (int m = 0; m < 3; ++m)
    for (int n = m; n < 3; ++n) add(B_U + m, B_G + n);          // UG
  for (int m = 0; m < 3; ++m)
    for (int n = m; n < 3; ++n)
      for (int h = n; h < 3; ++h) add(B_U + m, B_U + n, B_U + h);  // U3
  for (int m = 0; m < 3; ++m)
    for (int n = m; n < 3; ++n)
      for (int h = n; h < 3; ++h) add(B_U + m, B_G + n, B_U + h);  // UGU
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n) add(D(m, n));                    // DVDL1
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n) add(D(m, n), B_P);               // DVDLP
  for (int l1 = 0; l1 < 9; ++l1)
    for (int l2 = 0; l2 < 9; ++l2) add(B_D + l1, B_D + l2);      // DVDL2
  add(B_T); add(B_R); add(B_H); add(B_M);                        // T1 D1 H1 M1
  add(B_T, B_T); add(B_R, B_R); add(B_H, B_H);                   // T2 D2 H2
  add(B_H, B_R); add(B_H, B_P);                                  // DH PH
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n) add(D(m, n), B_M);               // DVDL1M
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n) add(D(m, n), B_M, B_H);          // DVDL1MH
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n)
      for (int h = 0; h < 3; ++h) add(D(m, n), B_M, B_U + h);    // DVDL1MU
  for (int l1 = 0; l1 < 9; ++l1)
    for (int l2 = 0; l2 < 9; ++l2) add(B_D + l1, B_D + l2, B_M); // DVDL2M
  for (int m = 0; m < 3; ++m) add(B_H, B_U + m);                 // UH
  for (int m = 0; m < 3; ++m) add(B_H, B_G + m);                 // GH
  for (int m = 0; m < 3; ++m)
    for (int n = m; n < 3; ++n) add(B_R, B_H, B_U + m, B_U + n); // U2DH
  for (int m = 0; m < 3; ++m) add(B_DH + m);                     // DhDL1
  for (int m = 0; m < 3; ++m) add(B_DH + m, B_P);                // DhDLP
  for (int m = 0; m < 3; ++m) add(B_DT + m, B_K);                // DTDLK
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n) add(B_DT + m, B_K, B_U + n);     // DTDLKU
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n)
      for (int h = 0; h < 3; ++h) add(B_DT + m, B_K, D(n, h));   // DTDLKDVDL
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n)
      for (int h = 0; h < 3; ++h) add(B_DH + m, B_M, D(n, h));   // DHDLMDVDL
  return t;
}

struct IOStatFields {
  const double *g[3];  // current mass flux G
};

// The 28 per-cell quantities of cell (i, j, k) (0-based i, k; row j), column
// `col` of b (stride ST_TPB): the cell-centred U and G (x 0.5), p, D(m, n)
// with the reference's central differences, and the thermal values and
// gradients (zero without the energy equation).
__device__ __forceinline__ void io_cell_base(const TGDev &d, const IODev &io, const IOStatFields &f, int i, int j,
                                             int k, double (*b)[ST_TPB], int col) {
  const int nx = d.nx, nz = d.nz;
  const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
  const int kp = k + 1 == nz ? 0 : k + 1, km = k == 0 ? nz - 1 : k - 1;
  const int64_t sy = d.sy, sz = d.sz;
  const int64_t c = i + sy * j + sz * k;
  const int64_t oxp = ip - i, oxm = im - i, ozp = sz * (kp - k), ozm = sz * (km - k);
  const double *u = d.u, *v = d.v, *w = d.w;
  const double U0 = (u[c] + u[c + oxp]) * 0.5;
  const double Ujp0 = (u[c + sy] + u[c + sy + oxp]) * 0.5, Ujm0 = (u[c - sy] + u[c - sy + oxp]) * 0.5;
  const double Ukp0 = (u[c + ozp] + u[c + ozp + oxp]) * 0.5, Ukm0 = (u[c + ozm] + u[c + ozm + oxp]) * 0.5;
  const double U2 = (w[c] + w[c + ozp]) * 0.5;
  const double Uip2 = (w[c + oxp] + w[c + oxp + ozp]) * 0.5, Uim2 = (w[c + oxm] + w[c + oxm + ozp]) * 0.5;
  const double Ujp2 = (w[c + sy] + w[c + sy + ozp]) * 0.5, Ujm2 = (w[c - sy] + w[c - sy + ozp]) * 0.5;
  const double U1 = (v[c] + v[c + sy]) * 0.5;
  const double Uip1 = (v[c + oxp] + v[c + oxp + sy]) * 0.5, Uim1 = (v[c + oxm] + v[c + oxm + sy]) * 0.5;
  const double Ukp1 = (v[c + ozp] + v[c + ozp + sy]) * 0.5, Ukm1 = (v[c + ozm] + v[c + ozm + sy]) * 0.5;
  const double dycp = d.dyci[j + 1], dycj = d.dyci[j];
  b[B_1][col] = 1.0;
  b[B_U][col] = U0;
  b[B_U + 1][col] = U1;
  b[B_U + 2][col] = U2;
  b[B_P][col] = d.p[c];
  b[B_G][col] = (f.g[0][c] + f.g[0][c + oxp]) * 0.5;
  b[B_G + 1][col] = (f.g[1][c] + f.g[1][c + sy]) * 0.5;
  b[B_G + 2][col] = (f.g[2][c] + f.g[2][c + ozp]) * 0.5;
  b[B_D + 0][col] = (u[c + oxp] - u[c]) * d.dxi;
  b[B_D + 1][col] = ((Ujp0 - U0) * dycp + (U0 - Ujm0) * dycj) * 0.5;
  b[B_D + 2][col] = (Ukp0 - Ukm0) * d.dzi * 0.5;
  b[B_D + 3][col] = (Uip1 - Uim1) * d.dxi * 0.5;
  b[B_D + 4][col] = (v[c + sy] - v[c]) * d.dyfi[j];
  b[B_D + 5][col] = (Ukp1 - Ukm1) * d.dzi * 0.5;
  b[B_D + 6][col] = (Uip2 - Uim2) * d.dxi * 0.5;
  b[B_D + 7][col] = ((Ujp2 - U2) * dycp + (U2 - Ujm2) * dycj) * 0.5;
  b[B_D + 8][col] = (w[c + ozp] - w[c]) * d.dzi;
  if (!io.thermal) {
#pragma unroll
    for (int q = B_T; q < SI_NB; ++q) b[q][col] = 0.0;
    return;
  }
  const double *h = io.h, *T = io.T;
  b[B_T][col] = T[c];
  b[B_R][col] = io.D[c];
  b[B_H][col] = h[c];
  b[B_M][col] = io.mu[c];
  b[B_K][col] = io.kap[c];
  b[B_DH][col] = (h[c + oxp] - h[c + oxm]) * d.dxi * 0.5;
  b[B_DH + 1][col] = ((h[c + sy] - h[c]) * dycp + (h[c] - h[c - sy]) * dycj) * 0.5;
  b[B_DH + 2][col] = (h[c + ozp] - h[c + ozm]) * d.dzi * 0.5;
  b[B_DT][col] = (T[c + oxp] - T[c + oxm]) * d.dxi * 0.5;
  b[B_DT + 1][col] = ((T[c + sy] - T[c]) * dycp + (T[c] - T[c - sy]) * dycj) * 0.5;
  b[B_DT + 2][col] = (T[c + ozp] - T[c + ozm]) * d.dzi * 0.5;
}

__global__ void __launch_bounds__(ST_TPB) k_io_stats_part(TGDev d, IODev io, IOStatFields f, const uint32_t *terms,
                                                          double *part) {
  __shared__ double b[SI_NB][ST_TPB];
  __shared__ uint32_t st[SI_GS];
  __shared__ double red[ST_TPB / 32][SI_GS];
  const int j = blockIdx.x + 1, a0 = blockIdx.z * SI_GS;
  if (threadIdx.x < SI_GS) st[threadIdx.x] = terms[a0 + threadIdx.x];
  __syncthreads();
  const int nx = d.nx, nz = d.nz;
  const int k0 = (int)((int64_t)nz * blockIdx.y / ST_NBK), k1 = (int)((int64_t)nz * (blockIdx.y + 1) / ST_NBK);
  double acc[SI_GS];
#pragma unroll
  for (int a = 0; a < SI_GS; ++a) acc[a] = 0.0;
  const int ncell = nx * (k1 - k0), col = threadIdx.x;
  for (int t = threadIdx.x; t < ncell; t += ST_TPB) {
    io_cell_base(d, io, f, t % nx, j, k0 + t / nx, b, col);  // this thread's own column
#pragma unroll
    for (int a = 0; a < SI_GS; ++a) {
      const uint32_t q = st[a];
      acc[a] += ((b[q & 255u][col] * b[(q >> 8) & 255u][col]) * b[(q >> 16) & 255u][col]) * b[q >> 24][col];
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < SI_GS; ++a) {
    double v = acc[a];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][a] = v;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < SI_GS; a += ST_TPB) {
    double s = 0.0;
    for (int q = 0; q < ST_TPB / 32; ++q) s += red[q][a];
    part[((size_t)(j - 1) * ST_NBK + blockIdx.y) * SI_NV + a0 + a] = s;
  }
}

// Sum the k-chunk partials of each row in order, scale by 1/(nx nz) and
// (accumulate != 0) fold into the time average.
__global__ void k_io_stats_final(int nx, int nz, const double *part, double *xz, double *xzt, double coe2, double coe3,
                                 int accumulate) {
  const int j = blockIdx.x + 1;
  const double vl = 1.0 / ((double)nx * (double)nz);
  for (int a = threadIdx.x; a < SI_NV; a += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < ST_NBK; ++b) s += part[((size_t)(j - 1) * ST_NBK + b) * SI_NV + a];
    const double val = s * vl;
    xz[(size_t)(j - 1) * SI_NV + a] = val;
    if (accumulate) {
      double *t = xzt + (size_t)(j - 1) * SI_NV + a;
      *t = coe3 * *t + coe2 * val;
    }
  }
}

// Values per row and partials per row of the context's statistics.
int nv_of(const chapsim_ctx *c) { return c->domain == CHAPSIM_IIO ? SI_NV : ST_NV; }
size_t npart_of(const chapsim_ctx *c) {
  return (size_t)c->d.ny * ST_NBK * (c->domain == CHAPSIM_IIO ? SI_NV : ST_G0 + ST_G1);
}

}  // namespace

int stats_run(chapsim_ctx *c, int accumulate) {
  if (c->domain == CHAPSIM_IIO) {
    TGDev &d = c->d;
    const size_t np = npart_of(c), nv = (size_t)d.ny * SI_NV;
    if (!c->stats_buf) {
      void *p = nullptr;
      // partials, xz, xzt, then the factor table
      CK(cudaMalloc(&p, (np + 2 * nv) * sizeof(double) + SI_NV * sizeof(uint32_t)));
      c->allocs.push_back(p);
      c->stats_buf = (double *)p;
      CK(cudaMemsetAsync(p, 0, (np + 2 * nv) * sizeof(double), c->stream));
      const std::vector<uint32_t> t = io_terms();
      CK(cudaMemcpyAsync(c->stats_buf + np + 2 * nv, t.data(), SI_NV * sizeof(uint32_t), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaStreamSynchronize(c->stream));  // the host table goes out of scope
    }
    double *part = c->stats_buf, *xz = part + np, *xzt = xz + nv;
    const uint32_t *terms = reinterpret_cast<const uint32_t *>(xzt + nv);
    IOStatFields f;
    for (int m = 0; m < 3; ++m) f.g[m] = c->io.g[c->io_cur][m];
    k_io_stats_part<<<dim3(d.ny, ST_NBK, SI_NG), ST_TPB, 0, c->stream>>>(d, c->io, f, terms, part);
    LAUNCHED();
    double coe2 = 0.0, coe3 = 0.0;
    if (accumulate) {  // T_Asymptotic_Average
      c->nstatis += 1;
      coe2 = 1.0 / (double)c->nstatis;
      coe3 = (double)(c->nstatis - 1) / (double)c->nstatis;
    }
    k_io_stats_final<<<d.ny, 128, 0, c->stream>>>(d.nx, d.nz, part, xz, xzt, coe2, coe3, accumulate);
    LAUNCHED();
    return CHAPSIM_OK;
  }
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
  const size_t nv = (size_t)c->d.ny * nv_of(c);
  double *xzt = c->stats_buf + npart_of(c) + nv;
  CK(cudaMemsetAsync(xzt, 0, nv * sizeof(double), c->stream));
  return CHAPSIM_OK;
}

int stats_get(chapsim_ctx *c, int which, double *host, int64_t n) {
  TGDev &d = c->d;
  if (!c->stats_buf || n != (int64_t)d.ny * nv_of(c)) return CHAPSIM_ERR_ARG;
  const double *xz = c->stats_buf + npart_of(c);
  const double *src = which == 0 ? xz : xz + (size_t)d.ny * nv_of(c);
  CK(cudaMemcpyAsync(host, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAPSIM_OK;
}

}  // namespace chapsim
