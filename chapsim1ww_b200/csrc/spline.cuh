// Table cubic splines shared by the property engine and the IO energy
// path: the Forsythe-Malcolm-Moler spline of CUBIC_SPLINE
// (src/Flow_State.f90:1693-1787) built on the host, evaluated on the device
// with the binary search of NIST_SLEVAL_* (src/Flow_State.f90:1015-1070)
// started from a uniform bucket table.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace chapsim_spl {

// Spline of y over x: coefficients b, c, d (Forsythe, Malcolm & Moler),
// also packed per interval as one 32-byte record {y, b, c, d}.
struct Spline {
  const double *x, *y, *b, *c, *d;
  const double4 *ybcd;
  const int *blo;    // bucket -> first candidate interval
  const int2 *brng;  // bucket -> search range {blo[b], min(n - 1, blo[b + 1] + 3)}
  double x0, binv;
  double xlo, xhi;   // x[0] and x[n - 1], held by value for the range test
  int n, nb;
};

// Interval i with x[i] <= u < x[i+1] (u strictly inside the table); the
// bucket gives a short range for the same binary search as the reference.
__device__ __forceinline__ int spline_find(const Spline &s, double u) {
  int b = (int)((u - s.x0) * s.binv);
  b = b < 0 ? 0 : (b >= s.nb ? s.nb - 1 : b);
  const int2 rg = __ldg(s.brng + b);
  int i = rg.x, j = rg.y;
  while (j > i + 1) {
    const int k = (i + j) >> 1;
    if (u < __ldg(s.x + k)) j = k; else i = k;
  }
  return i;
}
__device__ __forceinline__ double spline_at(const Spline &s, int i, double u) {
  const double2 r0 = __ldg(reinterpret_cast<const double2 *>(s.ybcd + i));
  const double2 r1 = __ldg(reinterpret_cast<const double2 *>(s.ybcd + i) + 1);
  const double4 r = make_double4(r0.x, r0.y, r1.x, r1.y);
  const double dx = u - __ldg(s.x + i);
  return r.x + dx * (r.y + dx * (r.z + dx * r.w));
}
__device__ __forceinline__ double spline_eval(const Spline &s, double u) { return spline_at(s, spline_find(s, u), u); }

__device__ __forceinline__ bool inside(const Spline &s, double u) { return u > s.xlo && u < s.xhi; }


// Host restatement of CUBIC_SPLINE (Forsythe-Malcolm-Moler, 1977).
inline void fmm_spline(int n, const double *x, const double *y, double *b, double *c, double *d) {
  const int nm1 = n - 1;
  d[0] = x[1] - x[0];
  c[1] = (y[1] - y[0]) / d[0];
  for (int i = 1; i < nm1; ++i) {
    d[i] = x[i + 1] - x[i];
    b[i] = 2.0 * (d[i - 1] + d[i]);
    c[i + 1] = (y[i + 1] - y[i]) / d[i];
    c[i] = c[i + 1] - c[i];
  }
  b[0] = -d[0];
  b[n - 1] = -d[n - 2];
  c[0] = 0.0;
  c[n - 1] = 0.0;
  if (n > 3) {
    c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0]);
    c[n - 1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4]);
    c[0] = c[0] * d[0] * d[0] / (x[3] - x[0]);
    c[n - 1] = -c[n - 1] * d[n - 2] * d[n - 2] / (x[n - 1] - x[n - 4]);
  }
  for (int i = 1; i < n; ++i) {
    const double t = d[i - 1] / b[i - 1];
    b[i] = b[i] - t * d[i - 1];
    c[i] = c[i] - t * c[i - 1];
  }
  c[n - 1] = c[n - 1] / b[n - 1];
  for (int l = 1; l <= nm1; ++l) {
    const int i = n - 1 - l;
    c[i] = (c[i] - d[i] * c[i + 1]) / b[i];
  }
  b[n - 1] = (y[n - 1] - y[nm1 - 1]) / d[nm1 - 1] + d[nm1 - 1] * (c[nm1 - 1] + 2.0 * c[n - 1]);
  for (int i = 0; i < nm1; ++i) {
    b[i] = (y[i + 1] - y[i]) / d[i] - d[i] * (c[i + 1] + 2.0 * c[i]);
    d[i] = (c[i + 1] - c[i]) / d[i];
    c[i] = 3.0 * c[i];
  }
  c[n - 1] = 3.0 * c[n - 1];
  d[n - 1] = d[n - 2];
}

// Bucket table over nb uniform buckets of [x_1, x_n]: blo[b] = I(start_b) - 1
// with I(v) = max{i : x_i <= v}, so every u in bucket b satisfies
// x[blo[b]] <= u < x[min(n-1, blo[b+1] + 3)] (one interval of slack each way
// for rounding); the binary search between them finds the reference's i.
inline void bucket_table(int n, const double *x, int nb, double &x0, double &binv, std::vector<int> &blo) {
  x0 = x[0];
  binv = nb / (x[n - 1] - x[0]);
  blo.assign(nb + 1, 0);
  int i = 0;
  for (int b = 0; b <= nb; ++b) {
    const double start = x0 + b / binv;
    while (i + 1 < n && x[i + 1] <= start) ++i;
    int l = i - 1;
    l = l < 0 ? 0 : l;
    blo[b] = l < n - 2 ? l : n - 2;
  }
}


// Search range of each bucket for spline_find: {blo[b], min(n - 1, blo[b + 1] + 3)}.
inline std::vector<int2> bucket_ranges(const std::vector<int> &blo, int n, int nb) {
  std::vector<int2> rng(nb);
  for (int q = 0; q < nb; ++q) rng[q] = make_int2(blo[q], blo[q + 1] + 3 < n - 1 ? blo[q + 1] + 3 : n - 1);
  return rng;
}

// Build the spline of y over x on the host and upload x, y, b, c, d, the
// packed records and the bucket table; every allocation is appended to
// allocs (freed by the owner).
inline cudaError_t upload_spline(std::vector<void *> &allocs, const std::vector<double> &x,
                                 const std::vector<double> &y, Spline &s) {
  const int n = (int)x.size();
  std::vector<double> b(n), c(n), d(n);
  fmm_spline(n, x.data(), y.data(), b.data(), c.data(), d.data());
  std::vector<int> blo;
  const int nb = 4 * n;
  bucket_table(n, x.data(), nb, s.x0, s.binv, blo);
  void *p = nullptr;
  cudaError_t e;
  double *arr[5];
  const std::vector<double> *src[5] = {&x, &y, &b, &c, &d};
  for (int q = 0; q < 5; ++q) {
    if ((e = cudaMalloc(&p, n * sizeof(double))) != cudaSuccess) return e;
    allocs.push_back(p);
    arr[q] = (double *)p;
    if ((e = cudaMemcpy(p, src[q]->data(), n * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  }
  if ((e = cudaMalloc(&p, (nb + 1) * sizeof(int))) != cudaSuccess) return e;
  allocs.push_back(p);
  if ((e = cudaMemcpy(p, blo.data(), (nb + 1) * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  s.blo = (const int *)p;
  const std::vector<int2> rng = bucket_ranges(blo, n, nb);
  if ((e = cudaMalloc(&p, nb * sizeof(int2))) != cudaSuccess) return e;
  allocs.push_back(p);
  if ((e = cudaMemcpy(p, rng.data(), nb * sizeof(int2), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  s.brng = (const int2 *)p;
  s.xlo = x[0];
  s.xhi = x[n - 1];
  std::vector<double> rec((size_t)4 * n);
  for (int i = 0; i < n; ++i) { rec[4 * i] = y[i]; rec[4 * i + 1] = b[i]; rec[4 * i + 2] = c[i]; rec[4 * i + 3] = d[i]; }
  if ((e = cudaMalloc(&p, rec.size() * sizeof(double))) != cudaSuccess) return e;
  allocs.push_back(p);
  if ((e = cudaMemcpy(p, rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  s.ybcd = (const double4 *)p;
  s.x = arr[0]; s.y = arr[1]; s.b = arr[2]; s.c = arr[3]; s.d = arr[4];
  s.n = n;
  s.nb = nb;
  return cudaSuccess;
}

}  // namespace chapsim_spl
