// Block-cooperative mixed-radix Stockham FFT on shared memory.
//
// Replaces the vendored Temperton FFT99 (real, x) and CFFT99 (complex, z)
// transforms the reference's Poisson solver calls
// (src/possion3d_FFT99.f90:299,310,460,474).  Transform definitions follow the
// FFT99/CFFT99 documentation (libs/fft99/FFT99.f90:87-94,
// libs/fft99/CFFT99.f90:171-196): forward = sum x e^{-2 pi i jk/N}, inverse =
// sum C e^{+2 pi i jk/N}; normalisation is applied by the callers.  Unlike
// FFT99 (radices 2, 3, 5 only) every length whose prime factors are in
// {2, 3, 5, 7, 11} is supported; powers of two run as radix-8 stages (a
// 512-point line takes three stages).
//
// Algorithm: self-sorting Stockham decimation in time.  Stage s with radix R
// and Ns = product of earlier radices maps, for j in [0, N/R):
//   v_r = in[j + r N/R] * w^{r (j mod Ns) N/(Ns R)},  V = DFT_R(v),
//   out[(j / Ns) Ns R + (j mod Ns) + s' Ns] = V_s'.
#pragma once
#include <cuda_runtime.h>

namespace chapsim {

template <typename C> struct CTraits;
template <> struct CTraits<double2> { typedef double R; };
template <> struct CTraits<float2> { typedef float R; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// multiply by -i (sign < 0) or +i (sign > 0)
template <typename C> __device__ __forceinline__ C cmuli(C a, int sign) {
  C r;
  if (sign < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
  return r;
}

// twiddle w^m = exp(sign 2 pi i m / N) from the forward table exp(-2 pi i m/N)
template <typename C> __device__ __forceinline__ C twiddle(const C *tw, int m, int sign) {
  C t = tw[m];
  if (sign > 0) t.y = -t.y;
  return t;
}

// in-place 4-point DFT with root sign * i
template <typename C> __device__ __forceinline__ void dft4(C &x0, C &x1, C &x2, C &x3, int sign) {
  C s02 = cadd(x0, x2), d02 = csub(x0, x2);
  C s13 = cadd(x1, x3), d13 = cmuli(csub(x1, x3), sign);
  x0 = cadd(s02, s13);
  x2 = csub(s02, s13);
  x1 = cadd(d02, d13);
  x3 = csub(d02, d13);
}

template <typename C, int R>
__device__ __forceinline__ void dft_small(C *v, const C *tw, int n, int sign) {
  if (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    dft4(v[0], v[1], v[2], v[3], sign);
  } else if (R == 8) {
    // X_{2m} = DFT4(x_r + x_{r+4})_m, X_{2m+1} = DFT4((x_r - x_{r+4}) w^r)_m
    // with w = exp(sign 2 pi i / 8)
    typedef typename CTraits<C>::R T;
    const T h = (T)0.70710678118654752440;  // 1 / sqrt(2)
    C a0 = cadd(v[0], v[4]), a1 = cadd(v[1], v[5]), a2 = cadd(v[2], v[6]), a3 = cadd(v[3], v[7]);
    C b0 = csub(v[0], v[4]), b1 = csub(v[1], v[5]), b2 = csub(v[2], v[6]), b3 = csub(v[3], v[7]);
    // b1 w = b1 (1 + sign i) / sqrt 2, b2 w^2 = sign i b2, b3 w^3 = b3 (-1 + sign i) / sqrt 2
    C t1, t3;
    if (sign < 0) {
      t1.x = (b1.x + b1.y) * h; t1.y = (b1.y - b1.x) * h;
      t3.x = (b3.y - b3.x) * h; t3.y = -(b3.x + b3.y) * h;
    } else {
      t1.x = (b1.x - b1.y) * h; t1.y = (b1.x + b1.y) * h;
      t3.x = -(b3.x + b3.y) * h; t3.y = (b3.x - b3.y) * h;
    }
    b2 = cmuli(b2, sign);
    dft4(a0, a1, a2, a3, sign);
    dft4(b0, t1, b2, t3, sign);
    v[0] = a0; v[2] = a1; v[4] = a2; v[6] = a3;
    v[1] = b0; v[3] = t1; v[5] = b2; v[7] = t3;
  } else {
    // generic odd radix: V_s = sum_r v_r w_R^{rs}, w_R = table[(n/R) * m]
    C out[R];
    const int step = n / R;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      C acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) {
        int m = (r * s) % R;
        acc = cadd(acc, cmul(v[r], twiddle(tw, m * step, sign)));
      }
      out[s] = acc;
    }
#pragma unroll
    for (int s = 0; s < R; ++s) v[s] = out[s];
  }
}

// v_r *= w^{r m} for r = 1 .. R-1 (r m < n).  Radix 8 and 4 load w^m, w^2m
// (and w^4m) from the table and form the other powers as products of two
// table entries, each within a few ulps of the table value: 3 table loads
// instead of 7.  In the last stage of a line-major transform the lanes of a
// warp take consecutive m, so the load of w^{rm} touches r times as many
// cache lines as that of w^m; the products replace the widest of them.
template <typename C, int R>
__device__ __forceinline__ void twiddle_inputs(C *v, const C *__restrict__ tw, int m, int sign) {
  if (R == 8) {
    const C w1 = twiddle(tw, m, sign), w2 = twiddle(tw, 2 * m, sign), w4 = twiddle(tw, 4 * m, sign);
    const C w3 = cmul(w1, w2);
    v[1] = cmul(v[1], w1);
    v[2] = cmul(v[2], w2);
    v[3] = cmul(v[3], w3);
    v[4] = cmul(v[4], w4);
    v[5] = cmul(v[5], cmul(w1, w4));
    v[6] = cmul(v[6], cmul(w2, w4));
    v[7] = cmul(v[7], cmul(w3, w4));
  } else if (R == 4) {
    const C w1 = twiddle(tw, m, sign), w2 = twiddle(tw, 2 * m, sign);
    v[1] = cmul(v[1], w1);
    v[2] = cmul(v[2], w2);
    v[3] = cmul(v[3], cmul(w1, w2));
  } else {
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twiddle(tw, r * m, sign));
  }
}

// Shared-memory position of element p of a line-major buffer: the low three
// bits are XORed with bits 3..5, a permutation inside every aligned group of
// eight elements.  The Stockham stages write at stride R (radix 8: eight
// 16-byte elements, one bank group); swizzled, those writes and the
// contiguous reads both spread over all banks.  Buffers indexed this way are
// sized to a multiple of eight elements.
__device__ __forceinline__ int swz(int p) { return p ^ ((p >> 3) & 7); }

template <typename C, int R>
__device__ __forceinline__ void stockham_stage(const C *__restrict__ in, C *__restrict__ out, int nlines,
                                               int n, int lstride, int Ns, const C *__restrict__ tw,
                                               int sign) {
  const int nb = n / R;
  const int total = nlines * nb;
  const int tstep = n / (Ns * R);
  // power-of-two divisors (every stage of a power-of-two plan) by shifts
  const bool nb2 = (nb & (nb - 1)) == 0, ns2 = (Ns & (Ns - 1)) == 0;
  const int lnb = __ffs(nb) - 1, lns = __ffs(Ns) - 1;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = nb2 ? t >> lnb : t / nb;
    const int j = t - line * nb;
    const int jq = ns2 ? j >> lns : j / Ns;
    const int k = j - jq * Ns;
    const int l0 = line * lstride;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[swz(l0 + j + r * nb)];
    if (k != 0) twiddle_inputs<C, R>(v, tw, k * tstep, sign);
    dft_small<C, R>(v, tw, n, sign);
    const int base = l0 + jq * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[swz(base + r * Ns)] = v[r];
  }
}

// Transform nlines lines (each n complex values, stride lstride) held in
// shared memory buffer a at swizzled positions (swz of line * lstride + e);
// b is scratch of the same size.  Returns the buffer holding the result.
// Must be called by every thread of the block.
// BIG selects whether radices 7 and 11 are compiled in (they raise register
// use of every stage, so plans with only 2, 3, 4, 5, 8 use the small variant).
template <typename C, bool BIG>
__device__ C *fft_lines(C *a, C *b, int nlines, int n, int lstride, const int *rad, int nrad,
                        const C *__restrict__ tw, int sign) {
  int Ns = 1;
  for (int s = 0; s < nrad; ++s) {
    const int R = rad[s];
    switch (R) {
      case 2: stockham_stage<C, 2>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      case 3: stockham_stage<C, 3>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      case 4: stockham_stage<C, 4>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      case 8: stockham_stage<C, 8>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      case 5: stockham_stage<C, 5>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      case 7: if (BIG) stockham_stage<C, 7>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      case 11: if (BIG) stockham_stage<C, 11>(a, b, nlines, n, lstride, Ns, tw, sign); break;
      default: break;  // plans only contain the radices above
    }
    __syncthreads();
    C *t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

// The same stages on lines stored interleaved: element e of line l at
// buf[e * nl + l] (consecutive lines adjacent; nl a power of two).
// Consecutive threads take consecutive lines, so each stage's reads and
// writes are contiguous rows.  Per element the arithmetic is that of
// stockham_stage, except that every twiddle comes from the table: the lanes
// of a warp share the twiddle index, so each table load is one broadcast.
template <typename C, int R>
__device__ __forceinline__ void stockham_stage_il(const C *__restrict__ in, C *__restrict__ out, int nl, int n,
                                                  int Ns, const C *__restrict__ tw, int sign) {
  const int nb = n / R;
  const int total = nl * nb;
  const int tstep = n / (Ns * R);
  // nl is a power of two; Ns is one in every power-of-two stage
  const int lnl = __ffs(nl) - 1;
  const bool ns2 = (Ns & (Ns - 1)) == 0;
  const int lns = __ffs(Ns) - 1;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int j = t >> lnl;
    const int line = t & (nl - 1);
    const int jq = ns2 ? j >> lns : j / Ns;
    const int k = j - jq * Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[(j + r * nb) * nl + line];
    if (k != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twiddle(tw, r * k * tstep, sign));
    }
    dft_small<C, R>(v, tw, n, sign);
    const int base = jq * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[(base + r * Ns) * nl + line] = v[r];
  }
}

template <typename C, bool BIG>
__device__ C *fft_lines_il(C *a, C *b, int nl, int n, const int *rad, int nrad, const C *__restrict__ tw, int sign) {
  int Ns = 1;
  for (int s = 0; s < nrad; ++s) {
    const int R = rad[s];
    switch (R) {
      case 2: stockham_stage_il<C, 2>(a, b, nl, n, Ns, tw, sign); break;
      case 3: stockham_stage_il<C, 3>(a, b, nl, n, Ns, tw, sign); break;
      case 4: stockham_stage_il<C, 4>(a, b, nl, n, Ns, tw, sign); break;
      case 8: stockham_stage_il<C, 8>(a, b, nl, n, Ns, tw, sign); break;
      case 5: stockham_stage_il<C, 5>(a, b, nl, n, Ns, tw, sign); break;
      case 7: if (BIG) stockham_stage_il<C, 7>(a, b, nl, n, Ns, tw, sign); break;
      case 11: if (BIG) stockham_stage_il<C, 11>(a, b, nl, n, Ns, tw, sign); break;
      default: break;
    }
    __syncthreads();
    C *t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

}  // namespace chapsim
