// Thermal property engine: table cubic splines (THERM_PROP_UPDATE) and the
// learned property model (MLP h -> T, rho, mu, k, cp) with its GPU training
// and an error-gated BF16 tensor-core inference path.
//
// Reference (CHAPSim1WW, paths relative to the project root):
//   THERM_PROP_UPDATE   src/THERM_PROP_UPDATE.f90:129-205
//   NIST_SLEVAL_HT/T*   src/Flow_State.f90:1015-1070, 1420-1581
//   CUBIC_SPLINE        src/Flow_State.f90:1693-1787 (the published
//                       Forsythe-Malcolm-Moler spline, restated below)
//   table columns       src/Flow_State.f90:394-433
// The MLP has no counterpart in the reference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/chapsim.h"
#include "spline.cuh"

namespace {

using namespace chapsim_spl;

constexpr int NH = 64, NO = 5;
constexpr int NP = NH + NH + NH * NH + NH + NO * NH + NO;  // 4613
constexpr int O_W1 = 0, O_B1 = NH, O_W2 = 2 * NH, O_B2 = 2 * NH + NH * NH, O_W3 = O_B2 + NH, O_B3 = O_W3 + NO * NH;

struct PropsDev {
  Spline ht, hcp, td, tm, tk;
  int *err_count;
  // MLP inference
  const __nv_bfloat16 *w2b;  // [64][64] (row = output unit)
  const __nv_bfloat16 *w3b;  // [8][64], rows 5..7 zero
  const float *params;       // W1, b1, b2, b3 read in FP32
  double hmid, hhalf, mean[NO], stdv[NO];
  const int *gate;  // per h-bin: 1 = MLP, 0 = table
  double g0, ginv;
  int nbins;
};

// THERM_PROP_UPDATE for one cell; returns false when h or T is outside the
// table (cell left unchanged).
__device__ __forceinline__ bool table_props(const PropsDev &P, double h, double &T, double &rho, double &mu,
                                            double &k, double &cp) {
  if (!inside(P.ht, h)) return false;
  const int ih = spline_find(P.ht, h);  // cp shares the H grid and interval
  T = spline_at(P.ht, ih, h);
  if (!inside(P.tm, T)) return false;
  const int it = spline_find(P.tm, T);  // mu, k, rho share the T grid and interval
  mu = spline_at(P.tm, it, T);
  k = spline_at(P.tk, it, T);
  rho = spline_at(P.td, it, T);
  if (fabs(T - 1.0) < 1.0e-10) { mu = 1.0; k = 1.0; rho = 1.0; }
  cp = spline_at(P.hcp, ih, h);
  return true;
}

__global__ void k_props_table(PropsDev P, const double *__restrict__ h, double *T, double *rho, double *mu,
                              double *kk, double *cp, int64_t n) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const double hv = h[c];
    if (fabs(hv) < 1.0e-10) continue;  // reference leaves these cells unchanged
    double t, r, m, kv, cpv;
    if (!table_props(P, hv, t, r, m, kv, cpv)) {
      atomicAdd(P.err_count, 1);
      continue;
    }
    T[c] = t; rho[c] = r; mu[c] = m; kk[c] = kv;
    if (cp) cp[c] = cpv;
  }
}

// ---------------------------------------------------------------- MLP
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Hardware tanh approximation (tanh.approx.f32, sm_75+), used only in the
// BF16 inference path, whose weights and activations carry ~4e-3 relative
// precision anyway; training uses tanhf.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// MLP forward for the 16 cells of a warp (m16n8k16 BF16 tensor-core MMA, FP32
// accumulation): layer 1 in FP32 straight into A fragments, layer 2 as
// 4 x 8 MMAs against W2 in shared memory, its accumulators re-packed as the A
// fragments of layer 3 (N = 5 padded to 8).  out[] = standardised outputs of
// columns 2q, 2q+1 for rows g and g+8 (q = lane & 3, g = lane >> 2).
__device__ void mlp_warp(const PropsDev &P, const __nv_bfloat16 *sW2, const __nv_bfloat16 *sW3, float xg, float xg8,
                         float (&out)[4]) {
  const int lane = threadIdx.x & 31, q = lane & 3;
  const float *W1 = P.params + O_W1, *b1 = P.params + O_B1, *b2 = P.params + O_B2;
  uint32_t a[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const int c0 = kt * 16 + q * 2, c1 = c0 + 8;
    a[kt][0] = pack_bf16(tanh_fast(W1[c0] * xg + b1[c0]), tanh_fast(W1[c0 + 1] * xg + b1[c0 + 1]));
    a[kt][1] = pack_bf16(tanh_fast(W1[c0] * xg8 + b1[c0]), tanh_fast(W1[c0 + 1] * xg8 + b1[c0 + 1]));
    a[kt][2] = pack_bf16(tanh_fast(W1[c1] * xg + b1[c1]), tanh_fast(W1[c1 + 1] * xg + b1[c1 + 1]));
    a[kt][3] = pack_bf16(tanh_fast(W1[c1] * xg8 + b1[c1]), tanh_fast(W1[c1 + 1] * xg8 + b1[c1 + 1]));
  }
  const int g = lane >> 2;
  float acc[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    const __nv_bfloat16 *wrow = sW2 + (nt * 8 + g) * NH;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(wrow + kt * 16 + q * 2);
      const uint32_t b1v = *reinterpret_cast<const uint32_t *>(wrow + kt * 16 + q * 2 + 8);
      mma_bf16(acc[nt], a[kt], b0, b1v);
    }
  }
  uint32_t a3[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const int n0 = 2 * kt, n1 = 2 * kt + 1;
    const int c0 = n0 * 8 + q * 2, c1 = n1 * 8 + q * 2;
    a3[kt][0] = pack_bf16(tanh_fast(acc[n0][0] + b2[c0]), tanh_fast(acc[n0][1] + b2[c0 + 1]));
    a3[kt][1] = pack_bf16(tanh_fast(acc[n0][2] + b2[c0]), tanh_fast(acc[n0][3] + b2[c0 + 1]));
    a3[kt][2] = pack_bf16(tanh_fast(acc[n1][0] + b2[c1]), tanh_fast(acc[n1][1] + b2[c1 + 1]));
    a3[kt][3] = pack_bf16(tanh_fast(acc[n1][2] + b2[c1]), tanh_fast(acc[n1][3] + b2[c1 + 1]));
  }
  out[0] = out[1] = out[2] = out[3] = 0.f;
  const __nv_bfloat16 *w3row = sW3 + g * NH;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const uint32_t b0 = *reinterpret_cast<const uint32_t *>(w3row + kt * 16 + q * 2);
    const uint32_t b1v = *reinterpret_cast<const uint32_t *>(w3row + kt * 16 + q * 2 + 8);
    mma_bf16(out, a3[kt], b0, b1v);
  }
}

constexpr int MI_WARPS = 4, MI_CELLS = MI_WARPS * 16;

// Property update with the learned model: MLP for all cells of the block,
// then per cell the reference's skip / range rules and the error gate (bins
// not cleared for the MLP take the table splines).
__global__ void __launch_bounds__(MI_WARPS * 32) k_props_mlp(PropsDev P, const double *__restrict__ h, double *T,
                                                              double *rho, double *mu, double *kk, double *cp,
                                                              int64_t n) {
  __shared__ __align__(16) __nv_bfloat16 sW2[NH * NH];
  __shared__ __align__(16) __nv_bfloat16 sW3[8 * NH];
  __shared__ float sout[MI_CELLS][8];
  for (int t = threadIdx.x; t < NH * NH; t += blockDim.x) sW2[t] = P.w2b[t];
  for (int t = threadIdx.x; t < 8 * NH; t += blockDim.x) sW3[t] = P.w3b[t];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const float *b3 = P.params + O_B3;
  for (int64_t base = (int64_t)blockIdx.x * MI_CELLS; base < n; base += (int64_t)gridDim.x * MI_CELLS) {
    const int64_t r0 = base + warp * 16 + g, r1 = r0 + 8;
    const float x0 = r0 < n ? (float)((h[r0] - P.hmid) / P.hhalf) : 0.f;
    const float x1 = r1 < n ? (float)((h[r1] - P.hmid) / P.hhalf) : 0.f;
    float o[4];
    mlp_warp(P, sW2, sW3, x0, x1, o);
    const int c = q * 2;
    sout[warp * 16 + g][c] = o[0];
    sout[warp * 16 + g][c + 1] = o[1];
    sout[warp * 16 + g + 8][c] = o[2];
    sout[warp * 16 + g + 8][c + 1] = o[3];
    __syncthreads();
    if (threadIdx.x < MI_CELLS) {
      const int64_t cidx = base + threadIdx.x;
      if (cidx < n) {
        const double hv = h[cidx];
        if (fabs(hv) >= 1.0e-10) {
          if (!(hv > P.ht.x[0] && hv < P.ht.x[P.ht.n - 1])) {
            atomicAdd(P.err_count, 1);
          } else {
            int bin = (int)((hv - P.g0) * P.ginv);
            bin = bin < 0 ? 0 : (bin >= P.nbins ? P.nbins - 1 : bin);
            double t, r, m, kv, cpv;
            bool ok = true;
            if (P.gate[bin]) {
              const float *so = sout[threadIdx.x];
              t = (so[0] + b3[0]) * P.stdv[0] + P.mean[0];
              r = (so[1] + b3[1]) * P.stdv[1] + P.mean[1];
              m = (so[2] + b3[2]) * P.stdv[2] + P.mean[2];
              kv = (so[3] + b3[3]) * P.stdv[3] + P.mean[3];
              cpv = (so[4] + b3[4]) * P.stdv[4] + P.mean[4];
            } else {
              ok = table_props(P, hv, t, r, m, kv, cpv);
              if (!ok) atomicAdd(P.err_count, 1);
            }
            if (ok) {
              T[cidx] = t; rho[cidx] = r; mu[cidx] = m; kk[cidx] = kv;
              if (cp) cp[cidx] = cpv;
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ MLP training
// One block = 128 samples (one per thread): FP32 forward, backward and the
// per-block gradient sums in a fixed order (deterministic), written as one
// partial gradient vector per block.
constexpr int TR_S = 128;
__global__ void __launch_bounds__(TR_S) k_mlp_grad(const float *__restrict__ params, const float *__restrict__ xs,
                                                   const float *__restrict__ ts, int nsamp, float *partials,
                                                   double *loss_part) {
  extern __shared__ __align__(16) float sm[];
  float *A1 = sm;                       // [TR_S][NH+1]
  float *A2 = A1 + TR_S * (NH + 1);     // [TR_S][NH+1]
  float *E = A2 + TR_S * (NH + 1);      // [TR_S][NO]
  float *W = E + TR_S * NO;             // parameters [NP]
  float *X = W + NP;                    // [TR_S]
  __shared__ double lred[TR_S];
  const int t = threadIdx.x;
  for (int p = t; p < NP; p += TR_S) W[p] = params[p];
  const int s = blockIdx.x * TR_S + t;
  const bool valid = s < nsamp;
  const float x = valid ? xs[s] : 0.f;
  X[t] = valid ? x : 0.f;
  __syncthreads();
  const float *W1 = W + O_W1, *b1 = W + O_B1, *W2 = W + O_W2, *b2 = W + O_B2, *W3 = W + O_W3, *b3 = W + O_B3;
  float a1[NH];
#pragma unroll
  for (int k = 0; k < NH; ++k) {
    a1[k] = tanhf(W1[k] * x + b1[k]);
    A1[t * (NH + 1) + k] = a1[k];
  }
  float y[NO];
#pragma unroll
  for (int o = 0; o < NO; ++o) y[o] = b3[o];
  for (int j = 0; j < NH; ++j) {
    float z = b2[j];
#pragma unroll
    for (int k = 0; k < NH; ++k) z += W2[j * NH + k] * a1[k];
    const float a2 = tanhf(z);
    A2[t * (NH + 1) + j] = a2;
#pragma unroll
    for (int o = 0; o < NO; ++o) y[o] += W3[o * NH + j] * a2;
  }
  const float scale = 2.0f / ((float)nsamp * NO);
  double l = 0.0;
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    const float e = valid ? (y[o] - ts[(size_t)s * NO + o]) : 0.f;
    l += (double)e * e;
    E[t * NO + o] = e * scale;
  }
  lred[t] = l;
  __syncthreads();
  float *G = partials + (size_t)blockIdx.x * NP;
  // gW3, gb3
  for (int idx = t; idx < NO * NH + NO; idx += TR_S) {
    float acc = 0.f;
    if (idx < NO * NH) {
      const int o = idx / NH, j = idx - o * NH;
      for (int r = 0; r < TR_S; ++r) acc += E[r * NO + o] * A2[r * (NH + 1) + j];
      G[O_W3 + idx] = acc;
    } else {
      const int o = idx - NO * NH;
      for (int r = 0; r < TR_S; ++r) acc += E[r * NO + o];
      G[O_B3 + o] = acc;
    }
  }
  __syncthreads();
  // d2 = (E W3) * (1 - a2^2), over this thread's row (in place of A2)
  for (int j = 0; j < NH; ++j) {
    float z = 0.f;
#pragma unroll
    for (int o = 0; o < NO; ++o) z += E[t * NO + o] * W3[o * NH + j];
    const float a2 = A2[t * (NH + 1) + j];
    A2[t * (NH + 1) + j] = z * (1.f - a2 * a2);
  }
  __syncthreads();
  // gW2 = D2^T A1, gb2
  for (int idx = t; idx < NH * NH + NH; idx += TR_S) {
    float acc = 0.f;
    if (idx < NH * NH) {
      const int j = idx / NH, k = idx - j * NH;
      for (int r = 0; r < TR_S; ++r) acc += A2[r * (NH + 1) + j] * A1[r * (NH + 1) + k];
      G[O_W2 + idx] = acc;
    } else {
      const int j = idx - NH * NH;
      for (int r = 0; r < TR_S; ++r) acc += A2[r * (NH + 1) + j];
      G[O_B2 + j] = acc;
    }
  }
  __syncthreads();
  // d1 = (D2 W2) * (1 - a1^2), own row (in place of A1)
  for (int k = 0; k < NH; ++k) {
    float z = 0.f;
    for (int j = 0; j < NH; ++j) z += A2[t * (NH + 1) + j] * W2[j * NH + k];
    const float a1v = A1[t * (NH + 1) + k];
    A1[t * (NH + 1) + k] = z * (1.f - a1v * a1v);
  }
  __syncthreads();
  // gW1, gb1
  if (t < NH) {
    float aw = 0.f, ab = 0.f;
    for (int r = 0; r < TR_S; ++r) {
      const float dd = A1[r * (NH + 1) + t];
      aw += dd * X[r];
      ab += dd;
    }
    G[O_W1 + t] = aw;
    G[O_B1 + t] = ab;
  }
  if (t == 0) {
    double acc = 0.0;
    for (int r = 0; r < TR_S; ++r) acc += lred[r];
    loss_part[blockIdx.x] = acc;
  }
}

// Sum the block partials in block order; optionally take one Adam step.
__global__ void k_mlp_reduce(const float *partials, int nblk, float *grad, float *params, float *m, float *v,
                             float lr, float b1, float b2, float bc1, float bc2, int adam) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NP) return;
  float g = 0.f;
  for (int b = 0; b < nblk; ++b) g += partials[(size_t)b * NP + p];
  grad[p] = g;
  if (adam) {
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    params[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + 1e-8f);
  }
}

__global__ void k_loss_sum(const double *lp, int nblk, int nsamp, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += lp[b];
    *out = s / ((double)nsamp * NO);
  }
}

__global__ void k_to_bf16(const float *params, __nv_bfloat16 *w2b, __nv_bfloat16 *w3b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < NH * NH) w2b[t] = __float2bfloat16_rn(params[O_W2 + t]);
  if (t < 8 * NH) w3b[t] = t < NO * NH ? __float2bfloat16_rn(params[O_W3 + t]) : __float2bfloat16_rn(0.f);
}

uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace

struct chapsim_props {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int n = 0;
  std::vector<double> H, T, D, M, K, CP;
  std::vector<void *> allocs;
  PropsDev P{};
  float *params = nullptr, *adam_m = nullptr, *adam_v = nullptr, *grad = nullptr;
  __nv_bfloat16 *w2b = nullptr, *w3b = nullptr;
  int *gate = nullptr;
  bool has_mlp = false;
};

#define PCK(call)                                                       \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) {                                            \
      pe->err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
      return CHAPSIM_ERR_CUDA;                                          \
    }                                                                   \
  } while (0)

static int palloc(chapsim_props *pe, void **p, size_t bytes) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    pe->err = "cudaMalloc failed";
    return CHAPSIM_ERR_NOMEM;
  }
  pe->allocs.push_back(*p);
  return CHAPSIM_OK;
}

static int upload_spline(chapsim_props *pe, const std::vector<double> &x, const std::vector<double> &y, Spline &s) {
  const int n = (int)x.size();
  std::vector<double> b(n), c(n), d(n);
  fmm_spline(n, x.data(), y.data(), b.data(), c.data(), d.data());
  std::vector<int> blo;
  const int nb = 4 * n;
  bucket_table(n, x.data(), nb, s.x0, s.binv, blo);
  void *p = nullptr;
  int rc;
  double *arr[5];
  const std::vector<double> *src[5] = {&x, &y, &b, &c, &d};
  for (int q = 0; q < 5; ++q) {
    if ((rc = palloc(pe, &p, n * sizeof(double)))) return rc;
    arr[q] = (double *)p;
    PCK(cudaMemcpy(p, src[q]->data(), n * sizeof(double), cudaMemcpyHostToDevice));
  }
  if ((rc = palloc(pe, &p, (nb + 1) * sizeof(int)))) return rc;
  PCK(cudaMemcpy(p, blo.data(), (nb + 1) * sizeof(int), cudaMemcpyHostToDevice));
  s.blo = (const int *)p;
  const std::vector<int2> rng = bucket_ranges(blo, n, nb);
  if ((rc = palloc(pe, &p, nb * sizeof(int2)))) return rc;
  PCK(cudaMemcpy(p, rng.data(), nb * sizeof(int2), cudaMemcpyHostToDevice));
  s.brng = (const int2 *)p;
  s.xlo = x[0];
  s.xhi = x[n - 1];
  std::vector<double> rec((size_t)4 * n);
  for (int i = 0; i < n; ++i) { rec[4 * i] = y[i]; rec[4 * i + 1] = b[i]; rec[4 * i + 2] = c[i]; rec[4 * i + 3] = d[i]; }
  if ((rc = palloc(pe, &p, rec.size() * sizeof(double)))) return rc;
  PCK(cudaMemcpy(p, rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice));
  s.ybcd = (const double4 *)p;
  s.x = arr[0]; s.y = arr[1]; s.b = arr[2]; s.c = arr[3]; s.d = arr[4];
  s.n = n;
  s.nb = nb;
  return CHAPSIM_OK;
}

static void props_free(chapsim_props *pe) {
  for (void *p : pe->allocs) cudaFree(p);
  pe->allocs.clear();
  if (pe->stream) cudaStreamDestroy(pe->stream);
  pe->stream = nullptr;
}

extern "C" {

int chapsim_props_create(const double *H, const double *T, const double *D, const double *M, const double *K,
                         const double *CP, int n, int device, chapsim_props **out) {
  if (!H || !T || !D || !M || !K || !CP || !out || n < 4) return CHAPSIM_ERR_ARG;
  *out = nullptr;
  for (int i = 1; i < n; ++i)
    if (!(H[i] > H[i - 1]) || !(T[i] > T[i - 1])) return CHAPSIM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CHAPSIM_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return CHAPSIM_ERR_ARG;
  chapsim_props *pe = new chapsim_props();
  pe->device = device;
  pe->n = n;
  pe->H.assign(H, H + n); pe->T.assign(T, T + n); pe->D.assign(D, D + n);
  pe->M.assign(M, M + n); pe->K.assign(K, K + n); pe->CP.assign(CP, CP + n);
  int rc = CHAPSIM_OK;
  void *p = nullptr;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&pe->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete pe;
    return CHAPSIM_ERR_CUDA;
  }
  if ((rc = upload_spline(pe, pe->H, pe->T, pe->P.ht)) || (rc = upload_spline(pe, pe->H, pe->CP, pe->P.hcp)) ||
      (rc = upload_spline(pe, pe->T, pe->D, pe->P.td)) || (rc = upload_spline(pe, pe->T, pe->M, pe->P.tm)) ||
      (rc = upload_spline(pe, pe->T, pe->K, pe->P.tk)))
    goto fail;
  if ((rc = palloc(pe, &p, 16 * sizeof(int)))) goto fail;
  pe->P.err_count = (int *)p;
  if ((rc = palloc(pe, &p, NP * sizeof(float)))) goto fail;
  pe->params = (float *)p;
  if ((rc = palloc(pe, &p, NP * sizeof(float)))) goto fail;
  pe->adam_m = (float *)p;
  if ((rc = palloc(pe, &p, NP * sizeof(float)))) goto fail;
  pe->adam_v = (float *)p;
  if ((rc = palloc(pe, &p, NP * sizeof(float)))) goto fail;
  pe->grad = (float *)p;
  if ((rc = palloc(pe, &p, NH * NH * sizeof(__nv_bfloat16)))) goto fail;
  pe->w2b = (__nv_bfloat16 *)p;
  if ((rc = palloc(pe, &p, 8 * NH * sizeof(__nv_bfloat16)))) goto fail;
  pe->w3b = (__nv_bfloat16 *)p;
  pe->P.params = pe->params;
  pe->P.w2b = pe->w2b;
  pe->P.w3b = pe->w3b;
  pe->P.hmid = 0.5 * (H[0] + H[n - 1]);
  pe->P.hhalf = 0.5 * (H[n - 1] - H[0]);
  for (int o = 0; o < NO; ++o) { pe->P.mean[o] = 0.0; pe->P.stdv[o] = 1.0; }
  pe->P.nbins = 1;
  pe->P.g0 = H[0];
  pe->P.ginv = 1.0 / (H[n - 1] - H[0]);
  if ((rc = palloc(pe, &p, 4096 * sizeof(int)))) goto fail;
  pe->gate = (int *)p;
  pe->P.gate = pe->gate;
  if (cudaMemset(pe->gate, 0, 4096 * sizeof(int)) != cudaSuccess) { rc = CHAPSIM_ERR_CUDA; goto fail; }
  if (cudaMemset(pe->params, 0, NP * sizeof(float)) != cudaSuccess) { rc = CHAPSIM_ERR_CUDA; goto fail; }
  *out = pe;
  return CHAPSIM_OK;
fail:
  props_free(pe);
  delete pe;
  return rc;
}

int chapsim_props_destroy(chapsim_props *pe) {
  if (!pe) return CHAPSIM_ERR_ARG;
  cudaSetDevice(pe->device);
  if (pe->stream) cudaStreamSynchronize(pe->stream);
  props_free(pe);
  delete pe;
  return CHAPSIM_OK;
}

const char *chapsim_props_last_error(const chapsim_props *pe) { return pe ? pe->err.c_str() : "null engine"; }

static int launch_update(chapsim_props *pe, int mode, const double *h, double *T, double *rho, double *mu, double *k,
                         double *cp, int64_t n) {
  if (n <= 0) return CHAPSIM_OK;
  if (mode == CHAPSIM_PROPS_TABLE) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_props_table<<<blocks, 256, 0, pe->stream>>>(pe->P, h, T, rho, mu, k, cp, n);
  } else {
    const int blocks = (int)std::min<int64_t>((n + MI_CELLS - 1) / MI_CELLS, 148 * 32);
    k_props_mlp<<<blocks, MI_WARPS * 32, 0, pe->stream>>>(pe->P, h, T, rho, mu, k, cp, n);
  }
  PCK(cudaGetLastError());
  return CHAPSIM_OK;
}

int chapsim_props_update(chapsim_props *pe, int mode, const double *h, double *T, double *rho, double *mu, double *k,
                         double *cp, int64_t n, int64_t *n_out_of_range) {
  if (!pe || !h || !T || !rho || !mu || !k || n < 0) return CHAPSIM_ERR_ARG;
  if (mode != CHAPSIM_PROPS_TABLE && mode != CHAPSIM_PROPS_MLP) return CHAPSIM_ERR_ARG;
  if (mode == CHAPSIM_PROPS_MLP && !pe->has_mlp) {
    pe->err = "no trained model: call chapsim_props_train or chapsim_props_set_params first";
    return CHAPSIM_ERR_STATE;
  }
  PCK(cudaSetDevice(pe->device));
  PCK(cudaMemsetAsync(pe->P.err_count, 0, sizeof(int), pe->stream));
  int rc = launch_update(pe, mode, h, T, rho, mu, k, cp, n);
  if (rc) return rc;
  int bad = 0;
  PCK(cudaMemcpyAsync(&bad, pe->P.err_count, sizeof(int), cudaMemcpyDeviceToHost, pe->stream));
  PCK(cudaStreamSynchronize(pe->stream));
  if (n_out_of_range) *n_out_of_range = bad;
  if (bad) {
    pe->err = std::to_string(bad) + " cells outside the property table (left unchanged)";
    return CHAPSIM_ERR_RANGE;
  }
  return CHAPSIM_OK;
}

static int refresh_bf16(chapsim_props *pe) {
  k_to_bf16<<<(NH * NH + 255) / 256, 256, 0, pe->stream>>>(pe->params, pe->w2b, pe->w3b);
  PCK(cudaGetLastError());
  return CHAPSIM_OK;
}

static size_t grad_smem() { return (size_t)(2 * TR_S * (NH + 1) + TR_S * NO + NP + TR_S) * sizeof(float); }

// partial gradients of a device batch; reduce (and optionally Adam)
static int grad_pass(chapsim_props *pe, const float *dx, const float *dt, int nsamp, float *partials, double *lpart,
                     double *dloss, int adam, float lr, int step) {
  const int nblk = (nsamp + TR_S - 1) / TR_S;
  k_mlp_grad<<<nblk, TR_S, grad_smem(), pe->stream>>>(pe->params, dx, dt, nsamp, partials, lpart);
  PCK(cudaGetLastError());
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_mlp_reduce<<<(NP + 255) / 256, 256, 0, pe->stream>>>(partials, nblk, pe->grad, pe->params, pe->adam_m,
                                                          pe->adam_v, lr, b1, b2, bc1, bc2, adam);
  PCK(cudaGetLastError());
  k_loss_sum<<<1, 32, 0, pe->stream>>>(lpart, nblk, nsamp, dloss);
  PCK(cudaGetLastError());
  return CHAPSIM_OK;
}

int chapsim_props_train(chapsim_props *pe, int nsamples, uint64_t seed, int steps, double lr, double *final_loss) {
  if (!pe || nsamples < TR_S || steps < 1 || !(lr > 0)) return CHAPSIM_ERR_ARG;
  PCK(cudaSetDevice(pe->device));
  PCK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem()));
  const int n = pe->n;
  // samples: h uniform strictly inside the table, targets from the splines
  std::vector<double> hs(nsamples);
  const double lo = pe->H[0], hi = pe->H[n - 1];
  for (int s = 0; s < nsamples; ++s) {
    const double u = (double)(splitmix64(splitmix64(seed) ^ (uint64_t)s) >> 11) * (1.0 / 9007199254740992.0);
    double hv = lo + (hi - lo) * (0.0005 + 0.999 * u);
    if (fabs(hv) < 1e-10) hv = 1e-9;
    hs[s] = hv;
  }
  std::vector<void *> tmp;
  auto talloc = [&](size_t bytes) -> void * {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    tmp.push_back(p);
    return p;
  };
  auto cleanup = [&]() { for (void *p : tmp) cudaFree(p); tmp.clear(); };
  double *dh = (double *)talloc(nsamples * sizeof(double));
  double *dout = (double *)talloc((size_t)nsamples * NO * sizeof(double));
  if (!dh || !dout) { cleanup(); pe->err = "cudaMalloc failed"; return CHAPSIM_ERR_NOMEM; }
  cudaMemcpy(dh, hs.data(), nsamples * sizeof(double), cudaMemcpyHostToDevice);
  PCK(cudaMemsetAsync(pe->P.err_count, 0, sizeof(int), pe->stream));
  int rc = launch_update(pe, CHAPSIM_PROPS_TABLE, dh, dout, dout + nsamples, dout + 2 * nsamples,
                         dout + 3 * nsamples, dout + 4 * nsamples, nsamples);
  if (rc) { cleanup(); return rc; }
  std::vector<double> tgt((size_t)nsamples * NO);
  cudaMemcpyAsync(tgt.data(), dout, tgt.size() * sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
  cudaStreamSynchronize(pe->stream);
  // standardisation
  for (int o = 0; o < NO; ++o) {
    double m = 0.0, v = 0.0;
    for (int s = 0; s < nsamples; ++s) m += tgt[(size_t)o * nsamples + s];
    m /= nsamples;
    for (int s = 0; s < nsamples; ++s) { const double e = tgt[(size_t)o * nsamples + s] - m; v += e * e; }
    pe->P.mean[o] = m;
    pe->P.stdv[o] = sqrt(v / nsamples) + 1e-12;
  }
  std::vector<float> xf(nsamples), tf((size_t)nsamples * NO);
  for (int s = 0; s < nsamples; ++s) {
    xf[s] = (float)((hs[s] - pe->P.hmid) / pe->P.hhalf);
    for (int o = 0; o < NO; ++o)
      tf[(size_t)s * NO + o] = (float)((tgt[(size_t)o * nsamples + s] - pe->P.mean[o]) / pe->P.stdv[o]);
  }
  // Xavier-style seeded init
  std::vector<float> w(NP, 0.f);
  auto rnd = [&](uint64_t i) {
    return (float)(-1.0 + 2.0 * ((double)(splitmix64(splitmix64(seed ^ 0xA5A5u) ^ i) >> 11) *
                                 (1.0 / 9007199254740992.0)));
  };
  for (int k = 0; k < NH; ++k) { w[O_W1 + k] = 2.0f * rnd(k); w[O_B1 + k] = 1.5f * rnd(100 + k); }
  for (int t = 0; t < NH * NH; ++t) w[O_W2 + t] = rnd(1000 + t) * sqrtf(6.0f / (2 * NH));
  for (int t = 0; t < NO * NH; ++t) w[O_W3 + t] = rnd(9000 + t) * sqrtf(6.0f / (NH + NO));
  float *dx = (float *)talloc(nsamples * sizeof(float));
  float *dtg = (float *)talloc((size_t)nsamples * NO * sizeof(float));
  const int nblk = (nsamples + TR_S - 1) / TR_S;
  float *partials = (float *)talloc((size_t)nblk * NP * sizeof(float));
  double *lpart = (double *)talloc(nblk * sizeof(double));
  double *dloss = (double *)talloc(sizeof(double));
  if (!dx || !dtg || !partials || !lpart || !dloss) { cleanup(); pe->err = "cudaMalloc failed"; return CHAPSIM_ERR_NOMEM; }
  cudaMemcpy(dx, xf.data(), xf.size() * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dtg, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(pe->params, w.data(), NP * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(pe->adam_m, 0, NP * sizeof(float));
  cudaMemset(pe->adam_v, 0, NP * sizeof(float));
  for (int st = 1; st <= steps; ++st) {
    const double frac = (double)(st - 1) / (double)steps;
    const float lrs = (float)(lr * (0.01 + 0.99 * 0.5 * (1.0 + cos(M_PI * frac))));
    rc = grad_pass(pe, dx, dtg, nsamples, partials, lpart, dloss, 1, lrs, st);
    if (rc) { cleanup(); return rc; }
  }
  // loss at the final parameters
  rc = grad_pass(pe, dx, dtg, nsamples, partials, lpart, dloss, 0, 0.f, 1);
  if (rc) { cleanup(); return rc; }
  double l = 0.0;
  cudaMemcpyAsync(&l, dloss, sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
  PCK(cudaStreamSynchronize(pe->stream));
  cleanup();
  if (final_loss) *final_loss = l;
  rc = refresh_bf16(pe);
  if (rc) return rc;
  pe->has_mlp = true;
  return CHAPSIM_OK;
}

int chapsim_props_gate(chapsim_props *pe, double tol, int nbins, int *n_mlp_bins, double *max_rel_err) {
  if (!pe || nbins < 1 || nbins > 4096 || !(tol >= 0)) return CHAPSIM_ERR_ARG;
  if (!pe->has_mlp) { pe->err = "no trained model"; return CHAPSIM_ERR_STATE; }
  PCK(cudaSetDevice(pe->device));
  const int n = pe->n;
  const int per = 8;  // evaluation points per table interval
  const int64_t m = (int64_t)(n - 1) * per;
  std::vector<double> hs(m);
  for (int64_t s = 0; s < m; ++s) {
    const int i = (int)(s / per), q = (int)(s % per);
    hs[s] = pe->H[i] + (pe->H[i + 1] - pe->H[i]) * (q + 0.5) / per;
    if (fabs(hs[s]) < 1e-10) hs[s] = 1e-9;
  }
  double *dh = nullptr, *da = nullptr, *db = nullptr;
  if (cudaMalloc(&dh, m * sizeof(double)) != cudaSuccess || cudaMalloc(&da, m * NO * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&db, m * NO * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dh); cudaFree(da); cudaFree(db);
    return CHAPSIM_ERR_NOMEM;
  }
  cudaMemcpy(dh, hs.data(), m * sizeof(double), cudaMemcpyHostToDevice);
  // all bins on the MLP for the measurement
  std::vector<int> ones(4096, 1);
  cudaMemcpy(pe->gate, ones.data(), 4096 * sizeof(int), cudaMemcpyHostToDevice);
  pe->P.nbins = 1;
  cudaMemsetAsync(pe->P.err_count, 0, sizeof(int), pe->stream);
  int rc = launch_update(pe, CHAPSIM_PROPS_TABLE, dh, da, da + m, da + 2 * m, da + 3 * m, da + 4 * m, m);
  if (!rc) rc = launch_update(pe, CHAPSIM_PROPS_MLP, dh, db, db + m, db + 2 * m, db + 3 * m, db + 4 * m, m);
  std::vector<double> A(m * NO), B(m * NO);
  cudaMemcpyAsync(A.data(), da, A.size() * sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
  cudaMemcpyAsync(B.data(), db, B.size() * sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
  cudaStreamSynchronize(pe->stream);
  cudaFree(dh); cudaFree(da); cudaFree(db);
  if (rc) return rc;
  double scale[NO];
  for (int o = 0; o < NO; ++o) {
    scale[o] = 0.0;
    for (int64_t s = 0; s < m; ++s) scale[o] = fmax(scale[o], fabs(A[o * m + s]));
    scale[o] = scale[o] > 0 ? scale[o] : 1.0;
  }
  std::vector<double> binerr(nbins, 0.0);
  const double g0 = pe->H[0], ginv = nbins / (pe->H[n - 1] - pe->H[0]);
  double worst = 0.0;
  for (int64_t s = 0; s < m; ++s) {
    int b = (int)((hs[s] - g0) * ginv);
    b = b < 0 ? 0 : (b >= nbins ? nbins - 1 : b);
    for (int o = 0; o < NO; ++o) {
      const double e = fabs(B[o * m + s] - A[o * m + s]) / scale[o];
      binerr[b] = fmax(binerr[b], e);
      worst = fmax(worst, e);
    }
  }
  std::vector<int> flags(4096, 0);
  int cnt = 0;
  for (int b = 0; b < nbins; ++b) {
    flags[b] = binerr[b] <= tol ? 1 : 0;
    cnt += flags[b];
  }
  cudaMemcpy(pe->gate, flags.data(), 4096 * sizeof(int), cudaMemcpyHostToDevice);
  pe->P.nbins = nbins;
  pe->P.g0 = g0;
  pe->P.ginv = ginv;
  if (n_mlp_bins) *n_mlp_bins = cnt;
  if (max_rel_err) *max_rel_err = worst;
  return CHAPSIM_OK;
}

int chapsim_props_get_params(const chapsim_props *pe, float *params, int nparams, double *norm, int nnorm) {
  if (!pe || !params || nparams != NP || !norm || nnorm != 2 + 2 * NO) return CHAPSIM_ERR_ARG;
  cudaSetDevice(pe->device);
  if (cudaMemcpy(params, pe->params, NP * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return CHAPSIM_ERR_CUDA;
  norm[0] = pe->P.hmid;
  norm[1] = pe->P.hhalf;
  for (int o = 0; o < NO; ++o) { norm[2 + o] = pe->P.mean[o]; norm[2 + NO + o] = pe->P.stdv[o]; }
  return CHAPSIM_OK;
}

int chapsim_props_set_params(chapsim_props *pe, const float *params, int nparams, const double *norm, int nnorm) {
  if (!pe || !params || nparams != NP || !norm || nnorm != 2 + 2 * NO) return CHAPSIM_ERR_ARG;
  PCK(cudaSetDevice(pe->device));
  PCK(cudaMemcpy(pe->params, params, NP * sizeof(float), cudaMemcpyHostToDevice));
  pe->P.hmid = norm[0];
  pe->P.hhalf = norm[1];
  for (int o = 0; o < NO; ++o) { pe->P.mean[o] = norm[2 + o]; pe->P.stdv[o] = norm[2 + NO + o]; }
  int rc = refresh_bf16(pe);
  if (rc) return rc;
  PCK(cudaStreamSynchronize(pe->stream));
  pe->has_mlp = true;
  return CHAPSIM_OK;
}

int chapsim_props_loss_grad(chapsim_props *pe, const float *x, const float *t, int n, double *loss, float *grad,
                            int nparams) {
  if (!pe || !x || !t || n < 1 || !loss || !grad || nparams != NP) return CHAPSIM_ERR_ARG;
  PCK(cudaSetDevice(pe->device));
  PCK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem()));
  const int nblk = (n + TR_S - 1) / TR_S;
  float *dx = nullptr, *dt = nullptr, *partials = nullptr;
  double *lpart = nullptr, *dloss = nullptr;
  if (cudaMalloc(&dx, n * sizeof(float)) != cudaSuccess || cudaMalloc(&dt, (size_t)n * NO * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&partials, (size_t)nblk * NP * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&lpart, nblk * sizeof(double)) != cudaSuccess || cudaMalloc(&dloss, sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dx); cudaFree(dt); cudaFree(partials); cudaFree(lpart); cudaFree(dloss);
    return CHAPSIM_ERR_NOMEM;
  }
  cudaMemcpy(dx, x, n * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dt, t, (size_t)n * NO * sizeof(float), cudaMemcpyHostToDevice);
  int rc = grad_pass(pe, dx, dt, n, partials, lpart, dloss, 0, 0.f, 1);
  if (!rc) {
    cudaMemcpyAsync(grad, pe->grad, NP * sizeof(float), cudaMemcpyDeviceToHost, pe->stream);
    cudaMemcpyAsync(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
    if (cudaStreamSynchronize(pe->stream) != cudaSuccess) rc = CHAPSIM_ERR_CUDA;
  }
  cudaFree(dx); cudaFree(dt); cudaFree(partials); cudaFree(lpart); cudaFree(dloss);
  return rc;
}

}  // extern "C"
