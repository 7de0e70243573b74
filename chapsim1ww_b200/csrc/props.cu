// Thermal property engine: table cubic splines (THERM_PROP_UPDATE) and the
// learned property model (polynomial base + MLP h -> T, rho, mu, k, cp) with
// its GPU training and an error-gated inference path on the sm_100a tensor
// cores (tcgen05, mlp_tc.cuh).
//
// Reference (CHAPSim1WW, paths relative to the project root):
//   THERM_PROP_UPDATE   src/THERM_PROP_UPDATE.f90:129-205
//   NIST_SLEVAL_HT/T*   src/Flow_State.f90:1015-1070, 1420-1581
//   CUBIC_SPLINE        src/Flow_State.f90:1693-1787 (the published
//                       Forsythe-Malcolm-Moler spline, restated below)
//   table columns       src/Flow_State.f90:394-433
// The learned model has no counterpart in the reference.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/chapsim.h"
#include "chapsim_internal.cuh"
#include "mlp_tc.cuh"
#include "spline.cuh"

namespace {

using namespace chapsim_spl;
using chapsim_mlp::NH;
using chapsim_mlp::NO;
using chapsim_mlp::NP;
using chapsim_mlp::O_B1;
using chapsim_mlp::O_B2;
using chapsim_mlp::O_B3;
using chapsim_mlp::O_W1;
using chapsim_mlp::O_W2;
using chapsim_mlp::O_W3;
constexpr int NNORM = 2 + 2 * NO + NO * chapsim_mlp::NBASE;  // hmid, hhalf, mean, std, base

struct PropsDev {
  Spline ht, hcp, td, tm, tk;
  int *err_count;
  int *dev_err;  // bounded-wait error word of the inference kernel
  chapsim_mlp::MlpDev M;
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
// Property update with the learned model: the model on every 128-cell tile
// (tensor cores), then per cell the reference's skip / range rules and the
// error gate, per output: an output whose bit is clear in the cell's h-bin
// comes from the table splines.
__global__ void __launch_bounds__(chapsim_mlp::TILE, 4)
    k_props_mlp_tc(PropsDev P, const double *__restrict__ h, double *T, double *rho, double *mu, double *kk,
                   double *cp, int64_t n) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  chapsim_mlp::Smem &s = chapsim_mlp::smem_of(smem_raw);
  const chapsim_mlp::MlpDev &M = P.M;
  chapsim_mlp::cta_setup(s, M);
  uint32_t phase = 0;
  const int64_t ntiles = (n + chapsim_mlp::TILE - 1) / chapsim_mlp::TILE;
  const unsigned need = cp ? 0x1Fu : chapsim_mlp::kStepMask;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t c = tile * chapsim_mlp::TILE + threadIdx.x;
    const double hv = c < n ? h[c] : 0.0;
    const double x = (hv - M.hmid) / M.hhalf;
    float y[NO];
    if (!chapsim_mlp::tile_eval(s, (float)x, y, phase, P.dev_err)) break;
    if (c >= n || fabs(hv) < 1.0e-10) continue;  // reference leaves these cells unchanged
    if (!(hv > P.ht.x[0] && hv < P.ht.x[P.ht.n - 1])) {
      atomicAdd(P.err_count, 1);
      continue;
    }
    double o[NO];
#pragma unroll
    for (int q = 0; q < NO; ++q) o[q] = chapsim_mlp::assemble(M, q, x, y[q]);
    const unsigned mask = chapsim_mlp::gate_mask(M, hv);
    if ((mask & need) != need) {
      double t, r, m, kv, cpv;
      if (!table_props(P, hv, t, r, m, kv, cpv)) {
        atomicAdd(P.err_count, 1);
        continue;
      }
      const double tab[NO] = {t, r, m, kv, cpv};
#pragma unroll
      for (int q = 0; q < NO; ++q)
        if (!(mask & (1u << q))) o[q] = tab[q];
    }
    T[c] = o[0]; rho[c] = o[1]; mu[c] = o[2]; kk[c] = o[3];
    if (cp) cp[c] = o[4];
  }
  chapsim_mlp::cta_teardown(s);
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
  uint16_t *wt = nullptr;  // BF16 hi / lo weight tiles of layers 2 and 3 (tensor-core operands)
  uint8_t *gate = nullptr;  // per h-bin output masks
  bool has_mlp = false;
  // per-output results of the last gate call
  int out_bins[NO] = {0, 0, 0, 0, 0};
  double out_err[NO] = {0, 0, 0, 0, 0};
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
  if ((rc = palloc(pe, &p, (2 * NH * NH + 2 * chapsim_mlp::NOP * NH) * sizeof(uint16_t)))) goto fail;
  pe->wt = (uint16_t *)p;
  if ((rc = palloc(pe, &p, chapsim_mlp::kMaxGateBins))) goto fail;
  pe->gate = (uint8_t *)p;
  if ((rc = palloc(pe, &p, sizeof(int)))) goto fail;
  pe->P.dev_err = (int *)p;
  if (cudaMemset(pe->P.dev_err, 0, sizeof(int)) != cudaSuccess) { rc = CHAPSIM_ERR_CUDA; goto fail; }
  {
    chapsim_mlp::MlpDev &M = pe->P.M;
    M.par = pe->params;
    M.wt = pe->wt;
    M.gate = pe->gate;
    M.hmid = 0.5 * (H[0] + H[n - 1]);
    M.hhalf = 0.5 * (H[n - 1] - H[0]);
    for (int o = 0; o < NO; ++o) {
      M.mean[o] = 0.0;
      M.stdv[o] = 1.0;
      for (int q = 0; q < chapsim_mlp::NBASE; ++q) M.base[o][q] = 0.0;
    }
    M.nbins = 1;
    M.g0 = H[0];
    M.ginv = 1.0 / (H[n - 1] - H[0]);
  }
  if (cudaMemset(pe->gate, 0, chapsim_mlp::kMaxGateBins) != cudaSuccess) { rc = CHAPSIM_ERR_CUDA; goto fail; }
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

static size_t mlp_smem() { return chapsim_mlp::kSmemBytes; }

static int launch_update(chapsim_props *pe, int mode, const double *h, double *T, double *rho, double *mu, double *k,
                         double *cp, int64_t n) {
  if (n <= 0) return CHAPSIM_OK;
  if (mode == CHAPSIM_PROPS_TABLE) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_props_table<<<blocks, 256, 0, pe->stream>>>(pe->P, h, T, rho, mu, k, cp, n);
  } else {
    PCK(cudaFuncSetAttribute(k_props_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_smem()));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, pe->device);
    const int64_t tiles = (n + chapsim_mlp::TILE - 1) / chapsim_mlp::TILE;
    const int blocks = (int)std::min<int64_t>(tiles, (int64_t)nsm * 4);
    k_props_mlp_tc<<<blocks, chapsim_mlp::TILE, mlp_smem(), pe->stream>>>(pe->P, h, T, rho, mu, k, cp, n);
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
  int bad = 0, werr = 0;
  PCK(cudaMemcpyAsync(&bad, pe->P.err_count, sizeof(int), cudaMemcpyDeviceToHost, pe->stream));
  PCK(cudaMemcpyAsync(&werr, pe->P.dev_err, sizeof(int), cudaMemcpyDeviceToHost, pe->stream));
  PCK(cudaStreamSynchronize(pe->stream));
  if (werr) {
    PCK(cudaMemsetAsync(pe->P.dev_err, 0, sizeof(int), pe->stream));
    pe->err = "tensor-core inference: a device-side wait gave up";
    return CHAPSIM_ERR_CUDA;
  }
  if (n_out_of_range) *n_out_of_range = bad;
  if (bad) {
    pe->err = std::to_string(bad) + " cells outside the property table (left unchanged)";
    return CHAPSIM_ERR_RANGE;
  }
  return CHAPSIM_OK;
}

// Rebuild the tensor-core weight tiles (BF16 hi / lo of W2 and W3 in the
// canonical operand layout) from the FP32 parameters on the device.
static int refresh_tiles(chapsim_props *pe) {
  std::vector<float> par(NP);
  PCK(cudaMemcpyAsync(par.data(), pe->params, NP * sizeof(float), cudaMemcpyDeviceToHost, pe->stream));
  PCK(cudaStreamSynchronize(pe->stream));
  std::vector<uint16_t> t(2 * NH * NH + 2 * chapsim_mlp::NOP * NH);
  chapsim_mlp::build_weight_tiles(par.data(), t.data());
  PCK(cudaMemcpyAsync(pe->wt, t.data(), t.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, pe->stream));
  PCK(cudaStreamSynchronize(pe->stream));
  return CHAPSIM_OK;
}

// Least-squares polynomial of degree NBASE-1 in x through (x_s, y_s):
// normal equations in FP64, solved by Gaussian elimination with partial
// pivoting (6 x 6, x in [-1, 1]).
static void poly_fit(const std::vector<double> &x, const double *y, double *coef) {
  constexpr int nb = chapsim_mlp::NBASE;
  double A[nb][nb + 1] = {};
  for (size_t s = 0; s < x.size(); ++s) {
    double pw[nb];
    pw[0] = 1.0;
    for (int q = 1; q < nb; ++q) pw[q] = pw[q - 1] * x[s];
    for (int r = 0; r < nb; ++r) {
      for (int q = 0; q < nb; ++q) A[r][q] += pw[r] * pw[q];
      A[r][nb] += pw[r] * y[s];
    }
  }
  for (int c = 0; c < nb; ++c) {
    int piv = c;
    for (int r = c + 1; r < nb; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    for (int q = 0; q <= nb; ++q) std::swap(A[c][q], A[piv][q]);
    for (int r = c + 1; r < nb; ++r) {
      const double f = A[r][c] / A[c][c];
      for (int q = c; q <= nb; ++q) A[r][q] -= f * A[c][q];
    }
  }
  for (int r = nb - 1; r >= 0; --r) {
    double v = A[r][nb];
    for (int q = r + 1; q < nb; ++q) v -= A[r][q] * coef[q];
    coef[r] = v / A[r][r];
  }
}

static double poly_at(const double *coef, double x) {
  double b = coef[chapsim_mlp::NBASE - 1];
  for (int q = chapsim_mlp::NBASE - 2; q >= 0; --q) b = b * x + coef[q];
  return b;
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
  // residual targets: a least-squares degree-5 polynomial in x per output,
  // then the residual standardised (mean, std)
  chapsim_mlp::MlpDev &M = pe->P.M;
  std::vector<double> xs(nsamples);
  for (int s = 0; s < nsamples; ++s) xs[s] = (hs[s] - M.hmid) / M.hhalf;
  for (int o = 0; o < NO; ++o) {
    double *y = tgt.data() + (size_t)o * nsamples;
    poly_fit(xs, y, M.base[o]);
    double m = 0.0, v = 0.0;
    for (int s = 0; s < nsamples; ++s) {
      y[s] -= poly_at(M.base[o], xs[s]);
      m += y[s];
    }
    m /= nsamples;
    for (int s = 0; s < nsamples; ++s) { const double e = y[s] - m; v += e * e; }
    M.mean[o] = m;
    M.stdv[o] = sqrt(v / nsamples) + 1e-12;
  }
  std::vector<float> xf(nsamples), tf((size_t)nsamples * NO);
  for (int s = 0; s < nsamples; ++s) {
    xf[s] = (float)xs[s];
    for (int o = 0; o < NO; ++o)
      tf[(size_t)s * NO + o] = (float)((tgt[(size_t)o * nsamples + s] - M.mean[o]) / M.stdv[o]);
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
  rc = refresh_tiles(pe);
  if (rc) return rc;
  pe->has_mlp = true;
  return CHAPSIM_OK;
}

int chapsim_props_gate(chapsim_props *pe, double tol, int nbins, int *n_mlp_bins, double *max_rel_err) {
  if (!pe || nbins < 1 || nbins > chapsim_mlp::kMaxGateBins || !(tol >= 0)) return CHAPSIM_ERR_ARG;
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
  // every output of every bin on the model for the measurement
  std::vector<uint8_t> all(chapsim_mlp::kMaxGateBins, 0x1F);
  cudaMemcpy(pe->gate, all.data(), all.size(), cudaMemcpyHostToDevice);
  pe->P.M.nbins = 1;
  cudaMemsetAsync(pe->P.err_count, 0, sizeof(int), pe->stream);
  int rc = launch_update(pe, CHAPSIM_PROPS_TABLE, dh, da, da + m, da + 2 * m, da + 3 * m, da + 4 * m, m);
  if (!rc) rc = launch_update(pe, CHAPSIM_PROPS_MLP, dh, db, db + m, db + 2 * m, db + 3 * m, db + 4 * m, m);
  std::vector<double> A(m * NO), B(m * NO);
  int werr = 0;
  cudaMemcpyAsync(A.data(), da, A.size() * sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
  cudaMemcpyAsync(B.data(), db, B.size() * sizeof(double), cudaMemcpyDeviceToHost, pe->stream);
  cudaMemcpyAsync(&werr, pe->P.dev_err, sizeof(int), cudaMemcpyDeviceToHost, pe->stream);
  cudaStreamSynchronize(pe->stream);
  cudaFree(dh); cudaFree(da); cudaFree(db);
  if (rc) return rc;
  if (werr) {
    cudaMemsetAsync(pe->P.dev_err, 0, sizeof(int), pe->stream);
    pe->err = "tensor-core inference: a device-side wait gave up";
    return CHAPSIM_ERR_CUDA;
  }
  // error of each output relative to its largest magnitude over the table
  double scale[NO];
  for (int o = 0; o < NO; ++o) {
    scale[o] = 0.0;
    for (int64_t s = 0; s < m; ++s) scale[o] = fmax(scale[o], fabs(A[o * m + s]));
    scale[o] = scale[o] > 0 ? scale[o] : 1.0;
  }
  std::vector<double> binerr((size_t)nbins * NO, 0.0);
  const double g0 = pe->H[0], ginv = nbins / (pe->H[n - 1] - pe->H[0]);
  for (int o = 0; o < NO; ++o) pe->out_err[o] = 0.0;
  for (int64_t s = 0; s < m; ++s) {
    int b = (int)((hs[s] - g0) * ginv);
    b = b < 0 ? 0 : (b >= nbins ? nbins - 1 : b);
    for (int o = 0; o < NO; ++o) {
      const double e = fabs(B[o * m + s] - A[o * m + s]) / scale[o];
      binerr[(size_t)b * NO + o] = fmax(binerr[(size_t)b * NO + o], e);
      pe->out_err[o] = fmax(pe->out_err[o], e);
    }
  }
  std::vector<uint8_t> flags(chapsim_mlp::kMaxGateBins, 0);
  int cnt = 0;
  for (int o = 0; o < NO; ++o) pe->out_bins[o] = 0;
  for (int b = 0; b < nbins; ++b) {
    unsigned mask = 0;
    for (int o = 0; o < NO; ++o)
      if (binerr[(size_t)b * NO + o] <= tol) {
        mask |= 1u << o;
        ++pe->out_bins[o];
      }
    flags[b] = (uint8_t)mask;
    cnt += (mask & chapsim_mlp::kStepMask) == chapsim_mlp::kStepMask;
  }
  cudaMemcpy(pe->gate, flags.data(), flags.size(), cudaMemcpyHostToDevice);
  pe->P.M.nbins = nbins;
  pe->P.M.g0 = g0;
  pe->P.M.ginv = ginv;
  double worst = 0.0;
  for (int o = 0; o < 4; ++o) worst = fmax(worst, pe->out_err[o]);
  if (n_mlp_bins) *n_mlp_bins = cnt;
  if (max_rel_err) *max_rel_err = worst;
  return CHAPSIM_OK;
}

int chapsim_props_gate_outputs(const chapsim_props *pe, int *bins, double *max_rel_err, int n) {
  if (!pe || !bins || !max_rel_err || n != NO) return CHAPSIM_ERR_ARG;
  for (int o = 0; o < NO; ++o) {
    bins[o] = pe->out_bins[o];
    max_rel_err[o] = pe->out_err[o];
  }
  return CHAPSIM_OK;
}

int chapsim_props_get_params(const chapsim_props *pe, float *params, int nparams, double *norm, int nnorm) {
  if (!pe || !params || nparams != NP || !norm || nnorm != NNORM) return CHAPSIM_ERR_ARG;
  cudaSetDevice(pe->device);
  if (cudaMemcpy(params, pe->params, NP * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return CHAPSIM_ERR_CUDA;
  const chapsim_mlp::MlpDev &M = pe->P.M;
  norm[0] = M.hmid;
  norm[1] = M.hhalf;
  for (int o = 0; o < NO; ++o) {
    norm[2 + o] = M.mean[o];
    norm[2 + NO + o] = M.stdv[o];
    for (int q = 0; q < chapsim_mlp::NBASE; ++q) norm[2 + 2 * NO + o * chapsim_mlp::NBASE + q] = M.base[o][q];
  }
  return CHAPSIM_OK;
}

int chapsim_props_set_params(chapsim_props *pe, const float *params, int nparams, const double *norm, int nnorm) {
  if (!pe || !params || nparams != NP || !norm || nnorm != NNORM) return CHAPSIM_ERR_ARG;
  PCK(cudaSetDevice(pe->device));
  PCK(cudaMemcpy(pe->params, params, NP * sizeof(float), cudaMemcpyHostToDevice));
  chapsim_mlp::MlpDev &M = pe->P.M;
  M.hmid = norm[0];
  M.hhalf = norm[1];
  for (int o = 0; o < NO; ++o) {
    M.mean[o] = norm[2 + o];
    M.stdv[o] = norm[2 + NO + o];
    for (int q = 0; q < chapsim_mlp::NBASE; ++q) M.base[o][q] = norm[2 + 2 * NO + o * chapsim_mlp::NBASE + q];
  }
  int rc = refresh_tiles(pe);
  if (rc) return rc;
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

namespace chapsim {

// The trained model of an engine, for a context that evaluates it in its own
// kernels (chapsim_set_props_mode): FP32 parameters, weight tiles, gate
// masks and the normalisation.  Device pointers stay owned by the engine.
int props_model(const chapsim_props *pe, chapsim_mlp::MlpDev *out, int *device) {
  if (!pe || !out) return CHAPSIM_ERR_ARG;
  if (!pe->has_mlp) return CHAPSIM_ERR_STATE;
  *out = pe->P.M;
  if (device) *device = pe->device;
  return CHAPSIM_OK;
}

// True when the engine was built on the table columns H, T, D, M, K given.
bool props_same_table(const chapsim_props *pe, const std::vector<double> *cols5) {
  const std::vector<double> *mine[5] = {&pe->H, &pe->T, &pe->D, &pe->M, &pe->K};
  for (int q = 0; q < 5; ++q)
    if (*mine[q] != cols5[q]) return false;
  return true;
}

}  // namespace chapsim
