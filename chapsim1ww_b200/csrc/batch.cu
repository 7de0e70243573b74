// Batched TG channels: n independent chapsim contexts of uneven sizes, one
// captured CUDA graph per time step holding every channel's three substeps as
// parallel branches (fork/join through events), and a launch-shape
// autotuner.  No counterpart in the reference, which advances one domain per
// job.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "chapsim_internal.cuh"

struct chapsim_batch {
  std::vector<chapsim_ctx *> ch;
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> ev;  // [0] fork, [1 + i] join of channel i
  cudaGraphExec_t graph = nullptr;
  int64_t kernels_per_step = 0;
  std::string err;
  int device = 0;
};

#define BCK(call)                                                      \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      b->err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
      return CHAPSIM_ERR_CUDA;                                         \
    }                                                                  \
  } while (0)

static void batch_free(chapsim_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  for (auto *c : b->ch)
    if (c) chapsim_destroy(c);
  b->ch.clear();
  for (auto e : b->ev)
    if (e) cudaEventDestroy(e);
  b->ev.clear();
  if (b->stream) cudaStreamDestroy(b->stream);
  b->stream = nullptr;
}

static void drop_graph(chapsim_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

extern "C" {

int chapsim_batch_create(const chapsim_config *cfgs, int n, chapsim_batch **out) {
  if (!cfgs || n < 1 || !out) return CHAPSIM_ERR_ARG;
  *out = nullptr;
  for (int i = 1; i < n; ++i)
    if (cfgs[i].device != cfgs[0].device) return CHAPSIM_ERR_ARG;  // one GPU per batch
  chapsim_batch *b = new chapsim_batch();
  b->device = cfgs[0].device;
  int rc = CHAPSIM_OK;
  for (int i = 0; i < n; ++i) {
    chapsim_ctx *c = nullptr;
    rc = chapsim_create(&cfgs[i], &c);
    if (rc) {
      batch_free(b);
      delete b;
      return rc;
    }
    b->ch.push_back(c);
  }
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    batch_free(b);
    delete b;
    return CHAPSIM_ERR_CUDA;
  }
  b->ev.assign(n + 1, nullptr);
  for (auto &e : b->ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      batch_free(b);
      delete b;
      return CHAPSIM_ERR_CUDA;
    }
  *out = b;
  return CHAPSIM_OK;
}

int chapsim_batch_destroy(chapsim_batch *b) {
  if (!b) return CHAPSIM_ERR_ARG;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_free(b);
  delete b;
  return CHAPSIM_OK;
}

const char *chapsim_batch_last_error(const chapsim_batch *b) { return b ? b->err.c_str() : "null batch"; }

int chapsim_batch_channel(chapsim_batch *b, int i, chapsim_ctx **ctx) {
  if (!b || !ctx || i < 0 || i >= (int)b->ch.size()) return CHAPSIM_ERR_ARG;
  *ctx = b->ch[i];
  return CHAPSIM_OK;
}

int chapsim_batch_init_random(chapsim_batch *b, uint64_t seed, double amp, int project) {
  if (!b) return CHAPSIM_ERR_ARG;
  for (size_t i = 0; i < b->ch.size(); ++i) {
    int rc = chapsim_init_random(b->ch[i], seed + i, amp, project);
    if (rc) {
      b->err = "channel " + std::to_string(i) + ": " + b->ch[i]->err;
      return rc;
    }
  }
  return CHAPSIM_OK;
}

// Time `reps` substeps of one channel (eager launches, events on its stream).
static int time_substeps(chapsim_ctx *c, int reps, float *ms) {
  cudaEvent_t a, e;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&e) != cudaSuccess) return CHAPSIM_ERR_CUDA;
  int rc = chapsim::launch_substep(c, 1);  // warm-up
  cudaEventRecord(a, c->stream);
  for (int r = 0; r < reps && !rc; ++r) rc = chapsim::launch_substep(c, 1 + r % 3);
  cudaEventRecord(e, c->stream);
  cudaEventSynchronize(e);
  cudaEventElapsedTime(ms, a, e);
  cudaEventDestroy(a);
  cudaEventDestroy(e);
  return rc;
}

// Time every candidate launch shape of one channel and keep the fastest.
// The fields the trial substeps overwrite are saved first; on every exit
// after the save (success or a failed trial) they are copied back and the
// save buffer is freed, so a failure never leaves trial state behind.
static int autotune_channel(chapsim_batch *b, chapsim_ctx *c, int reps) {
  const size_t n = (size_t)c->d.sz * c->d.nz;
  const size_t tsz = c->cfg.precision == CHAPSIM_MIXED ? sizeof(float) : sizeof(double);
  char *sp = nullptr;
  if (cudaMalloc((void **)&sp, n * (4 * sizeof(double) + 3 * tsz)) != cudaSuccess) {
    cudaGetLastError();
    b->err = "autotune: cannot allocate the save buffer";
    return CHAPSIM_ERR_NOMEM;
  }
  double *f[4] = {c->d.u, c->d.v, c->d.w, c->d.p};
  auto copy_all = [&](bool save) {
    bool ok = true;
    for (int q = 0; q < 4; ++q) {
      char *s = sp + q * n * sizeof(double);
      ok = ok && cudaMemcpyAsync(save ? (void *)s : (void *)f[q], save ? (const void *)f[q] : (const void *)s,
                                 n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess;
    }
    for (int q = 0; q < 3; ++q) {
      char *s = sp + 4 * n * sizeof(double) + q * n * tsz;
      ok = ok && cudaMemcpyAsync(save ? (void *)s : c->d.h0[q], save ? (const void *)c->d.h0[q] : (const void *)s,
                                 n * tsz, cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess;
    }
    return ok;
  };
  int rc = CHAPSIM_OK;
  if (!copy_all(true)) {
    cudaGetLastError();
    cudaFree(sp);
    b->err = "autotune: saving the channel state failed";
    return CHAPSIM_ERR_CUDA;
  }
  // candidate launch shapes: RHS z segment x transform rows per block,
  // then, with those fixed, the y-line block width of the Poisson solve
  const int nzc_c[] = {8, 16, 32, 64};
  const int lb_c[] = {0, 4, 8, 16};
  const int ys_c[] = {64, 128, 256};
  float best = 1e30f;
  int bn = c->rhs_nzc, bl = c->fft_lb, by = c->ys_bx;
  for (int nzc : nzc_c) {
    if (nzc > c->d.nz || rc) continue;
    for (int lb : lb_c) {
      c->rhs_nzc = nzc;
      c->fft_lb = lb;
      float ms = 0.f;
      if ((rc = time_substeps(c, reps, &ms))) break;
      if (ms < best) { best = ms; bn = nzc; bl = lb; }
    }
  }
  c->rhs_nzc = bn;
  c->fft_lb = bl;
  for (int ys : ys_c) {
    if (rc || ys == by) continue;
    c->ys_bx = ys;
    float ms = 0.f;
    if ((rc = time_substeps(c, reps, &ms))) break;
    if (ms < best) { best = ms; by = ys; }
  }
  c->ys_bx = by;
  // single exit: restore the saved state, then free the buffer
  const bool restored = copy_all(false) && cudaStreamSynchronize(c->stream) == cudaSuccess;
  if (!restored) cudaGetLastError();
  cudaFree(sp);
  if (c->step_graph) { cudaGraphExecDestroy(c->step_graph); c->step_graph = nullptr; }
  if (rc) return rc;
  if (!restored) {
    b->err = "autotune: restoring the channel state failed";
    return CHAPSIM_ERR_CUDA;
  }
  return CHAPSIM_OK;
}

int chapsim_batch_autotune(chapsim_batch *b, int reps) {
  if (!b || reps < 1) return CHAPSIM_ERR_ARG;
  BCK(cudaSetDevice(b->device));
  drop_graph(b);
  for (auto *c : b->ch) {
    const int rc = autotune_channel(b, c, reps);
    if (rc) return rc;
  }
  return CHAPSIM_OK;
}

static int capture(chapsim_batch *b) {
  cudaGraph_t g = nullptr;
  int64_t kernels = 0;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = CHAPSIM_OK;
  cudaEventRecord(b->ev[0], b->stream);
  for (size_t i = 0; i < b->ch.size() && !rc; ++i) {
    chapsim_ctx *c = b->ch[i];
    cudaStreamWaitEvent(c->stream, b->ev[0], 0);
    const int64_t before = c->launches;
    for (int ns = 1; ns <= 3 && !rc; ++ns) rc = chapsim::launch_substep(c, ns);
    kernels += c->launches - before;
    c->launches = before;
    cudaEventRecord(b->ev[1 + i], c->stream);
    cudaStreamWaitEvent(b->stream, b->ev[1 + i], 0);
  }
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    b->err = "capture failed";
    return rc;
  }
  if (e != cudaSuccess) {
    b->err = cudaGetErrorString(e);
    return CHAPSIM_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->graph = nullptr;
    b->err = cudaGetErrorString(e);
    return CHAPSIM_ERR_CUDA;
  }
  b->kernels_per_step = kernels;
  return CHAPSIM_OK;
}

int chapsim_batch_step(chapsim_batch *b, int nsteps) {
  if (!b || nsteps < 0) return CHAPSIM_ERR_ARG;
  BCK(cudaSetDevice(b->device));
  for (auto *c : b->ch)
    if (c->timing) { b->err = "phase timing is on for a channel"; return CHAPSIM_ERR_STATE; }
  if (!b->graph) {
    // channels' own work must be complete before their streams join the capture
    for (auto *c : b->ch) BCK(cudaStreamSynchronize(c->stream));
    int rc = capture(b);
    if (rc) return rc;
  }
  // order the graph after each channel's earlier work, and the channels'
  // later work (reductions, downloads) after the graph
  for (size_t i = 0; i < b->ch.size(); ++i) {
    BCK(cudaEventRecord(b->ev[1 + i], b->ch[i]->stream));
    BCK(cudaStreamWaitEvent(b->stream, b->ev[1 + i], 0));
  }
  for (int s = 0; s < nsteps; ++s) {
    BCK(cudaGraphLaunch(b->graph, b->stream));
    for (auto *c : b->ch) c->launches += b->kernels_per_step / (int64_t)b->ch.size();
  }
  BCK(cudaEventRecord(b->ev[0], b->stream));
  for (auto *c : b->ch) BCK(cudaStreamWaitEvent(c->stream, b->ev[0], 0));
  return CHAPSIM_OK;
}

int chapsim_batch_sync(chapsim_batch *b) {
  if (!b) return CHAPSIM_ERR_ARG;
  BCK(cudaStreamSynchronize(b->stream));
  for (auto *c : b->ch) {
    int rc = chapsim_sync(c);
    if (rc) { b->err = c->err; return rc; }
  }
  return CHAPSIM_OK;
}

int chapsim_batch_get_stream(const chapsim_batch *b, void **stream) {
  if (!b || !stream) return CHAPSIM_ERR_ARG;
  *stream = (void *)b->stream;
  return CHAPSIM_OK;
}

int chapsim_batch_kernels_per_step(const chapsim_batch *b, int64_t *count) {
  if (!b || !count) return CHAPSIM_ERR_ARG;
  *count = b->kernels_per_step;
  return CHAPSIM_OK;
}

}  // extern "C"
