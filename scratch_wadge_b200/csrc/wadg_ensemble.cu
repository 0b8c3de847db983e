// Batched ensemble of independent solves: one time step of every bin (a bin
// is the concatenation of all instances of one degree, see
// scratch_wadge_b200/ensemble.py) captured as one CUDA graph whose branches --
// one per bin, each on its bin's own stream -- run concurrently.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/wadg.h"

namespace wadg_internal {
void set_error(const std::string &msg);
}

struct wadg_ensemble {
  std::vector<wadg_app *> bins;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dt[2] = {0.0, 0.0};
  int parity = 0;  // buffer parity of the bins (fused stages flip it each step)
  int fused = 0;
};

namespace {
int efail(int code, const char *msg, cudaError_t e = cudaSuccess) {
  std::string m = msg;
  if (e != cudaSuccess) {
    m += ": ";
    m += cudaGetErrorString(e);
  }
  wadg_internal::set_error(m);
  return code;
}

int capture(wadg_ensemble *s, double dt) {
  const int p = s->parity;
  if (s->graph[p] && s->graph_dt[p] == dt) return WADG_OK;
  if (s->graph[p]) {
    cudaGraphExecDestroy(s->graph[p]);
    s->graph[p] = nullptr;
  }
  cudaError_t e = cudaStreamBeginCapture(s->master, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble capture", e);
  cudaEventRecord(s->fork, s->master);
  int r = WADG_OK;
  for (size_t b = 0; b < s->bins.size() && r == WADG_OK; ++b) {
    cudaStream_t bs = (cudaStream_t)wadg_app_stream(s->bins[b]);
    cudaStreamWaitEvent(bs, s->fork, 0);
    r = wadg_rk_run(s->bins[b], dt, 1, 0);  // 5 stages issued on the bin's stream
    cudaEventRecord(s->join[b], bs);
    cudaStreamWaitEvent(s->master, s->join[b], 0);
  }
  cudaGraph_t g;
  e = cudaStreamEndCapture(s->master, &g);
  // capture issued but did not execute the stages: restore the bins' parity
  for (auto *a : s->bins) wadg_app_set_parity(a, p);
  if (e != cudaSuccess) return r ? r : efail(WADG_ERR_CUDA, "ensemble end capture", e);
  if (r) {  // a stage failed to issue: drop the partial graph
    cudaGraphDestroy(g);
    return r;
  }
  e = cudaGraphInstantiate(&s->graph[p], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble instantiate", e);
  s->graph_dt[p] = dt;
  return WADG_OK;
}
}  // namespace

extern "C" {

int wadg_ensemble_create(int nbins, wadg_app **bins, wadg_ensemble **out) {
  if (nbins <= 0 || !bins || !out) return efail(WADG_ERR_INVALID, "invalid argument");
  *out = nullptr;
  wadg_ensemble *s = new wadg_ensemble;
  s->bins.assign(bins, bins + nbins);
  s->fused = wadg_app_get_fused(bins[0]) == WADG_STAGE_FUSED;
  for (auto *a : s->bins) {
    if (!a || (wadg_app_get_fused(a) == WADG_STAGE_FUSED) != s->fused) {
      delete s;
      return efail(WADG_ERR_INVALID, "bins must be non-null and share the stage variant");
    }
    wadg_app_set_parity(a, 0);
  }
  cudaError_t e = cudaStreamCreateWithFlags(&s->master, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming);
  s->join.resize(nbins, nullptr);
  for (int b = 0; b < nbins && e == cudaSuccess; ++b)
    e = cudaEventCreateWithFlags(&s->join[b], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    wadg_ensemble_destroy(s);
    return efail(WADG_ERR_CUDA, "ensemble streams/events", e);
  }
  *out = s;
  return WADG_OK;
}

int wadg_ensemble_destroy(wadg_ensemble *s) {
  if (!s) return WADG_OK;
  if (s->master) cudaStreamSynchronize(s->master);
  for (auto &g : s->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto &ev : s->join)
    if (ev) cudaEventDestroy(ev);
  if (s->fork) cudaEventDestroy(s->fork);
  if (s->master) cudaStreamDestroy(s->master);
  delete s;
  return WADG_OK;
}

int wadg_ensemble_run(wadg_ensemble *s, double dt, int nsteps) {
  if (!s || nsteps < 0) return efail(WADG_ERR_INVALID, "invalid argument");
  for (int t = 0; t < nsteps; ++t) {
    const int p = s->parity;
    int r = capture(s, dt);
    if (r) return r;
    cudaError_t e = cudaGraphLaunch(s->graph[p], s->master);
    if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble graph launch", e);
    if (s->fused) {
      s->parity = 1 - p;
      for (auto *a : s->bins) wadg_app_set_parity(a, s->parity);
    }
  }
  return WADG_OK;
}

int wadg_ensemble_sync(wadg_ensemble *s) {
  if (!s) return efail(WADG_ERR_INVALID, "null ensemble");
  cudaError_t e = cudaStreamSynchronize(s->master);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble sync", e);
  return WADG_OK;
}

int wadg_ensemble_time_run(wadg_ensemble *s, double dt, int nsteps, float *ms) {
  if (!s || !ms) return efail(WADG_ERR_INVALID, "invalid argument");
  // instantiate the graphs of both parities outside the timed region
  int r = capture(s, dt);
  if (r) return r;
  if (s->fused) {
    const int p = s->parity;
    s->parity = 1 - p;
    for (auto *a : s->bins) wadg_app_set_parity(a, s->parity);
    r = capture(s, dt);
    s->parity = p;
    for (auto *a : s->bins) wadg_app_set_parity(a, p);
    if (r) return r;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s->master);
  r = wadg_ensemble_run(s, dt, nsteps);
  cudaEventRecord(e1, s->master);
  cudaError_t e = cudaEventSynchronize(e1);
  if (!r && e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble time_run", e);
  return WADG_OK;
}

}  // extern "C"
