// Batched ensemble of independent solves, each with its own time step.
//
// A bin is one wadg_app holding the concatenation of all instances of one
// degree (scratch_wadge_b200/ensemble.py builds it: neighbour maps offset by
// the instance's first element, so the kernels walk the bin as one element
// list).  Every instance keeps its own step dt_i = T / n_i (the reference's
// dt = CFL hmin / C_N, euler.c:4180-4193, with the instance's wave speed,
// rounded to reach T) and runs n_i steps; the update kernel takes the step of
// element k from dtK[k].
//
// Work lists.  Per bin the volume + surface kernel walks a device list of
// batches (those that hold an element of an instance still running) and the
// update kernel a list of element groups (those that hold an element of such
// a batch).  When an instance has made its n_i
// steps its entries of dtK become 0 -- with the first LSRK coefficient 0, a
// stage with a zero step leaves Q, res and the projected traces as they are,
// so an element that shares a batch with a running instance stays frozen --
// and the lists are rebuilt without the batches it alone occupied.  The
// kernels read the list lengths from device memory, so one CUDA graph per
// time step (every bin on its own stream, concurrently) serves the whole run;
// between graph launches the host updates dtK and the lists on the master
// stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/wadg.h"
#include "wadg_app_impl.h"
#include "wadg_host.h"

namespace wadg_internal {
void set_error(const std::string &msg);
}

namespace {
struct Bin {
  wadg_app *app = nullptr;
  std::vector<int> off;      // instance element offsets (ninst + 1)
  std::vector<double> dt;    // step of each instance
  std::vector<int> nsteps;   // steps of each instance
  int Evs = 0, Eup = 0;      // elements per volume batch / update group
  double *dtK = nullptr;     // device: step of every element
  int *vlist = nullptr;      // device: active volume batches
  int *glist = nullptr;      // device: active update groups
  int *counts = nullptr;     // device: the two list lengths
  std::vector<int> hv, hg;   // host copies of the lists
};
}  // namespace

struct wadg_ensemble {
  std::vector<Bin> bins;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph = nullptr;
  int step = 0;       // time steps done
  int max_steps = 0;  // the longest instance's
};

namespace {
using wadg_internal::RK4A;
using wadg_internal::RK4B;

int efail(int code, const std::string &msg, cudaError_t e = cudaSuccess) {
  std::string m = msg;
  if (e != cudaSuccess) {
    m += ": ";
    m += cudaGetErrorString(e);
  }
  wadg_internal::set_error(m);
  return code;
}

// the lists of a bin for the instances still running after `step` steps:
// the volume batches that hold a running element, then the update groups
// that hold an element of those batches -- every element whose RHS the
// volume kernel overwrites (its traces in place) must be updated, which for a
// frozen element (step 0) rebuilds the same traces from its unchanged Q
void build_lists(Bin &b, int step) {
  const int K = b.app->K;
  std::vector<char> mark(K, 0);
  for (size_t i = 0; i + 1 < b.off.size(); ++i)
    if (step < b.nsteps[i]) std::fill(mark.begin() + b.off[i], mark.begin() + b.off[i + 1], 1);
  auto list = [&](int E, std::vector<int> &out) {
    out.clear();
    for (int k0 = 0, g = 0; k0 < K; k0 += E, ++g) {
      const int k1 = std::min(K, k0 + E);
      if (std::any_of(mark.begin() + k0, mark.begin() + k1, [](char c) { return c != 0; }))
        out.push_back(g);
    }
  };
  list(b.Evs, b.hv);
  std::fill(mark.begin(), mark.end(), 0);
  for (int g : b.hv)
    std::fill(mark.begin() + (size_t)g * b.Evs, mark.begin() + std::min(K, (g + 1) * b.Evs), 1);
  list(b.Eup, b.hg);
}

int upload_lists(Bin &b, cudaStream_t s) {
  const int n[2] = {(int)b.hv.size(), (int)b.hg.size()};
  cudaError_t e = cudaSuccess;
  if (n[0]) e = cudaMemcpyAsync(b.vlist, b.hv.data(), sizeof(int) * n[0], cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n[1])
    e = cudaMemcpyAsync(b.glist, b.hg.data(), sizeof(int) * n[1], cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b.counts, n, sizeof n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // n lives on this stack frame
  return e == cudaSuccess ? WADG_OK : efail(WADG_ERR_CUDA, "ensemble work lists", e);
}

// the per-element steps and the lists of the instances still running
int restart(wadg_ensemble *s) {
  for (auto &b : s->bins) {
    std::vector<double> h(b.app->K, 0.0);
    for (size_t i = 0; i + 1 < b.off.size(); ++i)
      if (b.nsteps[i] > 0) std::fill(h.begin() + b.off[i], h.begin() + b.off[i + 1], b.dt[i]);
    cudaError_t e = cudaMemcpyAsync(b.dtK, h.data(), sizeof(double) * h.size(),
                                    cudaMemcpyHostToDevice, s->master);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->master);
    if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble steps", e);
    build_lists(b, 0);
    if (int r = upload_lists(b, s->master)) return r;
  }
  s->step = 0;
  return WADG_OK;
}

int bin_stage(Bin &b, int st) {
  wadg_app *a = b.app;
  const int c = a->cur;
  int r = wadg_internal::volsurf_list(a->ctx, a->K, a->curved, a->vgeo, a->vfgeo, a->fgeo, a->mapPq,
                                      a->nrJ, a->nsJ, a->ntJ, a->Drq, a->Dsq, a->Dtq, a->VqLq,
                                      a->VfPq, a->uf[c], a->uq[c], b.vlist, b.counts);
  if (!r)
    r = wadg_internal::update_list(a->ctx, a->K, a->curved, a->Jq, a->VqPq, a->VfPq, RK4A[st],
                                   RK4B[st], b.dtK, a->uq[c], a->resQ, a->Q, a->uf[c], b.glist,
                                   b.counts + 1);
  return r;
}

// one time step of every bin (5 stages each), bins on their own streams
int capture(wadg_ensemble *s) {
  if (s->graph) return WADG_OK;
  cudaError_t e = cudaStreamBeginCapture(s->master, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble capture", e);
  cudaEventRecord(s->fork, s->master);
  int r = WADG_OK;
  for (size_t b = 0; b < s->bins.size() && r == WADG_OK; ++b) {
    cudaStream_t bs = s->bins[b].app->stream;
    cudaStreamWaitEvent(bs, s->fork, 0);
    for (int st = 0; st < 5 && r == WADG_OK; ++st) r = bin_stage(s->bins[b], st);
    cudaEventRecord(s->join[b], bs);
    cudaStreamWaitEvent(s->master, s->join[b], 0);
  }
  cudaGraph_t g;
  e = cudaStreamEndCapture(s->master, &g);
  if (e != cudaSuccess) return r ? r : efail(WADG_ERR_CUDA, "ensemble end capture", e);
  if (r) {  // a stage failed to issue: drop the partial graph
    cudaGraphDestroy(g);
    return r;
  }
  e = cudaGraphInstantiate(&s->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble instantiate", e);
  return WADG_OK;
}

// after step `step`: zero the steps of the instances that are done and drop
// the batches they alone occupied
int retire(wadg_ensemble *s) {
  for (auto &b : s->bins) {
    bool changed = false;
    for (size_t i = 0; i + 1 < b.off.size(); ++i)
      if (b.nsteps[i] == s->step) {
        const size_t n = (size_t)(b.off[i + 1] - b.off[i]);
        cudaError_t e = cudaMemsetAsync(b.dtK + b.off[i], 0, sizeof(double) * n, s->master);
        if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble retire", e);
        changed = true;
      }
    if (changed) {
      build_lists(b, s->step);
      if (int r = upload_lists(b, s->master)) return r;
    }
  }
  return WADG_OK;
}
}  // namespace

extern "C" {

int wadg_ensemble_create(int nbins, const wadg_ensemble_bin *desc, wadg_ensemble **out) {
  if (nbins <= 0 || !desc || !out) return efail(WADG_ERR_INVALID, "invalid argument");
  *out = nullptr;
  wadg_ensemble *s = new wadg_ensemble;
  s->bins.resize(nbins);
  cudaError_t e = cudaStreamCreateWithFlags(&s->master, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming);
  s->join.resize(nbins, nullptr);
  for (int b = 0; b < nbins && e == cudaSuccess; ++b)
    e = cudaEventCreateWithFlags(&s->join[b], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    wadg_ensemble_destroy(s);
    return efail(WADG_ERR_CUDA, "ensemble streams/events", e);
  }
  for (int b = 0; b < nbins; ++b) {
    const wadg_ensemble_bin &d = desc[b];
    Bin &B = s->bins[b];
    B.app = d.app;
    bool ok = d.app && d.ninst > 0 && d.offsets && d.dt && d.nsteps &&
              wadg_app_get_fused(d.app) != WADG_STAGE_FUSED && d.offsets[0] == 0 &&
              d.offsets[d.ninst] == d.app->K;
    for (int i = 0; ok && i < d.ninst; ++i)
      ok = d.offsets[i] < d.offsets[i + 1] && d.dt[i] > 0.0 && d.nsteps[i] >= 0;
    if (!ok) {
      B.app = nullptr;
      wadg_ensemble_destroy(s);
      return efail(WADG_ERR_INVALID,
                   "bin " + std::to_string(b) +
                       ": needs an app (not in the fused stage variant), ascending instance offsets "
                       "from 0 to its K, positive steps and non-negative step counts");
    }
    B.off.assign(d.offsets, d.offsets + d.ninst + 1);
    B.dt.assign(d.dt, d.dt + d.ninst);
    B.nsteps.assign(d.nsteps, d.nsteps + d.ninst);
    for (int n : B.nsteps) s->max_steps = std::max(s->max_steps, n);
    int g = 0;
    int r = wadg_kernel_shape(d.app->ctx, WADG_KERNEL_VOLSURF, d.app->curved, d.app->K, &B.Evs, &g);
    if (!r) r = wadg_kernel_shape(d.app->ctx, WADG_KERNEL_UPDATE, d.app->curved, d.app->K, &B.Eup, &g);
    if (r) {
      wadg_ensemble_destroy(s);
      return r;
    }
    const int K = d.app->K;
    e = cudaMalloc((void **)&B.dtK, sizeof(double) * K);
    if (e == cudaSuccess) e = cudaMalloc((void **)&B.vlist, sizeof(int) * ((K + B.Evs - 1) / B.Evs));
    if (e == cudaSuccess) e = cudaMalloc((void **)&B.glist, sizeof(int) * ((K + B.Eup - 1) / B.Eup));
    if (e == cudaSuccess) e = cudaMalloc((void **)&B.counts, sizeof(int) * 2);
    if (e != cudaSuccess) {
      wadg_ensemble_destroy(s);
      return efail(WADG_ERR_CUDA, "ensemble buffers", e);
    }
    wadg_app_set_parity(d.app, 0);
  }
  if (int r = restart(s)) {
    wadg_ensemble_destroy(s);
    return r;
  }
  *out = s;
  return WADG_OK;
}

int wadg_ensemble_destroy(wadg_ensemble *s) {
  if (!s) return WADG_OK;
  if (s->master) cudaStreamSynchronize(s->master);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  for (auto &b : s->bins) {
    if (b.dtK) cudaFree(b.dtK);
    if (b.vlist) cudaFree(b.vlist);
    if (b.glist) cudaFree(b.glist);
    if (b.counts) cudaFree(b.counts);
  }
  for (auto &ev : s->join)
    if (ev) cudaEventDestroy(ev);
  if (s->fork) cudaEventDestroy(s->fork);
  if (s->master) cudaStreamDestroy(s->master);
  delete s;
  return WADG_OK;
}

int wadg_ensemble_run(wadg_ensemble *s, int nsteps) {
  if (!s || nsteps < 0) return efail(WADG_ERR_INVALID, "invalid argument");
  if (int r = capture(s)) return r;
  for (int t = 0; t < nsteps && s->step < s->max_steps; ++t) {
    cudaError_t e = cudaGraphLaunch(s->graph, s->master);
    if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble graph launch", e);
    ++s->step;
    if (int r = retire(s)) return r;
  }
  return WADG_OK;
}

int wadg_ensemble_restart(wadg_ensemble *s) {
  if (!s) return efail(WADG_ERR_INVALID, "null ensemble");
  cudaError_t e = cudaStreamSynchronize(s->master);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble sync", e);
  return restart(s);
}

int wadg_ensemble_steps(const wadg_ensemble *s, int *done, int *max_steps) {
  if (!s) return efail(WADG_ERR_INVALID, "null ensemble");
  if (done) *done = s->step;
  if (max_steps) *max_steps = s->max_steps;
  return WADG_OK;
}

int wadg_ensemble_sync(wadg_ensemble *s) {
  if (!s) return efail(WADG_ERR_INVALID, "null ensemble");
  cudaError_t e = cudaStreamSynchronize(s->master);
  if (e != cudaSuccess) return efail(WADG_ERR_CUDA, "ensemble sync", e);
  return WADG_OK;
}

int wadg_ensemble_time_run(wadg_ensemble *s, int nsteps, float *ms) {
  if (!s || !ms) return efail(WADG_ERR_INVALID, "invalid argument");
  int r = capture(s);  // instantiate the graph outside the timed region
  if (r) return r;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s->master);
  r = wadg_ensemble_run(s, nsteps);
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
