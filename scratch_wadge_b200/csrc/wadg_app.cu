// Host driver: the reference's app_t / rk_step / rk_run (euler.c:2607-2796,
// 3610-3738) on device buffers owned by the library, with one LSRK-45 time
// step (5 stages x 3 kernels) captured as a CUDA graph.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/wadg.h"
#include "wadg_app_impl.h"

namespace wadg_internal {
void set_error(const std::string &msg);  // wadg_capi.cu
}

namespace {
using wadg_internal::RK4A;
using wadg_internal::RK4B;

int afail(int code, const char *msg, cudaError_t e = cudaSuccess) {
  std::string m = msg;
  if (e != cudaSuccess) {
    m += ": ";
    m += cudaGetErrorString(e);
  }
  wadg_internal::set_error(m);
  return code;
}
}  // namespace


namespace {

template <class T>
int upload(T **dst, const T *src, size_t n, cudaStream_t s) {
  cudaError_t e = cudaMalloc((void **)dst, sizeof(T) * (n ? n : 1));
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaMalloc", e);
  if (src) {
    e = cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaMemcpyAsync", e);
  } else {
    e = cudaMemsetAsync(*dst, 0, sizeof(T) * (n ? n : 1), s);
    if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaMemsetAsync", e);
  }
  return WADG_OK;
}

void free_all(wadg_app *a) {
  double *bufs[] = {a->vgeo, a->vfgeo, a->fgeo, a->Jq, a->nrJ, a->nsJ, a->ntJ, a->Drq, a->Dsq,
                    a->Dtq, a->Drstq, a->VqLq, a->VqPq, a->VfPq, a->Q, a->uq[0], a->uq[1],
                    a->uf[0], a->uf[1], a->resQ, a->rhsQf};
  for (double *b : bufs)
    if (b) cudaFree(b);
  if (a->mapPq) cudaFree(a->mapPq);
  if (a->check_work) cudaFree(a->check_work);
  for (auto &g : a->graph)
    if (g) cudaGraphExecDestroy(g);
  if (a->ctx) wadg_ctx_destroy(a->ctx);
  if (a->own_stream && a->stream) cudaStreamDestroy(a->stream);
}

// the reference's kernels on the current buffers (rk_step, euler.c:3610)
int vol(wadg_app *a) {
  const int K = a->K;
  double *rhsQ = a->uq[a->cur], *Qf = a->uf[a->cur];
  if (a->p.dim == 3)
    return a->curved ? wadg_euler_vol_3d_curved(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ,
                                                a->ntJ, a->Drq, a->Dsq, a->Dtq, a->Drstq, a->VqLq,
                                                a->VfPq, a->Q, Qf, rhsQ, a->rhsQf)
                     : wadg_euler_vol_3d(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ, a->ntJ,
                                         a->Drq, a->Dsq, a->Dtq, a->Drstq, a->VqLq, a->VfPq, a->Q,
                                         Qf, rhsQ, a->rhsQf);
  return a->curved ? wadg_euler_vol_2d_curved(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ,
                                              a->Drq, a->Dsq, a->VqLq, a->VfPq, a->Q, Qf, rhsQ,
                                              a->rhsQf)
                   : wadg_euler_vol_2d(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ, a->Drq,
                                       a->Dsq, a->VqLq, a->VfPq, a->Q, Qf, rhsQ, a->rhsQf);
}

int surf(wadg_app *a) {
  double *rhsQ = a->uq[a->cur], *Qf = a->uf[a->cur];
  return a->p.dim == 3 ? wadg_euler_surf_3d(a->ctx, a->K, a->fgeo, a->mapPq, a->VqLq, Qf,
                                            a->rhsQf, rhsQ)
                       : wadg_euler_surf_2d(a->ctx, a->K, a->fgeo, a->mapPq, a->VqLq, Qf,
                                            a->rhsQf, rhsQ);
}

// wadg: the curved update (weight-adjusted inverse mass and projection) on
// a curved app; false runs the affine update (used for the stage-0 projection)
int update(wadg_app *a, double rka, double rkb, double dt, bool wadg) {
  const int K = a->K;
  double *rhsQ = a->uq[a->cur], *Qf = a->uf[a->cur];
  if (a->p.dim == 3)
    return wadg ? wadg_euler_update_3d_curved(a->ctx, K, a->Jq, a->VqPq, a->VfPq, rka, rkb,
                                                   dt, rhsQ, a->resQ, a->Q, Qf)
                     : wadg_euler_update_3d(a->ctx, K, a->Jq, a->VqPq, a->VfPq, rka, rkb, dt,
                                            rhsQ, a->resQ, a->Q, Qf);
  return wadg ? wadg_euler_update_2d_curved(a->ctx, K, a->Jq, a->VqPq, a->VfPq, rka, rkb, dt,
                                                 rhsQ, a->resQ, a->Q, Qf)
                   : wadg_euler_update_2d(a->ctx, K, a->Jq, a->VqPq, a->VfPq, rka, rkb, dt, rhsQ,
                                          a->resQ, a->Q, Qf);
}

int stage3(wadg_app *a, double rka, double rkb, double dt) {
  int r = vol(a);
  if (!r) r = surf(a);
  if (!r) r = update(a, rka, rkb, dt, a->curved);
  return r;
}

// one fused stage: reads buffer cur, writes the other, then flips cur
int stage_fused(wadg_app *a, double rka, double rkb, double dt) {
  const int c = a->cur, n = 1 - c;
  int r = a->p.dim == 3
              ? wadg_euler_stage_3d(a->ctx, a->K, a->curved, a->vgeo, a->vfgeo, a->fgeo, a->mapPq,
                                    a->nrJ, a->nsJ, a->ntJ, a->Drq, a->Dsq, a->Dtq, a->VqLq,
                                    a->VfPq, a->VqPq, a->Jq, rka, rkb, dt, a->uq[c], a->uf[c],
                                    a->Q, a->resQ, a->uq[n], a->uf[n])
              : wadg_euler_stage_2d(a->ctx, a->K, a->curved, a->vgeo, a->vfgeo, a->fgeo, a->mapPq,
                                    a->nrJ, a->nsJ, a->Drq, a->Dsq, a->VqLq, a->VfPq, a->VqPq,
                                    a->Jq, rka, rkb, dt, a->uq[c], a->uf[c], a->Q, a->resQ,
                                    a->uq[n], a->uf[n]);
  if (!r) a->cur = n;
  return r;
}

// the volume + surface kernel on the current buffers (rhsQ: u~ in, RHS out)
int volsurf(wadg_app *a) {
  double *rhsQ = a->uq[a->cur], *Qf = a->uf[a->cur];
  return a->p.dim == 3
             ? wadg_euler_volsurf_3d(a->ctx, a->K, a->curved, a->vgeo, a->vfgeo, a->fgeo, a->mapPq,
                                     a->nrJ, a->nsJ, a->ntJ, a->Drq, a->Dsq, a->Dtq, a->VqLq,
                                     a->VfPq, Qf, rhsQ)
             : wadg_euler_volsurf_2d(a->ctx, a->K, a->curved, a->vgeo, a->vfgeo, a->fgeo, a->mapPq,
                                     a->nrJ, a->nsJ, a->Drq, a->Dsq, a->VqLq, a->VfPq, Qf, rhsQ);
}

int stage_volsurf(wadg_app *a, double rka, double rkb, double dt) {
  int r = volsurf(a);
  if (!r) r = update(a, rka, rkb, dt, a->curved);
  return r;
}

int stage(wadg_app *a, double rka, double rkb, double dt) {
  if (a->fused == WADG_STAGE_FUSED) return stage_fused(a, rka, rkb, dt);
  if (a->fused == WADG_STAGE_VOLSURF) return stage_volsurf(a, rka, rkb, dt);
  return stage3(a, rka, rkb, dt);
}

// capture one time step (5 stages) starting from buffer parity a->cur; the
// fused path flips the parity once per stage, so a step starting at parity p
// ends at 1-p and two graphs alternate
int capture_step(wadg_app *a, double dt) {
  const int p = a->cur;
  if (a->graph[p] && a->graph_dt[p] == dt && a->graph_fused[p] == a->fused) return WADG_OK;
  if (a->graph[p]) {
    cudaGraphExecDestroy(a->graph[p]);
    a->graph[p] = nullptr;
  }
  cudaGraph_t g;
  cudaError_t e = cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaStreamBeginCapture", e);
  int r = WADG_OK;
  for (int s = 0; s < 5 && r == WADG_OK; ++s) r = stage(a, RK4A[s], RK4B[s], dt);
  e = cudaStreamEndCapture(a->stream, &g);
  a->cur = p;  // capture does not execute: restore the parity
  if (r) return r;
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaStreamEndCapture", e);
  e = cudaGraphInstantiate(&a->graph[p], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaGraphInstantiate", e);
  a->graph_dt[p] = dt;
  a->graph_fused[p] = a->fused;
  return WADG_OK;
}

bool valid_map(const uint32_t *m, int K, int NfqNf, int Nf) {
  const size_t per = (size_t)NfqNf * Nf;
  for (size_t i = 0; i < (size_t)K * NfqNf; ++i) {
    const size_t e = m[i] / per, j = m[i] % per;
    if (e >= (size_t)K || j >= (size_t)NfqNf) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int wadg_app_create(const wadg_params *p, int K, int curved, const wadg_host_data *h,
                    wadg_app **out) {
  if (!p || !h || !out || K <= 0) return afail(WADG_ERR_INVALID, "invalid argument");
  *out = nullptr;
  wadg_app *a = new wadg_app;
  a->p = *p;
  a->K = K;
  a->curved = curved ? 1 : 0;
  a->Nq = p->Nq;
  a->NfqNf = p->Nfq * p->Nfaces;
  a->Nf = p->dim + 2;
  a->Nvgeo = p->dim * p->dim;
  a->Nfgeo = p->dim + 1;
  if (p->stream) {
    a->stream = (cudaStream_t)p->stream;
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete a;
      return afail(WADG_ERR_CUDA, "cudaStreamCreate", e);
    }
    a->own_stream = true;
  }
  wadg_params cp = *p;
  cp.stream = a->stream;
  int r = wadg_ctx_create(&cp, &a->ctx);
  if (r) {
    free_all(a);
    delete a;
    return r;
  }
  const bool d3 = p->dim == 3;
  if (!h->vgeo || !h->fgeo || !h->Jq || !h->mapPq || !h->nrJ || !h->nsJ || !h->Drq || !h->Dsq ||
      !h->VqLq || !h->VqPq || !h->VfPq || (curved && !h->vfgeo) || (d3 && (!h->ntJ || !h->Dtq))) {
    free_all(a);
    delete a;
    return afail(WADG_ERR_INVALID, "missing host array");
  }
  if ((unsigned long long)K * a->NfqNf * a->Nf > 0xffffffffULL) {
    free_all(a);
    delete a;
    return afail(WADG_ERR_INVALID, "K * NfqNf * Nfields exceeds the 32-bit range of mapPq");
  }
  if (!valid_map(h->mapPq, K, a->NfqNf, a->Nf)) {
    free_all(a);
    delete a;
    return afail(WADG_ERR_INVALID, "mapPq holds an index outside [0, K*NfqNf*Nfields)");
  }
  const size_t Nq = a->Nq, NfqNf = a->NfqNf, Nf = a->Nf;
  cudaStream_t s = a->stream;
  if ((r = upload(&a->vgeo, h->vgeo, K * Nq * a->Nvgeo, s)) ||
      (r = upload(&a->vfgeo, h->vfgeo, h->vfgeo ? K * NfqNf * a->Nvgeo : 1, s)) ||
      (r = upload(&a->fgeo, h->fgeo, K * NfqNf * a->Nfgeo, s)) ||
      (r = upload(&a->Jq, h->Jq, K * Nq, s)) ||
      (r = upload(&a->mapPq, h->mapPq, K * NfqNf, s)) ||
      (r = upload(&a->nrJ, h->nrJ, NfqNf, s)) || (r = upload(&a->nsJ, h->nsJ, NfqNf, s)) ||
      (r = upload(&a->ntJ, d3 ? h->ntJ : nullptr, NfqNf, s)) ||
      (r = upload(&a->Drq, h->Drq, Nq * Nq, s)) || (r = upload(&a->Dsq, h->Dsq, Nq * Nq, s)) ||
      (r = upload(&a->Dtq, d3 ? h->Dtq : nullptr, Nq * Nq, s)) ||
      (r = upload(&a->Drstq, (const double *)nullptr, 3 * Nq * Nq, s)) ||
      (r = upload(&a->VqLq, h->VqLq, Nq * NfqNf, s)) ||
      (r = upload(&a->VqPq, h->VqPq, Nq * Nq, s)) ||
      (r = upload(&a->VfPq, h->VfPq, NfqNf * Nq, s)) ||
      (r = upload(&a->Q, (const double *)nullptr, K * Nq * Nf, s)) ||
      (r = upload(&a->uq[0], (const double *)nullptr, K * Nq * Nf, s)) ||
      (r = upload(&a->uq[1], (const double *)nullptr, K * Nq * Nf, s)) ||
      (r = upload(&a->uf[1], (const double *)nullptr, K * NfqNf * Nf, s)) ||
      (r = upload(&a->resQ, (const double *)nullptr, K * Nq * Nf, s)) ||
      (r = upload(&a->uf[0], (const double *)nullptr, K * NfqNf * Nf, s)) ||
      (r = upload(&a->rhsQf, (const double *)nullptr, K * NfqNf * Nf, s)) ||
      (r = upload(&a->check_work, (const int *)nullptr, 2, s))) {
    free_all(a);
    delete a;
    return r;
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    free_all(a);
    delete a;
    return afail(WADG_ERR_CUDA, "upload", e);
  }
  *out = a;
  return WADG_OK;
}

int wadg_app_destroy(wadg_app *a) {
  if (!a) return WADG_OK;
  cudaStreamSynchronize(a->stream);
  free_all(a);
  delete a;
  return WADG_OK;
}

int wadg_app_set_state(wadg_app *a, const double *Q, const double *rhsQ, const double *Qf,
                       const double *resQ) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  const size_t nv = (size_t)a->K * a->Nq * a->Nf * sizeof(double);
  const size_t nf = (size_t)a->K * a->NfqNf * a->Nf * sizeof(double);
  struct {
    double *d;
    const double *h;
    size_t n;
  } c[] = {{a->Q, Q, nv}, {a->uq[a->cur], rhsQ, nv}, {a->uf[a->cur], Qf, nf}, {a->resQ, resQ, nv}};
  for (auto &x : c)
    if (x.h) {
      cudaError_t e = cudaMemcpyAsync(x.d, x.h, x.n, cudaMemcpyHostToDevice, a->stream);
      if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "set_state", e);
    }
  return WADG_OK;
}

int wadg_app_get_state(wadg_app *a, double *Q, double *rhsQ, double *Qf, double *resQ) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  const size_t nv = (size_t)a->K * a->Nq * a->Nf * sizeof(double);
  const size_t nf = (size_t)a->K * a->NfqNf * a->Nf * sizeof(double);
  struct {
    double *h;
    const double *d;
    size_t n;
  } c[] = {{Q, a->Q, nv}, {rhsQ, a->uq[a->cur], nv}, {Qf, a->uf[a->cur], nf}, {resQ, a->resQ, nv}};
  for (auto &x : c)
    if (x.h) {
      cudaError_t e = cudaMemcpyAsync(x.h, x.d, x.n, cudaMemcpyDeviceToHost, a->stream);
      if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "get_state", e);
    }
  cudaError_t e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "get_state sync", e);
  return WADG_OK;
}

int wadg_rk_step(wadg_app *a, double rka, double rkb, double dt) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  return stage(a, rka, rkb, dt);
}

// the state check of wadg_rk_run after `steps` steps
int check_after(wadg_app *a, int steps) {
  int nbad = 0;
  const int r = wadg_check_state(a->ctx, a->K, a->Q, a->check_work, &nbad, nullptr);
  if (r != WADG_ERR_STATE) return r;
  std::string m = "after step " + std::to_string(steps) + ": " + wadg_last_error();
  wadg_internal::set_error(m);
  return r;
}

int wadg_rk_run(wadg_app *a, double dt, int nsteps, int use_graph) {
  if (!a || nsteps < 0) return afail(WADG_ERR_INVALID, "invalid argument");
  for (int t = 0; t < nsteps; ++t) {
    if (use_graph) {
      const int p = a->cur;
      int r = capture_step(a, dt);
      if (r) return r;
      cudaError_t e = cudaGraphLaunch(a->graph[p], a->stream);
      if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "cudaGraphLaunch", e);
      if (a->fused == WADG_STAGE_FUSED) a->cur = 1 - p;  // 5 stages flip the parity once
    } else {
      for (int s = 0; s < 5; ++s)
        if (int r = stage(a, RK4A[s], RK4B[s], dt)) return r;
    }
    if (a->check_every > 0 && ((t + 1) % a->check_every == 0 || t + 1 == nsteps))
      if (int r = check_after(a, t + 1)) return r;
  }
  return WADG_OK;
}

int wadg_app_set_check_every(wadg_app *a, int nsteps) {
  if (!a || nsteps < 0) return afail(WADG_ERR_INVALID, "invalid argument");
  a->check_every = nsteps;
  return WADG_OK;
}

int wadg_app_check_state(wadg_app *a, int *nbad, int *first) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  return wadg_check_state(a->ctx, a->K, a->Q, a->check_work, nbad, first);
}

int wadg_app_set_fused(wadg_app *a, int variant) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  if (variant < WADG_STAGE_THREE || variant > WADG_STAGE_VOLSURF)
    return afail(WADG_ERR_INVALID, "unknown stage variant");
  a->fused = variant;
  return WADG_OK;
}

int wadg_app_solve_host(wadg_app *a, const double *Q0, const double *rhsQ0, const double *Qf0,
                        const double *resQ0, double dt, int nsteps, double *Q, double *rhsQ,
                        double *Qf, double *resQ) {
  if (!a || !Q0 || !rhsQ0 || !Qf0 || !Q) return afail(WADG_ERR_INVALID, "invalid argument");
  int r = wadg_app_set_state(a, Q0, rhsQ0, Qf0, resQ0);
  if (r) return r;
  if (!resQ0) {
    cudaError_t e = cudaMemsetAsync(a->resQ, 0, (size_t)a->K * a->Nq * a->Nf * sizeof(double),
                                    a->stream);
    if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "memset resQ", e);
  }
  if ((r = wadg_rk_run(a, dt, nsteps, 1))) return r;
  return wadg_app_get_state(a, Q, rhsQ, Qf, resQ);
}

int wadg_app_project(wadg_app *a) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  // the update kernel with a zero RHS and zero coefficients: Q unchanged,
  // resQ = 0, the traces = the entropy projection of Q.  The affine update
  // on curved meshes too: the reference's host builds the stage-0 traces with
  // VqPq alone (euler.c:3958-4133), not with the weight-adjusted projection
  // its curved update kernel applies in every later stage
  const size_t nvb = (size_t)a->K * a->Nq * a->Nf * sizeof(double);
  cudaError_t e;
  if ((e = cudaMemsetAsync(a->uq[a->cur], 0, nvb, a->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(a->resQ, 0, nvb, a->stream)) != cudaSuccess)
    return afail(WADG_ERR_CUDA, "memset", e);
  return update(a, 0.0, 0.0, 0.0, false);
}

int wadg_app_solve_host_q(wadg_app *a, const double *Q0, double dt, int nsteps, double *Q) {
  if (!a || !Q0 || !Q) return afail(WADG_ERR_INVALID, "invalid argument");
  int r = wadg_app_set_state(a, Q0, nullptr, nullptr, nullptr);
  if (!r) r = wadg_app_project(a);
  if (!r) r = wadg_rk_run(a, dt, nsteps, 1);
  if (!r) r = wadg_app_get_state(a, Q, nullptr, nullptr, nullptr);
  return r;
}

int wadg_app_sync(wadg_app *a) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  cudaError_t e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "sync", e);
  return WADG_OK;
}

int wadg_app_state_ptrs(wadg_app *a, double **Q, double **rhsQ, double **Qf, double **resQ,
                        double **rhsQf) {
  if (!a) return afail(WADG_ERR_INVALID, "null app");
  if (Q) *Q = a->Q;
  if (rhsQ) *rhsQ = a->uq[a->cur];
  if (Qf) *Qf = a->uf[a->cur];
  if (resQ) *resQ = a->resQ;
  if (rhsQf) *rhsQf = a->rhsQf;
  return WADG_OK;
}

int wadg_app_time_run(wadg_app *a, double dt, int nsteps, int use_graph, float *ms) {
  if (!a || !ms) return afail(WADG_ERR_INVALID, "invalid argument");
  if (use_graph) {  // instantiate both parities' graphs outside the timed region
    int r = capture_step(a, dt);
    if (r) return r;
    if (a->fused == WADG_STAGE_FUSED) {
      a->cur = 1 - a->cur;
      r = capture_step(a, dt);
      a->cur = 1 - a->cur;
      if (r) return r;
    }
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, a->stream);
  int r = wadg_rk_run(a, dt, nsteps, use_graph);
  cudaEventRecord(e1, a->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  if (!r && e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "time_run", e);
  return WADG_OK;
}

int wadg_app_time_kernels(wadg_app *a, double dt, int nstages, float *ms) {
  if (!a || !ms || nstages <= 0) return afail(WADG_ERR_INVALID, "invalid argument");
  cudaEvent_t ev[4];
  for (auto &x : ev) cudaEventCreate(&x);
  float tot[3] = {0, 0, 0};
  int r = WADG_OK;
  for (int s = 0; s < nstages && r == WADG_OK; ++s) {
    const double rka = RK4A[s % 5], rkb = RK4B[s % 5];
    cudaEventRecord(ev[0], a->stream);
    r = vol(a);
    cudaEventRecord(ev[1], a->stream);
    if (!r) r = surf(a);
    cudaEventRecord(ev[2], a->stream);
    if (!r) r = update(a, rka, rkb, dt, a->curved);
    cudaEventRecord(ev[3], a->stream);
    cudaError_t e = cudaEventSynchronize(ev[3]);
    if (e != cudaSuccess && !r) r = afail(WADG_ERR_CUDA, "time_kernels", e);
    if (!r)
      for (int q = 0; q < 3; ++q) {
        float t;
        cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
        tot[q] += t;
      }
  }
  for (auto &x : ev) cudaEventDestroy(x);
  if (r) return r;
  for (int q = 0; q < 3; ++q) ms[q] = tot[q];
  return WADG_OK;
}

int wadg_app_autotune(wadg_app *a, double dt, int nstages, int *warps, float *times) {
  if (!a || nstages <= 0) return afail(WADG_ERR_INVALID, "invalid argument");
  int cw[WADG_MAX_VOL_SHAPES], cr[WADG_MAX_VOL_SHAPES];
  const int n = wadg_vol_shapes(a->ctx, a->curved, cw, cr);
  if (n <= 0) return afail(WADG_ERR_UNSUPPORTED, "no volume kernel shapes");
  int best = 0;
  float best_ms = -1.0f;
  // the volume kernel's time, or (volume + surface variant) the volume +
  // surface kernel's
  const bool vs = a->fused == WADG_STAGE_VOLSURF;
  for (int i = 0; i < n; ++i) {
    int r = wadg_ctx_set_vol_shape(a->ctx, a->curved, cw[i], cr[i]);
    float ms[3] = {0, 0, 0};
    if (!r) r = vs ? wadg_app_time_volsurf(a, dt, 1, ms) : wadg_app_time_kernels(a, dt, 1, ms);
    if (!r) r = vs ? wadg_app_time_volsurf(a, dt, nstages, ms) : wadg_app_time_kernels(a, dt, nstages, ms);
    if (r) return r;
    if (times) times[i] = ms[0] / nstages;
    if (best_ms < 0.0f || ms[0] < best_ms) {
      best_ms = ms[0];
      best = i;
    }
  }
  // graphs captured with another shape are stale
  for (auto &g : a->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  if (warps) *warps = cw[best];
  return wadg_ctx_set_vol_shape(a->ctx, a->curved, cw[best], cr[best]);
}

int wadg_app_time_stage(wadg_app *a, double dt, int nstages, float *ms) {
  if (!a || !ms || nstages <= 0) return afail(WADG_ERR_INVALID, "invalid argument");
  const int fused = a->fused;
  a->fused = WADG_STAGE_FUSED;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, a->stream);
  int r = WADG_OK;
  for (int s = 0; s < nstages && r == WADG_OK; ++s) r = stage_fused(a, RK4A[s % 5], RK4B[s % 5], dt);
  cudaEventRecord(e1, a->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  if (!r && e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  a->fused = fused;
  if (r) return r;
  if (e != cudaSuccess) return afail(WADG_ERR_CUDA, "time_stage", e);
  return WADG_OK;
}

int wadg_app_time_volsurf(wadg_app *a, double dt, int nstages, float *ms) {
  if (!a || !ms || nstages <= 0) return afail(WADG_ERR_INVALID, "invalid argument");
  cudaEvent_t ev[3];
  for (auto &x : ev) cudaEventCreate(&x);
  float tot[2] = {0, 0};
  int r = WADG_OK;
  for (int s = 0; s < nstages && r == WADG_OK; ++s) {
    cudaEventRecord(ev[0], a->stream);
    r = volsurf(a);
    cudaEventRecord(ev[1], a->stream);
    if (!r) r = update(a, RK4A[s % 5], RK4B[s % 5], dt, a->curved);
    cudaEventRecord(ev[2], a->stream);
    cudaError_t e = cudaEventSynchronize(ev[2]);
    if (e != cudaSuccess && !r) r = afail(WADG_ERR_CUDA, "time_volsurf", e);
    if (!r)
      for (int q = 0; q < 2; ++q) {
        float t;
        cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
        tot[q] += t;
      }
  }
  for (auto &x : ev) cudaEventDestroy(x);
  if (r) return r;
  ms[0] = tot[0];
  ms[1] = tot[1];
  return WADG_OK;
}

void *wadg_app_stream(wadg_app *a) { return a ? (void *)a->stream : nullptr; }
wadg_ctx *wadg_app_ctx(wadg_app *a) { return a ? a->ctx : nullptr; }

int wadg_app_set_parity(wadg_app *a, int parity) {
  if (!a || (parity != 0 && parity != 1)) return afail(WADG_ERR_INVALID, "invalid argument");
  a->cur = parity;
  return WADG_OK;
}

int wadg_app_get_fused(wadg_app *a) { return a ? a->fused : 0; }

}  // extern "C"
