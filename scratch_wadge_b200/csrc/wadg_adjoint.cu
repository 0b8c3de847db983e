// Discrete adjoint of the LSRK-45 time loop (rk_run, euler.c:3672-3738) with
// checkpointing: the forward run stores Q every `every` steps; the reverse
// sweep walks the segments backwards, recomputes each segment's stages from
// its checkpoint into a tape (Q and the projected traces u~, uf~ at the start
// of every stage) and runs the stage adjoint kernels (wadg_adjoint_kernels.cuh)
// over the tape in reverse order.  The last segment's tape is written by the
// forward run itself, which computes those stages anyway.  Recompute and adjoint run on two streams
// with two tapes, so that the adjoint of segment s overlaps the recompute of
// segment s-1: the forward kernels fill the SMs the adjoint kernels leave
// idle (the pair kernel's last wave, the small per-element kernels).
//
// The first LSRK coefficient a_0 is 0, so a time step does not depend on the
// residual register left by the previous one: a checkpoint is Q alone.  The
// projected traces are a function of Q (the update kernel's projection), so
// the adjoint driver recomputes them from each checkpoint with the update
// kernel itself (coefficients 0, zero RHS), bit-identical to the values the
// forward run carried.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/wadg.h"
#include "wadg_adjoint_kernels.cuh"
#include "wadg_adjoint_mma.cuh"
#include "wadg_app_impl.h"
#include "wadg_host.h"

namespace wadg_internal {
void set_error(const std::string &msg);  // wadg_capi.cu
}

using namespace wadg;
using wadg_internal::RK4A;
using wadg_internal::RK4B;

struct wadg_adjoint {
  wadg_app *app = nullptr;
  int nsteps = 0, every = 0, nseg = 0;
  size_t nv = 0, nf = 0;  // doubles of a volume / face state array
  Phys phys{};
  double dt = 0.0;
  bool have_forward = false;
  double *ckpt = nullptr;                                      // (nseg + 1) x nv
  // the tape of the last segment (tape (nseg - 1) % 2) holds its stages: the
  // forward run writes it as it goes, so the reverse sweep need not
  // recompute that segment
  bool last_taped = false;
  // two tapes of 5*every stages: the VJP of one segment reads one while the
  // recompute of the previous segment fills the other
  double *tapeQ[2] = {nullptr, nullptr}, *tapeU[2] = {nullptr, nullptr},
         *tapeUf[2] = {nullptr, nullptr};
  cudaStream_t vs = nullptr;  // stream of the stage adjoint kernels
  cudaEvent_t evR[2] = {nullptr, nullptr}, evV[2] = {nullptr, nullptr}, evJoin = nullptr;
  double *Qbar = nullptr, *resbar = nullptr, *rhsbar = nullptr, *sfbar = nullptr;
  double *vbar = nullptr, *vfbar = nullptr;
  double *sQ = nullptr, *sR = nullptr, *suq = nullptr, *suf = nullptr, *srhsQf = nullptr;
  // transposes of the operators the adjoint applies transposed (column-major)
  double *VqPqT = nullptr, *VfPqT = nullptr, *VqLqT = nullptr;
};

namespace {

int jfail(int code, const std::string &msg, cudaError_t e = cudaSuccess) {
  std::string m = msg;
  if (e != cudaSuccess) m += std::string(": ") + cudaGetErrorString(e);
  wadg_internal::set_error(m);
  return code;
}

int ck(cudaError_t e, const char *what) {
  return e == cudaSuccess ? WADG_OK : jfail(WADG_ERR_CUDA, what, e);
}

int num_sms_adj() { return wadg_internal::sm_count(); }

constexpr int pickE(int target, int per) { return per >= target ? 1 : target / per; }

// warps per CTA of the pair VJP kernel: a multiple of its warps per element,
// as many as fit in 227 KB of shared memory, at most 12
template <int DIM, int N, bool CURVED>
constexpr int adjW() {
  using C1 = AdjPairsCfg<DIM, N, CURVED, 2>;
  constexpr int H = C1::H;
  constexpr size_t per_warp = sizeof(double) * (size_t)C1::per_elem * VolTile<DIM, N>::G / H;
  constexpr size_t w = (227 * 1024 - C1::fixed) / per_warp;
  constexpr int wc = w >= 12 ? 12 : (int)w;
  return wc < H ? H : (wc / H) * H;
}

template <class F>
int set_smem(F kern, size_t bytes, bool &done, const char *what) {
  if (done) return WADG_OK;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return jfail(WADG_ERR_CUDA, what, e);
  done = true;
  return WADG_OK;
}

template <int DIM, int N, bool CURVED>
int launch_seed(const wadg_adjoint *j, cudaStream_t s, double b, double dt) {
  const wadg_app *a = j->app;
  using C = AdjMmaCfg<DIM, N, CURVED>;
  auto kern = adj_seed_mma_kernel<DIM, N, CURVED>;
  static wadg_internal::PerDevice<bool> attr;
  if (int r = set_smem(kern, C::smem, attr.here(), "adjoint seed kernel smem attribute")) return r;
  kern<<<(a->K + C::EW - 1) / C::EW, C::threads, C::smem, s>>>(a->K, a->Jq, j->VqPqT, j->VqLqT, b,
                                                               dt, j->Qbar, j->resbar, j->rhsbar,
                                                               j->sfbar);
  return ck(cudaGetLastError(), "adjoint seed kernel");
}

// CTAs of the persistent pair VJP kernel over K elements (batches of C::E)
template <int DIM, int N, bool CURVED>
int pairs_grid(int K) {
  using C = AdjPairsCfg<DIM, N, CURVED, adjW<DIM, N, CURVED>()>;
  const int per_sm = (int)((227 * 1024) / C::smem) > 0 ? (int)((227 * 1024) / C::smem) : 1;
  const int batches = (K + C::E - 1) / C::E;
  return batches < num_sms_adj() * per_sm ? batches : num_sms_adj() * per_sm;
}

template <int DIM, int N, bool CURVED>
int launch_pairs(const wadg_adjoint *j, cudaStream_t s, const double *uq, const double *uf) {
  const wadg_app *a = j->app;
  constexpr int W = adjW<DIM, N, CURVED>();
  using C = AdjPairsCfg<DIM, N, CURVED, W>;
  static_assert(C::smem <= 227 * 1024, "pair VJP kernel does not fit in shared memory");
  auto kern = adj_pairs_kernel<DIM, N, CURVED, W>;
  static wadg_internal::PerDevice<bool> attr;
  if (int r = set_smem(kern, C::smem, attr.here(), "adjoint pair kernel smem attribute")) return r;
  const int grid = pairs_grid<DIM, N, CURVED>(a->K);
  kern<<<grid, C::threads, C::smem, s>>>(a->K, a->vgeo, a->vfgeo, a->fgeo, a->mapPq, a->nrJ,
                                                  a->nsJ, a->ntJ, a->Drq, a->Dsq, a->Dtq, a->VqLq,
                                                  a->VfPq, uq, uf, j->rhsbar, j->sfbar, j->vbar,
                                                  j->vfbar, j->phys);
  return ck(cudaGetLastError(), "adjoint pair kernel");
}

// projection adjoint of a stage; with seed_next, also the seed of the next
// stage of the reverse sweep (coefficient bn, step dtn)
template <int DIM, int N, bool CURVED>
int launch_proj(const wadg_adjoint *j, cudaStream_t s, const double *Qs, double ra, double rb,
                bool seed_next, double bn, double dtn) {
  const wadg_app *a = j->app;
  using C = AdjMmaCfg<DIM, N, CURVED>;
  auto kern = seed_next ? adj_proj_mma_kernel<DIM, N, CURVED, true>
                        : adj_proj_mma_kernel<DIM, N, CURVED, false>;
  static wadg_internal::PerDevice<bool> attr[2];
  if (int r = set_smem(kern, C::smem, attr[seed_next].here(), "adjoint projection kernel smem attribute"))
    return r;
  kern<<<(a->K + C::EW - 1) / C::EW, C::threads, C::smem, s>>>(
      a->K, a->Jq, j->VqPqT, j->VfPqT, Qs, j->vbar, j->vfbar, ra, rb, j->Qbar, j->resbar, j->phys,
      j->VqLqT, bn, dtn, j->rhsbar, j->sfbar);
  return ck(cudaGetLastError(), "adjoint projection kernel");
}

// the three launches of a stage adjoint: seed (unless the previous stage's
// projection kernel already seeded this one), pairs, projection (seeding the
// next stage when there is one)
struct StageStep {
  const double *Qs, *uq, *uf;
  double ra, rb, dt;
  bool seeded;           // rhsbar / sfbar already hold this stage's seed
  bool has_next;         // seed the next stage of the reverse sweep
  double bn, dtn;        // its coefficient and step
};

template <int DIM, int N, bool CURVED>
int stage_adjoint_t(const wadg_adjoint *j, cudaStream_t s, const StageStep &st) {
  int r = st.seeded ? WADG_OK : launch_seed<DIM, N, CURVED>(j, s, st.rb, st.dt);
  if (!r) r = launch_pairs<DIM, N, CURVED>(j, s, st.uq, st.uf);
  if (!r) r = launch_proj<DIM, N, CURVED>(j, s, st.Qs, st.ra, st.rb, st.has_next, st.bn, st.dtn);
  return r;
}

// adjoint of one stage at the taped state, on stream s: updates Qbar and
// resbar in place
int stage_adjoint(const wadg_adjoint *j, cudaStream_t s, const StageStep &st) {
  const wadg_app *a = j->app;
  const int dim = a->p.dim, N = a->p.N;
#define WADG_ADJ_CASE(D_, N_)                                                  \
  if (dim == D_ && N == N_)                                                    \
    return a->curved ? stage_adjoint_t<D_, N_, true>(j, s, st)                 \
                     : stage_adjoint_t<D_, N_, false>(j, s, st);
  WADG_ADJ_CASE(2, 1) WADG_ADJ_CASE(2, 2) WADG_ADJ_CASE(2, 3) WADG_ADJ_CASE(2, 4)
  WADG_ADJ_CASE(3, 1) WADG_ADJ_CASE(3, 2) WADG_ADJ_CASE(3, 3) WADG_ADJ_CASE(3, 4)
#undef WADG_ADJ_CASE
  return jfail(WADG_ERR_UNSUPPORTED, "degree not compiled");
}

}  // namespace

namespace wadg_internal {
// launch shape of the pair VJP kernel (wadg_kernel_shape)
int adj_pairs_shape(int dim, int N, bool curved, int K, int *E, int *grid) {
#define WADG_ADJ_SHAPE(D_, N_)                                                                     \
  if (dim == D_ && N == N_) {                                                                      \
    *E = curved ? AdjPairsCfg<D_, N_, true, adjW<D_, N_, true>()>::E                               \
                : AdjPairsCfg<D_, N_, false, adjW<D_, N_, false>()>::E;                            \
    *grid = curved ? pairs_grid<D_, N_, true>(K) : pairs_grid<D_, N_, false>(K);                   \
    return WADG_OK;                                                                                \
  }
  WADG_ADJ_SHAPE(2, 1) WADG_ADJ_SHAPE(2, 2) WADG_ADJ_SHAPE(2, 3) WADG_ADJ_SHAPE(2, 4)
  WADG_ADJ_SHAPE(3, 1) WADG_ADJ_SHAPE(3, 2) WADG_ADJ_SHAPE(3, 3) WADG_ADJ_SHAPE(3, 4)
#undef WADG_ADJ_SHAPE
  return jfail(WADG_ERR_UNSUPPORTED, "degree not compiled");
}
}  // namespace wadg_internal

namespace {

// the update kernel with a zero RHS and zero coefficients: Q unchanged, res = 0,
// u~ and uf~ = the entropy projection of Q (the traces the next stage reads)
int project(const wadg_app *a, double *Q, double *uq, double *uf, double *res, double fdt = 0.0) {
  const size_t nvb = (size_t)a->K * a->Nq * a->Nf * sizeof(double);
  if (fdt == 0.0) {
    if (int r = ck(cudaMemsetAsync(uq, 0, nvb, a->stream), "memset")) return r;
  }
  if (int r = ck(cudaMemsetAsync(res, 0, nvb, a->stream), "memset")) return r;
  if (a->p.dim == 3)
    return a->curved ? wadg_euler_update_3d_curved(a->ctx, a->K, a->Jq, a->VqPq, a->VfPq, 0.0, 0.0, fdt,
                                                   uq, res, Q, uf)
                     : wadg_euler_update_3d(a->ctx, a->K, a->Jq, a->VqPq, a->VfPq, 0.0, 0.0, fdt, uq,
                                            res, Q, uf);
  return a->curved ? wadg_euler_update_2d_curved(a->ctx, a->K, a->Jq, a->VqPq, a->VfPq, 0.0, 0.0, fdt,
                                                 uq, res, Q, uf)
                   : wadg_euler_update_2d(a->ctx, a->K, a->Jq, a->VqPq, a->VfPq, 0.0, 0.0, fdt, uq,
                                          res, Q, uf);
}

// volume + surface kernels on (uq -> RHS in uq, uf)
int rhs_kernels(const wadg_app *a, double *uq, double *uf, double *rhsQf) {
  int r;
  const int K = a->K;
  if (a->p.dim == 3) {
    r = a->curved ? wadg_euler_vol_3d_curved(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ, a->ntJ,
                                             a->Drq, a->Dsq, a->Dtq, a->Drstq, a->VqLq, a->VfPq,
                                             nullptr, uf, uq, rhsQf)
                  : wadg_euler_vol_3d(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ, a->ntJ, a->Drq,
                                      a->Dsq, a->Dtq, a->Drstq, a->VqLq, a->VfPq, nullptr, uf, uq,
                                      rhsQf);
    if (!r) r = wadg_euler_surf_3d(a->ctx, K, a->fgeo, a->mapPq, a->VqLq, uf, rhsQf, uq);
  } else {
    r = a->curved ? wadg_euler_vol_2d_curved(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ, a->Drq,
                                             a->Dsq, a->VqLq, a->VfPq, nullptr, uf, uq, rhsQf)
                  : wadg_euler_vol_2d(a->ctx, K, a->vgeo, a->vfgeo, a->nrJ, a->nsJ, a->Drq, a->Dsq,
                                      a->VqLq, a->VfPq, nullptr, uf, uq, rhsQf);
    if (!r) r = wadg_euler_surf_2d(a->ctx, K, a->fgeo, a->mapPq, a->VqLq, uf, rhsQf, uq);
  }
  return r;
}

int d2d(double *dst, const double *src, size_t n, cudaStream_t s) {
  return ck(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
}

void free_adj(wadg_adjoint *j) {
  double *bufs[] = {j->ckpt,     j->tapeQ[0], j->tapeU[0], j->tapeUf[0], j->tapeQ[1],
                    j->tapeU[1], j->tapeUf[1], j->Qbar,     j->resbar,    j->rhsbar,
                    j->sfbar,    j->vbar,      j->vfbar,    j->sQ,        j->sR,
                    j->suq,      j->suf,       j->srhsQf,   j->VqPqT,     j->VfPqT,
                    j->VqLqT};
  for (double *b : bufs)
    if (b) cudaFree(b);
  for (cudaEvent_t e : {j->evR[0], j->evR[1], j->evV[0], j->evV[1], j->evJoin})
    if (e) cudaEventDestroy(e);
  if (j->vs) cudaStreamDestroy(j->vs);
}

// run n time steps of size dt from the app's current state on its stream,
// taping (Q, u~, uf~) at the start of every stage into tape b; `last`: run
// the final stage too (the forward run needs its result, a recompute not)
int run_taped(wadg_adjoint *j, int n, int b, double dt, bool last) {
  wadg_app *a = j->app;
  cudaStream_t s = a->stream;
  int r;
  for (int t = 0; t < n; ++t)
    for (int st = 0; st < 5; ++st) {
      const size_t idx = (size_t)t * 5 + st;
      if ((r = d2d(j->tapeQ[b] + idx * j->nv, a->Q, j->nv, s)) ||
          (r = d2d(j->tapeU[b] + idx * j->nv, a->uq[a->cur], j->nv, s)) ||
          (r = d2d(j->tapeUf[b] + idx * j->nf, a->uf[a->cur], j->nf, s)))
        return r;
      if (!last && t == n - 1 && st == 4) break;
      if ((r = wadg_rk_step(a, RK4A[st], RK4B[st], dt))) return r;
    }
  return WADG_OK;
}

// recompute segment `seg` from its checkpoint on the app's stream, taping
// (Q, u~, uf~) at the start of every stage into tape b
int recompute(wadg_adjoint *j, int seg, int b) {
  wadg_app *a = j->app;
  cudaStream_t s = a->stream;
  const int n = std::min(j->every, j->nsteps - seg * j->every);
  int r;
  if ((r = d2d(a->Q, j->ckpt + seg * j->nv, j->nv, s))) return r;
  if ((r = project(a, a->Q, a->uq[a->cur], a->uf[a->cur], a->resQ))) return r;
  return run_taped(j, n, b, j->dt, false);
}

}  // namespace

extern "C" {

int wadg_adjoint_create(wadg_app *app, int nsteps, int every, wadg_adjoint **out) {
  if (!app || !out || nsteps < 0 || every <= 0)
    return jfail(WADG_ERR_INVALID, "invalid argument");
  *out = nullptr;
  if (RK4A[0] != 0.0) return jfail(WADG_ERR_UNSUPPORTED, "first LSRK coefficient must be 0");
  // the surface adjoint gathers the neighbour's contribution: mapPq must pair
  // face nodes both ways (mapPq(mapPq(j)) = j)
  {
    const size_t nmap = (size_t)app->K * app->NfqNf;
    std::vector<uint32_t> m(nmap);
    cudaError_t e = cudaMemcpy(m.data(), app->mapPq, nmap * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return jfail(WADG_ERR_CUDA, "read mapPq", e);
    const size_t blk = (size_t)app->NfqNf * app->Nf;
    for (size_t t = 0; t < nmap; ++t) {
      const size_t k = t / app->NfqNf, jn = t % app->NfqNf;
      const size_t idP = m[t], eP = idP / blk, jP = idP % blk;
      if (jP >= (size_t)app->NfqNf || eP >= (size_t)app->K || m[eP * app->NfqNf + jP] != jn + k * blk)
        return jfail(WADG_ERR_INVALID,
                     "mapPq is not a face pairing (mapPq(mapPq(j)) != j); the adjoint needs a "
                     "conforming mesh");
    }
  }
  wadg_adjoint *j = new wadg_adjoint;
  j->app = app;
  j->nsteps = nsteps;
  j->every = every;
  j->nseg = (nsteps + every - 1) / every;
  j->nv = (size_t)app->K * app->Nq * app->Nf;
  j->nf = (size_t)app->K * app->NfqNf * app->Nf;
  const double g = app->p.gamma;
  j->phys = Phys{g, g - 1.0, 1.0 / (2.0 * (g - 1.0)), app->p.tau, std::log(g - 1.0), 1.0 / (g - 1.0)};
  const size_t nst = (size_t)5 * (size_t)(every < nsteps ? every : (nsteps > 0 ? nsteps : 1));
  const size_t nst2 = j->nseg > 1 ? nst : 0;  // the second tape only when there are two segments
  struct {
    double **p;
    size_t n;
  } al[] = {{&j->ckpt, (j->nseg + 1) * j->nv}, {&j->tapeQ[0], nst * j->nv},
            {&j->tapeU[0], nst * j->nv},        {&j->tapeUf[0], nst * j->nf},
            {&j->tapeQ[1], nst2 * j->nv},       {&j->tapeU[1], nst2 * j->nv},
            {&j->tapeUf[1], nst2 * j->nf},      {&j->Qbar, j->nv},
            {&j->resbar, j->nv},                {&j->rhsbar, j->nv},
            {&j->sfbar, j->nf},                 {&j->vbar, j->nv},
            {&j->vfbar, j->nf},                 {&j->sQ, j->nv},
            {&j->sR, j->nv},                    {&j->suq, j->nv},
            {&j->suf, j->nf},                   {&j->srhsQf, j->nf}};
  for (auto &x : al) {
    if (x.n == 0) continue;
    cudaError_t e = cudaMalloc((void **)x.p, x.n * sizeof(double));
    if (e != cudaSuccess) {
      free_adj(j);
      delete j;
      return jfail(WADG_ERR_CUDA, "cudaMalloc (adjoint tape)", e);
    }
  }
  // transposed operators: one host round trip at creation
  {
    const int Nq = app->Nq, NF = app->NfqNf;
    struct {
      const double *src;
      double **dst;
      int rows, cols;
    } tr[] = {{app->VqPq, &j->VqPqT, Nq, Nq}, {app->VfPq, &j->VfPqT, NF, Nq}, {app->VqLq, &j->VqLqT, Nq, NF}};
    for (auto &x : tr) {
      std::vector<double> A((size_t)x.rows * x.cols), B(A.size());
      cudaError_t e = cudaMemcpy(A.data(), x.src, A.size() * sizeof(double), cudaMemcpyDeviceToHost);
      for (int c = 0; c < x.cols && e == cudaSuccess; ++c)
        for (int r = 0; r < x.rows; ++r) B[c + (size_t)r * x.cols] = A[r + (size_t)c * x.rows];
      if (e == cudaSuccess) e = cudaMalloc((void **)x.dst, B.size() * sizeof(double));
      if (e == cudaSuccess) e = cudaMemcpy(*x.dst, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        free_adj(j);
        delete j;
        return jfail(WADG_ERR_CUDA, "transposed operators", e);
      }
    }
  }
  {
    cudaError_t e = cudaStreamCreateWithFlags(&j->vs, cudaStreamNonBlocking);
    for (cudaEvent_t *ev : {&j->evR[0], &j->evR[1], &j->evV[0], &j->evV[1], &j->evJoin})
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      free_adj(j);
      delete j;
      return jfail(WADG_ERR_CUDA, "adjoint stream/events", e);
    }
  }
  *out = j;
  return WADG_OK;
}

int wadg_adjoint_destroy(wadg_adjoint *j) {
  if (!j) return WADG_OK;
  // does not touch the app, which may already be gone; cudaFree waits for
  // the device work that uses the buffers
  free_adj(j);
  delete j;
  return WADG_OK;
}

int wadg_adjoint_forward(wadg_adjoint *j, const double *Q0, double dt, double *QT) {
  if (!j || !Q0) return jfail(WADG_ERR_INVALID, "invalid argument");
  wadg_app *a = j->app;
  cudaStream_t s = a->stream;
  int r;
  j->last_taped = false;
  if ((r = d2d(a->Q, Q0, j->nv, s))) return r;
  if ((r = project(a, a->Q, a->uq[a->cur], a->uf[a->cur], a->resQ))) return r;
  for (int seg = 0; seg < j->nseg; ++seg) {
    if ((r = d2d(j->ckpt + seg * j->nv, a->Q, j->nv, s))) return r;
    const int n = std::min(j->every, j->nsteps - seg * j->every);
    // the last segment runs stage by stage into its tape (the states at the
    // start of its stages are the ones a recompute from its checkpoint
    // would produce, bit for bit); the others as graph-replayed steps
    if (seg == j->nseg - 1)
      r = run_taped(j, n, seg % 2, dt, true);
    else
      r = wadg_rk_run(a, dt, n, 1);
    if (r) return r;
  }
  j->last_taped = j->nseg > 0;
  if ((r = d2d(j->ckpt + j->nseg * j->nv, a->Q, j->nv, s))) return r;
  if (QT && (r = d2d(QT, a->Q, j->nv, s))) return r;
  j->dt = dt;
  j->have_forward = true;
  return WADG_OK;
}

int wadg_adjoint_reverse(wadg_adjoint *j, const double *QbarT, double *Qbar0) {
  if (!j || !QbarT || !Qbar0) return jfail(WADG_ERR_INVALID, "invalid argument");
  if (!j->have_forward) return jfail(WADG_ERR_INVALID, "wadg_adjoint_forward has not run");
  wadg_app *a = j->app;
  // two streams: the app's stream recomputes segments (forward kernels), the
  // adjoint's stream runs the stage adjoints; segment seg's adjoint overlaps
  // the recompute of segment seg-1 into the other tape
  cudaStream_t sr = a->stream, sv = j->vs;
  const double dt = j->dt;
  int r;
  // the adjoint stream starts after what the caller queued on the app's stream
  if ((r = ck(cudaEventRecord(j->evJoin, sr), "event")) ||
      (r = ck(cudaStreamWaitEvent(sv, j->evJoin, 0), "event")))
    return r;
  if ((r = d2d(j->Qbar, QbarT, j->nv, sv))) return r;
  if ((r = ck(cudaMemsetAsync(j->resbar, 0, j->nv * sizeof(double), sv), "memset"))) return r;
  const int last = j->nseg - 1;
  if (last >= 0) {
    // the forward run taped the last segment, unless a reverse sweep since
    // has refilled that tape with another segment
    if (!j->last_taped && (r = recompute(j, last, last % 2))) return r;
    if ((r = ck(cudaEventRecord(j->evR[last % 2], sr), "event"))) return r;
  }
  // with three segments or more, segment last - 2 refills the last one's tape
  j->last_taped = j->nseg > 0 && j->nseg <= 2;
  for (int seg = last; seg >= 0; --seg) {
    const int b = seg % 2;
    const int n = std::min(j->every, j->nsteps - seg * j->every);
    if ((r = ck(cudaStreamWaitEvent(sv, j->evR[b], 0), "event"))) return r;
    for (int idx = n * 5 - 1; idx >= 0; --idx) {
      const int st = idx % 5;
      // the stage before this one in the run (the next of the reverse sweep)
      // has coefficient RK4B[(st + 4) % 5]; the sweep's last stage seeds none
      const bool first = seg == last && idx == n * 5 - 1, final = seg == 0 && idx == 0;
      const StageStep step{j->tapeQ[b] + idx * j->nv, j->tapeU[b] + idx * j->nv,
                           j->tapeUf[b] + idx * j->nf, RK4A[st], RK4B[st], dt,
                           !first, !final, RK4B[(st + 4) % 5], dt};
      if ((r = stage_adjoint(j, sv, step))) return r;
    }
    if ((r = ck(cudaEventRecord(j->evV[b], sv), "event"))) return r;
    if (seg > 0) {
      const int nb = (seg - 1) % 2;  // the tape segment seg+1's adjoint read
      if (seg < last && (r = ck(cudaStreamWaitEvent(sr, j->evV[nb], 0), "event"))) return r;
      if ((r = recompute(j, seg - 1, nb))) return r;
      if ((r = ck(cudaEventRecord(j->evR[nb], sr), "event"))) return r;
    }
  }
  if ((r = d2d(Qbar0, j->Qbar, j->nv, sv))) return r;
  // leave the app at the final state of the forward run, and join the
  // adjoint stream into the app's stream
  if ((r = d2d(a->Q, j->ckpt + j->nseg * j->nv, j->nv, sr))) return r;
  if ((r = project(a, a->Q, a->uq[a->cur], a->uf[a->cur], a->resQ))) return r;
  if ((r = ck(cudaEventRecord(j->evJoin, sv), "event")) ||
      (r = ck(cudaStreamWaitEvent(sr, j->evJoin, 0), "event")))
    return r;
  return WADG_OK;
}

int wadg_adjoint_rhs(wadg_adjoint *j, const double *Q, double *R) {
  if (!j || !Q || !R) return jfail(WADG_ERR_INVALID, "invalid argument");
  const wadg_app *a = j->app;
  cudaStream_t s = a->stream;
  int r;
  if ((r = d2d(j->sQ, Q, j->nv, s))) return r;
  if ((r = project(a, j->sQ, j->suq, j->suf, j->sR))) return r;
  if ((r = rhs_kernels(a, j->suq, j->suf, j->srhsQf))) return r;
  // res = 0 * res + 1 * Minv rhs: the update kernel's inverse mass, exactly
  if ((r = project(a, j->sQ, j->suq, j->suf, j->sR, 1.0))) return r;
  return d2d(R, j->sR, j->nv, s);
}

int wadg_adjoint_rhs_vjp(wadg_adjoint *j, const double *Q, const double *w, double *Qbar) {
  if (!j || !Q || !w || !Qbar) return jfail(WADG_ERR_INVALID, "invalid argument");
  const wadg_app *a = j->app;
  cudaStream_t s = a->stream;
  int r;
  if ((r = d2d(j->sQ, Q, j->nv, s))) return r;
  if ((r = project(a, j->sQ, j->suq, j->suf, j->sR))) return r;
  // a stage with a = b = 0, dt = 1 and incoming adjoints (Qbar', resbar') =
  // (0, w) leaves Qbar = (dR/dQ)^T w
  if ((r = ck(cudaMemsetAsync(j->Qbar, 0, j->nv * sizeof(double), s), "memset"))) return r;
  if ((r = d2d(j->resbar, w, j->nv, s))) return r;
  const StageStep step{j->sQ, j->suq, j->suf, 0.0, 0.0, 1.0, false, false, 0.0, 0.0};
  if ((r = stage_adjoint(j, s, step))) return r;
  return d2d(Qbar, j->Qbar, j->nv, s);
}

}  // extern "C"
