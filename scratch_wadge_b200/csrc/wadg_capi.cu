// C ABI of the library: context, kernel entry points (one per OKL kernel of the
// reference), and the host driver (app / rk_step / rk_run).  See include/wadg.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wadg.h"
#include "wadg_host.h"
#include "wadg_diag.cuh"
#include "wadg_surf_mma.cuh"
#include "wadg_update_mma.cuh"
#include "wadg_stage.cuh"
#include "wadg_vol.cuh"

using namespace wadg;

struct wadg_ctx {
  int dim, N, Nq, Nfq, Nfaces;
  Phys phys;
  cudaStream_t stream;
  int vol_warps = 0;  // warps per CTA of the pair volume kernel; 0 = the default
  int vol_rows = 0;   // rows per lane of its node-to-thread map; 0 = the default
};

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) return fail(WADG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return WADG_OK;
}

int after_launch(const char *name) { return cuda_check(cudaGetLastError(), name); }

// warps per CTA of the pair-scheduled volume kernel: an even count, as many
// as fit in 227 KB of shared memory, at most `cap`
template <int DIM, int N, bool CURVED, int RR = 0>
constexpr int volpairsW_fit(int cap) {
  using C = VolPairsCfg<DIM, N, CURVED, 2, RR>;
  constexpr size_t per_warp = C::per_elem * VolTile<DIM, N, RR>::G / C::H;
  constexpr size_t w = (227 * 1024 - C::fixed) / per_warp;
  return w >= (size_t)cap ? cap : (w < 2 ? 2 : (int)(w & ~size_t(1)));
}

// the default shape: at most 12 warps (register budget ~170 per thread)
template <int DIM, int N, bool CURVED>
constexpr int volpairsW() {
  return volpairsW_fit<DIM, N, CURVED>(12);
}

int num_sms() { return wadg_internal::sm_count(); }

// CTAs of a persistent kernel over K elements in batches of E: one per batch,
// at most as many as are resident at once (shared memory per CTA `smem`); CTA
// b takes batches b, b + grid, b + 2 grid, ...
int persistent_grid(int K, int E, size_t smem) {
  const int per_sm = (int)((227 * 1024) / smem) > 0 ? (int)((227 * 1024) / smem) : 1;
  const int batches = (K + E - 1) / E;
  return batches < num_sms() * per_sm ? batches : num_sms() * per_sm;
}

// candidate CTA shapes of the pair volume kernel (warps per CTA; elements per
// CTA = warps / 2 * 32 / lanes per element): the default, then two and four
// warps fewer.  In 2D the second is 16 warps where they fit: four fields need
// fewer registers (128 per thread), and large 2D meshes run fastest at 16,
// small ones at 8
template <int DIM, int N, bool CURVED>
constexpr int volpairsW_cand(int i) {
  constexpr int W0 = volpairsW<DIM, N, CURVED>();
  constexpr int Wbig = DIM == 2 ? volpairsW_fit<DIM, N, CURVED>(16) : W0;
  if (i == 1 && Wbig > W0) return Wbig;
  return i == 0 ? W0 : (W0 - 2 * i >= 2 ? W0 - 2 * i : 0);
}

// The other node-to-thread maps: half and twice the default's lanes per
// element (about twice and half its rows per lane), each given to the kernels
// as RR = rows per lane.  A map is a candidate when it has as many lanes as
// intended (2 to 32), keeps a face node per lane in each warp's face half,
// pads no more node slots than the default, holds at most 4 rows per lane and
// fits a CTA of at least 4 warps in shared memory.  (Six rows per lane need
// more than 255 registers in 3D: 140-530 bytes of spills at every degree.)
// alt_rows<DIM, N, CURVED, j>(), j = 0 (half the lanes) or 1 (twice): its RR,
// or 0 when it is no candidate; its warps per CTA: the most that fit, up to 16
// with at most two rows per lane, else 8 (up to 255 registers per thread).
template <int DIM, int N, int RR>
struct NodeMap {  // VolTile's arithmetic, without its static checks
  static constexpr int Nq = Elem<DIM, N>::Nq;
  static constexpr int Lraw = RR > 0 ? (Nq + RR - 1) / RR : (Nq + 2) / 3;
  static constexpr int L = Lraw <= 1 ? 1 : Lraw <= 2 ? 2 : Lraw <= 4 ? 4 : Lraw <= 8 ? 8 : Lraw <= 16 ? 16 : 32;
  static constexpr int R = (Nq + L - 1) / L;
  static constexpr int pad = L * R - Nq;
};
template <int DIM, int N, bool CURVED, int RR>
constexpr int alt_warps() {
  return volpairsW_fit<DIM, N, CURVED, RR>(NodeMap<DIM, N, RR>::R <= 2 ? 16 : 8);
}
template <int DIM, int N, bool CURVED, int j>
constexpr int alt_rows() {
  constexpr int L0 = NodeMap<DIM, N, 0>::L, Lt = j == 0 ? L0 / 2 : 2 * L0;
  if constexpr (Lt < 2 || Lt > 32) {
    return 0;
  } else {
    constexpr int RR = (Elem<DIM, N>::Nq + Lt - 1) / Lt;
    using M = NodeMap<DIM, N, RR>;
    // (nf1: the smaller face half, the second warp's when there are two)
    constexpr int nf1 = Elem<DIM, N>::NfqNf / 2;
    constexpr int faces = nf1 >= M::L ? nf1 : Elem<DIM, N>::NfqNf;
    if constexpr (M::L != Lt || faces < M::L || M::pad > NodeMap<DIM, N, 0>::pad || M::R > 4) {
      return 0;
    } else {
      constexpr int W = alt_warps<DIM, N, CURVED, RR>();
      return (W >= 4 && VolPairsCfg<DIM, N, CURVED, W, RR>::smem <= 227 * 1024) ? RR : 0;
    }
  }
}

// SURF: the volume + surface kernel (rhsQf unused; fgeo, mapPq read)
template <int DIM, int N, bool CURVED, int W, bool SURF = false, int RR = 0>
int launch_vol_pairs_w(const wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                       const double *nrJ, const double *nsJ, const double *ntJ, const double *Drq,
                       const double *Dsq, const double *Dtq, const double *VqLq, const double *VfPq,
                       const double *Qf, double *rhsQ, double *rhsQf,
                       const double *fgeo = nullptr, const uint32_t *mapPq = nullptr,
                       const int *blist = nullptr, const int *nb = nullptr) {
  using C = VolPairsCfg<DIM, N, CURVED, W, RR>;
  static_assert(C::smem_vol <= 227 * 1024, "pair-scheduled volume kernel does not fit in shared memory");
  auto kern = vol_pairs_kernel<DIM, N, CURVED, W, SURF, RR>;
  static wadg_internal::PerDevice<bool> attr;
  if (!attr.here()) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_vol);
    if (e != cudaSuccess) return cuda_check(e, "volume kernel smem attribute");
    attr.here() = true;
  }
  const int grid = persistent_grid(K, C::E, C::smem_vol);
  kern<<<grid, C::threads, C::smem_vol, c->stream>>>(K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq,
                                                      VqLq, VfPq, Qf, rhsQ, rhsQf, c->phys, fgeo,
                                                      mapPq, blist, nb);
  return after_launch(SURF ? "volume + surface kernel" : "volume kernel");
}

// the volume + surface kernel in the context's CTA shape (wadg_ctx_set_vol_warps)
template <int DIM, int N, bool CURVED>
int launch_volsurf(const wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                   const double *fgeo, const uint32_t *mapPq, const double *nrJ,
                   const double *nsJ, const double *ntJ, const double *Drq, const double *Dsq,
                   const double *Dtq, const double *VqLq, const double *VfPq, const double *Qf,
                   double *rhsQ, const int *blist = nullptr, const int *nb = nullptr) {
  constexpr int A0 = alt_rows<DIM, N, CURVED, 0>(), A1 = alt_rows<DIM, N, CURVED, 1>();
  if constexpr (A0 > 0)
    if (c->vol_rows == A0)
      return launch_vol_pairs_w<DIM, N, CURVED, alt_warps<DIM, N, CURVED, A0>(), true, A0>(
          c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, nullptr, fgeo,
          mapPq, blist, nb);
  if constexpr (A1 > 0)
    if (c->vol_rows == A1)
      return launch_vol_pairs_w<DIM, N, CURVED, alt_warps<DIM, N, CURVED, A1>(), true, A1>(
          c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, nullptr, fgeo,
          mapPq, blist, nb);
  constexpr int W1 = volpairsW_cand<DIM, N, CURVED>(1), W2 = volpairsW_cand<DIM, N, CURVED>(2);
  if (W1 && c->vol_warps == W1)
    return launch_vol_pairs_w<DIM, N, CURVED, (W1 ? W1 : 2), true>(
        c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, nullptr, fgeo, mapPq,
        blist, nb);
  if (W2 && c->vol_warps == W2)
    return launch_vol_pairs_w<DIM, N, CURVED, (W2 ? W2 : 2), true>(
        c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, nullptr, fgeo, mapPq,
        blist, nb);
  return launch_vol_pairs_w<DIM, N, CURVED, volpairsW<DIM, N, CURVED>(), true>(
      c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, nullptr, fgeo, mapPq,
      blist, nb);
}

// the context's CTA shape (wadg_ctx_set_vol_warps), else the default
template <int DIM, int N, bool CURVED>
int launch_vol_pairs(const wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                     const double *nrJ, const double *nsJ, const double *ntJ, const double *Drq,
                     const double *Dsq, const double *Dtq, const double *VqLq, const double *VfPq,
                     const double *Qf, double *rhsQ, double *rhsQf) {
  constexpr int A0 = alt_rows<DIM, N, CURVED, 0>(), A1 = alt_rows<DIM, N, CURVED, 1>();
  if constexpr (A0 > 0)
    if (c->vol_rows == A0)
      return launch_vol_pairs_w<DIM, N, CURVED, alt_warps<DIM, N, CURVED, A0>(), false, A0>(
          c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf);
  if constexpr (A1 > 0)
    if (c->vol_rows == A1)
      return launch_vol_pairs_w<DIM, N, CURVED, alt_warps<DIM, N, CURVED, A1>(), false, A1>(
          c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf);
  constexpr int W1 = volpairsW_cand<DIM, N, CURVED>(1), W2 = volpairsW_cand<DIM, N, CURVED>(2);
  if (W1 && c->vol_warps == W1)
    return launch_vol_pairs_w<DIM, N, CURVED, (W1 ? W1 : 2)>(c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq,
                                                             Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf);
  if (W2 && c->vol_warps == W2)
    return launch_vol_pairs_w<DIM, N, CURVED, (W2 ? W2 : 2)>(c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq,
                                                             Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf);
  return launch_vol_pairs_w<DIM, N, CURVED, volpairsW<DIM, N, CURVED>()>(
      c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf);
}

template <int DIM, int N, bool CURVED>
int vol_warps_candidates(int *out) {
  int n = 0;
  for (int i = 0; i < 3; ++i)
    if (int w = volpairsW_cand<DIM, N, CURVED>(i)) out[n++] = w;
  return n;
}

// every compiled (warps, rows) shape: the default map's warps, then the
// other maps (rows > 0)
template <int DIM, int N, bool CURVED>
int vol_shapes(int *warps, int *rows) {
  int n = vol_warps_candidates<DIM, N, CURVED>(warps);
  for (int i = 0; i < n; ++i) rows[i] = 0;
  constexpr int A0 = alt_rows<DIM, N, CURVED, 0>(), A1 = alt_rows<DIM, N, CURVED, 1>();
  if constexpr (A0 > 0) {
    warps[n] = alt_warps<DIM, N, CURVED, A0>();
    rows[n++] = A0;
  }
  if constexpr (A1 > 0) {
    warps[n] = alt_warps<DIM, N, CURVED, A1>();
    rows[n++] = A1;
  }
  return n;
}

template <int DIM, int N, bool CURVED>
int launch_stage(const wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                 const double *fgeo, const uint32_t *mapPq, const double *nrJ, const double *nsJ,
                 const double *ntJ, const double *Drq, const double *Dsq, const double *Dtq,
                 const double *VqLq, const double *VfPq, const double *VqPq, const double *Jq,
                 double fa, double fb, double fdt, const double *uq, const double *uf, double *Q,
                 double *resQ, double *uq_out, double *uf_out) {
  if (uf_out == uf) return fail(WADG_ERR_INVALID, "stage: uf_out must not be uf");
  constexpr int W = stage_warps<DIM, N, CURVED, volpairsW<DIM, N, CURVED>()>();
  using C = VolPairsCfg<DIM, N, CURVED, W>;
  auto kern = stage_kernel<DIM, N, CURVED, W>;
  static wadg_internal::PerDevice<bool> attr;
  if (!attr.here()) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_vol);
    if (e != cudaSuccess) return cuda_check(e, "stage kernel smem attribute");
    attr.here() = true;
  }
  const int grid = persistent_grid(K, C::E, C::smem_vol);
  kern<<<grid, C::threads, C::smem_vol, c->stream>>>(K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ, Drq,
                                                  Dsq, Dtq, VqLq, VfPq, VqPq, Jq, fa, fb, fdt, uq,
                                                  uf, Q, resQ, uq_out, uf_out, c->phys);
  return after_launch("stage kernel");
}

template <int DIM, int N>
int launch_surf(const wadg_ctx *c, int K, const double *fgeo, const uint32_t *mapPq,
                const double *VqLq, const double *Qf, const double *rhsQf, double *rhsQ) {
  using C = SurfMmaCfg<DIM, N>;
  surf_mma_kernel<DIM, N><<<(K + C::EW - 1) / C::EW, C::threads, C::smem, c->stream>>>(
      K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ, c->phys);
  return after_launch("surf kernel");
}

// CTAs of the persistent update kernel: one per group of C::EW elements, at
// most as many as are resident at once (occupancy, cached per device)
template <int DIM, int N, bool CURVED>
int update_grid(int K, int *grid) {
  using C = UpdMmaCfg<DIM, N, CURVED>;
  auto kern = update_mma_kernel<DIM, N, CURVED>;
  static wadg_internal::PerDevice<int> per_sm_dev;
  int &per_sm = per_sm_dev.here();
  if (!per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
    if (e != cudaSuccess) return cuda_check(e, "update kernel smem attribute");
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, C::threads, C::smem);
    if (e != cudaSuccess) return cuda_check(e, "update kernel occupancy");
    per_sm = n < 1 ? 1 : n;
  }
  const int ctas = (K + C::EW - 1) / C::EW;
  *grid = ctas < num_sms() * per_sm ? ctas : num_sms() * per_sm;
  return WADG_OK;
}

// the launch shape of one kernel for K elements (wadg_kernel_shape)
template <int DIM, int N, bool CURVED, int W, int RR = 0>
void vol_shape(int K, int *E, int *grid) {
  using C = VolPairsCfg<DIM, N, CURVED, W, RR>;
  *E = C::E;
  *grid = persistent_grid(K, C::E, C::smem_vol);
}

template <int DIM, int N, bool CURVED>
int kernel_shape(const wadg_ctx *c, int kernel, int K, int *E, int *grid) {
  constexpr int W1 = volpairsW_cand<DIM, N, CURVED>(1), W2 = volpairsW_cand<DIM, N, CURVED>(2);
  constexpr int A0 = alt_rows<DIM, N, CURVED, 0>(), A1 = alt_rows<DIM, N, CURVED, 1>();
  if ((kernel == WADG_KERNEL_VOL || kernel == WADG_KERNEL_VOLSURF) && c->vol_rows) {
    if constexpr (A0 > 0)
      if (c->vol_rows == A0) vol_shape<DIM, N, CURVED, alt_warps<DIM, N, CURVED, A0>(), A0>(K, E, grid);
    if constexpr (A1 > 0)
      if (c->vol_rows == A1) vol_shape<DIM, N, CURVED, alt_warps<DIM, N, CURVED, A1>(), A1>(K, E, grid);
    return WADG_OK;
  }
  switch (kernel) {
    case WADG_KERNEL_VOL:
      if (W1 && c->vol_warps == W1) vol_shape<DIM, N, CURVED, (W1 ? W1 : 2)>(K, E, grid);
      else if (W2 && c->vol_warps == W2) vol_shape<DIM, N, CURVED, (W2 ? W2 : 2)>(K, E, grid);
      else vol_shape<DIM, N, CURVED, volpairsW<DIM, N, CURVED>()>(K, E, grid);
      return WADG_OK;
    case WADG_KERNEL_SURF:
      *E = SurfMmaCfg<DIM, N>::EW;
      *grid = (K + *E - 1) / *E;
      return WADG_OK;
    case WADG_KERNEL_UPDATE:
      *E = UpdMmaCfg<DIM, N, CURVED>::EW;
      return update_grid<DIM, N, CURVED>(K, grid);
    case WADG_KERNEL_VOLSURF:  // the same CTA shapes as the volume kernel
      if (W1 && c->vol_warps == W1) vol_shape<DIM, N, CURVED, (W1 ? W1 : 2)>(K, E, grid);
      else if (W2 && c->vol_warps == W2) vol_shape<DIM, N, CURVED, (W2 ? W2 : 2)>(K, E, grid);
      else vol_shape<DIM, N, CURVED, volpairsW<DIM, N, CURVED>()>(K, E, grid);
      return WADG_OK;
    case WADG_KERNEL_ADJ_PAIRS:
      return wadg_internal::adj_pairs_shape(DIM, N, CURVED, K, E, grid);
    case WADG_KERNEL_STAGE: {
      using C = VolPairsCfg<DIM, N, CURVED, stage_warps<DIM, N, CURVED, volpairsW<DIM, N, CURVED>()>()>;
      *E = C::E;
      *grid = persistent_grid(K, C::E, C::smem_vol);
      return WADG_OK;
    }
  }
  return fail(WADG_ERR_INVALID, "unknown kernel %d", kernel);
}

template <int DIM, int N, bool CURVED>
int launch_update(const wadg_ctx *c, int K, const double *Jq, const double *VqPq,
                  const double *VfPq, double fa, double fb, double fdt, double *rhsQ,
                  double *resQ, double *Q, double *Qf, const double *dtK = nullptr,
                  const int *glist = nullptr, const int *ng = nullptr) {
  using C = UpdMmaCfg<DIM, N, CURVED>;
  static_assert(C::smem <= 227 * 1024, "update kernel does not fit in shared memory");
  auto kern = update_mma_kernel<DIM, N, CURVED>;
  int grid = 0;
  if (int r = update_grid<DIM, N, CURVED>(K, &grid)) return r;
  kern<<<grid, C::threads, C::smem, c->stream>>>(K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q,
                                                 Qf, c->phys, dtK, glist, ng);
  return after_launch("update kernel");
}

// (dim, N) -> template instantiation
#define WADG_DISPATCH(c, CALL)                                 \
  do {                                                         \
    if ((c)->dim == 2) {                                       \
      switch ((c)->N) {                                        \
        case 1: { constexpr int D_ = 2, N_ = 1; CALL; }        \
        case 2: { constexpr int D_ = 2, N_ = 2; CALL; }        \
        case 3: { constexpr int D_ = 2, N_ = 3; CALL; }        \
        case 4: { constexpr int D_ = 2, N_ = 4; CALL; }        \
      }                                                        \
    } else {                                                   \
      switch ((c)->N) {                                        \
        case 1: { constexpr int D_ = 3, N_ = 1; CALL; }        \
        case 2: { constexpr int D_ = 3, N_ = 2; CALL; }        \
        case 3: { constexpr int D_ = 3, N_ = 3; CALL; }        \
        case 4: { constexpr int D_ = 3, N_ = 4; CALL; }        \
      }                                                        \
    }                                                          \
    return fail(WADG_ERR_UNSUPPORTED, "degree not compiled");  \
  } while (0)

int check_ctx(const wadg_ctx *c, int dim, int K) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  if (c->dim != dim) return fail(WADG_ERR_INVALID, "context is %dD, kernel is %dD", c->dim, dim);
  if (K < 0) return fail(WADG_ERR_INVALID, "K < 0");
  return WADG_OK;
}

bool any_null(std::initializer_list<const void *> ps) {
  for (auto p : ps)
    if (!p) return true;
  return false;
}

template <int DIM, int N> bool sizes_match(const wadg_params *p) {
  using El = Elem<DIM, N>;
  return p->Nq == El::Nq && p->Nfq == El::Nfq && p->Nfaces == El::Nfaces;
}

}  // namespace

namespace wadg_internal {
void set_error(const std::string &msg) { g_err = msg; }
}  // namespace wadg_internal

// dimension and face-point count of a context (used by wadg_noalloc.cu)
int wadg_ctx_sizes(const wadg_ctx *c, int *dim, int *NfqNf) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  *dim = c->dim;
  *NfqNf = c->Nfq * c->Nfaces;
  return WADG_OK;
}

// the stream a context's kernels run on (used by wadg_noalloc.cu)
cudaStream_t wadg_ctx_stream(const wadg_ctx *c) { return c ? c->stream : nullptr; }

namespace wadg_internal {
// The ensemble's stage kernels over work lists (wadg_ensemble.cu): the volume
// + surface kernel over the volume batches blist[0 .. *nb) (ascending batch
// indices of elems_per_batch(WADG_KERNEL_VOLSURF) elements), then the update
// over the groups glist[0 .. *ng) with the step of element k in dtK[k].
int volsurf_list(const wadg_ctx *c, int K, int curved, const double *vgeo, const double *vfgeo,
                 const double *fgeo, const uint32_t *mapPq, const double *nrJ, const double *nsJ,
                 const double *ntJ, const double *Drq, const double *Dsq, const double *Dtq,
                 const double *VqLq, const double *VfPq, const double *Qf, double *rhsQ,
                 const int *blist, const int *nb) {
  if (int r = check_ctx(c, c ? c->dim : 0, K)) return r;
  if (K == 0) return WADG_OK;
  if (curved)
    WADG_DISPATCH(c, return (launch_volsurf<D_, N_, true>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ,
                                                           Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, blist,
                                                           nb)));
  WADG_DISPATCH(c, return (launch_volsurf<D_, N_, false>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ,
                                                          Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, blist,
                                                          nb)));
}

int update_list(const wadg_ctx *c, int K, int curved, const double *Jq, const double *VqPq,
                const double *VfPq, double fa, double fb, const double *dtK, double *rhsQ,
                double *resQ, double *Q, double *Qf, const int *glist, const int *ng) {
  if (int r = check_ctx(c, c ? c->dim : 0, K)) return r;
  if (K == 0) return WADG_OK;
  if (curved)
    WADG_DISPATCH(c, return (launch_update<D_, N_, true>(c, K, Jq, VqPq, VfPq, fa, fb, 0.0, rhsQ, resQ,
                                                          Q, Qf, dtK, glist, ng)));
  WADG_DISPATCH(c, return (launch_update<D_, N_, false>(c, K, Jq, VqPq, VfPq, fa, fb, 0.0, rhsQ, resQ,
                                                         Q, Qf, dtK, glist, ng)));
}
}  // namespace wadg_internal

// per-element integrals (wadg_euler_3d_compute_aux, wadg_element_entropy)
template <int DIM, int N, bool ENTROPY>
int launch_integral(const wadg_ctx *c, int K, const double *Jq, const double *wq, const double *Q,
                    double *out) {
  const size_t threads = (size_t)K * 32;
  element_integral_kernel<DIM, N, ENTROPY><<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(
      K, Jq, wq, Q, out, c->phys);
  return after_launch("element integral kernel");
}

// halo pack: slot g of the send buffer gets the face trace at field-strided
// index src[g] (all fields), laid out as the receiver's ghost pseudo-elements
// (slot g -> face point g % NF of pseudo-element g / NF); padding slots
// (src = 0xffffffff) and indices past the end of Qf get zeros
__global__ void halo_pack_kernel(int n, int NF, int Nf, size_t nQf, const uint32_t *__restrict__ src,
                                 const double *__restrict__ Qf, double *__restrict__ buf) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const uint32_t sidx = src[g];
  const bool ok = sidx != 0xffffffffu && (size_t)sidx + (size_t)(Nf - 1) * NF < nQf;
  double *out = buf + (size_t)(g / NF) * NF * Nf + g % NF;
  for (int f = 0; f < Nf; ++f) out[(size_t)f * NF] = ok ? Qf[(size_t)sidx + (size_t)f * NF] : 0.0;
}

// failure detection: one thread per node of Q [K][Nf][Nq]; a node is bad when
// a field is not finite, rho <= 0 or the pressure is <= 0.  work[0] counts the
// bad nodes, work[1] keeps the smallest bad flat index k * Nq + i
template <int DIM>
__global__ void check_state_kernel(int K, int Nq, const double *__restrict__ Q, double gm1,
                                   int *__restrict__ work) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)K * Nq) return;
  const int k = (int)(t / Nq), i = (int)(t % Nq);
  const double *q = Q + (size_t)k * Nq * (DIM + 2) + i;
  const double rho = q[0], E = q[(size_t)(DIM + 1) * Nq];
  bool finite = isfinite(rho) && isfinite(E);
  double m2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double m = q[(size_t)(1 + d) * Nq];
    finite = finite && isfinite(m);
    m2 = fma(m, m, m2);
  }
  const double p = gm1 * (E - 0.5 * m2 / rho);
  if (!finite || !(rho > 0.0) || !(p > 0.0)) {
    atomicAdd(&work[0], 1);
    atomicMin(&work[1], (int)t);
  }
}

template <int DIM, int N, bool CURVED>
int launch_entropy_rhs(const wadg_ctx *c, int K, const double *wq, const double *Jq,
                       const double *VqPq, const double *Q, const double *rhs, double *out) {
  entropy_rhs_kernel<DIM, N, CURVED><<<(K + 7) / 8, 256, 0, c->stream>>>(K, wq, Jq, VqPq, Q, rhs,
                                                                         out, c->phys);
  return after_launch("entropy RHS kernel");
}

extern "C" {

const char *wadg_last_error(void) { return g_err.c_str(); }

int wadg_supported_degrees(int dim) { return (dim == 2 || dim == 3) ? 0x1e : 0; }

int wadg_ctx_create(const wadg_params *p, wadg_ctx **out) {
  if (!p || !out) return fail(WADG_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->dim != 2 && p->dim != 3) return fail(WADG_ERR_INVALID, "dim must be 2 or 3");
  bool ok = false;
  if (p->dim == 2) {
    switch (p->N) {
      case 1: ok = sizes_match<2, 1>(p); break;
      case 2: ok = sizes_match<2, 2>(p); break;
      case 3: ok = sizes_match<2, 3>(p); break;
      case 4: ok = sizes_match<2, 4>(p); break;
      default: return fail(WADG_ERR_UNSUPPORTED, "2D degree %d not compiled", p->N);
    }
  } else {
    switch (p->N) {
      case 1: ok = sizes_match<3, 1>(p); break;
      case 2: ok = sizes_match<3, 2>(p); break;
      case 3: ok = sizes_match<3, 3>(p); break;
      case 4: ok = sizes_match<3, 4>(p); break;
      default: return fail(WADG_ERR_UNSUPPORTED, "3D degree %d not compiled", p->N);
    }
  }
  if (!ok)
    return fail(WADG_ERR_UNSUPPORTED, "sizes Nq=%d Nfq=%d Nfaces=%d do not match degree %d", p->Nq,
                p->Nfq, p->Nfaces, p->N);
  if (!(p->gamma > 1.0)) return fail(WADG_ERR_INVALID, "gamma must be > 1");
  wadg_ctx *c = new wadg_ctx;
  c->dim = p->dim;
  c->N = p->N;
  c->Nq = p->Nq;
  c->Nfq = p->Nfq;
  c->Nfaces = p->Nfaces;
  c->phys.gamma = p->gamma;
  c->phys.gm1 = p->gamma - 1.0;
  c->phys.cbeta = 1.0 / (2.0 * (p->gamma - 1.0));
  c->phys.tau = p->tau;
  c->phys.lgm1 = log(p->gamma - 1.0);
  c->phys.igm1 = 1.0 / (p->gamma - 1.0);
  c->stream = (cudaStream_t)p->stream;
  *out = c;
  return WADG_OK;
}

int wadg_ctx_destroy(wadg_ctx *ctx) {
  delete ctx;
  return WADG_OK;
}

int wadg_ctx_set_stream(wadg_ctx *ctx, void *stream) {
  if (!ctx) return fail(WADG_ERR_INVALID, "null context");
  ctx->stream = (cudaStream_t)stream;
  return WADG_OK;
}

int wadg_vol_warps_candidates(const wadg_ctx *ctx, int curved, int *out) {
  if (!ctx || !out) return -fail(WADG_ERR_INVALID, "null argument");
  const wadg_ctx *c = ctx;
  if (curved) {
    WADG_DISPATCH(c, return (vol_warps_candidates<D_, N_, true>(out)));
  } else {
    WADG_DISPATCH(c, return (vol_warps_candidates<D_, N_, false>(out)));
  }
}

int wadg_ctx_set_vol_warps(wadg_ctx *ctx, int curved, int warps) {
  if (!ctx) return fail(WADG_ERR_INVALID, "null context");
  if (warps != 0) {
    int cand[3];
    const int n = wadg_vol_warps_candidates(ctx, curved, cand);
    bool ok = false;
    for (int i = 0; i < n; ++i) ok = ok || cand[i] == warps;
    if (!ok) return fail(WADG_ERR_INVALID, "%d warps per CTA is not a compiled shape", warps);
  }
  ctx->vol_warps = warps;
  ctx->vol_rows = 0;
  return WADG_OK;
}

int wadg_vol_shapes(const wadg_ctx *ctx, int curved, int *warps, int *rows) {
  if (!ctx || !warps || !rows) return -fail(WADG_ERR_INVALID, "null argument");
  const wadg_ctx *c = ctx;
  if (curved) {
    WADG_DISPATCH(c, return (vol_shapes<D_, N_, true>(warps, rows)));
  } else {
    WADG_DISPATCH(c, return (vol_shapes<D_, N_, false>(warps, rows)));
  }
}

int wadg_ctx_set_vol_shape(wadg_ctx *ctx, int curved, int warps, int rows) {
  if (!ctx) return fail(WADG_ERR_INVALID, "null context");
  if (rows == 0) return wadg_ctx_set_vol_warps(ctx, curved, warps);
  int w[WADG_MAX_VOL_SHAPES], r[WADG_MAX_VOL_SHAPES];
  const int n = wadg_vol_shapes(ctx, curved, w, r);
  for (int i = 0; i < n; ++i)
    if (w[i] == warps && r[i] == rows) {
      ctx->vol_warps = warps;
      ctx->vol_rows = rows;
      return WADG_OK;
    }
  return fail(WADG_ERR_INVALID, "%d warps x %d rows per lane is not a compiled shape", warps, rows);
}

int wadg_ctx_get_vol_rows(const wadg_ctx *ctx) { return ctx ? ctx->vol_rows : -1; }

int wadg_ctx_get_vol_warps(const wadg_ctx *ctx) { return ctx ? ctx->vol_warps : -1; }

int wadg_kernel_shape(const wadg_ctx *ctx, int kernel, int curved, int K, int *elems_per_batch,
                      int *grid) {
  if (!ctx || !elems_per_batch || !grid) return fail(WADG_ERR_INVALID, "null argument");
  if (K < 0) return fail(WADG_ERR_INVALID, "K < 0");
  const wadg_ctx *c = ctx;
  if (curved) {
    WADG_DISPATCH(c, return (kernel_shape<D_, N_, true>(c, kernel, K, elems_per_batch, grid)));
  }
  WADG_DISPATCH(c, return (kernel_shape<D_, N_, false>(c, kernel, K, elems_per_batch, grid)));
}

// ------------------------------------------------------------------ diagnostics

int wadg_euler_3d_compute_aux(wadg_ctx *c, int K, const double *Jq, const double *wq,
                              const double *Q, double *aux) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  if (K < 0) return fail(WADG_ERR_INVALID, "K < 0");
  if (K == 0) return WADG_OK;
  if (any_null({Jq, wq, Q, aux})) return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_integral<D_, N_, false>(c, K, Jq, wq, Q, aux)));
}

int wadg_element_entropy(wadg_ctx *c, int K, const double *Jq, const double *wq, const double *Q,
                         double *S) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  if (K < 0) return fail(WADG_ERR_INVALID, "K < 0");
  if (K == 0) return WADG_OK;
  if (any_null({Jq, wq, Q, S})) return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_integral<D_, N_, true>(c, K, Jq, wq, Q, S)));
}

int wadg_halo_pack(wadg_ctx *c, int n, const uint32_t *src, const double *Qf, size_t nQf,
                   double *buf) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  const int NF = c->Nfq * c->Nfaces, Nf = c->dim + 2;
  if (n < 0 || n % NF) return fail(WADG_ERR_INVALID, "slot count must be a multiple of NfqNf");
  if (n == 0) return WADG_OK;
  if (any_null({src, Qf, buf})) return fail(WADG_ERR_INVALID, "null pointer argument");
  halo_pack_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, NF, Nf, nQf, src, Qf, buf);
  return after_launch("halo pack kernel");
}

int wadg_check_state(wadg_ctx *c, int K, const double *Q, int *work, int *nbad, int *first) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  if (K < 0) return fail(WADG_ERR_INVALID, "K < 0");
  if (nbad) *nbad = 0;
  if (first) *first = -1;
  if (K == 0) return WADG_OK;
  if (any_null({Q, work})) return fail(WADG_ERR_INVALID, "null pointer argument");
  if ((long long)K * c->Nq >= 0x7f000000LL) return fail(WADG_ERR_INVALID, "K * Nq too large for a state check");
  // work[1] starts at 0x7f7f7f7f, above every node index (byte-wise memset)
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(int), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(work + 1, 0x7f, sizeof(int), c->stream);
  if (e != cudaSuccess) return cuda_check(e, "state check memset");
  const long long n = (long long)K * c->Nq;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (c->dim == 2)
    check_state_kernel<2><<<blocks, 256, 0, c->stream>>>(K, c->Nq, Q, c->phys.gm1, work);
  else
    check_state_kernel<3><<<blocks, 256, 0, c->stream>>>(K, c->Nq, Q, c->phys.gm1, work);
  if (int r = after_launch("state check kernel")) return r;
  int h[2] = {0, 0};
  e = cudaMemcpyAsync(h, work, sizeof h, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_check(e, "state check copy");
  if (nbad) *nbad = h[0];
  if (h[0] == 0) return WADG_OK;
  if (first) *first = h[1];
  return fail(WADG_ERR_STATE, "non-physical state: %d node(s) with a non-finite field, rho <= 0 or p <= 0; "
              "first at element %d, node %d", h[0], h[1] / c->Nq, h[1] % c->Nq);
}

int wadg_entropy_rhs(wadg_ctx *c, int K, int curved, const double *wq, const double *Jq,
                     const double *VqPq, const double *Q, const double *rhs, double *out) {
  if (!c) return fail(WADG_ERR_INVALID, "null context");
  if (K < 0) return fail(WADG_ERR_INVALID, "K < 0");
  if (K == 0) return WADG_OK;
  if (any_null({wq, VqPq, Q, rhs, out}) || (curved && !Jq))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  if (curved) {
    WADG_DISPATCH(c, return (launch_entropy_rhs<D_, N_, true>(c, K, wq, Jq, VqPq, Q, rhs, out)));
  }
  WADG_DISPATCH(c, return (launch_entropy_rhs<D_, N_, false>(c, K, wq, Jq, VqPq, Q, rhs, out)));
}

// ------------------------------------------------------------------ 3D
int wadg_euler_vol_3d(wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                      const double *nrJ, const double *nsJ, const double *ntJ, const double *Drq,
                      const double *Dsq, const double *Dtq, const double *Drstq,
                      const double *VqLq, const double *VfPq, const double *Q, const double *Qf,
                      double *rhsQ, double *rhsQf) {
  (void)Drstq; (void)Q; (void)vfgeo;
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_vol_pairs<D_, N_, false>(c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq,
                                                    Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf)));
}

int wadg_euler_vol_3d_curved(wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                             const double *nrJ, const double *nsJ, const double *ntJ,
                             const double *Drq, const double *Dsq, const double *Dtq,
                             const double *Drstq, const double *VqLq, const double *VfPq,
                             const double *Q, const double *Qf, double *rhsQ, double *rhsQf) {
  (void)Drstq; (void)Q;
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_vol_pairs<D_, N_, true>(c, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq,
                                                   Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf)));
}

int wadg_euler_surf_3d(wadg_ctx *c, int K, const double *fgeo, const uint32_t *mapPq,
                       const double *VqLq, const double *Qf, double *rhsQf, double *rhsQ) {
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_surf<D_, N_>(c, K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ)));
}

int wadg_euler_update_3d(wadg_ctx *c, int K, const double *Jq, const double *VqPq,
                         const double *VfPq, double fa, double fb, double fdt, double *rhsQ,
                         double *resQ, double *Q, double *Qf) {
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({Jq, VqPq, VfPq, rhsQ, resQ, Q, Qf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_update<D_, N_, false>(c, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ,
                                                         resQ, Q, Qf)));
}

int wadg_euler_update_3d_curved(wadg_ctx *c, int K, const double *Jq, const double *VqPq,
                                const double *VfPq, double fa, double fb, double fdt,
                                double *rhsQ, double *resQ, double *Q, double *Qf) {
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({Jq, VqPq, VfPq, rhsQ, resQ, Q, Qf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_update<D_, N_, true>(c, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ,
                                                        resQ, Q, Qf)));
}

// ------------------------------------------------------------------ 2D
int wadg_euler_vol_2d(wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                      const double *nrJ, const double *nsJ, const double *Drq, const double *Dsq,
                      const double *VqLq, const double *VfPq, const double *Q, const double *Qf,
                      double *rhsQ, double *rhsQf) {
  (void)Q; (void)vfgeo;
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, Qf, rhsQ, rhsQf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_vol_pairs<D_, N_, false>(c, K, vgeo, vfgeo, nrJ, nsJ, nullptr, Drq,
                                                    Dsq, nullptr, VqLq, VfPq, Qf, rhsQ, rhsQf)));
}

int wadg_euler_vol_2d_curved(wadg_ctx *c, int K, const double *vgeo, const double *vfgeo,
                             const double *nrJ, const double *nsJ, const double *Drq,
                             const double *Dsq, const double *VqLq, const double *VfPq,
                             const double *Q, const double *Qf, double *rhsQ, double *rhsQf) {
  (void)Q;
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, vfgeo, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, Qf, rhsQ, rhsQf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_vol_pairs<D_, N_, true>(c, K, vgeo, vfgeo, nrJ, nsJ, nullptr, Drq,
                                                   Dsq, nullptr, VqLq, VfPq, Qf, rhsQ, rhsQf)));
}

int wadg_euler_surf_2d(wadg_ctx *c, int K, const double *fgeo, const uint32_t *mapPq,
                       const double *VqLq, const double *Qf, const double *rhsQf, double *rhsQ) {
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_surf<D_, N_>(c, K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ)));
}

int wadg_euler_update_2d(wadg_ctx *c, int K, const double *Jq, const double *VqPq,
                         const double *VfPq, double fa, double fb, double fdt, double *rhsQ,
                         double *resQ, double *Q, double *Qf) {
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({Jq, VqPq, VfPq, rhsQ, resQ, Q, Qf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_update<D_, N_, false>(c, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ,
                                                         resQ, Q, Qf)));
}

int wadg_euler_update_2d_curved(wadg_ctx *c, int K, const double *Jq, const double *VqPq,
                                const double *VfPq, double fa, double fb, double fdt,
                                double *rhsQ, double *resQ, double *Q, double *Qf) {
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({Jq, VqPq, VfPq, rhsQ, resQ, Q, Qf}))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  WADG_DISPATCH(c, return (launch_update<D_, N_, true>(c, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ,
                                                        resQ, Q, Qf)));
}

// ------------------------------------------------------------ fused stage
int wadg_euler_stage_3d(wadg_ctx *c, int K, int curved, const double *vgeo, const double *vfgeo,
                        const double *fgeo, const uint32_t *mapPq, const double *nrJ,
                        const double *nsJ, const double *ntJ, const double *Drq, const double *Dsq,
                        const double *Dtq, const double *VqLq, const double *VfPq,
                        const double *VqPq, const double *Jq, double fa, double fb, double fdt,
                        const double *rhsQ_in, const double *Qf_in, double *Q, double *resQ,
                        double *rhsQ_out, double *Qf_out) {
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, fgeo, mapPq, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, VqPq, Jq, rhsQ_in,
                Qf_in, Q, resQ, rhsQ_out, Qf_out}) || (curved && !vfgeo))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  // the state may be updated in place; the traces need a second buffer
  if (Qf_in == Qf_out)
    return fail(WADG_ERR_INVALID, "stage: Qf_out must not be Qf_in");
  if (curved)
    WADG_DISPATCH(c, return (launch_stage<D_, N_, true>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                         ntJ, Drq, Dsq, Dtq, VqLq, VfPq, VqPq, Jq,
                                                         fa, fb, fdt, rhsQ_in, Qf_in, Q, resQ,
                                                         rhsQ_out, Qf_out)));
  WADG_DISPATCH(c, return (launch_stage<D_, N_, false>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                        ntJ, Drq, Dsq, Dtq, VqLq, VfPq, VqPq, Jq,
                                                        fa, fb, fdt, rhsQ_in, Qf_in, Q, resQ,
                                                        rhsQ_out, Qf_out)));
}

int wadg_euler_volsurf_3d(wadg_ctx *c, int K, int curved, const double *vgeo,
                          const double *vfgeo, const double *fgeo, const uint32_t *mapPq,
                          const double *nrJ, const double *nsJ, const double *ntJ,
                          const double *Drq, const double *Dsq, const double *Dtq,
                          const double *VqLq, const double *VfPq, const double *Qf, double *rhsQ) {
  if (int r = check_ctx(c, 3, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, fgeo, mapPq, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ}) ||
      (curved && !vfgeo))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  if (curved)
    WADG_DISPATCH(c, return (launch_volsurf<D_, N_, true>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                           ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ)));
  WADG_DISPATCH(c, return (launch_volsurf<D_, N_, false>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                          ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ)));
}

int wadg_euler_volsurf_2d(wadg_ctx *c, int K, int curved, const double *vgeo,
                          const double *vfgeo, const double *fgeo, const uint32_t *mapPq,
                          const double *nrJ, const double *nsJ, const double *Drq,
                          const double *Dsq, const double *VqLq, const double *VfPq,
                          const double *Qf, double *rhsQ) {
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, fgeo, mapPq, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, Qf, rhsQ}) || (curved && !vfgeo))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  if (curved)
    WADG_DISPATCH(c, return (launch_volsurf<D_, N_, true>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                           nullptr, Drq, Dsq, nullptr, VqLq, VfPq,
                                                           Qf, rhsQ)));
  WADG_DISPATCH(c, return (launch_volsurf<D_, N_, false>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                          nullptr, Drq, Dsq, nullptr, VqLq, VfPq,
                                                          Qf, rhsQ)));
}

int wadg_euler_stage_2d(wadg_ctx *c, int K, int curved, const double *vgeo, const double *vfgeo,
                        const double *fgeo, const uint32_t *mapPq, const double *nrJ,
                        const double *nsJ, const double *Drq, const double *Dsq,
                        const double *VqLq, const double *VfPq, const double *VqPq,
                        const double *Jq, double fa, double fb, double fdt,
                        const double *rhsQ_in, const double *Qf_in, double *Q, double *resQ,
                        double *rhsQ_out, double *Qf_out) {
  if (int r = check_ctx(c, 2, K)) return r;
  if (K == 0) return WADG_OK;
  if (any_null({vgeo, fgeo, mapPq, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, VqPq, Jq, rhsQ_in, Qf_in, Q,
                resQ, rhsQ_out, Qf_out}) || (curved && !vfgeo))
    return fail(WADG_ERR_INVALID, "null pointer argument");
  // the state may be updated in place; the traces need a second buffer
  if (Qf_in == Qf_out)
    return fail(WADG_ERR_INVALID, "stage: Qf_out must not be Qf_in");
  if (curved)
    WADG_DISPATCH(c, return (launch_stage<D_, N_, true>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                         nullptr, Drq, Dsq, nullptr, VqLq, VfPq,
                                                         VqPq, Jq, fa, fb, fdt, rhsQ_in, Qf_in, Q,
                                                         resQ, rhsQ_out, Qf_out)));
  WADG_DISPATCH(c, return (launch_stage<D_, N_, false>(c, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                                        nullptr, Drq, Dsq, nullptr, VqLq, VfPq,
                                                        VqPq, Jq, fa, fb, fdt, rhsQ_in, Qf_in, Q,
                                                        resQ, rhsQ_out, Qf_out)));
}

}  // extern "C"
