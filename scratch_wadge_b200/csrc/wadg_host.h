// Internal host helpers shared by the kernel launchers.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wadg_internal {

// A kernel's dynamic shared-memory limit (cudaFuncSetAttribute) and the
// device's SM count belong to one device: a process that drives several GPUs
// has to set and query them on each.  PerDevice<T> keeps one value per
// device ordinal, taken on the calling thread's current device.
constexpr int kMaxDevices = 256;

inline int current_device() {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess) return -1;
  return d;
}

template <class T>
struct PerDevice {
  T v[kMaxDevices] = {};
  // the slot of the current device; an ordinal beyond the table (or no
  // device) gets a fresh default value on every call, so that whatever is
  // cached there is recomputed rather than wrongly reused
  T &here() {
    const int d = current_device();
    if (d >= 0 && d < kMaxDevices) return v[d];
    static thread_local T fresh;
    fresh = T{};
    return fresh;
  }
};

// SMs of the current device
inline int sm_count() {
  static PerDevice<int> n;
  int &c = n.here();
  if (!c) {
    const int d = current_device();
    if (d < 0 || cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, d) != cudaSuccess ||
        c <= 0)
      c = 148;
  }
  return c;
}

}  // namespace wadg_internal

struct wadg_ctx;
namespace wadg_internal {
// the ensemble's stage kernels over work lists (wadg_capi.cu)
int volsurf_list(const wadg_ctx *c, int K, int curved, const double *vgeo, const double *vfgeo,
                 const double *fgeo, const uint32_t *mapPq, const double *nrJ, const double *nsJ,
                 const double *ntJ, const double *Drq, const double *Dsq, const double *Dtq,
                 const double *VqLq, const double *VfPq, const double *Qf, double *rhsQ,
                 const int *blist, const int *nb);
int update_list(const wadg_ctx *c, int K, int curved, const double *Jq, const double *VqPq,
                const double *VfPq, double fa, double fb, const double *dtK, double *rhsQ,
                double *resQ, double *Q, double *Qf, const int *glist, const int *ng);

// launch shape (elements per batch, CTAs) of the adjoint's pair VJP kernel
// for K elements (wadg_adjoint.cu)
int adj_pairs_shape(int dim, int N, bool curved, int K, int *E, int *grid);

}  // namespace wadg_internal
