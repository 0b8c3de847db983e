// One LSRK stage without any device allocation by the library.
//
// rk_step needs a face-row buffer (rhsQf) between the volume and the surface
// kernel.  wadg_app allocates it with cudaMalloc; this entry point instead
// keeps it in a fixed array of device memory that is part of the library
// image, for callers that may not allocate: a host program that owns all
// device memory through its own pool (as the reference's driver does with
// device_malloc, euler.c:131-156) and hands the library only its own
// buffers, or code that must not call cudaMalloc/cudaFree in its time loop
// because they synchronise the device and can fail mid-run.
//
// The array is WADG_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB) and is resident
// on every GPU that loads the library until the process exits.  All calls
// share it and it keeps the last call's contents; nothing in it has to start
// at zero, because the volume kernel writes every entry the surface kernel
// then reads.  Calls whose execution overlaps on the GPU (different streams,
// or several host threads) race on it: serialise them.
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "../../include/wadg.h"

namespace wadg_internal {
void set_error(const std::string &msg);  // wadg_capi.cu
}
int wadg_ctx_sizes(const wadg_ctx *c, int *dim, int *NfqNf);  // wadg_capi.cu
cudaStream_t wadg_ctx_stream(const wadg_ctx *c);                // wadg_capi.cu

namespace {

__device__ __align__(256) double g_noalloc_scratch[WADG_NOALLOC_SCRATCH_DOUBLES];

constexpr int kMaxDevices = 64;
std::atomic<double *> g_scratch_ptr[kMaxDevices];

int nfail(int code, const std::string &msg) {
  wadg_internal::set_error(msg);
  return code;
}

// The device address of the scratch array on the current device.  In host
// code `g_noalloc_scratch` names a host-side stand-in, not device memory, so
// the address is looked up with that device current.  The lookup is repeated
// on every call whose stream is not being captured (a context torn down and
// made again, e.g. by cudaDeviceReset, reloads the module at a new address);
// during a capture the address found by the last call on this device is
// used, so the first call on a device has to come before any capture.
int scratch_on_current_device(cudaStream_t stream, double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return nfail(WADG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return nfail(WADG_ERR_UNSUPPORTED, "device ordinal out of range");
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cs);
  if (e != cudaSuccess)
    return nfail(WADG_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  double *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (cs == cudaStreamCaptureStatusNone || !p) {
    void *a = nullptr;
    e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
    if (e != cudaSuccess)
      return nfail(WADG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    p = static_cast<double *>(a);
    g_scratch_ptr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return WADG_OK;
}

}  // namespace

extern "C" int wadg_rk_stage_noalloc(wadg_ctx *ctx, int K, int curved, const double *vgeo,
                                     const double *vfgeo, const double *fgeo,
                                     const uint32_t *mapPq, const double *nrJ, const double *nsJ,
                                     const double *ntJ, const double *Drq, const double *Dsq,
                                     const double *Dtq, const double *VqLq, const double *VqPq,
                                     const double *VfPq, const double *Jq, double fa, double fb,
                                     double fdt, double *rhsQ, double *resQ, double *Q,
                                     double *Qf) {
  if (!ctx) return nfail(WADG_ERR_INVALID, "null context");
  if (K < 0) return nfail(WADG_ERR_INVALID, "K < 0");
  if (K == 0) return WADG_OK;
  int dim = 0, NfqNf = 0;
  if (int r = wadg_ctx_sizes(ctx, &dim, &NfqNf)) return r;
  const size_t need = (size_t)K * (size_t)NfqNf * (size_t)(dim + 2);
  if (need > (size_t)WADG_NOALLOC_SCRATCH_DOUBLES)
    return nfail(WADG_ERR_INVALID,
                 "K = " + std::to_string(K) + " needs " + std::to_string(need) +
                     " doubles of face-row scratch; the fixed array holds " +
                     std::to_string((size_t)WADG_NOALLOC_SCRATCH_DOUBLES) +
                     " (use wadg_app or the kernel entry points with your own rhsQf)");
  double *rhsQf = nullptr;
  if (int r = scratch_on_current_device(wadg_ctx_stream(ctx), &rhsQf)) return r;

  int r;
  if (dim == 3) {
    r = curved ? wadg_euler_vol_3d_curved(ctx, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq,
                                          nullptr, VqLq, VfPq, Q, Qf, rhsQ, rhsQf)
               : wadg_euler_vol_3d(ctx, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, nullptr,
                                   VqLq, VfPq, Q, Qf, rhsQ, rhsQf);
    if (!r) r = wadg_euler_surf_3d(ctx, K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ);
    if (!r)
      r = curved ? wadg_euler_update_3d_curved(ctx, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf)
                 : wadg_euler_update_3d(ctx, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf);
  } else {
    r = curved ? wadg_euler_vol_2d_curved(ctx, K, vgeo, vfgeo, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, Q,
                                          Qf, rhsQ, rhsQf)
               : wadg_euler_vol_2d(ctx, K, vgeo, vfgeo, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, Q, Qf,
                                   rhsQ, rhsQf);
    if (!r) r = wadg_euler_surf_2d(ctx, K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ);
    if (!r)
      r = curved ? wadg_euler_update_2d_curved(ctx, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf)
                 : wadg_euler_update_2d(ctx, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf);
  }
  return r;
}
