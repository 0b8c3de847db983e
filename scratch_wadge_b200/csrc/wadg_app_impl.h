// Internal: the host driver's state (wadg_app) and the LSRK-45 tables,
// shared by the driver (wadg_app.cu) and the discrete adjoint
// (wadg_adjoint.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wadg.h"

namespace wadg_internal {
// LSRK-45 (Carpenter & Kennedy) coefficients, euler.c:2779-2796
constexpr double RK4A[5] = {0.0, -567301805773.0 / 1357537059087.0,
                        -2404267990393.0 / 2016746695238.0,
                        -3550918686646.0 / 2091501179385.0,
                        -1275806237668.0 / 842570457699.0};
constexpr double RK4B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                        2277821191437.0 / 14882151754819.0};
}  // namespace wadg_internal

struct wadg_app {
  wadg_ctx *ctx = nullptr;
  wadg_params p{};
  int K = 0, curved = 0;
  int Nq = 0, NfqNf = 0, Nf = 0, Nvgeo = 0, Nfgeo = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // geometry and operators
  double *vgeo = nullptr, *vfgeo = nullptr, *fgeo = nullptr, *Jq = nullptr;
  uint32_t *mapPq = nullptr;
  double *nrJ = nullptr, *nsJ = nullptr, *ntJ = nullptr, *Drq = nullptr, *Dsq = nullptr,
         *Dtq = nullptr, *Drstq = nullptr, *VqLq = nullptr, *VqPq = nullptr, *VfPq = nullptr;
  // solver state; the entropy-projected state (rhsQ, Qf) is double-buffered
  // for the fused stage kernel: buffer `cur` holds the current stage's
  double *Q = nullptr, *resQ = nullptr, *rhsQf = nullptr;
  double *uq[2] = {nullptr, nullptr}, *uf[2] = {nullptr, nullptr};
  int cur = 0;
  int fused = 0;
  // graphs of one time step, one per starting buffer parity (fused path)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // failure detection: device work words of wadg_check_state, and how often
  // wadg_rk_run checks the state (every `check_every` steps; 0 = never)
  int *check_work = nullptr;
  int check_every = 0;
  double graph_dt[2] = {0.0, 0.0};
  int graph_fused[2] = {-1, -1};
};
