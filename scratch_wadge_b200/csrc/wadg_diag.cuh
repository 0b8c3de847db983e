// Per-element diagnostics: the kinetic energy of
// euler_3d_compute_aux (Euler3D.okl:3888-3934) and the entropy integral the
// reference's driver sums on the host (euler.c:4135-4156, 4276-4315).
//   KE_k = sum_i 1/2 |m_i|^2 / rho_i  J_ik w_i
//   S_k  = sum_i w_i J_ik (-rho_i s_i),  s = log((gamma-1) rhoe / rho^gamma)
// One warp per element: lanes take nodes i = lane, lane + 32, ..., and a fixed
// butterfly reduces them (deterministic; the reference's tree over
// ceil(Nq) to a power of two differs only in rounding).
#pragma once

#include "wadg_device.cuh"

namespace wadg {

template <int DIM, int N, bool ENTROPY>
__global__ void __launch_bounds__(256)
element_integral_kernel(int K, const double *__restrict__ Jq, const double *__restrict__ wq,
                        const double *__restrict__ Q, double *__restrict__ out, Phys P) {
  using El = Elem<DIM, N>;
  constexpr int Nq = El::Nq, Nf = El::Nfields;
  const int k = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= K) return;  // the whole warp leaves together
  double acc = 0.0;
  for (int i = lane; i < Nq; i += 32) {
    const double *q = Q + (size_t)k * Nq * Nf + i;
    const double rho = q[0], E = q[(DIM + 1) * Nq];
    double m2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) m2 = fma(q[(1 + d) * Nq], q[(1 + d) * Nq], m2);
    const double wJ = Jq[(size_t)k * Nq + i] * wq[i];
    if (ENTROPY) {
      const double rhoe = E - 0.5 * m2 / rho;
      const double s = log(P.gm1 * rhoe / pow(rho, P.gamma));
      acc += wJ * (-rho * s);
    } else {
      acc += 0.5 * m2 / rho * wJ;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[k] = acc;
}

// The entropy balance of the RHS: D_k = sum_i w_i v~_i . rhs_i, with rhs the
// RHS of the volume and surface kernels (before the inverse mass) and v~ the
// entropy variables of the projected state the volume kernel read: the
// projection the update kernel applies to v = V(Q) (affine: VqPq v, WADG:
// VqPq((VqPq(v J))/J); V(U(v~)) = v~).  Flux differencing makes the volume
// terms of sum_k D_k vanish on a periodic mesh, so sum_k D_k = 0 without the
// Lax-Friedrichs penalty (tau = 0) and is positive with it (entropy
// dissipated).  The reference tracks the entropy itself on the host
// (euler.c:4135-4156); this is its rate, per element, on the device.
// One warp per element; V(Q) and the projection in shared memory.
template <int DIM, int N, bool CURVED>
__global__ void __launch_bounds__(256)
entropy_rhs_kernel(int K, const double *__restrict__ wq, const double *__restrict__ Jq,
                   const double *__restrict__ VqPq, const double *__restrict__ Q,
                   const double *__restrict__ rhs, double *__restrict__ out, Phys P) {
  using El = Elem<DIM, N>;
  constexpr int Nq = El::Nq, Nf = El::Nfields, W = 8;
  __shared__ double sv[W][2][Nf][Nq];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * W + warp;
  if (k >= K) return;  // the whole warp leaves together
  double (*A)[Nq] = sv[warp][0];
  double (*B)[Nq] = sv[warp][1];
  for (int i = lane; i < Nq; i += 32) {
    double U[Nf], V[Nf];
#pragma unroll
    for (int f = 0; f < Nf; ++f) U[f] = Q[(size_t)k * Nq * Nf + f * Nq + i];
    VU<DIM>(U, V, P);
    const double J = CURVED ? Jq[(size_t)k * Nq + i] : 1.0;
#pragma unroll
    for (int f = 0; f < Nf; ++f) A[f][i] = CURVED ? V[f] * J : V[f];
  }
  __syncwarp();
  auto project = [&](double (*X)[Nq], int i, double *o) {
#pragma unroll
    for (int f = 0; f < Nf; ++f) o[f] = 0.0;
    for (int j = 0; j < Nq; ++j) {
      const double w = __ldg(VqPq + i + j * Nq);
#pragma unroll
      for (int f = 0; f < Nf; ++f) o[f] = fma(w, X[f][j], o[f]);
    }
  };
  if (CURVED) {
    for (int i = lane; i < Nq; i += 32) {
      double t[Nf];
      project(A, i, t);
      const double J = Jq[(size_t)k * Nq + i];
#pragma unroll
      for (int f = 0; f < Nf; ++f) B[f][i] = t[f] / J;
    }
    __syncwarp();
  }
  double acc = 0.0;
  for (int i = lane; i < Nq; i += 32) {
    double v[Nf];
    project(CURVED ? B : A, i, v);
    double d = 0.0;
#pragma unroll
    for (int f = 0; f < Nf; ++f) d = fma(v[f], rhs[(size_t)k * Nq * Nf + f * Nq + i], d);
    acc = fma(wq[i], d, acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[k] = acc;
}

}  // namespace wadg
