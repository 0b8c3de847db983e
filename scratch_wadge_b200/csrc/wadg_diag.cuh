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

}  // namespace wadg
