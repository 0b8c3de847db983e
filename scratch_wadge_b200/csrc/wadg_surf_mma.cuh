// Surface kernel (wadg_euler_surf_*) with its lift on the FP64 tensor cores.
// Same arithmetic as the reference's surface kernels (Euler3Daffine.okl:421-552,
// Euler3D.okl:3242-3473, Euler2D.okl:1357-1495): at every face point the
// entropy-conservative flux F_S(u-, u+).nJ with the Lax-Friedrichs penalty
// tau/4 max(lam-, lam+) sJ (u+ - u-), plus the volume kernel's face-row
// contribution rhsQf; then the lift rhsQ += VqLq sf.
//
// One CTA per group of 8 elements, one thread per face point of the group
// (the neighbour gathers of all 8 elements are in flight together).  The face
// values go to shared memory as SF[face node][f*8 + e], the B operand of the
// lift Op[Nq x NfqNf] * SF[NfqNf x 8Nf]; one warp per m-tile of 8 volume
// nodes runs it as mma.sync m8n8k4 f64 with the element's rhsQ as the
// accumulator (loaded and stored in the fragment layout).  The node-per-row
// lift it replaces issued a shared load per FMA and a dependent weight load
// per face node.
#pragma once

#include "wadg_update_mma.cuh"

namespace wadg {

template <int DIM, int N>
struct SurfMmaCfg {
  using El = Elem<DIM, N>;
  static constexpr int Nq = El::Nq, NF = El::NfqNf, Nf = El::Nfields;
  static constexpr int EW = 8;
  static constexpr int KSF = (NF + 3) / 4;  // k-steps of the lift
  static constexpr int KPF = 4 * KSF;       // rows of SF (zero beyond NF)
  static constexpr int MQ = (Nq + 7) / 8;   // m-tiles of the lift
  static constexpr int LD = mma_ld(Nf * EW);
  static constexpr int warps_f = (EW * NF + 31) / 32;
  static constexpr int warps = warps_f > MQ ? warps_f : MQ;
  static constexpr int threads = 32 * warps;
  // register cap from the launch bounds: about 1024 threads per SM (3D N=3:
  // 2 CTAs of 12 warps; uncapped 0.103 ms, 1024: 0.068 ms, 1536: 0.072 ms)
  static constexpr int min_ctas = 1024 / threads > 0 ? 1024 / threads : 1;
  static constexpr size_t smem = sizeof(double) * KPF * LD;
};

template <int DIM, int N>
__global__ void __launch_bounds__(SurfMmaCfg<DIM, N>::threads, SurfMmaCfg<DIM, N>::min_ctas)
surf_mma_kernel(int K, const double *__restrict__ fgeo, const uint32_t *__restrict__ mapPq,
                const double *__restrict__ VqLq, const double *__restrict__ Qf,
                const double *__restrict__ rhsQf, double *__restrict__ rhsQ, Phys P) {
  using C = SurfMmaCfg<DIM, N>;
  using El = Elem<DIM, N>;
  constexpr int Nq = C::Nq, NF = C::NF, Nf = C::Nf, EW = C::EW, KSF = C::KSF, KPF = C::KPF,
                LD = C::LD, NFG = El::Nfgeo;
  extern __shared__ double SF[];
  const int k0 = blockIdx.x * EW;
  const int ne = min(EW, K - k0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // ---- surface flux at the group's face points -> SF
  for (int t = threadIdx.x; t < EW * NF; t += C::threads) {
    const int e = t / NF, j = t - e * NF;
    double sf[Nf];
    if (e < ne) {
      const int k = k0 + e;
      const size_t idM = j + (size_t)k * NF * Nf;
      const size_t idP = mapPq[j + (size_t)k * NF];
      const double *fg = fgeo + (size_t)k * NF * NFG + j;
      double nJ[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) nJ[d] = fg[d * NF];
      const double sJ = fg[DIM * NF];
      double UM[Nf], UP[Nf];
#pragma unroll
      for (int f = 0; f < Nf; ++f) {
        UM[f] = Qf[idM + f * NF];
        UP[f] = Qf[idP + f * NF];
      }
      double kM, kP, c2M, c2P;
      const NodeState<DIM> M = node_state_surf<DIM>(UM, 1, P, kM, c2M);
      const NodeState<DIM> Pp = node_state_surf<DIM>(UP, 1, P, kP, c2P);
      double F[Nf];
      ecflux_n_nolog<DIM>(M, Pp, nJ, P, F);
      // wave speeds |u| + sqrt(gamma p / rho)
      const double lamM = fsqrt(kM) + fsqrt(c2M);
      const double lamP = fsqrt(kP) + fsqrt(c2P);
      const double tau = (DIM == 3) ? P.tau : 1.0;
      const double Lfc = tau * 0.25 * fmax(lamM, lamP) * sJ;
      const double *rf = rhsQf + idM;
#pragma unroll
      for (int f = 0; f < Nf; ++f) sf[f] = 0.5 * F[f] + rf[f * NF] - Lfc * (UP[f] - UM[f]);
    } else {
#pragma unroll
      for (int f = 0; f < Nf; ++f) sf[f] = 0.0;
    }
#pragma unroll
    for (int f = 0; f < Nf; ++f) SF[j * LD + f * EW + e] = sf[f];
  }
  for (int t = threadIdx.x; t < (KPF - NF) * LD; t += C::threads) SF[NF * LD + t] = 0.0;
  __syncthreads();

  // ---- lift: rhsQ(m, :) += VqLq(m, :) SF, rhsQ as the accumulator
  for (int mt = warp; mt < C::MQ; mt += C::warps) {
    const int m = mt * 8 + (lane >> 2);
    bool ok[2];
    double *row[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int e = 2 * (lane & 3) + i;
      ok[i] = m < Nq && e < ne;
      row[i] = rhsQ + (size_t)(k0 + (ok[i] ? e : 0)) * Nq * Nf + (ok[i] ? m : 0);
    }
    double D[Nf][2];
#pragma unroll
    for (int f = 0; f < Nf; ++f)
#pragma unroll
      for (int i = 0; i < 2; ++i) D[f][i] = ok[i] ? row[i][f * Nq] : 0.0;
    const double *sb = SF + (lane & 3) * LD + (lane >> 2);
#pragma unroll 4
    for (int ks = 0; ks < KSF; ++ks) {
      const int k = ks * 4 + (lane & 3);
      const double a = (m < Nq && k < NF) ? __ldg(VqLq + m + (size_t)k * Nq) : 0.0;
      double b[Nf];
#pragma unroll
      for (int f = 0; f < Nf; ++f) b[f] = sb[ks * 4 * LD + f * EW];
#pragma unroll
      for (int f = 0; f < Nf; ++f) dmma884(D[f][0], D[f][1], a, b[f]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
      if (ok[i])
#pragma unroll
        for (int f = 0; f < Nf; ++f) row[i][f * Nq] = D[f][i];
  }
}

}  // namespace wadg
