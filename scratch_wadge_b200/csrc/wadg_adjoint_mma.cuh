// The seed and projection kernels of a stage adjoint with their operator
// products on the FP64 tensor cores (the layout of wadg_update_mma.cuh: a
// group of 8 elements per CTA, X[node][f*8 + e] in shared memory, one warp
// per 8-row m-tile, mma.sync m8n8k4 f64, the nonlinear epilogues on the
// lanes' fragments).
//
// seed:  w = dt (resbar + b Qbar); rhsbar = Minv^T w; sfbar = VqLq^T rhsbar
//        affine Minv = -2 diag(1/J) VqPq        (Euler3Daffine.okl:555-620)
//        WADG   Minv = VqPq diag(1/J) (-2 VqPq)  (Euler3D.okl:2527-2620)
// proj:  x = VqPq^T vbar + VfPq^T vfbar (one product over the stacked
//        [vbar; vfbar]); WADG: x <- J VqPq^T((VqPq^T x) / J); the adjoint of
//        V(Q) and the LSRK adjoint update, Qbar += dV/dQ^T x,
//        resbar = a (resbar + b Qbar); then (SEED) the seed of the next stage
//        of the reverse sweep from the updated adjoints.
// The transposed operators are the ones the adjoint stores once: VqPqT
// [Nq x Nq], VfPqT [Nq x NfqNf], VqLqT [NfqNf x Nq], column-major.
#pragma once

#include "wadg_adjoint_kernels.cuh"  // gas_of
#include "wadg_adjoint_math.cuh"
#include "wadg_update_mma.cuh"

namespace wadg {

template <int DIM, int N, bool CURVED>
struct AdjMmaCfg {
  using U = UpdMmaCfg<DIM, N, CURVED>;
  static constexpr int Nq = U::Nq, NF = U::NF, Nf = U::Nf, EW = U::EW, KS = U::KS, KP = U::KP,
                       MQ = U::MQ, LD = U::LD;
  static constexpr int MF = (NF + 7) / 8;           // m-tiles of VqLq^T
  static constexpr int KS1 = (Nq + NF + 3) / 4;     // k-steps over [vbar; vfbar]
  static constexpr int KP1 = 4 * KS1;
  static constexpr int WARPS = MQ < 2 ? 2 : (MQ > 6 ? 6 : MQ);
  static constexpr int threads = 32 * WARPS;
  // X [KP1 rows] | T1 [KP] | T2 [KP]; the seed uses X as W, T1 as R, T2
  static constexpr size_t smem = sizeof(double) * (KP1 + 2 * KP) * LD;
  static_assert(MQ <= WARPS, "the projection gives each warp one m-tile");
};

// A fragments of [VqPq^T | VfPq^T] (Nq x (Nq + NF)) for m-tile mt
template <int KS1, int Nq, int NF>
__device__ __forceinline__ void load_afrag_proj(const double *__restrict__ VqPqT,
                                                const double *__restrict__ VfPqT, int mt, int lane,
                                                double *a) {
  const int m = mt * 8 + (lane >> 2);
#pragma unroll
  for (int ks = 0; ks < KS1; ++ks) {
    const int k = ks * 4 + (lane & 3);
    double v = 0.0;
    if (m < Nq) {
      if (k < Nq)
        v = __ldg(VqPqT + m + (size_t)k * Nq);
      else if (k < Nq + NF)
        v = __ldg(VfPqT + m + (size_t)(k - Nq) * Nq);
    }
    a[ks] = v;
  }
}

// the seed of a group once W holds its (scaled) w: affine W = -2 w / J,
// WADG W = w.  Every warp calls it; it synchronises.  W, R, Y: [KP][LD]
// shared buffers (their pad rows are zeroed here); R ends up holding rhsbar.
template <int DIM, int N, bool CURVED>
__device__ __forceinline__ void seed_group(int k0, int ne, int warp, int lane, double *W,
                                           double *R, double *Y, const double *__restrict__ Jq,
                                           const double *__restrict__ VqPqT,
                                           const double *__restrict__ VqLqT,
                                           double *__restrict__ rhsbar,
                                           double *__restrict__ sfbar) {
  using C = AdjMmaCfg<DIM, N, CURVED>;
  constexpr int Nq = C::Nq, NF = C::NF, Nf = C::Nf, EW = C::EW, KS = C::KS, KP = C::KP,
                LD = C::LD, MQ = C::MQ, MF = C::MF, NW = C::WARPS;
  for (int t = threadIdx.x; t < (KP - Nq) * LD; t += C::threads) {
    W[Nq * LD + t] = 0.0;
    R[Nq * LD + t] = 0.0;
    Y[Nq * LD + t] = 0.0;
  }
  __syncthreads();
  double a[KS], D[Nf][2];
  const double *B = W;
  if (CURVED) {  // Y = -2 (VqPq^T w) / J
    for (int mt = warp; mt < MQ; mt += NW) {
      load_afrag<KS, Nq>(VqPqT, Nq, Nq, mt, lane, a);
      mtile_gemm<KS, Nf, LD>(a, W, lane, D);
      mtile_store<Nq, Nf, LD, true>(Y, mt, lane, D, -2.0, Jq, k0, ne);
    }
    __syncthreads();
    B = Y;
  }
  // rhsbar = VqPq^T B, to global and to R
  for (int mt = warp; mt < MQ; mt += NW) {
    load_afrag<KS, Nq>(VqPqT, Nq, Nq, mt, lane, a);
    mtile_gemm<KS, Nf, LD>(a, B, lane, D);
    const int m = mt * 8 + (lane >> 2);
    if (m < Nq)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int e = 2 * (lane & 3) + i;
        const bool ok = e < ne;
#pragma unroll
        for (int f = 0; f < Nf; ++f) {
          R[m * LD + f * EW + e] = ok ? D[f][i] : 0.0;
          if (ok) rhsbar[(size_t)(k0 + e) * Nq * Nf + f * Nq + m] = D[f][i];
        }
      }
  }
  __syncthreads();
  // sfbar = VqLq^T rhsbar
  for (int mt = warp; mt < MF; mt += NW) {
    load_afrag<KS, Nq>(VqLqT, NF, NF, mt, lane, a);
    mtile_gemm<KS, Nf, LD>(a, R, lane, D);
    const int fn = mt * 8 + (lane >> 2);
    if (fn < NF)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int e = 2 * (lane & 3) + i;
        if (e < ne)
#pragma unroll
          for (int f = 0; f < Nf; ++f) sfbar[(size_t)(k0 + e) * NF * Nf + f * NF + fn] = D[f][i];
      }
  }
}

// W(m, f*8 + e) = scaled seed w of the lane's (node, element) pairs
template <int Nq, int Nf, int LD, bool CURVED>
__device__ __forceinline__ void put_seed(double *W, int m, int lane, int ne, const double (*w)[Nf],
                                         const double *J) {
  if (m >= Nq) return;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int e = 2 * (lane & 3) + i;
    const bool ok = e < ne;
#pragma unroll
    for (int f = 0; f < Nf; ++f)
      W[m * LD + f * 8 + e] = ok ? (CURVED ? w[i][f] : -2.0 * w[i][f] / J[i]) : 0.0;
  }
}

template <int DIM, int N, bool CURVED>
__global__ void __launch_bounds__(AdjMmaCfg<DIM, N, CURVED>::threads)
adj_seed_mma_kernel(int K, const double *__restrict__ Jq, const double *__restrict__ VqPqT,
                    const double *__restrict__ VqLqT, double b, double dt,
                    const double *__restrict__ Qbar, const double *__restrict__ resbar,
                    double *__restrict__ rhsbar, double *__restrict__ sfbar) {
  using C = AdjMmaCfg<DIM, N, CURVED>;
  constexpr int Nq = C::Nq, Nf = C::Nf, EW = C::EW, KP = C::KP, KP1 = C::KP1, LD = C::LD,
                MQ = C::MQ, NW = C::WARPS;
  extern __shared__ double smem[];
  double *W = smem, *R = smem + KP1 * LD, *Y = R + KP * LD;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k0 = blockIdx.x * EW, ne = min(EW, K - k0);
  for (int mt = warp; mt < MQ; mt += NW) {
    const int m = mt * 8 + (lane >> 2);
    double w[2][Nf], J[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int e = 2 * (lane & 3) + i;
      const bool ok = m < Nq && e < ne;
      const size_t id = (size_t)(k0 + e) * Nq * Nf + m;
      J[i] = ok ? Jq[(size_t)(k0 + e) * Nq + m] : 1.0;
#pragma unroll
      for (int f = 0; f < Nf; ++f)
        w[i][f] = ok ? dt * fma(b, Qbar[id + f * Nq], resbar[id + f * Nq]) : 0.0;
    }
    put_seed<Nq, Nf, LD, CURVED>(W, m, lane, ne, w, J);
  }
  seed_group<DIM, N, CURVED>(k0, ne, warp, lane, W, R, Y, Jq, VqPqT, VqLqT, rhsbar, sfbar);
}

template <int DIM, int N, bool CURVED, bool SEED>
__global__ void __launch_bounds__(AdjMmaCfg<DIM, N, CURVED>::threads)
adj_proj_mma_kernel(int K, const double *__restrict__ Jq, const double *__restrict__ VqPqT,
                    const double *__restrict__ VfPqT, const double *__restrict__ Qs,
                    const double *__restrict__ vbar, const double *__restrict__ vfbar, double a_,
                    double b_, double *__restrict__ Qbar, double *__restrict__ resbar, Phys P,
                    const double *__restrict__ VqLqT, double bn, double dtn,
                    double *__restrict__ rhsbar, double *__restrict__ sfbar) {
  using C = AdjMmaCfg<DIM, N, CURVED>;
  constexpr int Nq = C::Nq, NF = C::NF, Nf = C::Nf, EW = C::EW, KS = C::KS, KP = C::KP,
                KS1 = C::KS1, KP1 = C::KP1, LD = C::LD, MQ = C::MQ, NW = C::WARPS;
  extern __shared__ double smem[];
  double *X = smem, *T1 = smem + KP1 * LD, *T2 = T1 + KP * LD;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k0 = blockIdx.x * EW, ne = min(EW, K - k0);

  // ---- the epilogue's operands of the warp's (node, element) pairs, loaded
  // first so that they arrive while the block is staged and multiplied
  const int m = warp * 8 + (lane >> 2);
  double Us[2][Nf], qbs[2][Nf], rbs[2][Nf], J[2];
  if (warp < MQ) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int e = 2 * (lane & 3) + i;
      const bool ok = m < Nq && e < ne;
      const size_t id = (size_t)(k0 + e) * Nq * Nf + m;
      J[i] = ok ? Jq[(size_t)(k0 + e) * Nq + m] : 1.0;
#pragma unroll
      for (int f = 0; f < Nf; ++f) {
        Us[i][f] = ok ? Qs[id + f * Nq] : 1.0;
        qbs[i][f] = ok ? Qbar[id + f * Nq] : 0.0;
        rbs[i][f] = ok ? resbar[id + f * Nq] : 0.0;
      }
    }
  }
  // ---- stage [vbar; vfbar] as X[k][f*8 + e] (rows beyond Nq + NF zero):
  // every load of the thread in flight before the stores
  {
    constexpr int T1N = EW * Nf * Nq, T2N = EW * Nf * NF;
    constexpr int I1 = (T1N + C::threads - 1) / C::threads, I2 = (T2N + C::threads - 1) / C::threads;
    double v1[I1], v2[I2];
#pragma unroll
    for (int it = 0; it < I1; ++it) {
      const int t = threadIdx.x + it * C::threads;
      v1[it] = (t < T1N && t / (Nf * Nq) < ne) ? vbar[(size_t)k0 * Nf * Nq + t] : 0.0;
    }
#pragma unroll
    for (int it = 0; it < I2; ++it) {
      const int t = threadIdx.x + it * C::threads;
      v2[it] = (t < T2N && t / (Nf * NF) < ne) ? vfbar[(size_t)k0 * Nf * NF + t] : 0.0;
    }
#pragma unroll
    for (int it = 0; it < I1; ++it) {
      const int t = threadIdx.x + it * C::threads;
      if (t < T1N) {
        const int e = t / (Nf * Nq), rem = t - e * (Nf * Nq), f = rem / Nq, n = rem - f * Nq;
        X[n * LD + f * EW + e] = v1[it];
      }
    }
#pragma unroll
    for (int it = 0; it < I2; ++it) {
      const int t = threadIdx.x + it * C::threads;
      if (t < T2N) {
        const int e = t / (Nf * NF), rem = t - e * (Nf * NF), f = rem / NF, n = rem - f * NF;
        X[(Nq + n) * LD + f * EW + e] = v2[it];
      }
    }
  }
  for (int t = threadIdx.x; t < (KP1 - Nq - NF) * LD; t += C::threads) X[(Nq + NF) * LD + t] = 0.0;
  if (CURVED)
    for (int t = threadIdx.x; t < (KP - Nq) * LD; t += C::threads) {
      T1[Nq * LD + t] = 0.0;
      T2[Nq * LD + t] = 0.0;
    }
  __syncthreads();

  // ---- x = VqPq^T vbar + VfPq^T vfbar
  double D[Nf][2];
  {
    double a1[KS1];
    // one m-tile per warp (MQ <= WARPS for the compiled degrees)
    if (warp < MQ) {
      load_afrag_proj<KS1, Nq, NF>(VqPqT, VfPqT, warp, lane, a1);
      mtile_gemm<KS1, Nf, LD>(a1, X, lane, D);
    }
  }
  if (CURVED) {  // x <- J VqPq^T((VqPq^T x) / J)
    if (warp < MQ) mtile_store<Nq, Nf, LD, false>(T1, warp, lane, D, 1.0, Jq, k0, ne);
    __syncthreads();
    double a[KS];
    if (warp < MQ) {
      load_afrag<KS, Nq>(VqPqT, Nq, Nq, warp, lane, a);
      mtile_gemm<KS, Nf, LD>(a, T1, lane, D);
      mtile_store<Nq, Nf, LD, true>(T2, warp, lane, D, 1.0, Jq, k0, ne);
    }
    __syncthreads();
    if (warp < MQ) {
      mtile_gemm<KS, Nf, LD>(a, T2, lane, D);
    }
  }
  // ---- adjoint of V(Q) and the LSRK adjoint update
  double wn[2][Nf];
  if (warp < MQ) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int e = 2 * (lane & 3) + i;
      const bool ok = m < Nq && e < ne;
      const size_t id = (size_t)(k0 + e) * Nq * Nf + m;
#pragma unroll
      for (int f = 0; f < Nf; ++f) wn[i][f] = 0.0;
      if (!ok) continue;
      double x[Nf], Ub[Nf];
#pragma unroll
      for (int f = 0; f < Nf; ++f) x[f] = CURVED ? D[f][i] * J[i] : D[f][i];
      adj::VU_vjp<DIM>(Us[i], x, gas_of(P), Ub);
#pragma unroll
      for (int f = 0; f < Nf; ++f) {
        const double qb = qbs[i][f];
        const double rt = fma(b_, qb, rbs[i][f]);
        const double rn = a_ * rt, qn = qb + Ub[f];
        resbar[id + f * Nq] = rn;
        Qbar[id + f * Nq] = qn;
        wn[i][f] = dtn * fma(bn, qn, rn);
      }
    }
  }
  if (SEED) {
    __syncthreads();  // every warp is done with X, T1, T2
    if (warp < MQ) put_seed<Nq, Nf, LD, CURVED>(X, m, lane, ne, wn, J);
    seed_group<DIM, N, CURVED>(k0, ne, warp, lane, X, T1, T2, Jq, VqPqT, VqLqT, rhsbar, sfbar);
  }
}

}  // namespace wadg
