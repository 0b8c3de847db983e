// The row-per-thread volume kernel of one LSRK stage (the surface and update
// kernels are in wadg_surf_mma.cuh and wadg_update_mma.cuh), templated on
// dimension and degree.  One CTA handles E consecutive elements; everything an
// element reads more than once is staged in shared memory.
#pragma once

#include "wadg_device.cuh"

namespace wadg {

// ---------------------------------------------------------------- volume
// rhsQ_i = sum_j (Q_x F_S(u_i,u_j))_ij + 1/2 sum_f VqLq_if F_S(u_i,uf_f).nJ_f
// rhsQf_f = -1/2 sum_j VfPq_fj F_S(uf_f,u_j).nJ_f
// (Euler3Daffine.okl:152-417, Euler3D.okl:2123-2523, Euler2D.okl:235-1353)
//
// Prologue: one thread per node converts the staged conservative state into
// the per-node flux state (rho, velocity, beta, log rho, log beta) once, so the
// pair loops do no divisions by rho, no pressure recovery and no logarithms.
// Rows: threads [0, E*Nq) own volume rows, threads [E*Nq, E*NN) own face rows;
// each accumulates its row in registers in the reference's j order.
template <int DIM, int N, bool CURVED, int E>
struct VolCfg {
  using El = Elem<DIM, N>;
  static constexpr int threads = E * El::NN;
  static constexpr size_t smem_state = sizeof(double) * E * El::NS * El::NN;
  static constexpr size_t smem_geo = sizeof(double) * E * El::Nvgeo * (CURVED ? El::NN : 1);
  static constexpr size_t smem = smem_state + smem_geo;
};

template <int DIM, int N, bool CURVED, int E>
__global__ void __launch_bounds__(VolCfg<DIM, N, CURVED, E>::threads)
vol_kernel(int K, const double *__restrict__ vgeo, const double *__restrict__ vfgeo,
           const double *__restrict__ nrJ, const double *__restrict__ nsJ,
           const double *__restrict__ ntJ, const double *__restrict__ Drq,
           const double *__restrict__ Dsq, const double *__restrict__ Dtq,
           const double *__restrict__ VqLq, const double *__restrict__ VfPq,
           const double *__restrict__ Qf, double *__restrict__ rhsQ,
           double *__restrict__ rhsQf, Phys P) {
  using El = Elem<DIM, N>;
  constexpr int Nq = El::Nq, NfqNf = El::NfqNf, Nfq = El::Nfq, NN = El::NN, NS = El::NS;
  constexpr int Nf = El::Nfields, NG = El::Nvgeo, NGN = CURVED ? NN : 1;
  extern __shared__ double smem[];
  double (*st)[NS][NN] = reinterpret_cast<double (*)[NS][NN]>(smem);
  double (*sg)[NG][NGN] = reinterpret_cast<double (*)[NG][NGN]>(smem + E * NS * NN);

  const int k0 = blockIdx.x * E;

  for (int t = threadIdx.x; t < E * NN; t += blockDim.x) {
    const int e = t / NN, n = t % NN, k = k0 + e;
    if (k >= K) continue;
    NodeState<DIM> s = (n < Nq) ? node_state<DIM>(rhsQ + (size_t)k * Nq * Nf + n, Nq, P)
                                : node_state<DIM>(Qf + (size_t)k * NfqNf * Nf + (n - Nq), NfqNf, P);
    st[e][0][n] = s.rho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) st[e][1 + d][n] = s.vel[d];
    st[e][DIM + 1][n] = s.beta;
    st[e][DIM + 2][n] = s.lrho;
    st[e][DIM + 3][n] = s.lbeta;
    if (CURVED) {
#pragma unroll
      for (int c = 0; c < NG; ++c)
        sg[e][c][n] = (n < Nq) ? vgeo[(size_t)k * Nq * NG + c * Nq + n]
                               : vfgeo[(size_t)k * NfqNf * NG + c * NfqNf + (n - Nq)];
    } else if (n < NG) {
      // affine: geometric factors of the first quadrature node (:205)
      sg[e][n][0] = vgeo[(size_t)k * Nq * NG + n * Nq];
    }
  }
  __syncthreads();

  const int t = threadIdx.x;
  const bool volrow = t < E * Nq;
  const int e = volrow ? t / Nq : (t - E * Nq) / NfqNf;
  const int row = volrow ? t % Nq : Nq + (t - E * Nq) % NfqNf;
  const int k = k0 + e;
  if (k >= K) return;

  auto load = [&](int n) {
    NodeState<DIM> s;
    s.rho = st[e][0][n];
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.vel[d] = st[e][1 + d][n];
    s.beta = st[e][DIM + 1][n];
    s.lrho = st[e][DIM + 2][n];
    s.lbeta = st[e][DIM + 3][n];
    return s;
  };
  // direction G^T r for reference direction r (G rows: r-, s-, t-factors)
  auto contract = [&](const double *G, const double *r, double *n) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      double v = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) v = fma(G[a * DIM + d], r[a], v);
      n[d] = v;
    }
  };

  const NodeState<DIM> A = load(row);
  double Gi[NG];
#pragma unroll
  for (int c = 0; c < NG; ++c) Gi[c] = CURVED ? sg[e][c][row] : sg[e][c][0];
  double acc[Nf];
#pragma unroll
  for (int f = 0; f < Nf; ++f) acc[f] = 0.0;

  if (volrow) {
    const int i = row;
    for (int j = 0; j < Nq; ++j) {
      const NodeState<DIM> B = load(j);
      double r[DIM], G[NG], nv[DIM], F[Nf];
      r[0] = __ldg(Drq + i + j * Nq);
      r[1] = __ldg(Dsq + i + j * Nq);
      if (DIM == 3) r[DIM - 1] = __ldg(Dtq + i + j * Nq);
#pragma unroll
      for (int c = 0; c < NG; ++c) G[c] = CURVED ? 0.5 * (Gi[c] + sg[e][c][j]) : Gi[c];
      contract(G, r, nv);
      ecflux_n<DIM>(A, B, nv, P, F);
#pragma unroll
      for (int f = 0; f < Nf; ++f) acc[f] += F[f];
    }
    for (int j = 0; j < NfqNf; ++j) {
      const NodeState<DIM> B = load(Nq + j);
      const int fc = j / Nfq;
      double r[DIM], G[NG], nv[DIM], F[Nf];
      r[0] = __ldg(nrJ + fc * Nfq);
      r[1] = __ldg(nsJ + fc * Nfq);
      if (DIM == 3) r[DIM - 1] = __ldg(ntJ + fc * Nfq);
#pragma unroll
      for (int c = 0; c < NG; ++c) G[c] = CURVED ? 0.5 * (Gi[c] + sg[e][c][Nq + j]) : Gi[c];
      contract(G, r, nv);
      ecflux_n<DIM>(A, B, nv, P, F);
      const double w = 0.5 * __ldg(VqLq + i + j * Nq);
#pragma unroll
      for (int f = 0; f < Nf; ++f) acc[f] = fma(w, F[f], acc[f]);
    }
    double *out = rhsQ + (size_t)k * Nq * Nf + i;
#pragma unroll
    for (int f = 0; f < Nf; ++f) out[f * Nq] = acc[f];
  } else {
    const int i = row - Nq;
    const int fc = i / Nfq;
    double r[DIM];
    r[0] = __ldg(nrJ + fc * Nfq);
    r[1] = __ldg(nsJ + fc * Nfq);
    if (DIM == 3) r[DIM - 1] = __ldg(ntJ + fc * Nfq);
    double nv[DIM];
    contract(Gi, r, nv);
    for (int j = 0; j < Nq; ++j) {
      const NodeState<DIM> B = load(j);
      double F[Nf];
      if (CURVED) {
        double G[NG];
#pragma unroll
        for (int c = 0; c < NG; ++c) G[c] = 0.5 * (Gi[c] + sg[e][c][j]);
        contract(G, r, nv);
      }
      ecflux_n<DIM>(A, B, nv, P, F);
      const double w = -0.5 * __ldg(VfPq + i + j * NfqNf);
#pragma unroll
      for (int f = 0; f < Nf; ++f) acc[f] = fma(w, F[f], acc[f]);
    }
    double *out = rhsQf + (size_t)k * NfqNf * Nf + i;
#pragma unroll
    for (int f = 0; f < Nf; ++f) out[f * NfqNf] = acc[f];
  }
}

}  // namespace wadg
