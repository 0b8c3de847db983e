// LSRK update kernel (wadg_euler_update_*) with its projections on the FP64
// tensor cores.  Same arithmetic as the reference's update kernels
// (Euler3Daffine.okl:555-773, Euler3D.okl:2527-2884, Euler2D.okl:1498-2282):
//   affine: r = -2 VqPq rhs / J; res = a res + dt r; Q += b res; v = V(Q);
//           Qf = U(VfPq v); rhsQ = U(VqPq v)
//   WADG:   r = VqPq((-2 VqPq rhs)/J); ...; v~ = VqPq((VqPq(v J))/J);
//           Qf = U(VfPq v~); rhsQ = U(VqPq v~)
// but every operator application is a small GEMM over a group of 8 elements,
// Op[M x Nq] * X[Nq x (8 Nf)], issued as mma.sync m8n8k4 f64 (the FP64 MMA of
// sm_80 and later; tcgen05 has no f64 kind).  A node-per-thread matrix-vector
// product issues one shared-memory load per FMA and is bound by the LSU pipe;
// a fragment-tiled MMA loads one B value per 8 FMAs.
//
// One CTA works on one group of 8 elements at a time:
//   * the group's rhs block is staged in shared memory as X[node][f*8 + e]
//     (column n of the GEMM = field f of element e), so that one n-tile of 8
//     columns is one field of the 8 elements;
//   * a warp computes all Nf n-tiles of an m-tile of 8 output nodes (the
//     CTA's warps take the m-tiles round-robin), so a lane
//     ends up holding every field of its (node, element) pairs in registers —
//     the nonlinear epilogues (V(U), U(V), the LSRK update) run there, with no
//     round trip through shared memory;
//   * rows of X beyond Nq are zero and the operator's fragments beyond its
//     extent are zero, so the padding adds nothing.
// The row stride of X is = 4 or 12 (mod 16) doubles: a half warp's B-fragment
// load (4 k-rows x 4 columns) then hits 16 distinct banks.
#pragma once

#include "wadg_device.cuh"

namespace wadg {

// D(8x8) += A(8x4) B(4x8).  Lane l holds A(l/4, l%4), B(l%4, l/4) and
// D(l/4, 2(l%4)), D(l/4, 2(l%4)+1).
// (not volatile: independent MMAs may be interleaved by the scheduler)
__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

constexpr int mma_ld(int c) { return (c % 16 == 4 || c % 16 == 12) ? c : mma_ld(c + 1); }

template <int DIM, int N, bool CURVED>
struct UpdMmaCfg {
  using El = Elem<DIM, N>;
  static constexpr int Nq = El::Nq, NF = El::NfqNf, Nf = El::Nfields;
  static constexpr int EW = 8;                      // elements per warp (one n-tile per field)
  static constexpr int KS = (Nq + 3) / 4;           // k-steps of 4 nodes
  static constexpr int KP = 4 * KS;                 // rows of X (zero beyond Nq)
  static constexpr int MQ = (Nq + 7) / 8;           // m-tiles of the Nq x Nq products
  static constexpr int MO = (NF + Nq + 7) / 8;      // m-tiles of [VfPq; VqPq]
  static constexpr int LD = mma_ld(Nf * EW);        // row stride of X (doubles)
  static constexpr int BUF = KP * LD;               // one buffer
  // one CTA works on one group at a time, one warp per m-tile of the Nq x Nq
  // products (the output projection's MO m-tiles go round-robin)
  static constexpr int WARPS = MQ < 2 ? 2 : (MQ > 6 ? 6 : MQ);
  static constexpr int threads = 32 * WARPS;
  static constexpr size_t smem = sizeof(double) * 2 * BUF;
  // register cap from the launch bounds.  Up to 3 warps per CTA, 5 resident
  // CTAs per SM measured best (3D N=3 affine: 0.065 ms vs 0.067 uncapped and
  // 0.065 at 7; the latency of the per-group chain wants warps more than
  // registers).  At 6 warps (N=4 in 3D), 5 CTAs cap the registers at 64 and
  // spill: 3 CTAs measured best (curved N=4: 0.0885 ms vs 0.0965 at 5,
  // 0.100 at 2, 0.091 at 4)
  static constexpr int min_ctas = WARPS >= 6 ? 3 : 5;
};

// A fragments of rows [8 mt, 8 mt + 8) of an operator stored column-major
// (Op(m, k) = Op[m + k ld], rows < M, columns < Nq); zero outside
template <int KS, int Nq>
__device__ __forceinline__ void load_afrag(const double *__restrict__ Op, int ld, int M, int mt,
                                           int lane, double *a) {
  const int m = mt * 8 + (lane >> 2);
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const int k = ks * 4 + (lane & 3);
    a[ks] = (m < M && k < Nq) ? __ldg(Op + m + (size_t)k * ld) : 0.0;
  }
}

// the stacked operator [VfPq; VqPq] (NF + Nq rows)
template <int KS, int Nq, int NF>
__device__ __forceinline__ void load_afrag_out(const double *__restrict__ VfPq,
                                               const double *__restrict__ VqPq, int mt, int lane,
                                               double *a) {
  const int m = mt * 8 + (lane >> 2);
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const int k = ks * 4 + (lane & 3);
    double v = 0.0;
    if (k < Nq) {
      if (m < NF)
        v = __ldg(VfPq + m + (size_t)k * NF);
      else if (m < NF + Nq)
        v = __ldg(VqPq + (m - NF) + (size_t)k * Nq);
    }
    a[ks] = v;
  }
}

// D[f][i] = sum_k A(m, k) X(k, f*8 + e), m = 8 mt + lane/4, e = 2 (lane%4) + i
template <int KS, int Nf, int LD>
__device__ __forceinline__ void mtile_gemm(const double *a, const double *X, int lane,
                                           double (*D)[2]) {
  const double *xb = X + (lane & 3) * LD + (lane >> 2);
#pragma unroll
  for (int f = 0; f < Nf; ++f) D[f][0] = D[f][1] = 0.0;
  // k outer: the Nf accumulator chains are independent, so consecutive MMAs
  // do not wait on each other
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    double b[Nf];
#pragma unroll
    for (int f = 0; f < Nf; ++f) b[f] = xb[ks * 4 * LD + f * 8];
#pragma unroll
    for (int f = 0; f < Nf; ++f) dmma884(D[f][0], D[f][1], a[ks], b[f]);
  }
}

// Y(m, f*8 + e) = c D[f][i] / J(m, e) for the lane's rows < Nq (J = 1
// without a Jacobian; columns of elements past the end get 0)
template <int Nq, int Nf, int LD, bool DIVJ>
__device__ __forceinline__ void mtile_store(double *Y, int mt, int lane, const double (*D)[2],
                                            double c, const double *__restrict__ Jq, int k0,
                                            int ne) {
  const int m = mt * 8 + (lane >> 2);
  if (m >= Nq) return;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int e = 2 * (lane & 3) + i;
    const bool ok = e < ne;
    const double cJ = (DIVJ && ok) ? c * rcp(Jq[(size_t)(k0 + e) * Nq + m]) : 1.0;
#pragma unroll
    for (int f = 0; f < Nf; ++f) Y[m * LD + f * 8 + e] = ok ? (DIVJ ? cJ * D[f][i] : D[f][i]) : 0.0;
  }
}

// the CTA-wide barrier (the update kernel: one group per CTA)
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// the LSRK operands of a lane's two (node, element) pairs of m-tile mt
template <int Nq, int Nf>
__device__ __forceinline__ void load_lsrk(const double *__restrict__ resQ,
                                          const double *__restrict__ Q,
                                          const double *__restrict__ Jq, int k0, int ne, int mt,
                                          int lane, double (*res0)[Nf], double (*q0)[Nf],
                                          double *Jv) {
  const int m = mt * 8 + (lane >> 2);
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int e = 2 * (lane & 3) + i;
    const bool ok = m < Nq && e < ne;
    const size_t id = (size_t)(k0 + e) * Nq * Nf + m;
    Jv[i] = ok ? Jq[(size_t)(k0 + e) * Nq + m] : 1.0;
#pragma unroll
    for (int f = 0; f < Nf; ++f) {
      res0[i][f] = ok ? resQ[id + f * Nq] : 0.0;
      q0[i][f] = ok ? Q[id + f * Nq] : 1.0;
    }
  }
}

// The update of one group once X holds its RHS (rows < Nq; rows beyond are
// zero): r = M^{-1} rhs, the LSRK update of resQ and Q, v = V(Q) (WADG: the
// weight-adjusted projection of v), the next traces U(VfPq v) -> Qf_out and
// U(VqPq v) -> rhsQ_out.  res0/q0/Jv hold the LSRK operands of the warp's
// first m-tile (load_lsrk), loaded early by the caller; PRE = false: each
// m-tile loads its own after its product (fewer registers live across the
// MMAs; the caller's res0/q0/Jv are scratch).  The UW warps that share the
// group (warp = 0 .. UW-1 among them) call this; `sync` is their barrier.  It
// ends with the output stores (the caller synchronises before X or Y are
// written again).
template <int DIM, int N, bool CURVED, int UW = UpdMmaCfg<DIM, N, CURVED>::WARPS,
          bool PRE = true, typename SyncF = CtaSync>
__device__ __forceinline__ void update_group(
    int k0, int ne, int warp, int lane, double *X, double *Y, const double *__restrict__ Jq,
    const double *__restrict__ VqPq, const double *__restrict__ VfPq, double fa, double fb,
    double fdt, double *__restrict__ resQ, double *__restrict__ Q, double *__restrict__ rhsQ_out,
    double *__restrict__ Qf_out, const Phys &P, double (*res0)[DIM + 2], double (*q0)[DIM + 2],
    double *Jv, const double *__restrict__ dtK = nullptr, SyncF sync = SyncF()) {
  using C = UpdMmaCfg<DIM, N, CURVED>;
  constexpr int Nq = C::Nq, NF = C::NF, Nf = C::Nf, EW = C::EW, KS = C::KS, LD = C::LD,
                MQ = C::MQ, MO = C::MO, W = UW;
  bool ev[2];
  double dte[2];  // the step of the lane's two elements: fdt, or per element (dtK)
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    ev[i] = 2 * (lane & 3) + i < ne;
    dte[i] = (dtK && ev[i]) ? dtK[k0 + 2 * (lane & 3) + i] : fdt;
  }

  double a[KS], D[Nf][2];
  // ---- r = M^{-1} rhs (affine: -2 VqPq rhs / J; WADG: VqPq(-2 VqPq rhs / J))
  const double *R = X;  // the operand of the last product before the update
  if (CURVED) {
    for (int mt = warp; mt < MQ; mt += W) {
      load_afrag<KS, Nq>(VqPq, Nq, Nq, mt, lane, a);
      mtile_gemm<KS, Nf, LD>(a, X, lane, D);
      mtile_store<Nq, Nf, LD, true>(Y, mt, lane, D, -2.0, Jq, k0, ne);
    }
    sync();
    R = Y;
  }
  // the update proper; V(U) goes to the other buffer (affine: Y; WADG: X,
  // scaled by J for the projection that follows)
  double *Vb = CURVED ? X : Y;
  for (int mt = warp; mt < MQ; mt += W) {
    if (PRE && mt != warp) load_lsrk<Nq, Nf>(resQ, Q, Jq, k0, ne, mt, lane, res0, q0, Jv);
    const int m = mt * 8 + (lane >> 2);
    load_afrag<KS, Nq>(VqPq, Nq, Nq, mt, lane, a);
    mtile_gemm<KS, Nf, LD>(a, R, lane, D);
    if (!PRE) load_lsrk<Nq, Nf>(resQ, Q, Jq, k0, ne, mt, lane, res0, q0, Jv);
    if (m < Nq) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int e = 2 * (lane & 3) + i;
        const size_t id = (size_t)(k0 + e) * Nq * Nf + m;
        const double m2J = CURVED ? 0.0 : -2.0 * rcp(Jv[i]);  // -2 / J
        double U[Nf], V[Nf];
#pragma unroll
        for (int f = 0; f < Nf; ++f) {
          const double r = CURVED ? D[f][i] : m2J * D[f][i];
          const double res = fa * res0[i][f] + dte[i] * r;
          U[f] = q0[i][f] + fb * res;
          if (ev[i]) {
            resQ[id + f * Nq] = res;
            Q[id + f * Nq] = U[f];
          }
        }
        if (ev[i]) {
          VU<DIM>(U, V, P);
        } else {
#pragma unroll
          for (int f = 0; f < Nf; ++f) V[f] = 0.0;
        }
#pragma unroll
        for (int f = 0; f < Nf; ++f) Vb[m * LD + f * EW + e] = CURVED ? V[f] * Jv[i] : V[f];
      }
    }
  }
  sync();
  const double *Xo = Y;  // the operand of the output projection
  if (CURVED) {
    // v~ = VqPq((VqPq(v J)) / J): X -> Y -> X
    for (int mt = warp; mt < MQ; mt += W) {
      load_afrag<KS, Nq>(VqPq, Nq, Nq, mt, lane, a);
      mtile_gemm<KS, Nf, LD>(a, X, lane, D);
      mtile_store<Nq, Nf, LD, true>(Y, mt, lane, D, 1.0, Jq, k0, ne);
    }
    sync();
    for (int mt = warp; mt < MQ; mt += W) {
      load_afrag<KS, Nq>(VqPq, Nq, Nq, mt, lane, a);
      mtile_gemm<KS, Nf, LD>(a, Y, lane, D);
      mtile_store<Nq, Nf, LD, false>(X, mt, lane, D, 1.0, Jq, k0, ne);
    }
    sync();
    Xo = X;
  }

  // ---- Qf = U(VfPq v), rhsQ = U(VqPq v)
  for (int mt = warp; mt < MO; mt += W) {
    load_afrag_out<KS, Nq, NF>(VfPq, VqPq, mt, lane, a);
    mtile_gemm<KS, Nf, LD>(a, Xo, lane, D);
    const int m = mt * 8 + (lane >> 2);
    if (m >= NF + Nq) continue;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (!ev[i]) continue;
      const int e = 2 * (lane & 3) + i;
      double V[Nf], U[Nf];
#pragma unroll
      for (int f = 0; f < Nf; ++f) V[f] = D[f][i];
      UV<DIM>(V, U, P);
      double *out = m < NF ? Qf_out + (size_t)(k0 + e) * NF * Nf + m
                           : rhsQ_out + (size_t)(k0 + e) * Nq * Nf + (m - NF);
      const int ld = m < NF ? NF : Nq;
#pragma unroll
      for (int f = 0; f < Nf; ++f) out[f * ld] = U[f];
    }
  }
}

// stage the rhs block [e][f][node] of a group as X[node][f*8 + e] (columns of
// elements past the end get 0): loads first, then the barrier that frees X,
// then the stores; `between` runs after the loads are issued.  Threads tid =
// 0 .. THREADS-1 with the barrier `sync`; CG: the loads bypass L1 (the block
// was written earlier in the same launch, by other threads)
template <int Nq, int Nf, int LD, int THREADS, bool CG = false, typename F, typename SyncF = CtaSync>
__device__ __forceinline__ void stage_rhs(const double *rhs, int k0, int ne, double *X, F between,
                                          int tid = threadIdx.x, SyncF sync = SyncF()) {
  constexpr int EW = 8, TOT = EW * Nf * Nq, IT = (TOT + THREADS - 1) / THREADS;
  const double *src = rhs + (size_t)k0 * Nf * Nq;
  const int lim = ne * Nf * Nq;
  double v[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int t = tid + THREADS * it;
    v[it] = t < lim ? (CG ? __ldcg(src + t) : __ldg(src + t)) : 0.0;
  }
  between();
  sync();  // the previous group's last reads of X and Y are done
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int t = tid + THREADS * it;
    if (t < TOT) {
      const int e = t / (Nf * Nq), rem = t - e * (Nf * Nq);
      const int f = rem / Nq, n = rem - f * Nq;
      X[n * LD + f * EW + e] = v[it];
    }
  }
}

template <int DIM, int N, bool CURVED>
__global__ void __launch_bounds__(UpdMmaCfg<DIM, N, CURVED>::threads, UpdMmaCfg<DIM, N, CURVED>::min_ctas)
update_mma_kernel(int K, const double *__restrict__ Jq, const double *__restrict__ VqPq,
                  const double *__restrict__ VfPq, double fa, double fb, double fdt,
                  double *__restrict__ rhsQ, double *__restrict__ resQ, double *__restrict__ Q,
                  double *__restrict__ Qf, Phys P, const double *__restrict__ dtK = nullptr,
                  const int *__restrict__ blist = nullptr, const int *__restrict__ nblist = nullptr) {
  using C = UpdMmaCfg<DIM, N, CURVED>;
  constexpr int Nq = C::Nq, Nf = C::Nf, EW = C::EW, KP = C::KP, LD = C::LD, MQ = C::MQ;
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *X = smem;
  double *Y = X + C::BUF;
  // the padding rows stay zero for the whole launch
  for (int t = threadIdx.x; t < (KP - Nq) * LD; t += C::threads) {
    X[Nq * LD + t] = 0.0;
    Y[Nq * LD + t] = 0.0;
  }

  // the groups to run: all of them, or (a work list: the ensemble's active
  // instances) the group indices blist[0 .. *nblist); dtK: a step per element
  const int ngroups = blist ? *nblist : (K + EW - 1) / EW;
  for (int ig = blockIdx.x; ig < ngroups; ig += gridDim.x) {
    const int k0 = (blist ? blist[ig] : ig) * EW;
    const int ne = min(EW, K - k0);
    // the LSRK operands of this warp's first m-tile load alongside the rhs block
    double res0[2][Nf], q0[2][Nf], Jv[2];
    stage_rhs<Nq, Nf, LD, C::threads>(rhsQ, k0, ne, X, [&] {
      if (warp < MQ) load_lsrk<Nq, Nf>(resQ, Q, Jq, k0, ne, warp, lane, res0, q0, Jv);
    });
    __syncthreads();
    update_group<DIM, N, CURVED>(k0, ne, warp, lane, X, Y, Jq, VqPq, VfPq, fa, fb, fdt, resQ, Q,
                                 rhsQ, Qf, P, res0, q0, Jv, dtK);
  }
}

}  // namespace wadg
