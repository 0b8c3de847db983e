// One LSRK stage in one launch (wadg_euler_stage_*): rk_step of the reference
// (euler.c:3610-3666: euler_vol_3d, euler_surf_3d, euler_update_3d or their
// curved / 2D counterparts) as the volume + surface kernel followed, per group
// of 8 elements, by the tensor-core update.
//
// The CTA is the volume + surface kernel's (pair-scheduled element groups of
// H warps, each synchronising only among its own warps).  Volume groups are
// joined into update groups of 8 elements (one DMMA n-tile per field): 8 / G
// volume groups share one update when a group holds G < 8 elements, and a
// group of G >= 8 elements runs G / 8 updates one after another.  Per batch:
//   1. each volume group computes its elements' whole right-hand side (pairs,
//      surface flux and penalty, lift) and writes it to uq_out;
//   2. the update group's warps meet at their barrier, stage the RHS block
//      back (through L2) into the state blocks of its elements, which are
//      free now, and run update_group there: r = M^{-1} rhs, the LSRK update
//      of resQ and Q, V(U), the projections and U(V) into uq_out and uf_out.
// While one update group runs its latency-bound chain (DMMA, then V(U) /
// U(V)), the CTA's other groups run their flux pairs: the update's latency
// hides behind FP64 work instead of running as a launch of its own.
//
// Buffers: (uq, uf) hold the stage's entropy-projected state and traces;
// uq_out receives first the RHS and then the next stage's state, uf_out the
// next traces.  uf_out must differ from uf: an element's surface flux reads
// its neighbours' current traces while other groups already write the next
// ones.  uq_out may equal uq (an element's own state is read before its RHS
// is written).  Q and resQ are updated in place.
#pragma once

#include "wadg_update_mma.cuh"
#include "wadg_vol.cuh"

namespace wadg {

template <int DIM, int N, bool CURVED, int W>
struct StageCfg {
  using V = VolPairs<DIM, N, CURVED, W>;
  using U = UpdMmaCfg<DIM, N, CURVED>;
  static constexpr int G = V::G, H = V::H, NGRP = W / H;
  static constexpr int UPG = G >= 8 ? 1 : 8 / G;  // volume groups per update group
  static constexpr int SUB = G >= 8 ? G / 8 : 1;  // updates per volume group, one after another
  static constexpr int UW = UPG * H;              // warps of an update group
  static constexpr int NUG = NGRP / UPG;          // update groups per CTA
  // named barriers: 1 .. NGRP for the volume groups (H = 2), then the update groups
  static constexpr int BAR0 = H == 1 ? 1 : 1 + NGRP;
  static_assert(G % 8 == 0 || 8 % G == 0, "element groups of a power of two");
  static_assert(NGRP % UPG == 0, "whole update groups per CTA");
  static_assert(UPG == 1 || BAR0 + NUG - 1 <= 15, "named barriers");
  // X and Y of an update over the state blocks of its elements
  static_assert(2 * U::BUF <= (G >= 8 ? G : 8) * V::SE, "update buffers fit the state blocks");
};

// warps per CTA of the stage kernel: the volume kernel's default, lowered
// until update groups tile the CTA
template <int DIM, int N, bool CURVED, int W0>
constexpr int stage_warps() {
  using T = VolTile<DIM, N>;
  constexpr int UPG = T::G >= 8 ? 1 : 8 / T::G;
  int w = W0;
  while (w > T::H * UPG && (w / T::H) % UPG != 0) w -= T::H;
  return w;
}

template <int DIM, int N, bool CURVED, int W>
__global__ void __launch_bounds__(32 * W, 1)
stage_kernel(int K, const double *__restrict__ vgeo, const double *__restrict__ vfgeo,
             const double *__restrict__ fgeo, const uint32_t *__restrict__ mapPq,
             const double *__restrict__ nrJ, const double *__restrict__ nsJ,
             const double *__restrict__ ntJ, const double *__restrict__ Drq,
             const double *__restrict__ Dsq, const double *__restrict__ Dtq,
             const double *__restrict__ VqLq, const double *__restrict__ VfPq,
             const double *__restrict__ VqPq, const double *__restrict__ Jq, double fa,
             double fb, double fdt, const double *uq, const double *__restrict__ uf,
             double *__restrict__ Q, double *__restrict__ resQ, double *uq_out,
             double *__restrict__ uf_out, Phys P) {
  using S = StageCfg<DIM, N, CURVED, W>;
  using V = typename S::V;
  using U = typename S::U;
  constexpr int Nq = V::Nq, NF = V::NF, Nf = V::Nf, R = V::R, L = V::L, E = V::E, H = V::H,
                G = V::G, GT = 32 * H, UW = S::UW, UPG = S::UPG, SUB = S::SUB;
  constexpr bool PRE = V::C::PREFETCH;
  extern __shared__ double smem[];
  V v(smem);
  v.load_tables(nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp / H, tq = threadIdx.x - q * GT;
  const int pu = q / UPG, wu = warp - pu * UW, tu = threadIdx.x - pu * UW * 32;
  // first element of the update group within a batch
  const int ubase = pu * UPG * G;
  auto gsync = [&] {
    if (H == 1)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;\n" ::"r"(1 + q), "r"(GT) : "memory");
  };
  auto usync = [&] {
    if (UPG == 1)
      gsync();
    else
      asm volatile("bar.sync %0, %1;\n" ::"r"(S::BAR0 + pu), "r"(32 * UW) : "memory");
  };
  auto prefetch_group = [&](int kb) {
    const int kq = kb + q * G;
    if (kq < K) {
      const int n = min(K - kq, G) * NF * Nf;
      const double *src = uf + (size_t)kq * NF * Nf;
      double *dst = v.sPre + (size_t)q * G * NF * Nf;
      for (int t = tq; t < n; t += GT) cp_async8(dst + t, src + t);
    }
    cp_async_commit();
  };
  __syncthreads();  // the tables are shared by every group
  const int nb = (K + E - 1) / E;
  if (PRE) prefetch_group(min(blockIdx.x, nb) * E);

  for (int ib = blockIdx.x; ib < nb; ib += gridDim.x) {
    const int k0 = ib * E;
    if (PRE) cp_async_wait_all();
    // an update group whose elements all lie past the end has nothing to do;
    // its volume groups leave together
    if (k0 + ubase >= K) break;
    // a volume group past the end (but not its update group) only joins the
    // update; it must not read element K-1's state, which its owner may
    // already have overwritten
    const bool vact = k0 + q * G < K;
    if (vact) {
      gsync();  // the group's traces staged
      v.template prologue_group<false, GT>(K, k0, q * G, tq, vgeo, vfgeo, uq, uf, P,
                                           PRE ? v.sPre : nullptr);
      gsync();
    }
    const int knext = ib + gridDim.x < nb ? (ib + gridDim.x) * E : K;
    if (PRE) prefetch_group(knext);  // the next batch's traces, during the pairs
    if (vact) {
      double acc[R][Nf];
      v.group_pairs(acc, P, q * G, tq, GT, gsync);
      gsync();
      v.template surface<GT>(K, k0, q * G, tq, fgeo, mapPq, uf, P);
      gsync();
      v.lift(acc);
      v.park_rows(acc);
      gsync();
      const int k = k0 + v.e;
      if (k < K && v.h == 0) {
        const double *rowbuf = v.sSt + v.e * V::SE;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = v.l + L * r;
          if (i < Nq) {
            double *out = uq_out + (size_t)k * Nq * Nf + i;
#pragma unroll
            for (int f = 0; f < Nf; ++f) out[f * Nq] = H == 2 ? acc[r][f] + rowbuf[f * Nq + i] : acc[r][f];
          }
        }
      }
    }
    // ---- the update of the group's elements, 8 at a time
    usync();  // their RHS written; their state blocks free
    double *X = v.sSt + (size_t)ubase * V::SE;
    double *Y = X + U::BUF;
    for (int t = tu; t < (U::KP - Nq) * U::LD; t += 32 * UW) {
      X[Nq * U::LD + t] = 0.0;
      Y[Nq * U::LD + t] = 0.0;
    }
#pragma unroll 1
    for (int s = 0; s < SUB; ++s) {
      const int ku = k0 + ubase + s * 8;
      if (ku >= K) break;
      const int ne = min(8, K - ku);
      // (the LSRK operands load after each m-tile's product: registers are
      // scarce here, and the CTA's other groups hide the latency)
      double res0[2][Nf], q0[2][Nf], Jv[2];
      stage_rhs<Nq, Nf, U::LD, 32 * UW, true>(uq_out, ku, ne, X, [] {}, tu, usync);
      usync();
      update_group<DIM, N, CURVED, UW, false>(ku, ne, wu, lane, X, Y, Jq, VqPq, VfPq, fa, fb, fdt,
                                              resQ, Q, uq_out, uf_out, P, res0, q0, Jv, nullptr,
                                              usync);
      usync();  // X and Y read: the next update, or the next batch's states
    }
  }
}

}  // namespace wadg
