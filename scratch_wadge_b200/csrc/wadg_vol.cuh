// Volume flux-differencing kernel, pair-scheduled (the default volume kernel).
//
// Same mathematics as vol_kernel (wadg_kernels.cuh), organised so that every
// volume-face pair (i, f) is evaluated once: F_S(u_i, uf_f).nJ_f feeds both
// the volume row i (weight 1/2 VqLq_if) and the face row f (weight
// -1/2 VfPq_fi).  The reference evaluates it twice, once per row
// (Euler3Daffine.okl:327-362 and :387-406); the flux is symmetric in its two
// states, so the sums are the same.
//
// Layout.  A group of L lanes owns one element; lane l owns the R volume rows
// i = l + L*r (register accumulators; the padding row, if any, computes on a
// clamped index and is never stored).  Two warps share each group of G = 32/L
// elements: warp h walks half of the volume columns j and half of the face
// steps s.  At face step s lane l takes face node f = (l + s) mod NfqNf, so the
// L lanes of a group always touch L distinct face rows; each adds its R
// contributions to its warp's copy of the face-row accumulators in shared
// memory, and a __syncwarp between steps orders the read-modify-writes.  The
// schedule is fixed, so results are deterministic (no atomics).  Warps stay
// converged throughout so that ecflux_n_warp can vote on the log-mean branch.
//
// Persistent CTAs: operator tables are staged in shared memory once per CTA;
// the face weights in a rotated layout [r][s][l] so that the lanes of a step
// read consecutive words.
#pragma once

#include "wadg_device.cuh"

namespace wadg {

template <int DIM, int N> struct VolTile {
  using El = Elem<DIM, N>;
  static constexpr int Lraw = (El::Nq + 2) / 3;
  static constexpr int L = Lraw <= 1 ? 1 : Lraw <= 2 ? 2 : Lraw <= 4 ? 4 : Lraw <= 8 ? 8 : Lraw <= 16 ? 16 : 32;
  static constexpr int R = (El::Nq + L - 1) / L;
  static constexpr int G = 32 / L;  // elements per warp group
  static_assert(El::NfqNf >= L, "face schedule needs NfqNf >= L");
};

template <int DIM, int N, bool CURVED, int W>
struct VolPairsCfg {
  using El = Elem<DIM, N>;
  using T = VolTile<DIM, N>;
  static constexpr int H = 2;                         // warps per element group
  static constexpr int threads = 32 * W;
  static constexpr int E = (W / H) * T::G;            // elements per batch
  // element strides in doubles: the state stride is 4 mod 8 and the stride of
  // an element's pair of face accumulators (H*SA) is 4 mod 8, so the G groups
  // of a warp start 8 banks apart (conflict-free broadcasts, two wavefronts
  // for a step's consecutive face rows)
  static constexpr int pad4of8(int x) { return ((x + 3) / 8) * 8 + 4; }   // == 4 mod 8
  static constexpr int pad2of4(int x) { return ((x + 1) / 4) * 4 + 2; }   // == 2 mod 4
  static constexpr int NGS = CURVED ? El::Nvgeo : 0;  // geometric factors per node
  static constexpr int SE = pad4of8((El::NS + NGS) * El::NN);
  static constexpr int SA = pad2of4(El::Nfields * El::NfqNf);
  static constexpr int SN = El::Nfaces * DIM + El::Nvgeo;
  static constexpr int nD = DIM * El::Nq * El::Nq;
  static constexpr int nW = T::R * El::NfqNf * T::L;
  static constexpr size_t fixed = sizeof(double) * (size_t)(nD + 2 * nW + El::Nfaces * DIM);
  static constexpr size_t per_elem = sizeof(double) * (size_t)(SE + H * SA + SN);
  static constexpr size_t smem = fixed + E * per_elem;
  static_assert(SE >= El::Nfields * El::Nq, "row buffer reuses the state region");
};

template <int DIM, int N, bool CURVED, int W>
__global__ void __launch_bounds__(32 * W, 1)
vol_pairs_kernel(int K, const double *__restrict__ vgeo, const double *__restrict__ vfgeo,
                 const double *__restrict__ nrJ, const double *__restrict__ nsJ,
                 const double *__restrict__ ntJ, const double *__restrict__ Drq,
                 const double *__restrict__ Dsq, const double *__restrict__ Dtq,
                 const double *__restrict__ VqLq, const double *__restrict__ VfPq,
                 const double *__restrict__ Qf, double *__restrict__ rhsQ,
                 double *__restrict__ rhsQf, Phys P) {
  using El = Elem<DIM, N>;
  using T = VolTile<DIM, N>;
  using C = VolPairsCfg<DIM, N, CURVED, W>;
  constexpr int Nq = El::Nq, NF = El::NfqNf, Nfq = El::Nfq, NN = El::NN, NS = El::NS;
  constexpr int Nf = El::Nfields, NG = El::Nvgeo, L = T::L, R = T::R, G = T::G, E = C::E;
  constexpr int SE = C::SE, SA = C::SA, SN = C::SN, H = C::H;

  extern __shared__ double smem[];
  double *sD = smem;                       // Drq | Dsq | Dtq, column-major
  double *sW1 = sD + C::nD;                // [R][NF][L]  1/2 VqLq(i, f), 0 on padding rows
  double *sW2 = sW1 + C::nW;               // [R][NF][L] -1/2 VfPq(f, i), 0 on padding rows
  double *sNr = sW2 + C::nW;               // reference normals [Nfaces][DIM]
  double *sSt = sNr + El::Nfaces * DIM;    // [E][SE]      node states (+ geometric factors)
  double *sAcc = sSt + E * SE;             // [E][H][SA]   face-row accumulators, one per warp
  double *sNrm = sAcc + E * H * SA;        // [E][SN]      per-face nJ (affine) + G

  const int tid = threadIdx.x;
  for (int t = tid; t < Nq * Nq; t += blockDim.x) {
    sD[t] = Drq[t];
    sD[Nq * Nq + t] = Dsq[t];
    if (DIM == 3) sD[2 * Nq * Nq + t] = Dtq[t];
  }
  for (int t = tid; t < C::nW; t += blockDim.x) {
    const int l = t % L, s = (t / L) % NF, r = t / (L * NF);
    const int i = l + L * r;
    int f = l + s;
    if (f >= NF) f -= NF;
    sW1[t] = i < Nq ? 0.5 * VqLq[i + f * Nq] : 0.0;
    sW2[t] = i < Nq ? -0.5 * VfPq[f + i * NF] : 0.0;
  }
  for (int t = tid; t < El::Nfaces; t += blockDim.x) {
    sNr[t * DIM + 0] = nrJ[t * Nfq];
    sNr[t * DIM + 1] = nsJ[t * Nfq];
    if (DIM == 3) sNr[t * DIM + 2] = ntJ[t * Nfq];
  }

  const int warp = tid >> 5, lane = tid & 31;
  const int h = warp % H;
  const int g = lane / L, l = lane % L;
  const int e = (warp / H) * G + g;

  for (int k0 = blockIdx.x * E; k0 < K; k0 += gridDim.x * E) {
    __syncthreads();  // tables ready / previous batch done with shared memory
    // ---- node states of the batch (one thread per node); elements past the
    // end replicate the last element so that every lane computes on valid data
    for (int t = tid; t < E * NN; t += blockDim.x) {
      const int ee = t / NN, n = t % NN;
      const int k = min(k0 + ee, K - 1);
      const NodeState<DIM> s = (n < Nq) ? node_state<DIM>(rhsQ + (size_t)k * Nq * Nf + n, Nq, P)
                                        : node_state<DIM>(Qf + (size_t)k * NF * Nf + (n - Nq), NF, P);
      double *st = sSt + ee * SE;
      st[0 * NN + n] = s.rho;
#pragma unroll
      for (int d = 0; d < DIM; ++d) st[(1 + d) * NN + n] = s.vel[d];
      st[(DIM + 1) * NN + n] = s.beta;
      st[(DIM + 2) * NN + n] = s.lrho;
      st[(DIM + 3) * NN + n] = s.lbeta;
      if (CURVED) {
#pragma unroll
        for (int c = 0; c < NG; ++c)
          st[(NS + c) * NN + n] = (n < Nq) ? vgeo[(size_t)k * Nq * NG + c * Nq + n]
                                           : vfgeo[(size_t)k * NF * NG + c * NF + (n - Nq)];
      }
    }
    for (int t = tid; t < E * H * SA; t += blockDim.x) sAcc[t] = 0.0;
    if (!CURVED) {
      for (int t = tid; t < E; t += blockDim.x) {
        const int k = min(k0 + t, K - 1);
        double Gk[NG];
#pragma unroll
        for (int c = 0; c < NG; ++c) Gk[c] = vgeo[(size_t)k * Nq * NG + c * Nq];  // node 0 (:205)
        double *nm = sNrm + t * SN;
#pragma unroll
        for (int c = 0; c < NG; ++c) nm[El::Nfaces * DIM + c] = Gk[c];
        for (int fc = 0; fc < El::Nfaces; ++fc)
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            double v = 0.0;
#pragma unroll
            for (int a = 0; a < DIM; ++a) v = fma(Gk[a * DIM + d], sNr[fc * DIM + a], v);
            nm[fc * DIM + d] = v;
          }
      }
    }
    __syncthreads();

    const int k = k0 + e;
    const bool kval = k < K;
    double *st = sSt + e * SE;
    double *acc_f = sAcc + (e * H + h) * SA;
    auto load = [&](int n) {
      NodeState<DIM> s;
      s.rho = st[n];
#pragma unroll
      for (int d = 0; d < DIM; ++d) s.vel[d] = st[(1 + d) * NN + n];
      s.beta = st[(DIM + 1) * NN + n];
      s.lrho = st[(DIM + 2) * NN + n];
      s.lbeta = st[(DIM + 3) * NN + n];
      return s;
    };

    NodeState<DIM> A[R];
    int ir[R];
    double acc[R][Nf];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      ir[r] = min(l + L * r, Nq - 1);  // padding row computes on a clamped index
      A[r] = load(ir[r]);
#pragma unroll
      for (int q = 0; q < Nf; ++q) acc[r][q] = 0.0;
    }
    double Ge[NG];
    if (!CURVED) {
#pragma unroll
      for (int c = 0; c < NG; ++c) Ge[c] = sNrm[e * SN + El::Nfaces * DIM + c];
    }

    // ---- volume-volume pairs: warp h takes columns [j0, j1)
    const int j0 = h ? Nq / 2 : 0, j1 = h ? Nq : Nq / 2;
    for (int j = j0; j < j1; ++j) {
      const NodeState<DIM> B = load(j);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = ir[r];
        double rr[DIM], nv[DIM], F[Nf];
#pragma unroll
        for (int a = 0; a < DIM; ++a) rr[a] = sD[a * Nq * Nq + i + j * Nq];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < DIM; ++a) {
            const double gad = CURVED ? 0.5 * (st[(NS + a * DIM + d) * NN + i] + st[(NS + a * DIM + d) * NN + j])
                                      : Ge[a * DIM + d];
            v = fma(gad, rr[a], v);
          }
          nv[d] = v;
        }
        ecflux_n_warp<DIM>(A[r], B, nv, P, F);
#pragma unroll
        for (int q = 0; q < Nf; ++q) acc[r][q] += F[q];
      }
    }

    // ---- volume-face pairs, each evaluated once: warp h takes steps [s0, s1)
    const int s0 = h ? NF / 2 : 0, s1 = h ? NF : NF / 2;
    for (int s = s0; s < s1; ++s) {
      int f = l + s;
      if (f >= NF) f -= NF;
      const NodeState<DIM> B = load(Nq + f);
      const int fc = f / Nfq;
      double nv[DIM];
      if (!CURVED) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) nv[d] = sNrm[e * SN + fc * DIM + d];
      }
      double af[Nf];
#pragma unroll
      for (int q = 0; q < Nf; ++q) af[q] = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (CURVED) {
          const int i = ir[r];
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            double v = 0.0;
#pragma unroll
            for (int a = 0; a < DIM; ++a)
              v = fma(0.5 * (st[(NS + a * DIM + d) * NN + i] + st[(NS + a * DIM + d) * NN + Nq + f]),
                      sNr[fc * DIM + a], v);
            nv[d] = v;
          }
        }
        double F[Nf];
        ecflux_n_warp<DIM>(A[r], B, nv, P, F);
        const double w1 = sW1[(r * NF + s) * L + l];
        const double w2 = sW2[(r * NF + s) * L + l];
#pragma unroll
        for (int q = 0; q < Nf; ++q) {
          acc[r][q] = fma(w1, F[q], acc[r][q]);
          af[q] = fma(w2, F[q], af[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < Nf; ++q) acc_f[q * NF + f] += af[q];
      __syncwarp();
    }

    // ---- combine the two warps' partial rows; write rows and face rows
    __syncthreads();  // all pairs done: the state region becomes the row buffer
    double *rowbuf = st;  // [Nf][Nq] partial rows of warp 1
    if (h == 1) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = l + L * r;
        if (i < Nq) {
#pragma unroll
          for (int q = 0; q < Nf; ++q) rowbuf[q * Nq + i] = acc[r][q];
        }
      }
    }
    __syncthreads();
    if (kval) {
      if (h == 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = l + L * r;
          if (i < Nq) {
            double *out = rhsQ + (size_t)k * Nq * Nf + i;
#pragma unroll
            for (int q = 0; q < Nf; ++q) out[q * Nq] = acc[r][q] + rowbuf[q * Nq + i];
          }
        }
      }
      const double *a0 = sAcc + (e * H + 0) * SA, *a1 = sAcc + (e * H + 1) * SA;
      double *outf = rhsQf + (size_t)k * NF * Nf;
      for (int t = h * L + l; t < NF * Nf; t += H * L) outf[t] = a0[t] + a1[t];
    }
  }
}

}  // namespace wadg
