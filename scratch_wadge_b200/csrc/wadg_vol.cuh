// Pair-scheduled volume kernel (the default volume kernel) and the fused
// stage kernel built on it.
//
// The reference's volume kernels (one thread per row, Euler3Daffine.okl:152-417),
// organised so that every volume-face pair (i, f) is evaluated once: F_S(u_i, uf_f).nJ_f feeds both
// the volume row i (weight 1/2 VqLq_if) and the face row f (weight
// -1/2 VfPq_fi).  The reference evaluates it twice, once per row
// (Euler3Daffine.okl:327-362 and :387-406); the flux is symmetric in its two
// states, so the sums are the same.
//
// Layout.  A group of L lanes owns one element; lane l owns the R volume rows
// i = l + L*r (register accumulators; the padding row, if any, computes on a
// clamped index and is never stored).  Two warps share each group of G = 32/L
// elements (one where a half of the face nodes would be fewer than L): warp h
// walks half of the volume columns j and its own half of the face nodes,
// [f0_h, f0_h + n_h).  At face step s lane l takes face node
// f = f0_h + (l + s) mod n_h, so the L lanes of a group always touch L distinct
// face rows, and the two warps never the same one: both add their R
// contributions to one copy of the face-row accumulators in shared memory, a
// __syncwarp between steps ordering the read-modify-writes.  The schedule is
// fixed, so results are deterministic (no atomics).  Warps stay converged
// throughout so that ecflux_n_warp can vote on the log-mean branch.
//
// Persistent CTAs: operator tables are staged in shared memory once per CTA;
// the face weights in a rotated layout [r][s][l] so that the lanes of a step
// read consecutive words.  In the volume kernel's batch loop the warps of an
// element group synchronise only among themselves (named barriers): a
// group's shared memory is its own, so no group waits for another.
#pragma once

#include "wadg_device.cuh"

namespace wadg {

// Node-to-thread map: L lanes per element, R rows per lane.  RR = 0: about
// three rows per lane (L = the power of two >= Nq/3); RR > 0: about RR rows
// (an autotuner candidate where it pads less, e.g. 2D N=4: Nq = 16 fills
// L = 4 x 4 or 8 x 2 exactly, against 8 x 3 = 24 slots by default)
template <int DIM, int N, int RR = 0> struct VolTile {
  using El = Elem<DIM, N>;
  static constexpr int Lraw = RR > 0 ? (El::Nq + RR - 1) / RR : (El::Nq + 2) / 3;
  static constexpr int L = Lraw <= 1 ? 1 : Lraw <= 2 ? 2 : Lraw <= 4 ? 4 : Lraw <= 8 ? 8 : Lraw <= 16 ? 16 : 32;
  static constexpr int R = (El::Nq + L - 1) / L;
  static constexpr int G = 32 / L;  // elements per warp group
  static_assert(El::NfqNf >= L, "face schedule needs NfqNf >= L");
  // face halves of the two warps of an element (the second may be empty)
  static constexpr int nf0 = (El::NfqNf + 1) / 2, nf1 = El::NfqNf - nf0;
  static constexpr int H = nf1 >= L ? 2 : 1;  // warps per element group
  __host__ __device__ static constexpr int nf(int h) { return H == 1 ? El::NfqNf : (h ? nf1 : nf0); }
  __host__ __device__ static constexpr int f0(int h) { return h ? nf0 : 0; }
};

template <int DIM, int N, bool CURVED, int W, int RR = 0>
struct VolPairsCfg {
  using El = Elem<DIM, N>;
  using T = VolTile<DIM, N, RR>;
  static constexpr int H = T::H;                      // warps per element group
  static constexpr int threads = 32 * W;
  static constexpr int E = (W / H) * T::G;            // elements per batch
  // element strides in doubles: the state stride and the face-accumulator
  // stride are 4 mod 8, so the G groups of a warp start 8 banks apart
  // (conflict-free broadcasts, two wavefronts for a step's consecutive face rows)
  static constexpr int pad4of8(int x) { return ((x + 3) / 8) * 8 + 4; }   // == 4 mod 8
  static constexpr int pad2of4(int x) { return ((x + 1) / 4) * 4 + 2; }   // == 2 mod 4
  static constexpr int NGS = CURVED ? El::Nvgeo : 0;  // geometric factors per node
  static constexpr int mx(int a, int b) { return a > b ? a : b; }
  // the state block of an element is reused after the pair phase for the row
  // buffer and the update's staging arrays (3 x Nfields x Nq)
  static constexpr int SE = pad4of8(mx((El::NS + NGS) * El::NN, 3 * El::Nfields * El::Nq));
  static constexpr int SA = pad4of8(El::Nfields * El::NfqNf);
  static constexpr int SN = El::Nfaces * DIM + El::Nvgeo;
  static constexpr int nD = DIM * El::Nq * El::Nq;
  static constexpr int nW = T::R * El::NfqNf * T::L;
  static constexpr size_t fixed = sizeof(double) * (size_t)(nD + 2 * nW + El::Nfaces * DIM);
  static constexpr size_t per_elem = sizeof(double) * (size_t)(SE + SA + SN);
  static constexpr size_t smem = fixed + E * per_elem;
  // the volume kernel stages the next batch's face traces (cp.async) while it
  // computes the current one, where shared memory has room for them
  static constexpr size_t pre = sizeof(double) * (size_t)E * El::Nfields * El::NfqNf;
  static constexpr bool PREFETCH = smem + pre <= 227 * 1024;
  static constexpr size_t smem_vol = smem + (PREFETCH ? pre : 0);
};

// Shared-memory carve-up and the two phases common to both kernels.
template <int DIM, int N, bool CURVED, int W, int RR = 0>
struct VolPairs {
  using El = Elem<DIM, N>;
  using T = VolTile<DIM, N, RR>;
  using C = VolPairsCfg<DIM, N, CURVED, W, RR>;
  static constexpr int Nq = El::Nq, NF = El::NfqNf, Nfq = El::Nfq, NN = El::NN, NS = El::NS;
  static constexpr int Nf = El::Nfields, NG = El::Nvgeo, L = T::L, R = T::R, G = T::G, E = C::E;
  static constexpr int SE = C::SE, SA = C::SA, SN = C::SN, H = C::H;

  double *sD, *sW1, *sW2, *sNr, *sSt, *sAcc, *sNrm, *sPre;
  int tid, h, g, l, e;

  __device__ __forceinline__ VolPairs(double *smem) {
    sD = smem;                     // Drq | Dsq | Dtq, column-major
    sW1 = sD + C::nD;              // [h][R][n_h][L]  1/2 VqLq(i, f), 0 on padding rows
    sW2 = sW1 + C::nW;             // [h][R][n_h][L] -1/2 VfPq(f, i), 0 on padding rows
    sNr = sW2 + C::nW;             // reference normals [Nfaces][DIM]
    sSt = sNr + El::Nfaces * DIM;  // [E][SE]     node states (+ geometric factors)
    sAcc = sSt + E * SE;           // [E][SA]     face-row accumulators
    sNrm = sAcc + E * SA;          // [E][SN]     per-face nJ (affine) + G
    sPre = sNrm + E * SN;          // [E][Nf][NF] staged face traces (volume kernel, PREFETCH)
    tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    h = warp % H;
    g = lane / L;
    l = lane % L;
    e = (warp / H) * G + g;
  }

  __device__ __forceinline__ void load_tables(const double *nrJ, const double *nsJ,
                                              const double *ntJ, const double *Drq,
                                              const double *Dsq, const double *Dtq,
                                              const double *VqLq, const double *VfPq) {
    for (int t = tid; t < Nq * Nq; t += blockDim.x) {
      sD[t] = Drq[t];
      sD[Nq * Nq + t] = Dsq[t];
      if (DIM == 3) sD[2 * Nq * Nq + t] = Dtq[t];
    }
    for (int t = tid; t < C::nW; t += blockDim.x) {
      int hh = 0, u = t;
      if (H == 2 && u >= R * L * T::nf(0)) {
        hh = 1;
        u -= R * L * T::nf(0);
      }
      const int n_ = T::nf(hh);
      const int ll = u % L, s = (u / L) % n_, r = u / (L * n_);
      const int i = ll + L * r;
      int ff = ll + s;
      if (ff >= n_) ff -= n_;
      const int f = T::f0(hh) + ff;
      sW1[t] = i < Nq ? 0.5 * VqLq[i + f * Nq] : 0.0;
      sW2[t] = i < Nq ? -0.5 * VfPq[f + i * NF] : 0.0;
    }
    for (int t = tid; t < El::Nfaces; t += blockDim.x) {
      sNr[t * DIM + 0] = nrJ[t * Nfq];
      sNr[t * DIM + 1] = nsJ[t * Nfq];
      if (DIM == 3) sNr[t * DIM + 2] = ntJ[t * Nfq];
    }
  }

  // Node states of one element group's batch elements [e0, e0 + G), by TS
  // threads t0, t0 + TS, ...; elements past the end replicate the last
  // element so that every lane computes on valid data.  ufs: the group's
  // face traces already staged in shared memory, or null.  The states carry
  // no logarithms unless LOGS (fill_logs adds them where a group needs
  // them).  A thread's nodes go in chunks of four whose
  // loads (global for the volume nodes) are all issued before their node
  // states are computed.  The chunks run in a loop, not unrolled: unrolled,
  // the 3D affine volume + surface kernel spilled registers (20 -> 64 bytes)
  // and lost 2 %; rolled it gains 1.8 % there, 3 % in the affine volume
  // kernel, and the same 2-7 % as unrolled in the curved and 2D kernels
  template <bool LOGS, int TS>
  __device__ __forceinline__ void prologue_group(int K, int k0, int e0, int t0, const double *vgeo,
                                                 const double *vfgeo, const double *uq,
                                                 const double *uf, const Phys &P,
                                                 const double *ufs) {
    constexpr int NT = (G * NN + TS - 1) / TS;
    // the thread's nodes in chunks of CH: a chunk's loads all in flight, few
    // registers held
    constexpr int CH = 4;  // 2, 3 and 4 measured: 4 is 0.3-2 % ahead
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += CH) {
      double u[CH][Nf];
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int t = t0 + (c0 + j) * TS;
        if (c0 + j < NT && t < G * NN) {
          const int ee = e0 + t / NN, n = t % NN;
          const int k = min(k0 + ee, K - 1);
          // staged traces only for the group's own elements (a clamped
          // element's copy may sit in another group's range)
          const int kk = k - k0;
          const double *fsrc = (ufs && kk >= e0 && kk < e0 + G) ? ufs + (size_t)kk * NF * Nf
                                                               : uf + (size_t)k * NF * Nf;
          const double *src = (n < Nq) ? uq + (size_t)k * Nq * Nf + n : fsrc + (n - Nq);
          const int stride = (n < Nq) ? Nq : NF;
#pragma unroll
          for (int f = 0; f < Nf; ++f) u[j][f] = src[f * stride];
        } else {
#pragma unroll
          for (int f = 0; f < Nf; ++f) u[j][f] = 1.0;
        }
      }
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int t = t0 + (c0 + j) * TS;
        if (c0 + j < NT && t < G * NN) {
          const int ee = e0 + t / NN, n = t % NN;
          const int k = min(k0 + ee, K - 1);
          const NodeState<DIM> s = node_state<DIM, LOGS>(u[j], 1, P);
          double *st = sSt + ee * SE;
          st[0 * NN + n] = s.rho;
#pragma unroll
          for (int d = 0; d < DIM; ++d) st[(1 + d) * NN + n] = 0.5 * s.vel[d];  // stored halved
          st[(DIM + 1) * NN + n] = s.beta;
          if (LOGS) {
            st[(DIM + 2) * NN + n] = s.lrho;
            st[(DIM + 3) * NN + n] = s.lbeta;
          }
          if (CURVED) {  // geometric factors stored halved: a pair's average
                         // (G_i + G_j)/2 is then one addition, with the same bits
#pragma unroll
            for (int c = 0; c < NG; ++c)
              st[(NS + c) * NN + n] = 0.5 * ((n < Nq) ? vgeo[(size_t)k * Nq * NG + c * Nq + n]
                                                      : vfgeo[(size_t)k * NF * NG + c * NF + (n - Nq)]);
          }
        }
      }
    }
    for (int t = t0; t < G * SA; t += TS) sAcc[e0 * SA + t] = 0.0;
    if (!CURVED) {
      for (int t = e0 + t0; t < e0 + G; t += TS) {
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
  }

  // a node's state as the pair phase keeps it: velocity stored halved (u/2)
  __device__ __forceinline__ NodeState<DIM> load(const double *st, int n) const {
    NodeState<DIM> s;
    s.rho = st[n];
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.vel[d] = st[(1 + d) * NN + n];
    s.beta = st[(DIM + 1) * NN + n];
    s.lrho = st[(DIM + 2) * NN + n];
    s.lbeta = st[(DIM + 3) * NN + n];
    return s;
  }

  // all flux pairs of element e: this warp's half of the volume columns and of
  // the face nodes; rows into acc (registers), face rows into the element's
  // face accumulators
  // SMALL: every pair of the warp's elements has u < SMALL_U (small_pairs),
  // so the fluxes take the u^2 series without a vote
  template <bool SMALL>
  __device__ __forceinline__ void pairs(double (&acc)[R][Nf], const Phys &P) const {
    const double *st = sSt + e * SE;
    double *acc_f = sAcc + e * SA;
    NodeState<DIM> A[R];
    int ir[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      ir[r] = min(l + L * r, Nq - 1);  // padding row computes on a clamped index
      A[r] = load(st, ir[r]);
#pragma unroll
      for (int q = 0; q < Nf; ++q) acc[r][q] = 0.0;
    }
    double Ge[NG];
    if (!CURVED) {
#pragma unroll
      for (int c = 0; c < NG; ++c) Ge[c] = sNrm[e * SN + El::Nfaces * DIM + c];
    }

    // volume-volume pairs: warp h takes columns [j0, j1)
    const int j0 = (H == 2 && h) ? Nq / 2 : 0, j1 = (H == 2 && !h) ? Nq / 2 : Nq;
    for (int j = j0; j < j1; ++j) {
      const NodeState<DIM> B = load(st, j);
      double nv[R][DIM], F[R][Nf];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = ir[r];
        double rr[DIM];
#pragma unroll
        for (int a = 0; a < DIM; ++a) rr[a] = sD[a * Nq * Nq + i + j * Nq];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < DIM; ++a) {
            const double gad = CURVED ? st[(NS + a * DIM + d) * NN + i] + st[(NS + a * DIM + d) * NN + j]
                                      : Ge[a * DIM + d];
            v = fma(gad, rr[a], v);
          }
          nv[r][d] = v;
        }
      }
      ecflux_n_warp_hR<DIM, R, SMALL>(A, B, nv, P, F);
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < Nf; ++q) acc[r][q] += F[r][q];
    }

    // volume-face pairs, each evaluated once: warp h takes its face nodes
    const int nfh = T::nf(h), f0h = T::f0(h);
    const double *w1h = sW1 + R * L * f0h, *w2h = sW2 + R * L * f0h;
    for (int s = 0; s < nfh; ++s) {
      int ff = l + s;
      if (ff >= nfh) ff -= nfh;
      const int f = f0h + ff;
      const NodeState<DIM> B = load(st, Nq + f);
      const int fc = f / Nfq;
      double nv[DIM];
      if (!CURVED) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) nv[d] = sNrm[e * SN + fc * DIM + d];
      }
      double af[Nf];
#pragma unroll
      for (int q = 0; q < Nf; ++q) af[q] = 0.0;
      double nvr[R][DIM], F[R][Nf];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (CURVED) {
          const int i = ir[r];
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            double v = 0.0;
#pragma unroll
            for (int a = 0; a < DIM; ++a)
              v = fma(st[(NS + a * DIM + d) * NN + i] + st[(NS + a * DIM + d) * NN + Nq + f],
                      sNr[fc * DIM + a], v);
            nvr[r][d] = v;
          }
        } else {
#pragma unroll
          for (int d = 0; d < DIM; ++d) nvr[r][d] = nv[d];
        }
      }
      ecflux_n_warp_hR<DIM, R, SMALL>(A, B, nvr, P, F);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double w1 = w1h[(r * nfh + s) * L + l];
        const double w2 = w2h[(r * nfh + s) * L + l];
#pragma unroll
        for (int q = 0; q < Nf; ++q) {
          acc[r][q] = fma(w1, F[r][q], acc[r][q]);
          af[q] = fma(w2, F[r][q], af[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < Nf; ++q) acc_f[q * NF + f] += af[q];
      __syncwarp();
    }
  }

  // surface flux + Lax-Friedrichs penalty at the face points of the group's
  // batch elements [e0, e0 + G) (the TS threads t0, t0 + TS, ... of the
  // group), added to the face-row accumulators: sf = rhsQf + 1/2
  // F_S(u-, u+).nJ - tau/4 max(lam-, lam+) sJ (u+ - u-) (Euler3D.okl:3256-3346,
  // Euler2D.okl:1373-1453).  The minus state is the pair phase's node state
  // (velocity stored halved) and the trace in uf; the plus trace is gathered
  // from uf through mapPq (the neighbour indices of all of a thread's face
  // points are loaded first).
  template <int TS>
  __device__ __forceinline__ void surface(int K, int k0, int e0, int t0,
                                          const double *__restrict__ fgeo,
                                          const uint32_t *__restrict__ mapPq,
                                          const double *__restrict__ uf, const Phys &P) const {
    constexpr int NFG = El::Nfgeo, NPT = (G * NF + TS - 1) / TS;
    uint32_t idP[NPT];
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
      const int t = t0 + u * TS, k = k0 + e0 + t / NF;
      idP[u] = (t < G * NF && k < K) ? mapPq[t % NF + (size_t)k * NF] : 0u;
    }
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
      const int t = t0 + u * TS;
      const int ee = e0 + t / NF, f = t % NF, k = k0 + ee;
      if (t >= G * NF || k >= K) continue;
      const size_t idM = f + (size_t)k * NF * Nf;
      const double *fg = fgeo + (size_t)k * NF * NFG + f;
      double nJ[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) nJ[d] = fg[d * NF];
      const double sJ = fg[DIM * NF];
      double UM[Nf], UP[Nf];
#pragma unroll
      for (int q = 0; q < Nf; ++q) {
        UM[q] = uf[idM + q * NF];
        UP[q] = uf[idP[u] + q * NF];
      }
      NodeState<DIM> M = load(sSt + ee * SE, Nq + f);
#pragma unroll
      for (int d = 0; d < DIM; ++d) M.vel[d] *= 2.0;  // the pair phase's states hold u/2
      double kM, kP, c2M, c2P;
      node_state_surf<DIM>(UM, 1, P, kM, c2M);
      const NodeState<DIM> Pp = node_state_surf<DIM>(UP, 1, P, kP, c2P);
      double F[Nf];
      ecflux_n_nolog<DIM>(M, Pp, nJ, P, F);
      const double lamM = fsqrt(kM) + fsqrt(c2M);
      const double lamP = fsqrt(kP) + fsqrt(c2P);
      const double tau = (DIM == 3) ? P.tau : 1.0;
      const double Lfc = tau * 0.25 * fmax(lamM, lamP) * sJ;
      double *a0 = sAcc + ee * SA;
#pragma unroll
      for (int q = 0; q < Nf; ++q) a0[q * NF + f] = a0[q * NF + f] + 0.5 * F[q] - Lfc * (UP[q] - UM[q]);
    }
  }

  // lift: rows += VqLq sf on the rotated weights (VqLq = 2 W1), the warps of
  // the group splitting the face nodes as in the pair phase
  __device__ __forceinline__ void lift(double (&acc)[R][Nf]) const {
    const double *sf = sAcc + e * SA;
    const int nfh = T::nf(h), f0h = T::f0(h);
    const double *w1h = sW1 + R * L * f0h;
    for (int s = 0; s < nfh; ++s) {
      int ff = l + s;
      if (ff >= nfh) ff -= nfh;
      const int f = f0h + ff;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double w = 2.0 * w1h[(r * nfh + s) * L + l];
#pragma unroll
        for (int q = 0; q < Nf; ++q) acc[r][q] = fma(w, sf[q * NF + f], acc[r][q]);
      }
    }
  }

  // warp 1 parks its partial rows in element e's state block ([Nf][Nq]);
  // call between two __syncthreads
  // the per-node logarithms of the batch elements [e0, e0 + ne) (threads t0,
  // t0 + ts, ...), from the stored density and beta: the same values the
  // prologue's node_state would have stored
  __device__ __forceinline__ void fill_logs(int e0, int ne, int t0, int ts) const {
    for (int t = t0; t < ne * NN; t += ts) {
      double *st = sSt + (e0 + t / NN) * SE;
      const int n = t % NN;
      st[(DIM + 2) * NN + n] = log(st[n]);
      st[(DIM + 3) * NN + n] = log(st[(DIM + 1) * NN + n]);
    }
  }

  // The pair phase of the group (H warps, threads t0 .. t0 + ts - 1 over
  // the batch elements [e0, e0 + G), `gsync` its barrier), after a prologue
  // without logarithms: where every pair of the group's elements is nearly
  // equal (small_pairs) the pairs take the u^2 series with no vote and need
  // no logarithm; otherwise the logarithms are filled in first (they feed
  // the log-difference branch).
  template <typename Sync>
  __device__ __forceinline__ void group_pairs(double (&acc)[R][Nf], const Phys &P, int e0, int t0,
                                              int ts, Sync gsync) const {
    if (small_pairs<DIM, NN, L>(sSt + e * SE, l)) {
      pairs<true>(acc, P);
    } else {
      fill_logs(e0, G, t0, ts);
      gsync();
      pairs<false>(acc, P);
    }
  }

  __device__ __forceinline__ void park_rows(const double (&acc)[R][Nf]) const {
    double *rowbuf = sSt + e * SE;
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
  }
};

// SURF = false: the volume kernel (euler_vol_*): rhsQ <- the volume rows,
// rhsQf <- the face rows.  SURF = true: the volume and the surface kernel of
// a stage in one launch: after the pairs, the group adds the surface flux and
// penalty to its face rows (gathering the neighbours' traces from Qf through
// mapPq; Qf is only read, so every element's traces are final) and lifts
// them into its rows; rhsQ <- the whole right-hand side the surface kernel
// would leave, rhsQf is not written (fgeo and mapPq unused when false)
template <int DIM, int N, bool CURVED, int W, bool SURF = false, int RR = 0>
__global__ void __launch_bounds__(32 * W, 1)
vol_pairs_kernel(int K, const double *__restrict__ vgeo, const double *__restrict__ vfgeo,
                 const double *__restrict__ nrJ, const double *__restrict__ nsJ,
                 const double *__restrict__ ntJ, const double *__restrict__ Drq,
                 const double *__restrict__ Dsq, const double *__restrict__ Dtq,
                 const double *__restrict__ VqLq, const double *__restrict__ VfPq,
                 const double *__restrict__ Qf, double *__restrict__ rhsQ,
                 double *__restrict__ rhsQf, Phys P, const double *__restrict__ fgeo = nullptr,
                 const uint32_t *__restrict__ mapPq = nullptr,
                 const int *__restrict__ blist = nullptr, const int *__restrict__ nblist = nullptr) {
  using V = VolPairs<DIM, N, CURVED, W, RR>;
  constexpr int Nq = V::Nq, NF = V::NF, Nf = V::Nf, R = V::R, L = V::L, E = V::E, H = V::H;
  extern __shared__ double smem[];
  V v(smem);
  v.load_tables(nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq);
  constexpr bool PRE = V::C::PREFETCH;
  // After the tables, the H warps of an element group touch only their own
  // G elements' shared memory (states, face rows, normals, staged traces),
  // so within the batch loop they synchronise among themselves (a named
  // barrier per group) and never wait for the CTA's other groups.
  constexpr int G = V::G, GT = 32 * H;
  const int q = (threadIdx.x >> 5) / H, tq = threadIdx.x - q * GT;
  auto gsync = [&] {
    if (H == 1)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;\n" ::"r"(1 + q), "r"(GT) : "memory");
  };
  // stage the group's elements from kq on (face traces, a contiguous range
  // of Qf) into shared memory
  auto prefetch_group = [&](int kq) {
    if (kq < K) {
      const int n = min(K - kq, G) * NF * Nf;
      const double *src = Qf + (size_t)kq * NF * Nf;
      double *dst = v.sPre + (size_t)q * G * NF * Nf;
      for (int t = tq; t < n; t += GT) cp_async8(dst + t, src + t);
    }
    cp_async_commit();
  };
  __syncthreads();  // the tables are shared by every group
  // The work: batches of E elements, all of them or (a work list: the
  // ensemble's active instances) the ascending batch indices blist[0 ..
  // *nblist), each cut into its NG group slices of G elements.  The groups
  // take the slices independently: in round i group q of CTA b takes slice
  // (i NG + q) grid + b, so a last, partial round leaves the busy groups
  // spread over every SM (rather than whole CTAs busy and the other SMs
  // idle).  Every slice is G consecutive elements, so the elements that
  // share a warp, and the results, do not depend on the schedule.
  constexpr int NG = W / H;
  const int nb = blist ? *nblist : (K + E - 1) / E;
  const int ns = nb * NG, sstep = (int)gridDim.x * NG;
  auto slice = [&](int g) {  // first element of slice g (K past the end)
    if (g >= ns) return K;
    const int cb = g / NG;
    return (blist ? blist[cb] : cb) * E + (g - cb * NG) * G;
  };
  const int g0 = q * (int)gridDim.x + (int)blockIdx.x;
  if (PRE) prefetch_group(slice(g0));

  for (int gi = g0; gi < ns; gi += sstep) {
    const int kg = slice(gi);
    if (PRE) cp_async_wait_all();
    // a slice whose elements all lie past the end (of a partial last batch)
    // has nothing to compute, and must not read element K-1's input, which
    // the group owning it may already have overwritten with its RHS
    if (kg >= K) break;
    // the helpers index the group's elements as k0 + q G + (0 .. G-1)
    const int k0 = kg - q * G;
    gsync();  // the group's traces staged / its previous slice done with its shared memory
    v.template prologue_group<false, GT>(K, k0, q * G, tq, vgeo, vfgeo, rhsQ, Qf, P,
                                         PRE ? v.sPre : nullptr);
    gsync();
    if (PRE) prefetch_group(slice(gi + sstep));  // the next slice's traces, during the pairs
    double acc[R][Nf];
    v.group_pairs(acc, P, q * G, tq, GT, gsync);
    gsync();  // the group's pairs done: its state block becomes the row buffer
    if (SURF) {
      v.template surface<GT>(K, k0, q * G, tq, fgeo, mapPq, Qf, P);
      gsync();  // face rows complete (and the states read): lift, then park
      v.lift(acc);
    }
    v.park_rows(acc);
    gsync();
    const int k = k0 + v.e;
    if (k < K) {
      const double *rowbuf = v.sSt + v.e * V::SE;
      if (v.h == 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = v.l + L * r;
          if (i < Nq) {
            double *out = rhsQ + (size_t)k * Nq * Nf + i;
#pragma unroll
            for (int q = 0; q < Nf; ++q) out[q * Nq] = H == 2 ? acc[r][q] + rowbuf[q * Nq + i] : acc[r][q];
          }
        }
      }
      if (!SURF) {
        const double *a0 = v.sAcc + v.e * V::SA;
        double *outf = rhsQf + (size_t)k * NF * Nf;
        for (int t = v.h * L + v.l; t < NF * Nf; t += H * L) outf[t] = a0[t];
      }
    }
  }
}

}  // namespace wadg
