// Discrete adjoint of one LSRK stage of the entropy-stable RHS: device kernels.
//
// The stage (rk_step, euler.c:3610-3666, with the three kernels of
// Euler3Daffine.okl / Euler3D.okl / Euler2D.okl) maps (Q, res) to
//   res' = a res + dt R(Q),   Q' = Q + b res',
//   R(Q) = Minv rhs(u~(Q), uf~(Q)),
// where u~ = U(VqPq V(Q)) and uf~ = U(VfPq V(Q)) are the entropy-projected
// traces the previous update wrote (the WADG projection on curved elements),
// rhs is the volume + surface flux differencing and Minv the affine or
// weight-adjusted inverse mass.  Its adjoint, given (Qbar', resbar'):
//   r = resbar' + b Qbar',  resbar = a r,  Qbar = Qbar' + (dR/dQ)^T (dt r).
// Three kernels evaluate it:
//   adj_seed_mma_kernel  w = dt r, rhsbar = Minv^T w, sfbar = VqLq^T rhsbar
//                        (the adjoint of the lift rhsQ += VqLq sf;
//                        wadg_adjoint_mma.cuh)
//   adj_pairs_kernel     the VJP of every two-point flux evaluation
//                        (volume-volume, volume-face and surface, with the
//                        Lax-Friedrichs penalty), then the adjoints of the
//                        primitive recovery and of U(V~) at each volume and
//                        face node: vbar, vfbar (this file)
//   adj_proj_mma_kernel  the adjoint of the entropy projection and of V(Q), and
//                        the LSRK adjoint update of Qbar and resbar; in a
//                        reverse sweep it also seeds the next stage (so the
//                        seed kernel runs only for the sweep's first stage;
//                        wadg_adjoint_mma.cuh).
// Neighbour contributions of the surface term are gathered, not scattered:
// face node j adds the P-side derivative of the evaluation made at its
// neighbour m = mapPq(j), which needs sfbar at m -- computed, for every
// element, before the pair kernel starts -- and mapPq(m) = j (a conforming
// face pairing; checked on the host).
#pragma once

#include "wadg_adjoint_math.cuh"
#include "wadg_device.cuh"
#include "wadg_vol.cuh"

namespace wadg {

// node state of the pair VJP: NodeState plus 1/rho and 1/beta
template <int DIM> struct AdjNode {
  double rho, vel[DIM], beta, lrho, lbeta, irho, ibeta;
};

// F(u) = sum_{k<=8} u^k/(2k+1) and dF/du
__device__ __forceinline__ void polyF_d(double u, double &F, double &dF) {
  const double c[9] = {1.0, 1.0 / 3.0, 1.0 / 5.0, 1.0 / 7.0, 1.0 / 9.0,
                       1.0 / 11.0, 1.0 / 13.0, 1.0 / 15.0, 1.0 / 17.0};
  F = c[8];
  dF = 0.0;
#pragma unroll
  for (int k = 7; k >= 0; --k) {
    dF = fma(dF, u, F);
    F = fma(F, u, c[k]);
  }
}
// G(u) = 1/F(u) to degree 8 (the coefficients of polyG) and dG/du
__device__ __forceinline__ void polyG_d(double u, double &G, double &dG) {
  const double c[9] = {1.0, -1.0 / 3.0, -4.0 / 45.0, -44.0 / 945.0, -428.0 / 14175.0,
                       -10196.0 / 467775.0, -10719068.0 / 638512875.0,
                       -25865068.0 / 1915538625.0, -5472607916.0 / 488462349375.0};
  G = c[8];
  dG = 0.0;
#pragma unroll
  for (int k = 7; k >= 0; --k) {
    dG = fma(dG, u, G);
    G = fma(G, u, c[k]);
  }
}

// Vector-Jacobian product of the contracted two-point flux F_S(a, b).n
// (ecflux_n; Euler3Daffine.okl:107-148, Euler2D.okl:139-161) with the
// adjoint c of its Nfields components, split into the part that depends on
// the two states only (FluxCore: the means and their partial derivatives)
// and a reverse sweep per (n, c) that adds the adjoints of a's and b's
// primitive states (rho, velocity, beta) to ba and bb.
//
// Log-mean derivatives (L(a,b) = (a-b)/(log a - log b), s = a+b, f = (a-b)/s,
// u = f^2):
//   log form:    dL/da = (1 - L/a)/(log a - log b), dL/db = (L/b - 1)/(log a - log b)
//   series form: L = s/2 G(u): dL/da = G/2 + G'(u) f (1-f), dL/db = G/2 - G' f (1+f)
// and for 1/L (the inverse-temperature mean, 1/L = 2F(u)/s):
//   log form:    d(1/L)/da = (1/a - 1/L)/(a-b), d(1/L)/db = (1/L - 1/b)/(a-b)
//   series form: d(1/L)/da = 2/s^2 (-F + 2F' f(1-f)), d(1/L)/db = 2/s^2 (-F - 2F' f(1+f))
// with the same branch switch (u < 1e-2) as the forward flux.
template <int DIM> struct FluxCore {
  double rl, rla, rlb, ibl, ibla, iblb, pa, isb, ubar[DIM], vv;
};

__device__ __forceinline__ void rl_series(double sr, double fr, double G, double dG, double &rl,
                                          double &rla, double &rlb) {
  rl = 0.5 * sr * G;
  const double t = dG * fr;
  rla = fma(-t, fr, fma(0.5, G, t));
  rlb = fma(-t, fr, fma(0.5, G, -t));
}
__device__ __forceinline__ void ibl_series(double isb, double fb, double F, double dF,
                                           double &ibl, double &ibla, double &iblb) {
  ibl = 2.0 * isb * F;
  const double t2 = 2.0 * isb * isb, t = 2.0 * dF * fb;
  ibla = t2 * (fma(-t, fb, t) - F);
  iblb = t2 * (fma(-t, fb, -t) - F);
}

// WARP = true: must be called by all 32 lanes of a converged warp; when every
// lane has u < 1e-6 for both means (nearly equal states, e.g. the whole
// Taylor-Green field) the series are truncated at u^2 (remainders below
// 1e-18 relative in the means and 1e-13 in their u-derivatives, which enter
// multiplied by f < 1e-3).  SMALL = true: the caller has established u <
// SMALL_U (4e-6) for every pair of the warp's elements (small_pairs); the
// truncated series without a vote (remainders below 1e-17 in the means and
// 2e-11 in the derivatives, which enter multiplied by f < 2e-3).
template <int DIM, bool WARP, bool SMALL = false>
__device__ __forceinline__ FluxCore<DIM> flux_core(const AdjNode<DIM> &a, const AdjNode<DIM> &b) {
  FluxCore<DIM> k;
  const double sr = a.rho + b.rho, dr = a.rho - b.rho;
  const double sb = a.beta + b.beta, db = a.beta - b.beta;
  const double isr = rcp1(sr);  // forms only the series argument and f(1 -+ f)
  k.isb = rcp(sb);
  const double fr = dr * isr, fb = db * k.isb;
  const double ur = fr * fr, ub = fb * fb;
  if (SMALL || (WARP && __all_sync(0xffffffffu, fmax(ur, ub) < 1e-6))) {
    rl_series(sr, fr, fma(fma(ur, -4.0 / 45.0, -1.0 / 3.0), ur, 1.0), fma(ur, -8.0 / 45.0, -1.0 / 3.0),
              k.rl, k.rla, k.rlb);
    ibl_series(k.isb, fb, fma(fma(ub, 1.0 / 5.0, 1.0 / 3.0), ub, 1.0), fma(ub, 2.0 / 5.0, 1.0 / 3.0),
               k.ibl, k.ibla, k.iblb);
  } else if (WARP && __all_sync(0xffffffffu, fmax(ur, ub) < 1e-2)) {
    // every lane in the degree-8 series range for both means: the same
    // series as below, with no per-lane branch
    double G, dG, F, dF;
    polyG_d(ur, G, dG);
    rl_series(sr, fr, G, dG, k.rl, k.rla, k.rlb);
    polyF_d(ub, F, dF);
    ibl_series(k.isb, fb, F, dF, k.ibl, k.ibla, k.iblb);
  } else {
    if (ur < 1e-2) {
      double G, dG;
      polyG_d(ur, G, dG);
      rl_series(sr, fr, G, dG, k.rl, k.rla, k.rlb);
    } else {
      const double ild = rcp(a.lrho - b.lrho);
      k.rl = dr * ild;
      k.rla = fma(-k.rl, a.irho, 1.0) * ild;
      k.rlb = fma(k.rl, b.irho, -1.0) * ild;
    }
    if (ub < 1e-2) {
      double F, dF;
      polyF_d(ub, F, dF);
      ibl_series(k.isb, fb, F, dF, k.ibl, k.ibla, k.iblb);
    } else {
      const double idb = rcp(db);
      k.ibl = (a.lbeta - b.lbeta) * idb;
      k.ibla = (a.ibeta - k.ibl) * idb;
      k.iblb = (k.ibl - b.ibeta) * idb;
    }
  }
  k.pa = 0.5 * sr * k.isb;
  k.vv = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    k.ubar[d] = 0.5 * (a.vel[d] + b.vel[d]);
    k.vv = fma(a.vel[d], b.vel[d], k.vv);
  }
  return k;
}

// reverse sweep for one direction n and adjoint c; BSIDE = false skips b's adjoint
template <int DIM, bool BSIDE>
__device__ __forceinline__ void flux_rev(const FluxCore<DIM> &k, const AdjNode<DIM> &a,
                                         const AdjNode<DIM> &b, const double *n, const double *c,
                                         const Phys &P, double *ba, double *bb) {
  double un = 0.0, cu = 0.0, cn = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    un = fma(k.ubar[d], n[d], un);
    cu = fma(c[1 + d], k.ubar[d], cu);
    cn = fma(c[1 + d], n[d], cn);
  }
  const double h = fma(k.ibl, P.cbeta, 0.5 * k.vv);
  const double f4 = fma(k.rl, h, k.pa);
  const double F0 = k.rl * un;
  const double cE = c[DIM + 1];
  const double F0b = c[0] + cu;
  const double f4b = cE * un;
  const double unb = fma(F0b, k.rl, cE * f4);
  const double rlbar = fma(F0b, un, f4b * h);
  const double iblbar = f4b * k.rl * P.cbeta;
  const double vvb = 0.5 * f4b * k.rl;
  const double pab = cn + f4b;
  const double prho = 0.5 * pab * k.isb, pbeta = -pab * k.pa * k.isb;
  ba[0] = fma(rlbar, k.rla, ba[0] + prho);
  ba[DIM + 1] = fma(iblbar, k.ibla, ba[DIM + 1] + pbeta);
  if (BSIDE) {
    bb[0] = fma(rlbar, k.rlb, bb[0] + prho);
    bb[DIM + 1] = fma(iblbar, k.iblb, bb[DIM + 1] + pbeta);
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double hb = 0.5 * fma(c[1 + d], F0, unb * n[d]);
    ba[1 + d] = fma(vvb, b.vel[d], ba[1 + d] + hb);
    if (BSIDE) bb[1 + d] = fma(vvb, a.vel[d], bb[1 + d] + hb);
  }
}

template <int DIM, bool WARP, bool SMALL = false>
__device__ __forceinline__ void ecflux_vjp(const AdjNode<DIM> &a, const AdjNode<DIM> &b,
                                           const double *n, const double *c, const Phys &P,
                                           double *ba, double *bb) {
  const FluxCore<DIM> k = flux_core<DIM, WARP, SMALL>(a, b);
  flux_rev<DIM, true>(k, a, b, n, c, P, ba, bb);
}

// adjoint of the primitive recovery (rho, u = m/rho, beta = rho/(2p)) at a
// node: primitive adjoint pb -> conservative adjoint Ub; with p = rho/(2 beta),
// d beta/d(rho, m, E) = -2 beta^2/rho * dp/d(.) + (beta/rho, 0, 0)
template <int DIM>
__device__ __forceinline__ void prim_vjp_dev(const AdjNode<DIM> &s, const double *pb,
                                             const Phys &P, double *Ub) {
  double kin = 0.0, pu = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    kin = fma(s.vel[d], s.vel[d], kin);
    pu = fma(pb[1 + d], s.vel[d], pu);
  }
  const double q = -2.0 * s.beta * s.beta * s.irho * pb[DIM + 1];  // beta-bar * d beta / dp
  Ub[0] = pb[0] + pb[DIM + 1] * s.beta * s.irho + q * P.gm1 * 0.5 * kin - pu * s.irho;
#pragma unroll
  for (int d = 0; d < DIM; ++d) Ub[1 + d] = fma(pb[1 + d], s.irho, -q * P.gm1 * s.vel[d]);
  Ub[DIM + 1] = q * P.gm1;
}

// wave speed lambda = |u| + sqrt(gamma p / rho) = |u| + sqrt(gamma / (2 beta))
// and (GRAD) its gradient with respect to the conservative state
template <int DIM, bool GRAD>
__device__ __forceinline__ double lambda_dev(const AdjNode<DIM> &s, const Phys &P, double *dl) {
  double kin = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) kin = fma(s.vel[d], s.vel[d], kin);
  const double un = fsqrt(kin), c = fsqrt(0.5 * P.gamma * s.ibeta);
  if (GRAD) {
    // d|u|/drho = -|u|/rho, d|u|/dm = u/(|u| rho); dc = gamma/(2c) (dp/rho - p/rho^2)
    const double k = 0.5 * P.gamma * rcp(c) * s.irho;
    const double iun = un > 0.0 ? rcp(un) : 0.0;
    const double p_over_rho = 0.5 * s.ibeta;
    dl[0] = fma(k, fma(P.gm1 * 0.5, kin, -p_over_rho), -un * s.irho);
#pragma unroll
    for (int d = 0; d < DIM; ++d) dl[1 + d] = s.vel[d] * s.irho * fma(-k, P.gm1 * s.rho, iun);
    dl[DIM + 1] = k * P.gm1;
  }
  return un + c;
}

template <int DIM>
__device__ __forceinline__ AdjNode<DIM> adj_node(const double *q, int stride, const Phys &P) {
  const NodeState<DIM> s = node_state<DIM>(q, stride, P);
  AdjNode<DIM> a;
  a.rho = s.rho;
#pragma unroll
  for (int d = 0; d < DIM; ++d) a.vel[d] = s.vel[d];
  a.beta = s.beta;
  a.lrho = s.lrho;
  a.lbeta = s.lbeta;
  a.irho = rcp(s.rho);
  a.ibeta = rcp(s.beta);
  return a;
}

__device__ __forceinline__ adj::Gas gas_of(const Phys &P) {
  return adj::Gas{P.gamma, P.gm1, P.cbeta, P.lgm1, P.igm1};
}

// ------------------------------------------------------------------ pairs
// Layout as the pair-scheduled volume kernel (wadg_vol.cuh): a group of L
// lanes owns an element, lane l owns the volume rows i = l + L r, whose state,
// seed rhsbar(i) and primitive adjoint stay in registers.  The column partner
// of a step is staggered, j = j0 + (l + s) mod n, so the L lanes of a group
// touch L distinct columns and add their column adjoints to shared memory
// without conflicts (__syncwarp between steps).  With H = 2 the two warps of
// an element take disjoint halves of the columns, so they never write the
// same column; the row adjoints of the two warps are combined at the end.
// Every ordered volume pair (i, j) is one VJP (seed rhsbar(i), direction
// D_ij); every volume-face pair (i, f) is one VJP with the combined seed
// 1/2 VqLq(i,f) rhsbar(i) - 1/2 VfPq(f,i) sfbar(f), the two uses of that
// flux in the forward volume kernel.
template <int DIM, int N, bool CURVED, int W>
struct AdjPairsCfg {
  using El = Elem<DIM, N>;
  using T = VolTile<DIM, N>;
  static constexpr int Nq = El::Nq, NF = El::NfqNf, NN = El::NN, Nf = El::Nfields;
  static constexpr int L = T::L, R = T::R, G = T::G;
  static constexpr int nv0 = (Nq + 1) / 2, nv1 = Nq - nv0, nf0 = (NF + 1) / 2, nf1 = NF - nf0;
  static constexpr int H = (nv1 >= L && nf1 >= L) ? 2 : 1;
  static constexpr int NSA = DIM + 6;               // AdjNode fields
  static constexpr int NGS = CURVED ? El::Nvgeo : 0; // geometric factors per node
  static constexpr int NB = DIM + 2;                // primitive adjoint components
  static constexpr int threads = 32 * W;
  static constexpr int E = (W / H) * T::G;
  static constexpr int pad4of8(int x) { return ((x + 3) / 8) * 8 + 4; }
  static constexpr int SST = (NSA + NGS) * NN;  // node states (+ geometric factors)
  static constexpr int SSF = Nf * NF;           // sfbar of the face nodes
  static constexpr int SBR = NB * NN;           // column adjoints
  static constexpr int SN = El::Nfaces * DIM + El::Nvgeo;
  static constexpr int per_elem = pad4of8(SST + SSF + SBR + SN);
  static constexpr int nTD = DIM * R * Nq * L;
  static constexpr int nTW = R * NF * L;
  static constexpr size_t fixed = sizeof(double) * (size_t)(nTD + 2 * nTW + El::Nfaces * DIM);
  static constexpr size_t smem_core = fixed + sizeof(double) * (size_t)E * per_elem;
  // the next batch's face traces are staged (cp.async) during the pair phase
  // where shared memory has room for them
  static constexpr size_t pre = sizeof(double) * (size_t)E * Nf * NF;
  static constexpr bool PREFETCH = smem_core + pre <= 227 * 1024;
  static constexpr size_t smem = smem_core + (PREFETCH ? pre : 0);
  static_assert(W % H == 0, "warps per CTA must be a multiple of the warps per element");
};

template <int DIM, int N, bool CURVED, int W>
__global__ void __launch_bounds__(32 * W, 1)
adj_pairs_kernel(int K, const double *__restrict__ vgeo, const double *__restrict__ vfgeo,
                 const double *__restrict__ fgeo, const uint32_t *__restrict__ mapPq,
                 const double *__restrict__ nrJ, const double *__restrict__ nsJ,
                 const double *__restrict__ ntJ, const double *__restrict__ Drq,
                 const double *__restrict__ Dsq, const double *__restrict__ Dtq,
                 const double *__restrict__ VqLq, const double *__restrict__ VfPq,
                 const double *__restrict__ uq, const double *__restrict__ uf,
                 const double *__restrict__ rhsbar, const double *__restrict__ sfbar,
                 double *__restrict__ vbar, double *__restrict__ vfbar, Phys P) {
  using C = AdjPairsCfg<DIM, N, CURVED, W>;
  using El = Elem<DIM, N>;
  constexpr int Nq = C::Nq, NF = C::NF, NN = C::NN, Nf = C::Nf, L = C::L, R = C::R, G = C::G;
  constexpr int H = C::H, E = C::E, NSA = C::NSA, NB = C::NB, NG = El::Nvgeo, Nfq = El::Nfq;
  constexpr int NFG = El::Nfgeo;
  extern __shared__ double smem[];
  double *tD = smem;                 // [h][a][r][s][l]
  double *tW1 = tD + C::nTD;         // [h][r][s][l]  1/2 VqLq(i, f)
  double *tW2 = tW1 + C::nTW;        // [h][r][s][l] -1/2 VfPq(f, i)
  double *sNr = tW2 + C::nTW;        // [Nfaces][DIM]
  double *sEl = sNr + El::Nfaces * DIM;
  double *sPre = sEl + E * C::per_elem;  // [E][Nf][NF] staged face traces (PREFETCH)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int h = warp % H, g = lane / L, l = lane % L;
  const int e = (warp / H) * G + g;
  auto nv = [](int hh) { return H == 1 ? Nq : (hh ? C::nv1 : C::nv0); };
  auto nf = [](int hh) { return H == 1 ? NF : (hh ? C::nf1 : C::nf0); };
  auto cv = [](int hh) { return hh ? C::nv0 : 0; };
  auto cf = [](int hh) { return hh ? C::nf0 : 0; };

  // tables
  for (int t = tid; t < C::nTD; t += blockDim.x) {
    int hh = 0, u = t;
    if (H == 2 && u >= DIM * R * L * C::nv0) {
      hh = 1;
      u -= DIM * R * L * C::nv0;
    }
    const int n_ = nv(hh);
    const int ll = u % L, s = (u / L) % n_, r = (u / (L * n_)) % R, a = u / (L * n_ * R);
    const int i = ll + L * r;
    int jj = ll + s;
    if (jj >= n_) jj -= n_;
    const int j = cv(hh) + jj;
    const double *D = a == 0 ? Drq : (a == 1 ? Dsq : Dtq);
    tD[t] = i < Nq ? D[i + j * Nq] : 0.0;
  }
  for (int t = tid; t < C::nTW; t += blockDim.x) {
    int hh = 0, u = t;
    if (H == 2 && u >= R * L * C::nf0) {
      hh = 1;
      u -= R * L * C::nf0;
    }
    const int n_ = nf(hh);
    const int ll = u % L, s = (u / L) % n_, r = u / (L * n_);
    const int i = ll + L * r;
    int ff = ll + s;
    if (ff >= n_) ff -= n_;
    const int f = cf(hh) + ff;
    tW1[t] = i < Nq ? 0.5 * VqLq[i + f * Nq] : 0.0;
    tW2[t] = i < Nq ? -0.5 * VfPq[f + i * NF] : 0.0;
  }
  for (int t = tid; t < El::Nfaces; t += blockDim.x) {
    sNr[t * DIM + 0] = nrJ[t * Nfq];
    sNr[t * DIM + 1] = nsJ[t * Nfq];
    if (DIM == 3) sNr[t * DIM + 2] = ntJ[t * Nfq];
  }
  const double *tDh = tD + DIM * R * L * cv(h);
  const double *tW1h = tW1 + R * L * cf(h), *tW2h = tW2 + R * L * cf(h);
  const adj::Gas gas = gas_of(P);

  constexpr bool PRE = C::PREFETCH;
  // After the tables, the H warps of an element group touch only their own
  // G elements' shared memory, so within the batch loop they synchronise
  // among themselves (a named barrier per group), never with other groups.
  const int q = warp / H, tq = tid - q * 32 * H, e0 = q * G;
  constexpr int GT = 32 * H;
  auto gsync = [&] {
    if (H == 1)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;\n" ::"r"(1 + q), "r"(GT) : "memory");
  };
  // stage the group's elements of batch kb (face traces) into shared memory
  auto prefetch = [&](int kb) {
    const int kq = kb + e0;
    if (kq < K) {
      const int n = min(K - kq, G) * NF * Nf;
      const double *src = uf + (size_t)kq * NF * Nf;
      double *dst = sPre + (size_t)e0 * NF * Nf;
      for (int t = tq; t < n; t += GT) cp_async8(dst + t, src + t);
    }
    cp_async_commit();
  };
  __syncthreads();  // the tables are shared by every group
  if (PRE) prefetch(blockIdx.x * E);

  for (int k0 = blockIdx.x * E; k0 < K; k0 += gridDim.x * E) {
    if (PRE) cp_async_wait_all();
    gsync();  // the group's traces staged / its previous batch done with its shared memory
    // ---- prologue: node states, face seeds, zeroed column adjoints, normals
    // (the thread's nodes in chunks of four, each chunk's loads in flight
    // before its node states are computed, the chunks in a rolled loop:
    // reverse sweep 152.3 -> 148.0 ms at K=3072 against unrolled chunks of two)
    {
      constexpr int NT = (G * NN + GT - 1) / GT, CH = 4;
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += CH) {
        double u[CH][Nf];
#pragma unroll
        for (int j = 0; j < CH; ++j) {
          const int t = tq + (c0 + j) * GT;
          if (c0 + j < NT && t < G * NN) {
            const int ee = e0 + t / NN, n = t % NN;
            const int k = min(k0 + ee, K - 1);
            // staged traces only for the group's own elements (a clamped
            // element's copy may sit in another group's range)
            const int kk = k - k0;
            const double *fsrc = (PRE && kk >= e0 && kk < e0 + G) ? sPre + (size_t)kk * NF * Nf
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
          const int t = tq + (c0 + j) * GT;
          if (c0 + j < NT && t < G * NN) {
            const int ee = e0 + t / NN, n = t % NN;
            const int k = min(k0 + ee, K - 1);
            const AdjNode<DIM> s = adj_node<DIM>(u[j], 1, P);
            double *st = sEl + ee * C::per_elem;
            st[0 * NN + n] = s.rho;
#pragma unroll
            for (int d = 0; d < DIM; ++d) st[(1 + d) * NN + n] = s.vel[d];
            st[(DIM + 1) * NN + n] = s.beta;
            st[(DIM + 2) * NN + n] = s.lrho;
            st[(DIM + 3) * NN + n] = s.lbeta;
            st[(DIM + 4) * NN + n] = s.irho;
            st[(DIM + 5) * NN + n] = s.ibeta;
            if (CURVED) {
#pragma unroll
              for (int c = 0; c < NG; ++c)
                st[(NSA + c) * NN + n] = (n < Nq) ? vgeo[(size_t)k * Nq * NG + c * Nq + n]
                                                  : vfgeo[(size_t)k * NF * NG + c * NF + (n - Nq)];
            }
          }
        }
      }
    }
    for (int t = tq; t < G * C::SSF; t += GT) {
      const int ee = e0 + t / C::SSF, u = t % C::SSF;
      const int k = min(k0 + ee, K - 1);
      sEl[ee * C::per_elem + C::SST + u] = sfbar[(size_t)k * NF * Nf + u];
    }
    for (int t = tq; t < G * C::SBR; t += GT) {
      const int ee = e0 + t / C::SBR, u = t % C::SBR;
      sEl[ee * C::per_elem + C::SST + C::SSF + u] = 0.0;
    }
    if (!CURVED) {
      for (int t = e0 + tq; t < e0 + G; t += GT) {
        const int k = min(k0 + t, K - 1);
        double Gk[NG];
#pragma unroll
        for (int c = 0; c < NG; ++c) Gk[c] = vgeo[(size_t)k * Nq * NG + c * Nq];  // node 0 (:205)
        double *nm = sEl + t * C::per_elem + C::SST + C::SSF + C::SBR;
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
    gsync();
    if (PRE) prefetch(k0 + gridDim.x * E);  // the next batch's traces, during the pairs

    // ---- pairs
    const double *st = sEl + e * C::per_elem;
    const double *sfb = st + C::SST;
    double *bar = sEl + e * C::per_elem + C::SST + C::SSF;
    const double *nm = st + C::SST + C::SSF + C::SBR;
    auto load = [&](int n) {
      AdjNode<DIM> s;
      s.rho = st[n];
#pragma unroll
      for (int d = 0; d < DIM; ++d) s.vel[d] = st[(1 + d) * NN + n];
      s.beta = st[(DIM + 1) * NN + n];
      s.lrho = st[(DIM + 2) * NN + n];
      s.lbeta = st[(DIM + 3) * NN + n];
      s.irho = st[(DIM + 4) * NN + n];
      s.ibeta = st[(DIM + 5) * NN + n];
      return s;
    };
    const int kq = min(k0 + e, K - 1);
    AdjNode<DIM> A[R];
    int ir[R];
    double cr[R][Nf], rb[R][NB];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = l + L * r;
      ir[r] = min(i, Nq - 1);  // padding row: clamped state, zero seed
      A[r] = load(ir[r]);
#pragma unroll
      for (int q = 0; q < Nf; ++q)
        cr[r][q] = i < Nq ? rhsbar[(size_t)kq * Nq * Nf + q * Nq + i] : 0.0;
#pragma unroll
      for (int q = 0; q < NB; ++q) rb[r][q] = 0.0;
    }
    double Ge[NG];
    if (!CURVED) {
#pragma unroll
      for (int c = 0; c < NG; ++c) Ge[c] = nm[El::Nfaces * DIM + c];
    }

    // the pair loops: with a vote per pair (SM = false) or, where every pair
    // of the warp's elements is nearly equal (small_pairs), without
    auto pair_loops = [&](auto small_tag) {
    constexpr bool SM = decltype(small_tag)::value;
    // volume-volume pairs over this warp's column half
    {
      const int n_ = nv(h), j0 = cv(h);
      for (int s = 0; s < n_; ++s) {
        int jj = l + s;
        if (jj >= n_) jj -= n_;
        const int j = j0 + jj;
        const AdjNode<DIM> B = load(j);
        double cb[NB];
#pragma unroll
        for (int q = 0; q < NB; ++q) cb[q] = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          double rr[DIM], nvd[DIM];
#pragma unroll
          for (int a = 0; a < DIM; ++a) rr[a] = tDh[((a * R + r) * n_ + s) * L + l];
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            double v = 0.0;
#pragma unroll
            for (int a = 0; a < DIM; ++a) {
              const double gad = CURVED ? 0.5 * (st[(NSA + a * DIM + d) * NN + ir[r]] +
                                                 st[(NSA + a * DIM + d) * NN + j])
                                        : Ge[a * DIM + d];
              v = fma(gad, rr[a], v);
            }
            nvd[d] = v;
          }
          ecflux_vjp<DIM, !SM, SM>(A[r], B, nvd, cr[r], P, rb[r], cb);
        }
#pragma unroll
        for (int q = 0; q < NB; ++q) bar[q * NN + j] += cb[q];
        __syncwarp();
      }
    }
    // volume-face pairs over this warp's face half
    {
      const int n_ = nf(h), f0 = cf(h);
      for (int s = 0; s < n_; ++s) {
        int ff = l + s;
        if (ff >= n_) ff -= n_;
        const int f = f0 + ff;
        const AdjNode<DIM> B = load(Nq + f);
        const int fc = f / Nfq;
        double cfs[Nf], nvd[DIM];
#pragma unroll
        for (int q = 0; q < Nf; ++q) cfs[q] = sfb[q * NF + f];
        if (!CURVED) {
#pragma unroll
          for (int d = 0; d < DIM; ++d) nvd[d] = nm[fc * DIM + d];
        }
        double cb[NB];
#pragma unroll
        for (int q = 0; q < NB; ++q) cb[q] = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (CURVED) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
              double v = 0.0;
#pragma unroll
              for (int a = 0; a < DIM; ++a)
                v = fma(0.5 * (st[(NSA + a * DIM + d) * NN + ir[r]] +
                               st[(NSA + a * DIM + d) * NN + Nq + f]),
                        sNr[fc * DIM + a], v);
              nvd[d] = v;
            }
          }
          const double w1 = tW1h[(r * n_ + s) * L + l];
          const double w2 = tW2h[(r * n_ + s) * L + l];
          double c[Nf];
#pragma unroll
          for (int q = 0; q < Nf; ++q) c[q] = fma(w1, cr[r][q], w2 * cfs[q]);
          ecflux_vjp<DIM, !SM, SM>(A[r], B, nvd, c, P, rb[r], cb);
        }
#pragma unroll
        for (int q = 0; q < NB; ++q) bar[q * NN + Nq + f] += cb[q];
        __syncwarp();
      }
    }
    };
    if (small_pairs<DIM, NN, L>(st, l))
      pair_loops(BoolTag<true>());
    else
      pair_loops(BoolTag<false>());
    // row adjoints into the column adjoints, one warp of the element at a time
#pragma unroll
    for (int hh = 0; hh < H; ++hh) {
      gsync();
      if (h == hh) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = l + L * r;
          if (i < Nq) {
#pragma unroll
            for (int q = 0; q < NB; ++q) bar[q * NN + i] += rb[r][q];
          }
        }
      }
    }
    gsync();

    // ---- per node: surface term (face nodes), primitive recovery and U(V~) adjoints
    for (int t = tq; t < G * NN; t += GT) {
      const int ee = e0 + t / NN, n = t % NN, k = k0 + ee;
      if (k >= K) continue;
      const double *ste = sEl + ee * C::per_elem;
      const double *bt = ste + C::SST + C::SSF;
      AdjNode<DIM> own;
      own.rho = ste[n];
#pragma unroll
      for (int d = 0; d < DIM; ++d) own.vel[d] = ste[(1 + d) * NN + n];
      own.beta = ste[(DIM + 1) * NN + n];
      own.lrho = ste[(DIM + 2) * NN + n];
      own.lbeta = ste[(DIM + 3) * NN + n];
      own.irho = ste[(DIM + 4) * NN + n];
      own.ibeta = ste[(DIM + 5) * NN + n];
      double pb[NB], U[Nf], Ub[Nf], Vb[Nf];
#pragma unroll
      for (int q = 0; q < NB; ++q) pb[q] = bt[q * NN + n];
      if (n < Nq) {
        const double *qv = uq + (size_t)k * Nq * Nf + n;
#pragma unroll
        for (int f = 0; f < Nf; ++f) U[f] = qv[f * Nq];
        prim_vjp_dev<DIM>(own, pb, P, Ub);
      } else {
        // surface flux + Lax-Friedrichs penalty (Euler3Daffine.okl:421-552,
        // Euler3D.okl:3242-3473, Euler2D.okl:1357-1495):
        //   sf_j = 1/2 F_S(u_j, u_P).nJ_j - tau/4 max(lam_j, lam_P) sJ_j (u_P - u_j).
        // Face point j enters its own evaluation (as the minus side) and its
        // neighbour m's (as the plus side); the flux is symmetric in its two
        // states, so both are the a-side adjoint of one F_S(u_j, u_m) with
        // the two (direction, seed) pairs (nJ_j/2, sfbar_j) and (nJ_m/2, sfbar_m).
        const int j = n - Nq;
        const size_t idM = (size_t)k * NF * Nf + j;
        const size_t idP = mapPq[(size_t)k * NF + j];
        const size_t eP = idP / (size_t)(NF * Nf), jP = idP - eP * (size_t)(NF * Nf);
        double UP[Nf], cM[Nf], cP[Nf], nM[DIM], nP[DIM];
#pragma unroll
        for (int f = 0; f < Nf; ++f) {
          U[f] = uf[idM + f * NF];
          UP[f] = uf[idP + f * NF];
          cM[f] = ste[C::SST + f * NF + j];  // this element's sfbar, staged in shared memory
          cP[f] = sfbar[idP + f * NF];
        }
        const double *fgM = fgeo + (size_t)k * NF * NFG + j;
        const double *fgP = fgeo + eP * NF * NFG + jP;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          nM[d] = 0.5 * fgM[d * NF];
          nP[d] = 0.5 * fgP[d * NF];
        }
        const double sJM = fgM[DIM * NF], sJP = fgP[DIM * NF];
        const AdjNode<DIM> nb = adj_node<DIM>(UP, 1, P);
        const FluxCore<DIM> core = flux_core<DIM, false>(own, nb);
        flux_rev<DIM, false>(core, own, nb, nM, cM, P, pb, nullptr);
        flux_rev<DIM, false>(core, own, nb, nP, cP, P, pb, nullptr);
        prim_vjp_dev<DIM>(own, pb, P, Ub);
        double dl[Nf];
        const double lamM = lambda_dev<DIM, true>(own, P, dl);
        const double lamP = lambda_dev<DIM, false>(nb, P, nullptr);
        const double tq = (DIM == 3 ? P.tau : 1.0) * 0.25;
        const double lmax = fmax(lamM, lamP);
        double LbM = 0.0, LbP = 0.0;
#pragma unroll
        for (int f = 0; f < Nf; ++f) {
          const double du = UP[f] - U[f];
          Ub[f] = fma(tq * lmax, sJM * cM[f] - sJP * cP[f], Ub[f]);
          LbM = fma(-cM[f], du, LbM);  // adjoint of the own penalty scale
          LbP = fma(cP[f], du, LbP);   // ... and of the neighbour's (its jump is u_j - u_P)
        }
        // the max takes the branch the forward took (`lamM > lamP ? lamM : lamP`):
        // the own evaluation picks j when lam_j > lam_P; the neighbour's picks
        // j unless lam_P > lam_j
        const double gsel = (lamM > lamP ? LbM * sJM : 0.0) + (lamP > lamM ? 0.0 : LbP * sJP);
#pragma unroll
        for (int f = 0; f < Nf; ++f) Ub[f] = fma(tq * gsel, dl[f], Ub[f]);
      }
      adj::UV_vjp_U<DIM>(U, Ub, gas, Vb);
      if (n < Nq) {
        double *o = vbar + (size_t)k * Nq * Nf + n;
#pragma unroll
        for (int f = 0; f < Nf; ++f) o[f * Nq] = Vb[f];
      } else {
        double *o = vfbar + (size_t)k * NF * Nf + (n - Nq);
#pragma unroll
        for (int f = 0; f < Nf; ++f) o[f * NF] = Vb[f];
      }
    }
  }
}

}  // namespace wadg
