// Device building blocks of the entropy-stable flux-differencing RHS:
// compile-time element sizes, FP64 reciprocal, log-mean, two-point EC flux,
// conservative <-> entropy variables.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wadg {

// Element sizes of the reference's operator builder for cubature degree 2N
// (tri_cubature / tet_cubature tables of node_data.h as used by
// build_ref_ops_2D/3D, operators.cpp:104-341).
template <int DIM, int N> struct Sizes;
template <> struct Sizes<2, 1> { static constexpr int Np = 3,  Nq = 3,  Nfq = 2;  };
template <> struct Sizes<2, 2> { static constexpr int Np = 6,  Nq = 6,  Nfq = 3;  };
template <> struct Sizes<2, 3> { static constexpr int Np = 10, Nq = 12, Nfq = 4;  };
template <> struct Sizes<2, 4> { static constexpr int Np = 15, Nq = 16, Nfq = 5;  };
template <> struct Sizes<3, 1> { static constexpr int Np = 4,  Nq = 4,  Nfq = 3;  };
template <> struct Sizes<3, 2> { static constexpr int Np = 10, Nq = 11, Nfq = 6;  };
template <> struct Sizes<3, 3> { static constexpr int Np = 20, Nq = 23, Nfq = 12; };
template <> struct Sizes<3, 4> { static constexpr int Np = 35, Nq = 44, Nfq = 16; };

template <int DIM, int N> struct Elem {
  static constexpr int Nfaces = DIM + 1;
  static constexpr int Nq = Sizes<DIM, N>::Nq;
  static constexpr int Nfq = Sizes<DIM, N>::Nfq;
  static constexpr int NfqNf = Nfq * Nfaces;
  static constexpr int Nfields = DIM + 2;
  static constexpr int Nvgeo = DIM * DIM;
  static constexpr int Nfgeo = DIM + 1;
  static constexpr int NN = Nq + NfqNf;   // volume + face nodes
  static constexpr int NS = DIM + 4;      // rho, velocity, beta, log rho, log beta
};

// 8-byte asynchronous global -> shared copies (cp.async, sm_80 and later):
// the copies of a block are in flight together, occupying no registers, while
// the issuing threads go on computing; commit + wait completes them
__device__ __forceinline__ void cp_async8(double *dst_smem, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

struct Phys {
  double gamma;
  double gm1;     // gamma - 1
  double cbeta;   // 1 / (2 (gamma - 1))
  double tau;     // LF penalty scale of the surface kernel
  double lgm1;    // log(gamma - 1)
  double igm1;    // 1 / (gamma - 1)
};

// 1/x: Newton-Raphson refinement (two steps, quadratic convergence) of the
// hardware reciprocal estimate rcp.approx.ftz.f64.  Accurate to a few ulp for
// the positive, normal-range arguments it is used on (sums of densities and
// inverse temperatures, log differences).
__device__ __forceinline__ double rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  return y;
}

// 1/x with one Newton-Raphson step: relative error ~1e-14, for quantities
// that only feed a series argument or a branch test (the log-mean's u), never
// a result directly.
__device__ __forceinline__ double rcp1(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// Log-mean of a, b > 0: (a - b) / (log a - log b).
//
// The reference (Euler3Daffine.okl:43-71, Euler2D.okl:36-67) evaluates
// (a + b) / (2F) with F = log(xi)/(2f), f = (xi-1)/(xi+1), xi = a/b, and
// replaces F by its Taylor series F(u) = sum_k u^k/(2k+1), u = f^2, when u is
// small.  Here log a and log b are computed once per node, so
//   * for u < 1e-2 the series is used (degree 8 in u: truncation below 1e-18
//     relative, so this branch is accurate to rounding over a wider range than
//     the reference's 1e-4 / 1e-3 switch, where the log-difference would lose
//     digits to cancellation);
//   * otherwise (a+b)/(2F) = (a-b)/(log a - log b), where |log a - log b| >=
//     0.2 keeps the cancellation error of the difference below ~1e-14.
// Both branches agree with the reference's to rounding (parity tests hold
// them to 1e-12 relative).
__device__ __forceinline__ double polyF(double u) {  // sum_{k<=8} u^k/(2k+1)
  double p = 1.0 / 17.0;
  p = fma(p, u, 1.0 / 15.0);
  p = fma(p, u, 1.0 / 13.0);
  p = fma(p, u, 1.0 / 11.0);
  p = fma(p, u, 1.0 / 9.0);
  p = fma(p, u, 1.0 / 7.0);
  p = fma(p, u, 1.0 / 5.0);
  p = fma(p, u, 1.0 / 3.0);
  return fma(p, u, 1.0);
}
// 1/F(u) to degree 8 (coefficients of the series reciprocal, exact rationals)
__device__ __forceinline__ double polyG(double u) {
  double p = -5472607916.0 / 488462349375.0;
  p = fma(p, u, -25865068.0 / 1915538625.0);
  p = fma(p, u, -10719068.0 / 638512875.0);
  p = fma(p, u, -10196.0 / 467775.0);
  p = fma(p, u, -428.0 / 14175.0);
  p = fma(p, u, -44.0 / 945.0);
  p = fma(p, u, -4.0 / 45.0);
  p = fma(p, u, -1.0 / 3.0);
  return fma(p, u, 1.0);
}

__device__ __forceinline__ double logmean(double a, double b, double la, double lb) {
  const double d = a - b, s = a + b;
  if (d * d < 1e-2 * (s * s)) {
    const double f = d * rcp(s);
    return 0.5 * s * polyG(f * f);
  }
  return d * rcp(la - lb);
}

// 1 / logmean(a, b), and 1/(a+b) through `isum`
__device__ __forceinline__ double inv_logmean(double a, double b, double la, double lb,
                                              double &isum) {
  const double d = a - b, s = a + b;
  isum = rcp(s);
  if (d * d < 1e-2 * (s * s)) {
    const double f = d * isum;
    return 2.0 * isum * polyF(f * f);
  }
  return (la - lb) * rcp(d);
}

// Per-node state of the two-point flux: everything of euler3d_flux /
// euler2d_flux (Euler3Daffine.okl:107-148, Euler2D.okl:139-161) that depends
// on one node only.
template <int DIM> struct NodeState {
  double rho, vel[DIM], beta, lrho, lbeta;
};

// from conservative variables q[f*stride]; beta = rho / (2p)
// (Euler3Daffine.okl:22-26 pfun/beta, Euler2D.okl:19-21)
// LOGS = false: lrho and lbeta are left 0 (the caller fills them where the
// log-difference branch of the log-mean may be taken)
template <int DIM, bool LOGS = true>
__device__ __forceinline__ NodeState<DIM> node_state(const double *q, int stride, const Phys &P) {
  NodeState<DIM> s;
  s.rho = q[0];
  const double ir = rcp(s.rho);
  double kin = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.vel[d] = q[(1 + d) * stride] * ir;
    kin = fma(s.vel[d], s.vel[d], kin);
  }
  const double E = q[(DIM + 1) * stride];
  const double p = P.gm1 * (E - 0.5 * s.rho * kin);
  s.beta = 0.5 * s.rho * rcp(p);
  s.lrho = LOGS ? log(s.rho) : 0.0;
  s.lbeta = LOGS ? log(s.beta) : 0.0;
  return s;
}

// Chandrashekar's entropy-conservative flux F_S(a, b) contracted with the
// direction n:  F.n  (the reference forms FxS, FyS, FzS and then
// FxS*nx + FyS*ny + FzS*nz; this is the same sum regrouped):
//   rholog = L(rho), betalog = L(beta), ubar = (ua+ub)/2,
//   pa = rhoavg / (2 betaavg),  un = ubar.n,
//   F0 = rholog un, Fm = F0 ubar + pa n,
//   FE = (rholog/(2(gamma-1) betalog) + pa + rholog (ua.ub)/2) un
// where ua.ub equals the reference's 2|ubar|^2 - avg(|u|^2).
template <int DIM>
__device__ __forceinline__ void ecflux_n(const NodeState<DIM> &a, const NodeState<DIM> &b,
                                         const double *n, const Phys &P, double *F) {
  double isb;
  const double ibl = inv_logmean(a.beta, b.beta, a.lbeta, b.lbeta, isb);
  const double rl = logmean(a.rho, b.rho, a.lrho, b.lrho);
  const double pa = 0.5 * (a.rho + b.rho) * isb;
  double ub[DIM], un = 0.0, vv = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    ub[d] = 0.5 * (a.vel[d] + b.vel[d]);
    un = fma(ub[d], n[d], un);
    vv = fma(a.vel[d], b.vel[d], vv);
  }
  const double f4 = fma(rl, fma(ibl, P.cbeta, 0.5 * vv), pa);
  const double F0 = rl * un;
  F[0] = F0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = fma(F0, ub[d], pa * n[d]);
  F[DIM + 1] = f4 * un;
}

// conservative -> entropy variables (Euler3Daffine.okl:73-93 / Euler2D.okl:69-87)
template <int DIM>
__device__ __forceinline__ void VU(const double *U, double *V, const Phys &P) {
  const double rho = U[0], E = U[DIM + 1];
  double m2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) m2 = fma(U[1 + d], U[1 + d], m2);
  const double rhoe = E - 0.5 * m2 * rcp(rho);
  // s = log((gamma-1) rhoe / rho^gamma), written with two logarithms
  const double s = log(P.gm1 * rhoe) - P.gamma * log(rho);
  const double irhoe = rcp(rhoe);
  V[0] = (-E + rhoe * (P.gamma + 1.0 - s)) * irhoe;
#pragma unroll
  for (int d = 0; d < DIM; ++d) V[1 + d] = U[1 + d] * irhoe;
  V[DIM + 1] = -rho * irhoe;
}

// entropy -> conservative variables (Euler3Daffine.okl:95-105 / Euler2D.okl:89-98)
template <int DIM>
__device__ __forceinline__ void UV(const double *V, double *U, const Phys &P) {
  const double Vl = V[DIM + 1];
  double vv = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) vv = fma(V[1 + d], V[1 + d], vv);
  const double h = 0.5 * vv * rcp(Vl);  // vv / (2 V_l)
  const double sV = P.gamma - V[0] + h;
  // rhoe = ((gamma-1)/(-V_l)^gamma)^(1/(gamma-1)) exp(-sV/(gamma-1)), as one
  // exponential: exp((log(gamma-1) - gamma log(-V_l) - sV) / (gamma-1)).
  // For air (gamma = 1.4) the power is (-V_l)^(-7/2) = 1 / ((-V_l)^3
  // sqrt(-V_l)): a square root and a reciprocal in place of the logarithm
  // (within a few ulp of the general form)
  double rhoe;
  if (P.gamma == 1.4) {
    const double mv = -Vl;
    rhoe = exp((P.lgm1 - sV) * P.igm1) * rcp(mv * mv * mv * sqrt(mv));
  } else {
    rhoe = exp((P.lgm1 - P.gamma * log(-Vl) - sV) * P.igm1);
  }
  U[0] = -rhoe * Vl;
#pragma unroll
  for (int d = 0; d < DIM; ++d) U[1 + d] = rhoe * V[1 + d];
  U[DIM + 1] = rhoe * (1.0 - h);
}

}  // namespace wadg

namespace wadg {

// Two-point flux for converged warps.  Same value as ecflux_n; the log-mean
// evaluation is chosen per warp when every lane agrees:
//   * all lanes have u = ((a-b)/(a+b))^2 < 1e-6 for both density and inverse
//     temperature (nearly equal states, e.g. the whole Taylor-Green field):
//     the series truncated at u^2, whose remainder is below 5e-20 relative;
//   * otherwise each lane takes the degree-8 series (u < 1e-2) or the
//     log-difference, as in logmean / inv_logmean.
// The branch test reuses f = (a-b)/(a+b), which the series needs anyway.
// Must be called by all 32 lanes of the warp.
__device__ __forceinline__ double polyF2(double u) { return fma(fma(u, 1.0 / 5.0, 1.0 / 3.0), u, 1.0); }
// 2 polyF2(u) and 2 polyF(u) with the factor 2 in the coefficients: scaling
// by 2 is exact and commutes with rounding, so these are the same bits as
// 2.0 * poly, one multiplication fewer where the result multiplies isb
__device__ __forceinline__ double polyF2x2(double u) { return fma(fma(u, 2.0 / 5.0, 2.0 / 3.0), u, 2.0); }
__device__ __forceinline__ double polyFx2(double u) {
  double p = 2.0 / 17.0;
  p = fma(p, u, 2.0 / 15.0);
  p = fma(p, u, 2.0 / 13.0);
  p = fma(p, u, 2.0 / 11.0);
  p = fma(p, u, 2.0 / 9.0);
  p = fma(p, u, 2.0 / 7.0);
  p = fma(p, u, 2.0 / 5.0);
  p = fma(p, u, 2.0 / 3.0);
  return fma(p, u, 2.0);
}
__device__ __forceinline__ double polyG2(double u) { return fma(fma(u, -4.0 / 45.0, -1.0 / 3.0), u, 1.0); }

template <int DIM>
__device__ __forceinline__ void ecflux_n_warp(const NodeState<DIM> &a, const NodeState<DIM> &b,
                                              const double *n, const Phys &P, double *F) {
  const double sr = a.rho + b.rho, dr = a.rho - b.rho;
  const double sb = a.beta + b.beta, db = a.beta - b.beta;
  // 1/(a+b) of the densities only forms the series argument ur (and its
  // branch test): one Newton step suffices; 1/(a+b) of beta enters pa and the
  // mean itself, so it gets two
  const double isr = rcp1(sr), isb = rcp(sb);
  const double fr = dr * isr, fb = db * isb;
  const double ur = fr * fr, ub = fb * fb;
  double rl, ibl;
  if (__all_sync(0xffffffffu, fmax(ur, ub) < 1e-6)) {
    rl = 0.5 * sr * polyG2(ur);
    ibl = 2.0 * isb * polyF2(ub);
  } else {
    rl = (ur < 1e-2) ? 0.5 * sr * polyG(ur) : dr * rcp(a.lrho - b.lrho);
    ibl = (ub < 1e-2) ? 2.0 * isb * polyF(ub) : (a.lbeta - b.lbeta) * rcp(db);
  }
  const double pa = 0.5 * sr * isb;
  double ub2[DIM], un = 0.0, vv = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    ub2[d] = 0.5 * (a.vel[d] + b.vel[d]);
    un = fma(ub2[d], n[d], un);
    vv = fma(a.vel[d], b.vel[d], vv);
  }
  const double f4 = fma(rl, fma(ibl, P.cbeta, 0.5 * vv), pa);
  const double F0 = rl * un;
  F[0] = F0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = fma(F0, ub2[d], pa * n[d]);
  F[DIM + 1] = f4 * un;
}

template <bool B> struct BoolTag {
  static constexpr bool value = B;
};

// Pairs of nearly equal states.  The log-mean series truncated at u^2 (u =
// ((a-b)/(a+b))^2) leaves a relative remainder below u^3/7 in F and below
// 0.05 u^3 in its reciprocal G: under 1e-17 -- a tenth of the rounding of the
// sum itself -- for u < SMALL_U.  small_pairs tells whether every pair that
// the warp's elements form, volume-volume and volume-face, has u < SMALL_U
// for the density and for beta: over an element's nodes u is largest for the
// extreme pair, ((max - min)/(max + min))^2.  The L lanes of an element group
// (lane l reads nodes l, l + L, ... of its state block `st`: rho at [n],
// beta at [(DIM+1) NN + n]) reduce by shuffles.  Must be called by all 32
// lanes of the warp.  A warp that passes runs its pair loops without any
// per-pair vote or branch (a loop body the compiler schedules across
// columns); on the Taylor-Green workload every element passes (largest u
// 2.9e-6), on the curved density wave none does (u up to 3e-2).
constexpr double SMALL_U = 4e-6;
template <int DIM, int NN, int L>
__device__ __forceinline__ bool small_pairs(const double *st, int l) {
  double rmin = st[0], rmax = rmin, bmin = st[(DIM + 1) * NN], bmax = bmin;
  for (int n = l; n < NN; n += L) {
    const double r = st[n], b = st[(DIM + 1) * NN + n];
    rmin = fmin(rmin, r);
    rmax = fmax(rmax, r);
    bmin = fmin(bmin, b);
    bmax = fmax(bmax, b);
  }
#pragma unroll
  for (int o = L / 2; o >= 1; o >>= 1) {
    rmin = fmin(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    bmin = fmin(bmin, __shfl_xor_sync(0xffffffffu, bmin, o));
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
  }
  const double fr = (rmax - rmin) / (rmax + rmin), fb = (bmax - bmin) / (bmax + bmin);
  // positive states only; a NaN fails the comparisons
  const bool ok = rmin > 0.0 && bmin > 0.0 && fr * fr < SMALL_U && fb * fb < SMALL_U;
  return __all_sync(0xffffffffu, ok);
}

// ecflux_n_warp_h for R row states a[r] against one column state b: one
// warp vote for all R pairs of every lane (the u^2 series when all of them
// have u < 1e-6; else the degree-8 series, without the per-lane choice of
// the log-difference, when all of them have u < 1e-2), then the R fluxes side
// by side -- independent chains in one basic block, which the scheduler
// interleaves.  Same value per pair as ecflux_n_warp_h to rounding.  Must be
// called by all 32 lanes of the warp.
// SMALL = true: the caller has established u < SMALL_U for every pair
// (small_pairs); the u^2 series, no vote.
template <int DIM, int R, bool SMALL = false>
__device__ __forceinline__ void ecflux_n_warp_hR(const NodeState<DIM> (&a)[R], const NodeState<DIM> &b,
                                                 const double (&n)[R][DIM], const Phys &P,
                                                 double (&F)[R][DIM + 2]) {
  double hsr[R], dr[R], db[R], isb[R], ur[R], ub[R];
  bool small = true, mid = true;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double sr = a[r].rho + b.rho, sb = a[r].beta + b.beta;
    dr[r] = a[r].rho - b.rho;
    db[r] = a[r].beta - b.beta;
    const double isr = rcp1(sr);
    isb[r] = rcp(sb);
    const double fr = dr[r] * isr, fb = db[r] * isb[r];
    ur[r] = fr * fr;
    ub[r] = fb * fb;
    hsr[r] = 0.5 * sr;
    small = small && fmax(ur[r], ub[r]) < 1e-6;
    mid = mid && fmax(ur[r], ub[r]) < 1e-2;
  }
  double rl[R], ibl[R];
  if (SMALL || __all_sync(0xffffffffu, small)) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rl[r] = hsr[r] * polyG2(ur[r]);
      ibl[r] = isb[r] * polyF2x2(ub[r]);
    }
  } else if (__all_sync(0xffffffffu, mid)) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rl[r] = hsr[r] * polyG(ur[r]);
      ibl[r] = isb[r] * polyFx2(ub[r]);
    }
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rl[r] = (ur[r] < 1e-2) ? hsr[r] * polyG(ur[r]) : dr[r] * rcp(a[r].lrho - b.lrho);
      ibl[r] = (ub[r] < 1e-2) ? isb[r] * polyFx2(ub[r]) : (a[r].lbeta - b.lbeta) * rcp(db[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double pa = hsr[r] * isb[r];
    double ubar[DIM], un = 0.0, hv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      ubar[d] = a[r].vel[d] + b.vel[d];
      un = fma(ubar[d], n[r][d], un);
      hv = fma(a[r].vel[d], b.vel[d], hv);
    }
    const double f4 = fma(rl[r], fma(ibl[r], P.cbeta, 2.0 * hv), pa);
    const double F0 = rl[r] * un;
    F[r][0] = F0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[r][1 + d] = fma(F0, ubar[d], pa * n[r][d]);
    F[r][DIM + 1] = f4 * un;
  }
}

// ecflux_n_warp for states whose velocity is stored halved (vel = u/2), the
// pair kernel's layout: ubar = a.vel + b.vel, (ua.ub)/2 = 2 (a.vel . b.vel),
// and (rho_a + rho_b)/2 is formed once for rholog and pa.  Same value to
// rounding.  Must be called by all 32 lanes of the warp.
template <int DIM>
__device__ __forceinline__ void ecflux_n_warp_h(const NodeState<DIM> &a, const NodeState<DIM> &b,
                                                const double *n, const Phys &P, double *F) {
  const double sr = a.rho + b.rho, dr = a.rho - b.rho;
  const double sb = a.beta + b.beta, db = a.beta - b.beta;
  const double isr = rcp1(sr), isb = rcp(sb);
  const double fr = dr * isr, fb = db * isb;
  const double ur = fr * fr, ub = fb * fb;
  const double hsr = 0.5 * sr;
  double rl, ibl;
  if (__all_sync(0xffffffffu, fmax(ur, ub) < 1e-6)) {
    rl = hsr * polyG2(ur);
    ibl = 2.0 * isb * polyF2(ub);
  } else {
    rl = (ur < 1e-2) ? hsr * polyG(ur) : dr * rcp(a.lrho - b.lrho);
    ibl = (ub < 1e-2) ? 2.0 * isb * polyF(ub) : (a.lbeta - b.lbeta) * rcp(db);
  }
  const double pa = hsr * isb;
  double ubar[DIM], un = 0.0, hv = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    ubar[d] = a.vel[d] + b.vel[d];
    un = fma(ubar[d], n[d], un);
    hv = fma(a.vel[d], b.vel[d], hv);
  }
  const double f4 = fma(rl, fma(ibl, P.cbeta, 2.0 * hv), pa);
  const double F0 = rl * un;
  F[0] = F0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = fma(F0, ubar[d], pa * n[d]);
  F[DIM + 1] = f4 * un;
}

}  // namespace wadg

namespace wadg {

// Two-point flux for states without precomputed logarithms (surface traces):
// the log branch of the log-mean evaluates log(a/b) itself, as the reference
// does; the series branches are those of logmean / inv_logmean.
template <int DIM>
__device__ __forceinline__ void ecflux_n_nolog(const NodeState<DIM> &a, const NodeState<DIM> &b,
                                               const double *n, const Phys &P, double *F) {
  const double sr = a.rho + b.rho, dr = a.rho - b.rho;
  const double sb = a.beta + b.beta, db = a.beta - b.beta;
  const double isr = rcp(sr), isb = rcp(sb);
  const double fr = dr * isr, fb = db * isb;
  const double ur = fr * fr, ub = fb * fb;
  const double rl = (ur < 1e-2) ? 0.5 * sr * polyG(ur) : dr / log(a.rho / b.rho);
  const double ibl = (ub < 1e-2) ? 2.0 * isb * polyF(ub) : log(a.beta / b.beta) / db;
  const double pa = 0.5 * sr * isb;
  double ub2[DIM], un = 0.0, vv = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    ub2[d] = 0.5 * (a.vel[d] + b.vel[d]);
    un = fma(ub2[d], n[d], un);
    vv = fma(a.vel[d], b.vel[d], vv);
  }
  const double f4 = fma(rl, fma(ibl, P.cbeta, 0.5 * vv), pa);
  const double F0 = rl * un;
  F[0] = F0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = fma(F0, ub2[d], pa * n[d]);
  F[DIM + 1] = f4 * un;
}

// sqrt(x) for x >= 0 (0 for x <= 0): the reciprocal square root estimate
// rsqrt.approx.f64 refined by two Newton-Raphson steps on y^-2 = x, then one
// Newton step on s^2 = x for s = x y; a few ulp, for the surface kernels'
// wave speeds (which only enter the penalty's max)
__device__ __forceinline__ double fsqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = y * fma(-0.5 * x * y, y, 1.5);
  y = y * fma(-0.5 * x * y, y, 1.5);
  double s = x * y;
  s = fma(0.5 * y, fma(-s, s, x), s);
  return x > 0.0 ? s : 0.0;
}

// node state of a conservative trace without the logarithms (for
// ecflux_n_nolog), with |u|^2 and the squared sound speed gamma p / rho of the
// surface penalty; reciprocals (rcp) in place of divisions
template <int DIM>
__device__ __forceinline__ NodeState<DIM> node_state_surf(const double *q, int stride, const Phys &P,
                                                          double &kin, double &c2) {
  NodeState<DIM> s;
  s.rho = q[0];
  const double ir = rcp(s.rho);
  kin = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.vel[d] = q[(1 + d) * stride] * ir;
    kin = fma(s.vel[d], s.vel[d], kin);
  }
  const double p = P.gm1 * (q[(DIM + 1) * stride] - 0.5 * s.rho * kin);
  s.beta = 0.5 * s.rho * rcp(p);
  c2 = P.gamma * p * ir;
  s.lrho = 0.0;
  s.lbeta = 0.0;
  return s;
}

// node state without the logarithms (for ecflux_n_nolog)
template <int DIM>
__device__ __forceinline__ NodeState<DIM> node_state_nolog(const double *q, int stride, const Phys &P) {
  NodeState<DIM> s;
  s.rho = q[0];
  const double ir = 1.0 / s.rho;
  double kin = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.vel[d] = q[(1 + d) * stride] * ir;
    kin = fma(s.vel[d], s.vel[d], kin);
  }
  const double p = P.gm1 * (q[(DIM + 1) * stride] - 0.5 * s.rho * kin);
  s.beta = s.rho / (2.0 * p);
  s.lrho = 0.0;
  s.lbeta = 0.0;
  return s;
}

}  // namespace wadg
