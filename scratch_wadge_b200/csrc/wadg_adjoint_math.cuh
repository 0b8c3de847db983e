// Derivatives for the discrete adjoint: vector-Jacobian products of the
// two-point entropy-conservative flux, of the primitive recovery, of the
// Lax-Friedrichs penalty and of the entropy-variable maps.  Host+device, so the
// same code is checked against finite differences on the CPU.
//
// Forward definitions (reference formulas, Euler3Daffine.okl:22-148,
// Euler2D.okl:19-161; conservative U = (rho, m, E)):
//   u = m/rho, p = (g-1)(E - |m|^2/(2 rho)), beta = rho/(2p)
//   L(a,b) = (a-b)/(log a - log b)          (log-mean, L(a,a) = a)
//   rl = L(rho_a, rho_b), ibl = 1/L(beta_a, beta_b)
//   pa = (rho_a+rho_b)/(2(beta_a+beta_b)), ub = (u_a+u_b)/2, un = ub.n
//   vv = u_a.u_b, f4 = rl (ibl/(2(g-1)) + vv/2) + pa
//   Fn = [rl un, rl un ub + pa n, f4 un]
//   lambda = |u| + sqrt(g p / rho)
//   V(U): rhoe = E - |m|^2/(2 rho), s = log((g-1) rhoe) - g log rho,
//         V = [(-E + rhoe (g+1-s))/rhoe, m/rhoe, -rho/rhoe]
//   U(V): sV = g - V1 + |Vm|^2/(2 Vl),
//         rhoe = exp((log(g-1) - g log(-Vl) - sV)/(g-1)),
//         U = [-rhoe Vl, rhoe Vm, rhoe (1 - |Vm|^2/(2 Vl))]
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define WADG_HD __host__ __device__ __forceinline__
#else
#define WADG_HD inline
#endif

namespace wadg {
namespace adj {

struct Gas {
  double gamma, gm1, cbeta, lgm1, igm1;  // g, g-1, 1/(2(g-1)), log(g-1), 1/(g-1)
};

// primitive state of a node (with logs for the log-mean)
template <int DIM> struct Prim {
  double rho, u[DIM], beta, lrho, lbeta;
};

// adjoint of a primitive state
template <int DIM> struct PrimBar {
  double rho, u[DIM], beta;
};

template <int DIM> WADG_HD void zero(PrimBar<DIM> &b) {
  b.rho = 0.0;
  for (int d = 0; d < DIM; ++d) b.u[d] = 0.0;
  b.beta = 0.0;
}

template <int DIM> WADG_HD Prim<DIM> prim(const double *U, const Gas &g) {
  Prim<DIM> s;
  s.rho = U[0];
  double kin = 0.0;
  for (int d = 0; d < DIM; ++d) {
    s.u[d] = U[1 + d] / s.rho;
    kin += s.u[d] * s.u[d];
  }
  const double p = g.gm1 * (U[DIM + 1] - 0.5 * s.rho * kin);
  s.beta = s.rho / (2.0 * p);
  s.lrho = log(s.rho);
  s.lbeta = log(s.beta);
  return s;
}

// series of F(u) = sum u^k/(2k+1) and of G = 1/F, with derivatives (degree 8)
WADG_HD void series_FG(double u, double &G, double &dG) {
  const double c[9] = {1.0, -1.0 / 3.0, -4.0 / 45.0, -44.0 / 945.0, -428.0 / 14175.0,
                       -10196.0 / 467775.0, -10719068.0 / 638512875.0,
                       -25865068.0 / 1915538625.0, -5472607916.0 / 488462349375.0};
  G = c[8];
  dG = 8.0 * c[8];
  for (int k = 7; k >= 1; --k) {
    G = G * u + c[k];
    dG = dG * u + k * c[k];
  }
  G = G * u + c[0];
}

// log-mean L(a, b) and its partials (La = dL/da, Lb = dL/db)
WADG_HD void logmean_d(double a, double b, double la, double lb, double &L, double &La,
                       double &Lb) {
  const double d = a - b, s = a + b;
  const double f = d / s, u = f * f;
  if (u < 1e-2) {
    // L = (s/2) G(u), u = (d/s)^2: du/da = 2f(1-f)/s, du/db = -2f(1+f)/s
    double G, dG;
    series_FG(u, G, dG);
    L = 0.5 * s * G;
    La = 0.5 * G + dG * f * (1.0 - f);
    Lb = 0.5 * G - dG * f * (1.0 + f);
  } else {
    const double ld = la - lb;
    L = d / ld;
    La = (1.0 - L / a) / ld;
    Lb = (L / b - 1.0) / ld;
  }
}

// VJP of Fn(a, b, n) (the flux contracted with the direction n): given the
// adjoint c of the Nf flux components, add the adjoints of a's and b's
// primitive states to ba, bb.
template <int DIM>
WADG_HD void flux_vjp(const Prim<DIM> &a, const Prim<DIM> &b, const double *n, const Gas &g,
                      const double *c, PrimBar<DIM> &ba, PrimBar<DIM> &bb) {
  double rl, rla, rlb, Lbt, Lba, Lbb;
  logmean_d(a.rho, b.rho, a.lrho, b.lrho, rl, rla, rlb);
  logmean_d(a.beta, b.beta, a.lbeta, b.lbeta, Lbt, Lba, Lbb);
  const double ibl = 1.0 / Lbt;
  const double sb = a.beta + b.beta, sr = a.rho + b.rho;
  const double pa = 0.5 * sr / sb;
  double ub[DIM], un = 0.0, vv = 0.0;
  for (int d = 0; d < DIM; ++d) {
    ub[d] = 0.5 * (a.u[d] + b.u[d]);
    un += ub[d] * n[d];
    vv += a.u[d] * b.u[d];
  }
  const double f4 = rl * (ibl * g.cbeta + 0.5 * vv) + pa;
  const double F0 = rl * un;
  // reverse sweep
  double F0b = c[0], pab = 0.0, ubb[DIM];
  for (int d = 0; d < DIM; ++d) {
    F0b += c[1 + d] * ub[d];
    ubb[d] = c[1 + d] * F0;
    pab += c[1 + d] * n[d];
  }
  const double f4b = c[DIM + 1] * un;
  const double unb = F0b * rl + c[DIM + 1] * f4;
  const double rlb_ = F0b * un + f4b * (ibl * g.cbeta + 0.5 * vv);
  const double iblb = f4b * rl * g.cbeta;
  const double vvb = f4b * rl * 0.5;
  pab += f4b;
  for (int d = 0; d < DIM; ++d) ubb[d] += unb * n[d];
  // to the node states
  const double dpa_drho = 0.5 / sb, dpa_dbeta = -pa / sb;
  ba.rho += rlb_ * rla + pab * dpa_drho;
  bb.rho += rlb_ * rlb + pab * dpa_drho;
  const double dibl = -ibl * ibl;
  ba.beta += iblb * dibl * Lba + pab * dpa_dbeta;
  bb.beta += iblb * dibl * Lbb + pab * dpa_dbeta;
  for (int d = 0; d < DIM; ++d) {
    ba.u[d] += 0.5 * ubb[d] + vvb * b.u[d];
    bb.u[d] += 0.5 * ubb[d] + vvb * a.u[d];
  }
}

// adjoint of the primitive recovery: primitive adjoint -> conservative adjoint
template <int DIM>
WADG_HD void prim_vjp(const double *U, const PrimBar<DIM> &pb, const Gas &g, double *Ub) {
  const double rho = U[0], E = U[DIM + 1];
  double u[DIM], kin = 0.0;
  for (int d = 0; d < DIM; ++d) {
    u[d] = U[1 + d] / rho;
    kin += u[d] * u[d];
  }
  const double p = g.gm1 * (E - 0.5 * rho * kin);
  // beta = rho/(2p): d/drho = 1/(2p) - rho/(2p^2) dp/drho, d/dm = -rho/(2p^2) dp/dm
  const double q = -rho / (2.0 * p * p);
  const double dp_drho = g.gm1 * 0.5 * kin;
  Ub[0] = pb.rho + pb.beta * (1.0 / (2.0 * p) + q * dp_drho);
  for (int d = 0; d < DIM; ++d) {
    Ub[0] -= pb.u[d] * u[d] / rho;
    Ub[1 + d] = pb.u[d] / rho + pb.beta * q * (-g.gm1 * u[d]);
  }
  Ub[DIM + 1] = pb.beta * q * g.gm1;
}

// wave speed lambda = |u| + sqrt(g p / rho) and its gradient w.r.t. U
template <int DIM>
WADG_HD double lambda_d(const double *U, const Gas &g, double *dl) {
  const double rho = U[0], E = U[DIM + 1];
  double u[DIM], kin = 0.0;
  for (int d = 0; d < DIM; ++d) {
    u[d] = U[1 + d] / rho;
    kin += u[d] * u[d];
  }
  const double p = g.gm1 * (E - 0.5 * rho * kin);
  const double un = sqrt(kin), c = sqrt(g.gamma * p / rho);
  // d|u|: d/drho = -|u|/rho, d/dm = u/(|u| rho) (0 at |u| = 0)
  // dc = g/(2c) (dp/rho - p/rho^2 drho)
  const double k = g.gamma / (2.0 * c);
  const double dp_drho = g.gm1 * 0.5 * kin;
  dl[0] = -un / rho + k * (dp_drho / rho - p / (rho * rho));
  for (int d = 0; d < DIM; ++d)
    dl[1 + d] = (un > 0.0 ? u[d] / (un * rho) : 0.0) + k * (-g.gm1 * u[d] / rho);
  dl[DIM + 1] = k * g.gm1 / rho;
  return un + c;
}

// adjoint of U(V): Ub -> Vb  (V at which U is evaluated)
template <int DIM>
WADG_HD void UV_vjp(const double *V, const double *Ub, const Gas &g, double *Vb) {
  const double Vl = V[DIM + 1];
  double vv = 0.0;
  for (int d = 0; d < DIM; ++d) vv += V[1 + d] * V[1 + d];
  const double sV = g.gamma - V[0] + vv / (2.0 * Vl);
  const double rhoe = exp((g.lgm1 - g.gamma * log(-Vl) - sV) * g.igm1);
  const double h = 1.0 - vv / (2.0 * Vl);
  double rb = -Ub[0] * Vl + Ub[DIM + 1] * h;
  for (int d = 0; d < DIM; ++d) rb += Ub[1 + d] * V[1 + d];
  const double t = rb * rhoe;  // adjoint of the exponent A
  Vb[0] = t * g.igm1;
  for (int d = 0; d < DIM; ++d)
    Vb[1 + d] = t * (-V[1 + d] / Vl) * g.igm1 + Ub[1 + d] * rhoe + Ub[DIM + 1] * rhoe * (-V[1 + d] / Vl);
  Vb[DIM + 1] = t * (-g.gamma / Vl + vv / (2.0 * Vl * Vl)) * g.igm1 - Ub[0] * rhoe +
                Ub[DIM + 1] * rhoe * vv / (2.0 * Vl * Vl);
}

// adjoint of U(V) at V = V(U), written in terms of U (no exp or log):
// with rhoe = E - |m|^2/(2 rho), u = m/rho, V_m = m/rhoe, V_l = -rho/rhoe,
// -V_m/V_l = u, 1/V_l = -rhoe/rho and |V_m|^2/(2 V_l^2) = |u|^2/2
template <int DIM>
WADG_HD void UV_vjp_U(const double *U, const double *Ub, const Gas &g, double *Vb) {
  const double rho = U[0], ir = 1.0 / rho;
  double u[DIM], u2 = 0.0;
  for (int d = 0; d < DIM; ++d) {
    u[d] = U[1 + d] * ir;
    u2 += u[d] * u[d];
  }
  const double rhoe = U[DIM + 1] - 0.5 * rho * u2;
  const double irhoe = 1.0 / rhoe;
  // rb = Ub . dU/d(rhoe) = Ub0 rho/rhoe + Ub_m m/rhoe + UbE (1 + rho |u|^2 / (2 rhoe))
  double rb = Ub[0] * rho * irhoe + Ub[DIM + 1] * (1.0 + 0.5 * rho * u2 * irhoe);
  for (int d = 0; d < DIM; ++d) rb += Ub[1 + d] * U[1 + d] * irhoe;
  const double t = rb * rhoe * g.igm1;  // adjoint of the exponent, over (gamma - 1)
  Vb[0] = t;
  for (int d = 0; d < DIM; ++d) Vb[1 + d] = t * u[d] + (Ub[1 + d] + Ub[DIM + 1] * u[d]) * rhoe;
  Vb[DIM + 1] = t * (g.gamma * rhoe * ir + 0.5 * u2) + (Ub[DIM + 1] * 0.5 * u2 - Ub[0]) * rhoe;
}

// adjoint of V(U): Vb -> Ub  (U at which V is evaluated)
template <int DIM>
WADG_HD void VU_vjp(const double *U, const double *Vb, const Gas &g, double *Ub) {
  const double rho = U[0], E = U[DIM + 1];
  double m2 = 0.0;
  for (int d = 0; d < DIM; ++d) m2 += U[1 + d] * U[1 + d];
  const double rhoe = E - 0.5 * m2 / rho;
  const double ir = 1.0 / rhoe, ir2 = ir * ir;
  // V1 = -E/rhoe + g + 1 - s, s = log((g-1) rhoe) - g log rho
  const double sb = -Vb[0];
  double rhoeb = Vb[0] * E * ir2 + sb * ir + Vb[DIM + 1] * rho * ir2;
  for (int d = 0; d < DIM; ++d) rhoeb -= Vb[1 + d] * U[1 + d] * ir2;
  Ub[0] = -Vb[DIM + 1] * ir + sb * (-g.gamma / rho) + rhoeb * 0.5 * m2 / (rho * rho);
  for (int d = 0; d < DIM; ++d) Ub[1 + d] = Vb[1 + d] * ir - rhoeb * U[1 + d] / rho;
  Ub[DIM + 1] = -Vb[0] * ir + rhoeb;
}

// forward helpers used by the checks
template <int DIM> WADG_HD void flux_fwd(const Prim<DIM> &a, const Prim<DIM> &b, const double *n,
                                         const Gas &g, double *F) {
  double rl, t1, t2, Lbt;
  logmean_d(a.rho, b.rho, a.lrho, b.lrho, rl, t1, t2);
  logmean_d(a.beta, b.beta, a.lbeta, b.lbeta, Lbt, t1, t2);
  const double ibl = 1.0 / Lbt;
  const double pa = 0.5 * (a.rho + b.rho) / (a.beta + b.beta);
  double ub[DIM], un = 0.0, vv = 0.0;
  for (int d = 0; d < DIM; ++d) {
    ub[d] = 0.5 * (a.u[d] + b.u[d]);
    un += ub[d] * n[d];
    vv += a.u[d] * b.u[d];
  }
  const double f4 = rl * (ibl * g.cbeta + 0.5 * vv) + pa;
  F[0] = rl * un;
  for (int d = 0; d < DIM; ++d) F[1 + d] = F[0] * ub[d] + pa * n[d];
  F[DIM + 1] = f4 * un;
}

template <int DIM> WADG_HD void V_of_U(const double *U, const Gas &g, double *V) {
  const double rho = U[0], E = U[DIM + 1];
  double m2 = 0.0;
  for (int d = 0; d < DIM; ++d) m2 += U[1 + d] * U[1 + d];
  const double rhoe = E - 0.5 * m2 / rho;
  const double s = log(g.gm1 * rhoe) - g.gamma * log(rho);
  V[0] = (-E + rhoe * (g.gamma + 1.0 - s)) / rhoe;
  for (int d = 0; d < DIM; ++d) V[1 + d] = U[1 + d] / rhoe;
  V[DIM + 1] = -rho / rhoe;
}

template <int DIM> WADG_HD void U_of_V(const double *V, const Gas &g, double *U) {
  const double Vl = V[DIM + 1];
  double vv = 0.0;
  for (int d = 0; d < DIM; ++d) vv += V[1 + d] * V[1 + d];
  const double sV = g.gamma - V[0] + vv / (2.0 * Vl);
  const double rhoe = exp((g.lgm1 - g.gamma * log(-Vl) - sV) * g.igm1);
  U[0] = -rhoe * Vl;
  for (int d = 0; d < DIM; ++d) U[1 + d] = rhoe * V[1 + d];
  U[DIM + 1] = rhoe * (1.0 - vv / (2.0 * Vl));
}

}  // namespace adj
}  // namespace wadg
