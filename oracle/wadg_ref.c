/*
 * ORACLE — test infrastructure only (see wadg_ref.h).  Plain-C restatement of
 * the reference kernels, element by element, in the reference's own loop and
 * summation order.  OpenMP runs elements in parallel; nothing depends on the
 * thread count.
 *
 * Literal constants follow the OKL source: `.5f`, `2.f` etc. are exact; the
 * log-mean series thresholds are the float constants 1e-4f (3D) and 1e-3f (2D)
 * written `1.fe-4` / `1.fe-3` in the OKL.
 */
#include "wadg_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXQ 512 /* largest Nq / NfqNfaces handled (3D N=9 has 220 / 3*55) */

/* ---------------------------------------------------------------- log-mean */
/* Euler3Daffine.okl:43-71 (3D, threshold 1e-4f, series to u^3) and
 * Euler2D.okl:36-67 with TESTING off (2D, threshold 1e-3f, series to u^4). */
double wadg_ref_logmean(int dim, double aL, double aR)
{
  const double xi = aL / aR;
  const double f = (xi - 1.0) / (xi + 1.0);
  const double u = f * f;
  const double u2 = u * u;
  double F = log(xi) / 2.0 / f;
  if (dim == 3)
  {
    if (fabs(u) < (double)1e-4f)
      F = 1.0 + u / 3.0 + u2 / 5.0 + u2 * u / 7.0;
  }
  else
  {
    if (fabs(u) < (double)1e-3f)
      F = 1.0 + u / 3.0 + u2 / 5.0 + u2 * u / 7.0 + u2 * u2 / 9.0;
  }
  return (aL + aR) / (2.0 * F);
}

#define AVG(a, b) (.5 * ((a) + (b)))

/* -------------------------------------------------- 3D two-point EC flux */
/* euler3d_flux, Euler3Daffine.okl:107-148 (Chandrashekar) */
static void flux3(double g, double rho_i, double rho_j, double u_i, double u_j,
                  double v_i, double v_j, double w_i, double w_j,
                  double beta_i, double beta_j, double *FxS, double *FyS,
                  double *FzS)
{
  const double rholog = wadg_ref_logmean(3, rho_i, rho_j);
  const double rhoavg = AVG(rho_i, rho_j);
  const double uavg = AVG(u_i, u_j);
  const double vavg = AVG(v_i, v_j);
  const double wavg = AVG(w_i, w_j);
  const double vnavg = 2.0 * (uavg * uavg + vavg * vavg + wavg * wavg) -
                       (AVG(u_i * u_i, u_j * u_j) + AVG(v_i * v_i, v_j * v_j) +
                        AVG(w_i * w_i, w_j * w_j));
  const double beta_avg = AVG(beta_i, beta_j);
  const double pa = rhoavg / (2.0 * beta_avg);
  const double f4aux =
      rholog / (2.0 * (g - 1.0) * wadg_ref_logmean(3, beta_i, beta_j)) + pa +
      .5 * rholog * vnavg;

  FxS[0] = rholog * uavg;
  FyS[0] = rholog * vavg;
  FzS[0] = rholog * wavg;
  FxS[1] = FxS[0] * uavg + pa;
  FyS[1] = FyS[0] * uavg;
  FzS[1] = FzS[0] * uavg;
  FxS[2] = FxS[0] * vavg;
  FyS[2] = FyS[0] * vavg + pa;
  FzS[2] = FzS[0] * vavg;
  FxS[3] = FxS[0] * wavg;
  FyS[3] = FyS[0] * wavg;
  FzS[3] = FzS[0] * wavg + pa;
  FxS[4] = f4aux * uavg;
  FyS[4] = f4aux * vavg;
  FzS[4] = f4aux * wavg;
}

/* pfun / beta macros, Euler3Daffine.okl:22-26 */
static inline double pfun3(double g, double rho, double u, double v, double w,
                           double E)
{
  return (g - 1.0) * (E - .5 * rho * (u * u + v * v + w * w));
}
static inline double beta3(double g, double rho, double u, double v, double w,
                           double E)
{
  return rho / (2.0 * pfun3(g, rho, u, v, w, E));
}

typedef struct
{
  double rho, u, v, w, E, beta;
} prim3;

static inline prim3 prim3_of(double g, const double *q, int stride)
{
  prim3 p;
  p.rho = q[0];
  p.u = q[stride] / p.rho;
  p.v = q[2 * stride] / p.rho;
  p.w = q[3 * stride] / p.rho;
  p.E = q[4 * stride];
  p.beta = beta3(g, p.rho, p.u, p.v, p.w, p.E);
  return p;
}

/* ------------------------------------------------------------------ vol 3D */
void wadg_ref_vol_3d(const wadg_ref_dims *d, int curved, int K,
                     const double *vgeo, const double *vfgeo,
                     const double *nrJ, const double *nsJ, const double *ntJ,
                     const double *Drq, const double *Dsq, const double *Dtq,
                     const double *VqLq, const double *VfPq, const double *Qf,
                     double *rhsQ, double *rhsQf)
{
  const int Nq = d->Nq, Nfq = d->Nfq, NfqNf = d->Nfq * d->Nfaces;
  const double g = d->gamma;

#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k)
  {
    prim3 pv[MAXQ], pf[MAXQ];
    /* the volume states come in through rhsQ (= u(VqPq v)), the face states
     * through Qf (Euler3Daffine.okl:232-256) */
    for (int i = 0; i < Nq; ++i)
      pv[i] = prim3_of(g, rhsQ + i + k * Nq * 5, Nq);
    for (int i = 0; i < NfqNf; ++i)
      pf[i] = prim3_of(g, Qf + i + k * NfqNf * 5, NfqNf);

    double outv[5 * MAXQ], outf[5 * MAXQ];

    /* affine geofacs: first quadrature node of the element (:205) */
    const double *G0 = vgeo + k * Nq * 9;
#define GA(c) (G0[(c)*Nq])

    for (int i = 0; i < Nq; ++i)
    {
      double divF[5] = {0, 0, 0, 0, 0};
      const prim3 a = pv[i];
      double Gi[9];
      for (int c = 0; c < 9; ++c)
        Gi[c] = curved ? vgeo[i + c * Nq + k * Nq * 9] : GA(c);

      for (int j = 0; j < Nq; ++j)
      {
        const int jid = i + j * Nq;
        const prim3 b = pv[j];
        double FxS[5], FyS[5], FzS[5];
        flux3(g, a.rho, b.rho, a.u, b.u, a.v, b.v, a.w, b.w, a.beta, b.beta,
              FxS, FyS, FzS);
        double G[9];
        for (int c = 0; c < 9; ++c)
          G[c] = curved ? .5 * (Gi[c] + vgeo[j + c * Nq + k * Nq * 9]) : Gi[c];
        /* G order: rxJ ryJ rzJ sxJ syJ szJ txJ tyJ tzJ */
        const double Dx = Drq[jid] * G[0] + Dsq[jid] * G[3] + Dtq[jid] * G[6];
        const double Dy = Drq[jid] * G[1] + Dsq[jid] * G[4] + Dtq[jid] * G[7];
        const double Dz = Drq[jid] * G[2] + Dsq[jid] * G[5] + Dtq[jid] * G[8];
        for (int jj = 0; jj < 5; ++jj)
          divF[jj] += Dx * FxS[jj] + Dy * FyS[jj] + Dz * FzS[jj];
      }

      for (int j = 0; j < NfqNf; ++j)
      {
        const double VqLq_ij = .5 * VqLq[i + j * Nq];
        const prim3 b = pf[j];
        double FxS[5], FyS[5], FzS[5];
        flux3(g, a.rho, b.rho, a.u, b.u, a.v, b.v, a.w, b.w, a.beta, b.beta,
              FxS, FyS, FzS);
        const int f = j / Nfq;
        const double nr = nrJ[f * Nfq], ns = nsJ[f * Nfq], nt = ntJ[f * Nfq];
        double G[9];
        for (int c = 0; c < 9; ++c)
          G[c] = curved ? .5 * (Gi[c] + vfgeo[j + c * NfqNf + k * NfqNf * 9])
                        : Gi[c];
        const double nxJ = G[0] * nr + G[3] * ns + G[6] * nt;
        const double nyJ = G[1] * nr + G[4] * ns + G[7] * nt;
        const double nzJ = G[2] * nr + G[5] * ns + G[8] * nt;
        for (int jj = 0; jj < 5; ++jj)
        {
          const double Fjj = FxS[jj] * nxJ + FyS[jj] * nyJ + FzS[jj] * nzJ;
          divF[jj] += VqLq_ij * Fjj;
        }
      }
      for (int jj = 0; jj < 5; ++jj)
        outv[i + jj * Nq] = divF[jj];
    }

    for (int i = 0; i < NfqNf; ++i)
    {
      double divF[5] = {0, 0, 0, 0, 0};
      const prim3 a = pf[i];
      const int f = i / Nfq;
      const double nr = nrJ[f * Nfq], ns = nsJ[f * Nfq], nt = ntJ[f * Nfq];
      double Gi[9];
      for (int c = 0; c < 9; ++c)
        Gi[c] = curved ? vfgeo[i + c * NfqNf + k * NfqNf * 9] : GA(c);
      for (int j = 0; j < Nq; ++j)
      {
        const double VfPq_ij = -.5 * VfPq[i + j * NfqNf];
        const prim3 b = pv[j];
        double FxS[5], FyS[5], FzS[5];
        flux3(g, a.rho, b.rho, a.u, b.u, a.v, b.v, a.w, b.w, a.beta, b.beta,
              FxS, FyS, FzS);
        double G[9];
        for (int c = 0; c < 9; ++c)
          G[c] = curved ? .5 * (Gi[c] + vgeo[j + c * Nq + k * Nq * 9]) : Gi[c];
        const double nxJ = G[0] * nr + G[3] * ns + G[6] * nt;
        const double nyJ = G[1] * nr + G[4] * ns + G[7] * nt;
        const double nzJ = G[2] * nr + G[5] * ns + G[8] * nt;
        for (int jj = 0; jj < 5; ++jj)
        {
          const double Fjj = FxS[jj] * nxJ + FyS[jj] * nyJ + FzS[jj] * nzJ;
          divF[jj] += VfPq_ij * Fjj;
        }
      }
      for (int jj = 0; jj < 5; ++jj)
        outf[i + jj * NfqNf] = divF[jj];
    }
#undef GA
    memcpy(rhsQ + k * Nq * 5, outv, sizeof(double) * Nq * 5);
    memcpy(rhsQf + k * NfqNf * 5, outf, sizeof(double) * NfqNf * 5);
  }
}

/* ----------------------------------------------------------------- surf 3D */
/* Euler3D.okl:3242-3473 (the lift phase is identical in Euler3Daffine.okl:
 * 512-551; the affine file also overwrites rhsQf with rho+, a debug store
 * that the next volume kernel discards, :508) */
void wadg_ref_surf_3d(const wadg_ref_dims *d, int K, const double *fgeo,
                      const uint32_t *mapPq, const double *VqLq,
                      const double *Qf, const double *rhsQf, double *rhsQ)
{
  const int Nq = d->Nq, NfqNf = d->Nfq * d->Nfaces;
  const double g = d->gamma, tau = d->tau;

#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k)
  {
    double sfS[5][MAXQ];
    for (int i = 0; i < NfqNf; ++i)
    {
      const int idM = i + k * NfqNf * 5;
      const int idP = (int)mapPq[i + k * NfqNf];
      const int fid = i + 4 * NfqNf * k;
      const double nxJ = fgeo[fid + 0 * NfqNf];
      const double nyJ = fgeo[fid + 1 * NfqNf];
      const double nzJ = fgeo[fid + 2 * NfqNf];
      const double sJ = fgeo[fid + 3 * NfqNf];
      const double *qM = Qf + idM, *qP = Qf + idP;
      const double rhoM = qM[0], rhouM = qM[NfqNf], rhovM = qM[2 * NfqNf],
                   rhowM = qM[3 * NfqNf], EM = qM[4 * NfqNf];
      const double rhoP = qP[0], rhouP = qP[NfqNf], rhovP = qP[2 * NfqNf],
                   rhowP = qP[3 * NfqNf], EP = qP[4 * NfqNf];
      const double uM = rhouM / rhoM, vM = rhovM / rhoM, wM = rhowM / rhoM;
      const double uP = rhouP / rhoP, vP = rhovP / rhoP, wP = rhowP / rhoP;
      const double betaM = beta3(g, rhoM, uM, vM, wM, EM);
      const double betaP = beta3(g, rhoP, uP, vP, wP, EP);
      double FxS[5], FyS[5], FzS[5];
      flux3(g, rhoM, rhoP, uM, uP, vM, vP, wM, wP, betaM, betaP, FxS, FyS,
            FzS);
      const double lamM = sqrt(uM * uM + vM * vM + wM * wM) +
                          sqrt(g * pfun3(g, rhoM, uM, vM, wM, EM) / rhoM);
      const double lamP = sqrt(uP * uP + vP * vP + wP * wP) +
                          sqrt(g * pfun3(g, rhoP, uP, vP, wP, EP) / rhoP);
      const double Lfc_sJ = tau * .25 * (lamM > lamP ? lamM : lamP) * sJ;
      const double dU[5] = {rhoP - rhoM, rhouP - rhouM, rhovP - rhovM,
                            rhowP - rhowM, EP - EM};
      const int id = i + k * 5 * NfqNf;
      for (int jj = 0; jj < 5; ++jj)
      {
        const double fn = FxS[jj] * nxJ + FyS[jj] * nyJ + FzS[jj] * nzJ;
        sfS[jj][i] = .5 * fn + rhsQf[id + jj * NfqNf] - Lfc_sJ * dU[jj];
      }
    }
    for (int i = 0; i < Nq; ++i)
    {
      double val[5] = {0, 0, 0, 0, 0};
      for (int j = 0; j < NfqNf; ++j)
      {
        const double VqLq_ij = VqLq[i + j * Nq];
        for (int jj = 0; jj < 5; ++jj)
          val[jj] += VqLq_ij * sfS[jj][j];
      }
      const int id = i + k * 5 * Nq;
      for (int jj = 0; jj < 5; ++jj)
        rhsQ[id + jj * Nq] += val[jj];
    }
  }
}

/* ------------------------------------------------- entropy variables (VU/UV) */
/* Euler3Daffine.okl:28-40 (sU, sV, rhoeU, rhoeV), :73-105 (VU, UV);
 * Euler2D.okl:24-33, :69-98 */
void wadg_ref_VU(int dim, double g, const double *U, double *V)
{
  if (dim == 3)
  {
    const double rho = U[0], rhou = U[1], rhov = U[2], rhow = U[3], E = U[4];
    const double rhoe = E - .5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
    const double s = log((g - 1.0) * rhoe / pow(rho, g));
    const double invrhoe = 1 / rhoe;
    V[0] = (-E + rhoe * (g + 1.0 - s)) * invrhoe;
    V[1] = rhou * invrhoe;
    V[2] = rhov * invrhoe;
    V[3] = rhow * invrhoe;
    V[4] = (-rho) * invrhoe;
  }
  else
  {
    const double rho = U[0], rhou = U[1], rhov = U[2], E = U[3];
    const double rhoe = E - .5 * (rhou * rhou + rhov * rhov) / rho;
    const double s = log((g - 1.0) * rhoe / pow(rho, g));
    const double invrhoe = 1 / rhoe;
    V[0] = (-E + rhoe * (g + 1.0 - s)) * invrhoe;
    V[1] = rhou * invrhoe;
    V[2] = rhov * invrhoe;
    V[3] = (-rho) * invrhoe;
  }
}

void wadg_ref_UV(int dim, double g, const double *V, double *U)
{
  if (dim == 3)
  {
    const double V1 = V[0], V2 = V[1], V3 = V[2], V4 = V[3], V5 = V[4];
    const double sV = g - V1 + (V2 * V2 + V3 * V3 + V4 * V4) / (2.0 * V5);
    const double rhoe = pow((g - 1.0) / pow(-V5, g), 1.0 / (g - 1.0)) *
                        exp(-sV / (g - 1.0));
    U[0] = rhoe * (-V5);
    U[1] = rhoe * (V2);
    U[2] = rhoe * (V3);
    U[3] = rhoe * (V4);
    U[4] = rhoe * (1.0 - (V2 * V2 + V3 * V3 + V4 * V4) / (2.0 * V5));
  }
  else
  {
    const double V1 = V[0], V2 = V[1], V3 = V[2], V4 = V[3];
    const double sV = g - V1 + (V2 * V2 + V3 * V3) / (2.0 * V4);
    const double rhoe = pow((g - 1.0) / pow(-V4, g), 1.0 / (g - 1.0)) *
                        exp(-sV / (g - 1.0));
    U[0] = rhoe * (-V4);
    U[1] = rhoe * (V2);
    U[2] = rhoe * (V3);
    U[3] = rhoe * (1.0 - (V2 * V2 + V3 * V3) / (2.0 * V4));
  }
}

/* ------------------------------------------------------------ update (any D) */
/* Affine: Euler3Daffine.okl:555-773, Euler2D.okl:1498-1725.
 * WADG:   Euler3D.okl:2527-2884, Euler2D.okl:1729-2282. */
static void update_any(const wadg_ref_dims *d, int Nf, int curved, int K,
                       const double *Jq, const double *VqPq, const double *VfPq,
                       double fa, double fb, double fdt, double *rhsQ,
                       double *resQ, double *Q, double *Qf)
{
  const int Nq = d->Nq, NfqNf = d->Nfq * d->Nfaces;
  const int dim = d->dim;
  const double g = d->gamma;

#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k)
  {
    double s[5][MAXQ], sV[5][MAXQ];
    for (int i = 0; i < Nq; ++i)
      for (int f = 0; f < Nf; ++f)
        s[f][i] = rhsQ[i + f * Nq + k * Nq * Nf];

    if (curved)
    {
      /* r = (-2 VqPq rhs) / J, then re-projected (WADG M^-1) */
      for (int i = 0; i < Nq; ++i)
      {
        const double Jqi = Jq[i + k * Nq];
        double r[5] = {0, 0, 0, 0, 0};
        for (int j = 0; j < Nq; ++j)
        {
          const double VqPq_ij = -2.0 * VqPq[i + j * Nq];
          for (int f = 0; f < Nf; ++f)
            r[f] += VqPq_ij * s[f][j];
        }
        for (int f = 0; f < Nf; ++f)
          sV[f][i] = r[f] / Jqi;
      }
    }

    for (int i = 0; i < Nq; ++i)
    {
      const double Jqi = Jq[i + k * Nq];
      double r[5] = {0, 0, 0, 0, 0};
      if (curved)
      {
        for (int j = 0; j < Nq; ++j)
        {
          const double VqPq_ij = VqPq[i + j * Nq];
          for (int f = 0; f < Nf; ++f)
            r[f] += VqPq_ij * sV[f][j];
        }
      }
      else
      {
        for (int j = 0; j < Nq; ++j)
        {
          const double VqPq_ij = -2.0 * VqPq[i + j * Nq];
          for (int f = 0; f < Nf; ++f)
            r[f] += VqPq_ij * s[f][j];
        }
        for (int f = 0; f < Nf; ++f)
          r[f] /= Jqi;
      }
      const int id = i + k * Nq * Nf;
      double U[5], V[5];
      for (int f = 0; f < Nf; ++f)
      {
        double res = resQ[id + f * Nq];
        res = fa * res + fdt * r[f];
        resQ[id + f * Nq] = res;
        double q = Q[id + f * Nq];
        q += fb * res;
        Q[id + f * Nq] = q;
        U[f] = q;
      }
      wadg_ref_VU(dim, g, U, V);
      if (curved)
        for (int f = 0; f < Nf; ++f)
          s[f][i] = V[f] * Jqi; /* premultiplied by J for WADG */
      else
        for (int f = 0; f < Nf; ++f)
          sV[f][i] = V[f];
    }

    if (curved)
    {
      /* weight-adjusted projection VqPq((VqPq (v J)) / J) */
      for (int i = 0; i < Nq; ++i)
      {
        const double Jqi = Jq[i + k * Nq];
        double r[5] = {0, 0, 0, 0, 0};
        for (int j = 0; j < Nq; ++j)
        {
          const double VqPq_ij = VqPq[i + j * Nq];
          for (int f = 0; f < Nf; ++f)
            r[f] += VqPq_ij * s[f][j];
        }
        for (int f = 0; f < Nf; ++f)
          sV[f][i] = r[f] / Jqi;
      }
      for (int i = 0; i < Nq; ++i)
      {
        double r[5] = {0, 0, 0, 0, 0};
        for (int j = 0; j < Nq; ++j)
        {
          const double VqPq_ij = VqPq[i + j * Nq];
          for (int f = 0; f < Nf; ++f)
            r[f] += VqPq_ij * sV[f][j];
        }
        for (int f = 0; f < Nf; ++f)
          s[f][i] = r[f];
      }
      /* the final stage reads the projected values from s */
      for (int i = 0; i < Nq; ++i)
        for (int f = 0; f < Nf; ++f)
          sV[f][i] = s[f][i];
    }

    /* face values u(VfPq v) and volume values u(VqPq v) */
    for (int i = 0; i < NfqNf; ++i)
    {
      double V[5] = {0, 0, 0, 0, 0}, U[5];
      for (int j = 0; j < Nq; ++j)
      {
        const double VfPq_ij = VfPq[i + j * NfqNf];
        for (int f = 0; f < Nf; ++f)
          V[f] += VfPq_ij * sV[f][j];
      }
      wadg_ref_UV(dim, g, V, U);
      for (int f = 0; f < Nf; ++f)
        Qf[i + f * NfqNf + k * NfqNf * Nf] = U[f];
    }
    for (int i = 0; i < Nq; ++i)
    {
      double V[5] = {0, 0, 0, 0, 0}, U[5];
      for (int j = 0; j < Nq; ++j)
      {
        const double VqPq_ij = VqPq[i + j * Nq];
        for (int f = 0; f < Nf; ++f)
          V[f] += VqPq_ij * sV[f][j];
      }
      wadg_ref_UV(dim, g, V, U);
      for (int f = 0; f < Nf; ++f)
        rhsQ[i + f * Nq + k * Nq * Nf] = U[f];
    }
  }
}

void wadg_ref_update_3d(const wadg_ref_dims *d, int curved, int K,
                        const double *Jq, const double *VqPq,
                        const double *VfPq, double fa, double fb, double fdt,
                        double *rhsQ, double *resQ, double *Q, double *Qf)
{
  update_any(d, 5, curved, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf);
}

void wadg_ref_update_2d(const wadg_ref_dims *d, int curved, int K,
                        const double *Jq, const double *VqPq,
                        const double *VfPq, double fa, double fb, double fdt,
                        double *rhsQ, double *resQ, double *Q, double *Qf)
{
  update_any(d, 4, curved, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf);
}

/* -------------------------------------------------- 2D two-point EC flux */
/* euler2d_flux with TESTING off, Euler2D.okl:139-161 */
static void flux2(double g, double rho_i, double rho_j, double u_i, double u_j,
                  double v_i, double v_j, double beta_i, double beta_j,
                  double *Fx, double *Fy)
{
  const double rholog = wadg_ref_logmean(2, rho_i, rho_j);
  const double rhoavg = AVG(rho_i, rho_j);
  const double uavg = AVG(u_i, u_j);
  const double vavg = AVG(v_i, v_j);
  const double vnavg = 2.0 * (uavg * uavg + vavg * vavg) -
                       (AVG(u_i * u_i, u_j * u_j) + AVG(v_i * v_i, v_j * v_j));
  const double beta_avg = AVG(beta_i, beta_j);
  const double pa = rhoavg / (2.0 * beta_avg);
  const double f4aux =
      rholog / (2.0 * (g - 1.0) * wadg_ref_logmean(2, beta_i, beta_j)) + pa +
      .5 * rholog * vnavg;
  Fx[0] = rholog * uavg;
  Fy[0] = rholog * vavg;
  Fx[1] = Fx[0] * uavg + pa;
  Fy[1] = Fy[0] * uavg;
  Fx[2] = Fy[1];
  Fy[2] = Fy[0] * vavg + pa;
  Fx[3] = f4aux * uavg;
  Fy[3] = f4aux * vavg;
}

/* pfun / beta, Euler2D.okl:19-21 */
static inline double pfun2(double g, double rho, double u, double v, double E)
{
  return (g - 1.0) * (E - .5 * rho * (u * u + v * v));
}
static inline double beta2(double g, double rho, double u, double v, double E)
{
  return 0.5 * rho / pfun2(g, rho, u, v, E);
}

typedef struct
{
  double rho, u, v, E, beta;
} prim2;

static inline prim2 prim2_of(double g, const double *q, int stride)
{
  prim2 p;
  p.rho = q[0];
  p.u = q[stride] / p.rho;
  p.v = q[2 * stride] / p.rho;
  p.E = q[3 * stride];
  p.beta = beta2(g, p.rho, p.u, p.v, p.E);
  return p;
}

/* ------------------------------------------------------------------ vol 2D */
/* affine: euler_vol_2d, Euler2D.okl:235-769 (geofacs of the first quadrature
 * node); curved: euler_vol_2d_curved, :773-1353 (pairwise averaged) */
void wadg_ref_vol_2d(const wadg_ref_dims *d, int curved, int K,
                     const double *vgeo, const double *vfgeo,
                     const double *nrJ, const double *nsJ,
                     const double *Drq, const double *Dsq,
                     const double *VqLq, const double *VfPq, const double *Qf,
                     double *rhsQ, double *rhsQf)
{
  const int Nq = d->Nq, Nfq = d->Nfq, NfqNf = d->Nfq * d->Nfaces;
  const double g = d->gamma;

#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k)
  {
    prim2 pv[MAXQ], pf[MAXQ];
    for (int i = 0; i < Nq; ++i)
      pv[i] = prim2_of(g, rhsQ + i + k * Nq * 4, Nq);
    for (int i = 0; i < NfqNf; ++i)
      pf[i] = prim2_of(g, Qf + i + k * NfqNf * 4, NfqNf);
    double outv[4 * MAXQ], outf[4 * MAXQ];
    const double *G0 = vgeo + k * Nq * 4;

    for (int i = 0; i < Nq; ++i)
    {
      double divF[4] = {0, 0, 0, 0};
      const prim2 a = pv[i];
      double Gi[4];
      for (int c = 0; c < 4; ++c)
        Gi[c] = curved ? vgeo[i + c * Nq + k * Nq * 4] : G0[c * Nq];
      for (int j = 0; j < Nq; ++j)
      {
        const int jid = i + j * Nq;
        const double Drq_ij = Drq[jid], Dsq_ij = Dsq[jid];
        const prim2 b = pv[j];
        double G[4];
        for (int c = 0; c < 4; ++c)
          G[c] = curved ? .5 * (Gi[c] + vgeo[j + c * Nq + k * Nq * 4]) : Gi[c];
        /* G order: rxJ ryJ sxJ syJ (operators_c.cpp:143-146) */
        double Fx[4], Fy[4];
        flux2(g, a.rho, b.rho, a.u, b.u, a.v, b.v, a.beta, b.beta, Fx, Fy);
        for (int jj = 0; jj < 4; ++jj)
          divF[jj] += Drq_ij * (Fx[jj] * G[0] + Fy[jj] * G[1]) +
                      Dsq_ij * (Fx[jj] * G[2] + Fy[jj] * G[3]);
      }
      for (int j = 0; j < NfqNf; ++j)
      {
        const double VqLq_ij = .5 * VqLq[i + j * Nq];
        const prim2 b = pf[j];
        double Fx[4], Fy[4];
        flux2(g, a.rho, b.rho, a.u, b.u, a.v, b.v, a.beta, b.beta, Fx, Fy);
        const int f = j / Nfq;
        const double nr = nrJ[f * Nfq], ns = nsJ[f * Nfq];
        double G[4];
        for (int c = 0; c < 4; ++c)
          G[c] = curved ? .5 * (Gi[c] + vfgeo[j + c * NfqNf + k * NfqNf * 4])
                        : Gi[c];
        for (int jj = 0; jj < 4; ++jj)
        {
          const double F = (Fx[jj] * G[0] + Fy[jj] * G[1]) * nr +
                           (Fx[jj] * G[2] + Fy[jj] * G[3]) * ns;
          divF[jj] += VqLq_ij * F;
        }
      }
      for (int jj = 0; jj < 4; ++jj)
        outv[i + jj * Nq] = divF[jj];
    }

    for (int i = 0; i < NfqNf; ++i)
    {
      double divF[4] = {0, 0, 0, 0};
      const prim2 a = pf[i];
      const int f = i / Nfq;
      const double nr = nrJ[f * Nfq], ns = nsJ[f * Nfq];
      double Gi[4];
      for (int c = 0; c < 4; ++c)
        Gi[c] = curved ? vfgeo[i + c * NfqNf + k * NfqNf * 4] : G0[c * Nq];
      for (int j = 0; j < Nq; ++j)
      {
        const double VfPq_ij = -.5 * VfPq[i + j * NfqNf];
        const prim2 b = pv[j];
        double Fx[4], Fy[4];
        flux2(g, a.rho, b.rho, a.u, b.u, a.v, b.v, a.beta, b.beta, Fx, Fy);
        double G[4];
        for (int c = 0; c < 4; ++c)
          G[c] = curved ? .5 * (Gi[c] + vgeo[j + c * Nq + k * Nq * 4]) : Gi[c];
        for (int jj = 0; jj < 4; ++jj)
        {
          const double F = (Fx[jj] * G[0] + Fy[jj] * G[1]) * nr +
                           (Fx[jj] * G[2] + Fy[jj] * G[3]) * ns;
          divF[jj] += VfPq_ij * F;
        }
      }
      for (int jj = 0; jj < 4; ++jj)
        outf[i + jj * NfqNf] = divF[jj];
    }
    memcpy(rhsQ + k * Nq * 4, outv, sizeof(double) * Nq * 4);
    memcpy(rhsQf + k * NfqNf * 4, outf, sizeof(double) * NfqNf * 4);
  }
}

/* ----------------------------------------------------------------- surf 2D */
/* Euler2D.okl:1357-1495; the penalty assumes tau = 1 (:1423-1425) */
void wadg_ref_surf_2d(const wadg_ref_dims *d, int K, const double *fgeo,
                      const uint32_t *mapPq, const double *VqLq,
                      const double *Qf, const double *rhsQf, double *rhsQ)
{
  const int Nq = d->Nq, NfqNf = d->Nfq * d->Nfaces;
  const double g = d->gamma;

#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k)
  {
    double sfS[4][MAXQ];
    for (int i = 0; i < NfqNf; ++i)
    {
      const int idM = i + k * NfqNf * 4;
      const int idP = (int)mapPq[i + k * NfqNf];
      const int fid = i + 3 * NfqNf * k;
      const double nxJ = fgeo[fid + 0 * NfqNf];
      const double nyJ = fgeo[fid + 1 * NfqNf];
      const double sJ = fgeo[fid + 2 * NfqNf];
      const double *qM = Qf + idM, *qP = Qf + idP;
      const double rhoM = qM[0], rhouM = qM[NfqNf], rhovM = qM[2 * NfqNf],
                   EM = qM[3 * NfqNf];
      const double rhoP = qP[0], rhouP = qP[NfqNf], rhovP = qP[2 * NfqNf],
                   EP = qP[3 * NfqNf];
      const double uM = rhouM / rhoM, vM = rhovM / rhoM;
      const double uP = rhouP / rhoP, vP = rhovP / rhoP;
      const double betaM = beta2(g, rhoM, uM, vM, EM);
      const double betaP = beta2(g, rhoP, uP, vP, EP);
      double Fx[4], Fy[4];
      flux2(g, rhoM, rhoP, uM, uP, vM, vP, betaM, betaP, Fx, Fy);
      const double lamM =
          sqrt(uM * uM + vM * vM) + sqrt(g * pfun2(g, rhoM, uM, vM, EM) / rhoM);
      const double lamP =
          sqrt(uP * uP + vP * vP) + sqrt(g * pfun2(g, rhoP, uP, vP, EP) / rhoP);
      const double Lfc_sJ = .25 * (lamM > lamP ? lamM : lamP) * sJ;
      const double dU[4] = {rhoP - rhoM, rhouP - rhouM, rhovP - rhovM, EP - EM};
      const int id = i + k * 4 * NfqNf;
      for (int jj = 0; jj < 4; ++jj)
      {
        const double fn = .5 * (Fx[jj] * nxJ + Fy[jj] * nyJ);
        sfS[jj][i] = fn + rhsQf[id + jj * NfqNf] - Lfc_sJ * dU[jj];
      }
    }
    for (int i = 0; i < Nq; ++i)
    {
      double val[4] = {0, 0, 0, 0};
      for (int j = 0; j < NfqNf; ++j)
      {
        const double VqLq_ij = VqLq[i + j * Nq];
        for (int jj = 0; jj < 4; ++jj)
          val[jj] += VqLq_ij * sfS[jj][j];
      }
      for (int jj = 0; jj < 4; ++jj)
        rhsQ[i + jj * Nq + k * 4 * Nq] += val[jj];
    }
  }
}
