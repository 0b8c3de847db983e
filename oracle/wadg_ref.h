/*
 * ORACLE — test infrastructure only.  A plain-C restatement of the reference's
 * entropy-stable flux-differencing kernels (okl/Euler3Daffine.okl,
 * okl/Euler3D.okl, okl/Euler2D.okl), used by the tests, smoke() and the CPU
 * baseline of bench.py as the checker.  The product never links it.
 *
 * Parity is pinned: the tests compare these functions with the reference's
 * own OKL kernels compiled from their sources (oracle/_ref/, see build.py),
 * and with golden vectors generated from them (tests/golden/).
 *
 * Array layouts are the reference's (euler.c:2798-2877, operators_c.cpp):
 *   Q, rhsQ, resQ [K][Nfields][Nq]; Qf, rhsQf [K][Nfields][NfqNfaces]
 *   vgeo [K][Nvgeo][Nq]; vfgeo [K][Nvgeo][NfqNfaces]; fgeo [K][Nfgeo][NfqNfaces]
 *   Jq [K][Nq]; operators column-major; mapPq [K][NfqNfaces] field-strided.
 */
#ifndef WADG_REF_H
#define WADG_REF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
  int dim;     /* 2 or 3 */
  int Nq;      /* volume quadrature points */
  int Nfq;     /* quadrature points per face */
  int Nfaces;  /* 3 or 4 */
  double gamma;
  double tau;  /* LF penalty scale (3D only; the 2D kernel hard-codes 1) */
} wadg_ref_dims;

/* Euler3Daffine.okl:152 (curved=0) and Euler3D.okl:2123 (curved=1) */
void wadg_ref_vol_3d(const wadg_ref_dims *d, int curved, int K,
                     const double *vgeo, const double *vfgeo,
                     const double *nrJ, const double *nsJ, const double *ntJ,
                     const double *Drq, const double *Dsq, const double *Dtq,
                     const double *VqLq, const double *VfPq, const double *Qf,
                     double *rhsQ, double *rhsQf);

/* Euler3Daffine.okl:421 / Euler3D.okl:3242 */
void wadg_ref_surf_3d(const wadg_ref_dims *d, int K, const double *fgeo,
                      const uint32_t *mapPq, const double *VqLq,
                      const double *Qf, const double *rhsQf, double *rhsQ);

/* Euler3Daffine.okl:555 (curved=0) and Euler3D.okl:2527 (curved=1) */
void wadg_ref_update_3d(const wadg_ref_dims *d, int curved, int K,
                        const double *Jq, const double *VqPq,
                        const double *VfPq, double fa, double fb, double fdt,
                        double *rhsQ, double *resQ, double *Q, double *Qf);

/* Euler2D.okl:235 (curved=0) and :773 (curved=1) */
void wadg_ref_vol_2d(const wadg_ref_dims *d, int curved, int K,
                     const double *vgeo, const double *vfgeo,
                     const double *nrJ, const double *nsJ,
                     const double *Drq, const double *Dsq,
                     const double *VqLq, const double *VfPq, const double *Qf,
                     double *rhsQ, double *rhsQf);

/* Euler2D.okl:1357 */
void wadg_ref_surf_2d(const wadg_ref_dims *d, int K, const double *fgeo,
                      const uint32_t *mapPq, const double *VqLq,
                      const double *Qf, const double *rhsQf, double *rhsQ);

/* Euler2D.okl:1498 (curved=0) and :1729 (curved=1) */
void wadg_ref_update_2d(const wadg_ref_dims *d, int curved, int K,
                        const double *Jq, const double *VqPq,
                        const double *VfPq, double fa, double fb, double fdt,
                        double *rhsQ, double *resQ, double *Q, double *Qf);

/* conservative <-> entropy variables, per node (Euler3Daffine.okl:73-105,
 * Euler2D.okl:69-98). U and V hold dim+2 values. */
void wadg_ref_VU(int dim, double gamma, const double *U, double *V);
void wadg_ref_UV(int dim, double gamma, const double *V, double *U);

/* log-mean (Euler3Daffine.okl:43-71, Euler2D.okl:36-67) */
double wadg_ref_logmean(int dim, double aL, double aR);

#ifdef __cplusplus
}
#endif

#endif
