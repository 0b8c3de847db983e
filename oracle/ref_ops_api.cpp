/*
 * Test infrastructure only (oracle): a C-callable wrapper around the
 * reference's own operator builder, compiled together with the reference
 * sources operators.cpp and operators_c.cpp into oracle/_ref/.  Nothing in the
 * product links this file; tests and the fixture generator in tests/golden/
 * load it with ctypes.
 *
 *   wadgref_refelem_sizes / wadgref_refelem_fill
 *       reference-element data of build_ref_ops_2D / build_ref_ops_3D
 *       (operators.cpp:104-213, 214-341) plus the hybridized operators that
 *       host_operators_new_2D / _3D assemble (operators_c.cpp:46-69, 212-241).
 *   wadgref_ops_new / wadgref_ops_free
 *       host_operators_new_2D / _3D on a caller-supplied mesh
 *       (operators_c.cpp:39, 205): geometric factors, Jq, maps.
 *   wadgref_geofacs
 *       the geometric factors, Jq and physical node coordinates that
 *       host_operators_new_2D / _3D build for a mesh given by its element
 *       vertex coordinates (build_geofacs_2D / _3D, operators.cpp:343-719),
 *       copied out in the layouts the kernels read.
 */
#include "operators.h"
#include "operators_c.h"

#include <cstring>

namespace
{
ref_elem_data *build(int dim, int N, int M)
{
  return dim == 2 ? build_ref_ops_2D(N, M, M) : build_ref_ops_3D(N, M, M);
}

void put(double *dst, const MatrixXd &m)
{
  /* Eigen default storage is column-major, the layout the kernels use */
  std::memcpy(dst, m.data(), sizeof(double) * (size_t)m.size());
}
void put(double *dst, const VectorXd &v)
{
  std::memcpy(dst, v.data(), sizeof(double) * (size_t)v.size());
}
} // namespace

extern "C" {

void wadgref_ops_free(host_operators_t *ops);

/* sizes[0..4] = Np, Nq, Nfq (per face), Nfaces, Nfq*Nfaces */
int wadgref_refelem_sizes(int dim, int N, int M, int *sizes)
{
  ref_elem_data *rd = build(dim, N, M);
  sizes[0] = (int)rd->r.size();
  sizes[1] = (int)rd->rq.size();
  sizes[2] = (int)rd->ref_rfq.size();
  sizes[3] = rd->Nfaces;
  sizes[4] = (int)rd->rfq.size();
  delete rd;
  return 0;
}

/*
 * out[k] receives array k (column-major), in this order; 2D leaves the t/Dt
 * entries untouched:
 *  0 r[Np] 1 s[Np] 2 t[Np] 3 rq[Nq] 4 sq[Nq] 5 tq[Nq] 6 wq[Nq]
 *  7 rfq[NfqNf] 8 sfq[NfqNf] 9 tfq[NfqNf] 10 wfq[NfqNf]
 *  11 nrJ[NfqNf] 12 nsJ[NfqNf] 13 ntJ[NfqNf]
 *  14 V[Np,Np] 15 Dr[Np,Np] 16 Ds[Np,Np] 17 Dt[Np,Np]
 *  18 Vq[Nq,Np] 19 Pq[Np,Nq] 20 Vfq[NfqNf,Np]
 *  21 ref_rfq[Nfq] 22 ref_sfq[Nfq]
 *  23 VqLq[Nq,NfqNf] 24 VqPq[Nq,Nq] 25 VfPq[NfqNf,Nq]
 *  26 Drq[Nq,Nq] 27 Dsq[Nq,Nq] 28 Dtq[Nq,Nq]
 */
int wadgref_refelem_fill(int dim, int N, int M, double **out)
{
  ref_elem_data *rd = build(dim, N, M);
  put(out[0], rd->r);
  put(out[1], rd->s);
  if (dim == 3)
    put(out[2], rd->t);
  put(out[3], rd->rq);
  put(out[4], rd->sq);
  if (dim == 3)
    put(out[5], rd->tq);
  put(out[6], rd->wq);
  put(out[7], rd->rfq);
  put(out[8], rd->sfq);
  if (dim == 3)
    put(out[9], rd->tfq);
  put(out[10], rd->wfq);
  put(out[11], rd->nrJ);
  put(out[12], rd->nsJ);
  if (dim == 3)
    put(out[13], rd->ntJ);
  put(out[14], rd->V);
  put(out[15], rd->Dr);
  put(out[16], rd->Ds);
  if (dim == 3)
    put(out[17], rd->Dt);
  put(out[18], rd->Vq);
  put(out[19], rd->Pq);
  put(out[20], rd->Vfq);
  put(out[21], rd->ref_rfq);
  if (dim == 3)
    put(out[22], rd->ref_sfq);
  delete rd;

  /* the hybridized operators exactly as host_operators_new_* assembles them;
   * a one-element mesh is enough since they do not depend on geometry */
  uint32_t EToE[4] = {0, 0, 0, 0};
  uint8_t EToF[4] = {0, 1, 2, 3};
  uint8_t EToO[4] = {0, 0, 0, 0};
  double EToVX2[6] = {-1, -1, 1, -1, -1, 1};
  double EToVX3[12] = {-1, -1, -1, 1, -1, -1, -1, 1, -1, -1, -1, 1};
  host_operators_t *ops =
      dim == 2 ? host_operators_new_2D(N, M, 1, EToE, EToF, EToO, EToVX2)
               : host_operators_new_3D(N, M, 1, EToE, EToF, EToO, EToVX3);
  const int Nq = ops->Nq, NfqNf = ops->Nfq * ops->Nfaces;
  std::memcpy(out[23], ops->VqLq, sizeof(double) * Nq * NfqNf);
  std::memcpy(out[24], ops->VqPq, sizeof(double) * Nq * Nq);
  std::memcpy(out[25], ops->VfPq, sizeof(double) * NfqNf * Nq);
  std::memcpy(out[26], ops->Drq, sizeof(double) * Nq * Nq);
  std::memcpy(out[27], ops->Dsq, sizeof(double) * Nq * Nq);
  if (dim == 3)
    std::memcpy(out[28], ops->Dtq, sizeof(double) * Nq * Nq);
  wadgref_ops_free(ops);
  return 0;
}

/* host_operators_new_2D/_3D on a mesh given as EToE/EToF/EToO/EToVX
 * (euler.c:2758-2766). The caller frees with wadgref_ops_free. */
host_operators_t *wadgref_ops_new(int dim, int N, int M, uint32_t E,
                                  uint32_t *EToE, uint8_t *EToF, uint8_t *EToO,
                                  double *EToVX)
{
  return dim == 2 ? host_operators_new_2D(N, M, E, EToE, EToF, EToO, EToVX)
                  : host_operators_new_3D(N, M, E, EToE, EToF, EToO, EToVX);
}

void wadgref_ops_free(host_operators_t *ops)
{
  free(ops->xyzq);
  free(ops->xyzf);
  free(ops->vfgeo);
  free(ops->wq);
  if (ops->dim == 3)
    free(ops->Drstq);
  host_operators_free(ops);
  free(ops);
}

/* EToVX: E columns of the element's vertex coordinates, vertex-major
 * (x0 y0 [z0] x1 y1 [z1] ...), as euler.c passes them.  Connectivity is
 * set to "every face its own neighbour": the maps are not copied out.
 * Outputs: vgeo [E][Nvgeo][Nq], vfgeo [E][Nvgeo][NfqNf],
 * fgeo [E][Nfgeo][NfqNf], Jq [E][Nq], xyzq [E][3][Nq] and
 * xyzf [E][3][NfqNf] (2D: the third row is left as allocated). */
int wadgref_geofacs(int dim, int N, int M, uint32_t E, double *EToVX, double *vgeo,
                    double *vfgeo, double *fgeo, double *Jq, double *xyzq, double *xyzf)
{
  const int nf = dim + 1;
  uint32_t *EToE = new uint32_t[(size_t)nf * E];
  uint8_t *EToF = new uint8_t[(size_t)nf * E];
  uint8_t *EToO = new uint8_t[(size_t)nf * E];
  for (uint32_t e = 0; e < E; ++e)
    for (int f = 0; f < nf; ++f)
    {
      EToE[f + nf * e] = e;
      EToF[f + nf * e] = (uint8_t)f;
      EToO[f + nf * e] = 0;
    }
  host_operators_t *ops = wadgref_ops_new(dim, N, M, E, EToE, EToF, EToO, EToVX);
  delete[] EToE;
  delete[] EToF;
  delete[] EToO;
  if (!ops)
    return 1;
  const size_t Nq = ops->Nq, NF = (size_t)ops->Nfq * ops->Nfaces;
  std::memcpy(vgeo, ops->vgeo, sizeof(double) * Nq * ops->Nvgeo * E);
  std::memcpy(vfgeo, ops->vfgeo, sizeof(double) * NF * ops->Nvgeo * E);
  std::memcpy(fgeo, ops->fgeo, sizeof(double) * NF * ops->Nfgeo * E);
  std::memcpy(Jq, ops->Jq, sizeof(double) * Nq * E);
  for (uint32_t e = 0; e < E; ++e)
    for (int d = 0; d < dim; ++d)
    {
      std::memcpy(xyzq + (e * 3 + d) * Nq, ops->xyzq + (e * 3 + d) * Nq, sizeof(double) * Nq);
      std::memcpy(xyzf + (e * 3 + d) * NF, ops->xyzf + (e * 3 + d) * NF, sizeof(double) * NF);
    }
  wadgref_ops_free(ops);
  return 0;
}

} /* extern "C" */
