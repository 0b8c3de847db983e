// GPU builder of the geometric data the kernels read: the work the reference
// does on the host in build_geofacs_2D / _3D (operators.cpp:343-719) and in
// build_maps + its periodic fix-up (operators.cpp:765-1025,
// euler.c:3004-3175).
//
// wadg_geofacs: one CTA per element.  The element's nodal coordinates are
// staged in shared memory; every threads' loop below is over the rows of one
// small operator product.
//   2D (operators.cpp:385-440): rxJ = ys, ryJ = -xs, sxJ = -yr, syJ = xr at
//      volume and face points, J = xr ys - yr xs, nxJ = rxJ nrJ + sxJ nsJ,
//      nyJ = ryJ nrJ + syJ nsJ, sJ = |n| J;
//   3D (operators.cpp:542-719): J and sJ from the cross-product form, the
//      metric terms from Kopriva's conservative curl form evaluated at degree
//      N+1 and interpolated back to degree N (so curved meshes satisfy the
//      discrete GCL), then to volume and face points;
//   both: Jq = VqPq J, and the physical coordinates of the quadrature points.
//
// wadg_match_faces: the neighbour of every face quadrature point, periodic in
// every direction, by physical coincidence: each point's position in the
// periodic box is quantised to 2^-21 of the box per coordinate, the quantised
// positions go into an open-addressing hash table (bounded linear probing,
// atomicCAS on the key), and every key must hold two points of two different
// elements, or, where the caller allows boundaries, one point, which becomes
// its own neighbour (the reference's idM == idP boundary points).  Anything
// else is reported as an error, as the host builder does.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/wadg.h"

namespace wadg_internal {
void set_error(const std::string &msg);  // wadg_capi.cu
}

namespace {

int gfail(int code, const std::string &msg, cudaError_t e = cudaSuccess) {
  std::string m = msg;
  if (e != cudaSuccess) m += std::string(": ") + cudaGetErrorString(e);
  wadg_internal::set_error(m);
  return code;
}

// out[v][i] = sum_j A[i + j lda] in[v][j], for the CTA's threads
__device__ __forceinline__ double dotc(const double *__restrict__ A, int lda, int i,
                                       const double *in, int n) {
  double s = 0.0;
  for (int j = 0; j < n; ++j) s = fma(__ldg(A + i + (size_t)j * lda), in[j], s);
  return s;
}

// the operator set as kernel parameters (Drq.. here are Vq Dr.., not the
// hybridized derivative operators of the volume kernel)
struct GeoOps {
  int dim, N, Np, Nq, NF, Np2;
  const double *Vq, *Vfq, *Drq, *Dsq, *Dtq, *Drf, *Dsf, *Dtf, *VqPq, *nrJ, *nsJ, *ntJ, *V12, *Dr2,
      *Ds2, *Dt2, *V21;
};

GeoOps to_dev(const wadg_geo_ops *o) {
  return GeoOps{o->dim,  o->N,    o->Np,   o->Nq,   o->NfqNf, o->Np2,  o->Vq,   o->Vfq,
                o->VqDr, o->VqDs, o->VqDt, o->VfDr, o->VfDs,  o->VfDt, o->VqPq, o->nrJ,
                o->nsJ,  o->ntJ,  o->V12,  o->Dr2,  o->Ds2,   o->Dt2,  o->V21};
}

__global__ void geofacs2d_kernel(GeoOps o, const double *__restrict__ x, double *__restrict__ vgeo,
                                 double *__restrict__ vfgeo, double *__restrict__ fgeo,
                                 double *__restrict__ Jq, double *__restrict__ xyzq,
                                 double *__restrict__ xyzf) {
  extern __shared__ double sm[];
  const int k = blockIdx.x, Np = o.Np, Nq = o.Nq, NF = o.NF;
  double *X = sm, *Y = X + Np, *J = Y + Np;
  for (int t = threadIdx.x; t < 2 * Np; t += blockDim.x) X[t] = x[(size_t)k * 2 * Np + t];
  __syncthreads();
  for (int i = threadIdx.x; i < Nq; i += blockDim.x) {
    const double xr = dotc(o.Drq, Nq, i, X, Np), yr = dotc(o.Drq, Nq, i, Y, Np);
    const double xs = dotc(o.Dsq, Nq, i, X, Np), ys = dotc(o.Dsq, Nq, i, Y, Np);
    double *vg = vgeo + (size_t)k * 4 * Nq + i;
    vg[0 * Nq] = ys;   // rxJ
    vg[1 * Nq] = -xs;  // ryJ
    vg[2 * Nq] = -yr;  // sxJ
    vg[3 * Nq] = xr;   // syJ
    J[i] = xr * ys - yr * xs;
    double *xq = xyzq + (size_t)k * 3 * Nq + i;
    xq[0] = dotc(o.Vq, Nq, i, X, Np);
    xq[Nq] = dotc(o.Vq, Nq, i, Y, Np);
    xq[2 * Nq] = 0.0;
  }
  for (int i = threadIdx.x; i < NF; i += blockDim.x) {
    const double xr = dotc(o.Drf, NF, i, X, Np), yr = dotc(o.Drf, NF, i, Y, Np);
    const double xs = dotc(o.Dsf, NF, i, X, Np), ys = dotc(o.Dsf, NF, i, Y, Np);
    const double rxJ = ys, ryJ = -xs, sxJ = -yr, syJ = xr;
    double *vg = vfgeo + (size_t)k * 4 * NF + i;
    vg[0 * NF] = rxJ;
    vg[1 * NF] = ryJ;
    vg[2 * NF] = sxJ;
    vg[3 * NF] = syJ;
    const double Jf = xr * ys - yr * xs;
    const double nxJ = rxJ * o.nrJ[i] + sxJ * o.nsJ[i];
    const double nyJ = ryJ * o.nrJ[i] + syJ * o.nsJ[i];
    const double nx = nxJ / Jf, ny = nyJ / Jf;
    double *fg = fgeo + (size_t)k * 3 * NF + i;
    fg[0] = nxJ;
    fg[NF] = nyJ;
    fg[2 * NF] = sqrt(nx * nx + ny * ny) * Jf;
    double *xf = xyzf + (size_t)k * 3 * NF + i;
    xf[0] = dotc(o.Vfq, NF, i, X, Np);
    xf[NF] = dotc(o.Vfq, NF, i, Y, Np);
    xf[2 * NF] = 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Nq; i += blockDim.x) Jq[(size_t)k * Nq + i] = dotc(o.VqPq, Nq, i, J, Nq);
}

// 3D: shared memory X[3][Np] | J[Nq] | x2[3][Np2] | d2[9][Np2] | P[9][Np2] |
// T[9][Np2] | G[9][Np]
__global__ void geofacs3d_kernel(GeoOps o, const double *__restrict__ x, double *__restrict__ vgeo,
                                 double *__restrict__ vfgeo, double *__restrict__ fgeo,
                                 double *__restrict__ Jq, double *__restrict__ xyzq,
                                 double *__restrict__ xyzf) {
  extern __shared__ double sm[];
  const int k = blockIdx.x, Np = o.Np, Nq = o.Nq, NF = o.NF, N2 = o.Np2;
  double *X = sm, *J = X + 3 * Np, *x2 = J + Nq, *d2 = x2 + 3 * N2, *P = d2 + 9 * N2,
         *T = P + 9 * N2, *G = T + 9 * N2;
  for (int t = threadIdx.x; t < 3 * Np; t += blockDim.x) X[t] = x[(size_t)k * 3 * Np + t];
  __syncthreads();
  const double *Xc[3] = {X, X + Np, X + 2 * Np};

  // J at the volume points, sJ at the face points (cross-product form), the
  // physical coordinates, and the coordinates at the degree N+1 nodes
  for (int i = threadIdx.x; i < Nq; i += blockDim.x) {
    double d[3][3];  // d[c][a]: d(coordinate c)/d(r, s, t)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      d[c][0] = dotc(o.Drq, Nq, i, Xc[c], Np);
      d[c][1] = dotc(o.Dsq, Nq, i, Xc[c], Np);
      d[c][2] = dotc(o.Dtq, Nq, i, Xc[c], Np);
    }
    const double xr = d[0][0], xs = d[0][1], xt = d[0][2], yr = d[1][0], ys = d[1][1],
                 yt = d[1][2], zr = d[2][0], zs = d[2][1], zt = d[2][2];
    J[i] = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
    double *xq = xyzq + (size_t)k * 3 * Nq + i;
#pragma unroll
    for (int c = 0; c < 3; ++c) xq[c * Nq] = dotc(o.Vq, Nq, i, Xc[c], Np);
  }
  for (int i = threadIdx.x; i < NF; i += blockDim.x) {
    double d[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      d[c][0] = dotc(o.Drf, NF, i, Xc[c], Np);
      d[c][1] = dotc(o.Dsf, NF, i, Xc[c], Np);
      d[c][2] = dotc(o.Dtf, NF, i, Xc[c], Np);
    }
    const double xr = d[0][0], xs = d[0][1], xt = d[0][2], yr = d[1][0], ys = d[1][1],
                 yt = d[1][2], zr = d[2][0], zs = d[2][1], zt = d[2][2];
    const double rxJ = ys * zt - zs * yt, sxJ = yt * zr - zt * yr, txJ = yr * zs - zr * ys;
    const double ryJ = xt * zs - xs * zt, syJ = xr * zt - xt * zr, tyJ = xs * zr - zs * xr;
    const double rzJ = xs * yt - xt * ys, szJ = xt * yr - xr * yt, tzJ = xr * ys - xs * yr;
    const double Jf = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
    const double nr = o.nrJ[i], ns = o.nsJ[i], nt = o.ntJ[i];
    const double nx = (rxJ * nr + sxJ * ns + txJ * nt) / Jf;
    const double ny = (ryJ * nr + syJ * ns + tyJ * nt) / Jf;
    const double nz = (rzJ * nr + szJ * ns + tzJ * nt) / Jf;
    fgeo[(size_t)k * 4 * NF + 3 * NF + i] = sqrt(nx * nx + ny * ny + nz * nz) * Jf;
    double *xf = xyzf + (size_t)k * 3 * NF + i;
#pragma unroll
    for (int c = 0; c < 3; ++c) xf[c * NF] = dotc(o.Vfq, NF, i, Xc[c], Np);
  }
  for (int t = threadIdx.x; t < 3 * N2; t += blockDim.x) {
    const int c = t / N2, i = t - c * N2;
    x2[t] = dotc(o.V12, N2, i, Xc[c], Np);
  }
  __syncthreads();

  // d2[3a + c] = D_a x2_c (a = r, s, t; c = x, y, z) at degree N+1
  for (int t = threadIdx.x; t < 9 * N2; t += blockDim.x) {
    const int v = t / N2, i = t - v * N2, a = v / 3, c = v - 3 * a;
    const double *D = a == 0 ? o.Dr2 : (a == 1 ? o.Ds2 : o.Dt2);
    d2[t] = dotc(D, N2, i, x2 + c * N2, N2);
  }
  __syncthreads();
  // the products the curl form differentiates:
  // P = ys z, yt z, yr z, xs z, xt z, xr z, ys x, yt x, yr x
  {
    const double *xr = d2, *yr = d2 + N2, *xs = d2 + 3 * N2, *ys = d2 + 4 * N2,
                 *xt = d2 + 6 * N2, *yt = d2 + 7 * N2;
    const double *X2 = x2, *Z2 = x2 + 2 * N2;
    for (int i = threadIdx.x; i < N2; i += blockDim.x) {
      P[0 * N2 + i] = ys[i] * Z2[i];
      P[1 * N2 + i] = yt[i] * Z2[i];
      P[2 * N2 + i] = yr[i] * Z2[i];
      P[3 * N2 + i] = xs[i] * Z2[i];
      P[4 * N2 + i] = xt[i] * Z2[i];
      P[5 * N2 + i] = xr[i] * Z2[i];
      P[6 * N2 + i] = ys[i] * X2[i];
      P[7 * N2 + i] = yt[i] * X2[i];
      P[8 * N2 + i] = yr[i] * X2[i];
    }
  }
  __syncthreads();
  // metric terms in the vgeo order rxJ ryJ rzJ sxJ syJ szJ txJ tyJ tzJ:
  //   rxJ = Dt P0 - Ds P1      sxJ = Dr P1 - Dt P2      txJ = Ds P2 - Dr P0
  //   ryJ = -(Dt P3 - Ds P4)   syJ = -(Dr P4 - Dt P5)   tyJ = -(Ds P5 - Dr P3)
  //   rzJ = -(Dt P6 - Ds P7)   szJ = -(Dr P7 - Dt P8)   tzJ = -(Ds P8 - Dr P6)
  for (int t = threadIdx.x; t < 9 * N2; t += blockDim.x) {
    const int c = t / N2, i = t - c * N2;
    const int row = c / 3, col = c - 3 * row;  // row: r, s, t; col: x, y, z
    const int base = 3 * col;                  // x: P0..2, y: P3..5, z: P6..8
    const double *Da, *Db;
    int pa, pb;
    if (row == 0) {
      Da = o.Dt2; pa = base + 0; Db = o.Ds2; pb = base + 1;
    } else if (row == 1) {
      Da = o.Dr2; pa = base + 1; Db = o.Dt2; pb = base + 2;
    } else {
      Da = o.Ds2; pa = base + 2; Db = o.Dr2; pb = base + 0;
    }
    const double v = dotc(Da, N2, i, P + pa * N2, N2) - dotc(Db, N2, i, P + pb * N2, N2);
    T[(row * 3 + col) * N2 + i] = col == 0 ? v : -v;
  }
  __syncthreads();
  // back to degree N; the vgeo order is rxJ ryJ rzJ sxJ syJ szJ txJ tyJ tzJ,
  // i.e. (row, col) = (c / 3, c % 3) in T
  for (int t = threadIdx.x; t < 9 * Np; t += blockDim.x) {
    const int c = t / Np, i = t - c * Np;
    G[t] = dotc(o.V21, Np, i, T + c * N2, N2);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 9 * Nq; t += blockDim.x) {
    const int c = t / Nq, i = t - c * Nq;
    vgeo[(size_t)k * 9 * Nq + t] = dotc(o.Vq, Nq, i, G + c * Np, Np);
  }
  for (int i = threadIdx.x; i < NF; i += blockDim.x) {
    double g[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      g[c] = dotc(o.Vfq, NF, i, G + c * Np, Np);
      vfgeo[(size_t)k * 9 * NF + c * NF + i] = g[c];
    }
    const double nr = o.nrJ[i], ns = o.nsJ[i], nt = o.ntJ[i];
    double *fg = fgeo + (size_t)k * 4 * NF + i;
    fg[0] = g[0] * nr + g[3] * ns + g[6] * nt;  // nxJ = rxJ nrJ + sxJ nsJ + txJ ntJ
    fg[NF] = g[1] * nr + g[4] * ns + g[7] * nt;
    fg[2 * NF] = g[2] * nr + g[5] * ns + g[8] * nt;
  }
  for (int i = threadIdx.x; i < Nq; i += blockDim.x) Jq[(size_t)k * Nq + i] = dotc(o.VqPq, Nq, i, J, Nq);
}

// ---------------------------------------------------------------- maps
constexpr unsigned long long kEmpty = ~0ull;
constexpr int kQBits = 21;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

struct Box {
  double lo[3], L[3];
};

// key of every face point from its position in the periodic box
__global__ void face_keys_kernel(int dim, int Np, int NF, const double *__restrict__ Vfq,
                                 const double *__restrict__ xa, Box box,
                                 unsigned long long *__restrict__ keys) {
  extern __shared__ double sm[];
  const int k = blockIdx.x;
  for (int t = threadIdx.x; t < dim * Np; t += blockDim.x) sm[t] = xa[(size_t)k * dim * Np + t];
  __syncthreads();
  for (int i = threadIdx.x; i < NF; i += blockDim.x) {
    unsigned long long key = 0;
    for (int d = 0; d < dim; ++d) {
      const double c = dotc(Vfq, NF, i, sm + d * Np, Np);
      double t = (c - box.lo[d]) / box.L[d];
      t -= floor(t);
      long long q = llrint(t * (double)(1ll << kQBits));
      if (q >= (1ll << kQBits)) q -= (1ll << kQBits);
      if (q < 0) q = 0;
      key |= (unsigned long long)q << (kQBits * d);
    }
    keys[(size_t)k * NF + i] = key;
  }
}

__global__ void insert_kernel(int n, const unsigned long long *__restrict__ keys,
                              unsigned long long *tkey, unsigned *tcnt, unsigned *ta, unsigned *tb,
                              unsigned tmask, int *flag) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const unsigned long long key = keys[p];
  unsigned h = (unsigned)mix64(key) & tmask;
  for (unsigned probe = 0; probe <= tmask; ++probe) {
    const unsigned long long prev = atomicCAS(&tkey[h], kEmpty, key);
    if (prev == kEmpty || prev == key) {
      const unsigned c = atomicAdd(&tcnt[h], 1u);
      if (c == 0)
        ta[h] = (unsigned)p;
      else if (c == 1)
        tb[h] = (unsigned)p;
      return;
    }
    h = (h + 1) & tmask;
  }
  atomicOr(flag, 2);  // table full (cannot happen at load 1/2)
}

__global__ void pair_kernel(unsigned tsize, int unpaired_self, const unsigned *__restrict__ tcnt,
                            const unsigned *__restrict__ ta, const unsigned *__restrict__ tb,
                            unsigned *partner, int *flag) {
  const unsigned h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= tsize) return;
  const unsigned c = tcnt[h];
  if (c == 0) return;
  if (c == 1 && unpaired_self) {  // a boundary point: its own neighbour
    partner[ta[h]] = ta[h];
    return;
  }
  if (c != 2) {
    atomicOr(flag, 1);
    return;
  }
  partner[ta[h]] = tb[h];
  partner[tb[h]] = ta[h];
}

__global__ void mapPq_kernel(int n, int NF, int Nfields, const unsigned *__restrict__ partner,
                             uint32_t *__restrict__ mapPq, int *flag) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const unsigned q = partner[p];
  if (q == 0xffffffffu || ((int)(q / NF) == p / NF && (int)q != p)) {
    atomicOr(flag, 4);
    mapPq[p] = (uint32_t)p;
    return;
  }
  mapPq[p] = (q % NF) + (q / NF) * (unsigned)(NF * Nfields);
}

struct Work {
  unsigned long long *keys, *tkey;
  unsigned *tcnt, *ta, *tb, *partner;
  int *flag;
  unsigned tsize;
  size_t bytes;
};

Work carve(void *base, int K, int NF) {
  const size_t n = (size_t)K * NF;
  unsigned t = 1;
  while (t < 2 * n) t <<= 1;
  Work w{};
  w.tsize = t;
  char *p = (char *)base;
  size_t off = 0;
  auto take = [&](size_t b) {
    char *q = p ? p + off : nullptr;
    off += (b + 255) & ~size_t(255);
    return q;
  };
  w.keys = (unsigned long long *)take(8 * n);
  w.tkey = (unsigned long long *)take(8 * (size_t)t);
  w.tcnt = (unsigned *)take(4 * (size_t)t);
  w.ta = (unsigned *)take(4 * (size_t)t);
  w.tb = (unsigned *)take(4 * (size_t)t);
  w.partner = (unsigned *)take(4 * n);
  w.flag = (int *)take(4);
  w.bytes = off;
  return w;
}

bool ops_ok(const wadg_geo_ops *o) {
  if (!o || (o->dim != 2 && o->dim != 3) || o->Np <= 0 || o->Nq <= 0 || o->NfqNf <= 0) return false;
  if (!o->Vq || !o->Vfq || !o->VqDr || !o->VqDs || !o->VfDr || !o->VfDs || !o->VqPq || !o->nrJ ||
      !o->nsJ)
    return false;
  if (o->dim == 3 && (o->Np2 <= 0 || !o->VqDt || !o->VfDt || !o->ntJ || !o->V12 || !o->Dr2 ||
                      !o->Ds2 || !o->Dt2 || !o->V21))
    return false;
  return true;
}

}  // namespace

extern "C" {

int wadg_geofacs(const wadg_geo_ops *ops, int K, const double *x, double *vgeo, double *vfgeo,
                 double *fgeo, double *Jq, double *xyzq, double *xyzf, void *stream) {
  if (!ops_ok(ops)) return gfail(WADG_ERR_INVALID, "wadg_geofacs: incomplete operator set");
  if (K < 0) return gfail(WADG_ERR_INVALID, "wadg_geofacs: K < 0");
  if (K == 0) return WADG_OK;
  if (!x || !vgeo || !vfgeo || !fgeo || !Jq || !xyzq || !xyzf)
    return gfail(WADG_ERR_INVALID, "wadg_geofacs: null pointer argument");
  const GeoOps o = to_dev(ops);
  cudaStream_t s = (cudaStream_t)stream;
  const int threads = 128;
  if (o.dim == 2) {
    const size_t smem = sizeof(double) * (2 * o.Np + o.Nq);
    geofacs2d_kernel<<<K, threads, smem, s>>>(o, x, vgeo, vfgeo, fgeo, Jq, xyzq, xyzf);
  } else {
    const size_t smem = sizeof(double) * (3 * o.Np + o.Nq + 30 * o.Np2 + 9 * o.Np);
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(geofacs3d_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return gfail(WADG_ERR_CUDA, "wadg_geofacs: smem attribute", e);
    }
    geofacs3d_kernel<<<K, threads, smem, s>>>(o, x, vgeo, vfgeo, fgeo, Jq, xyzq, xyzf);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return gfail(WADG_ERR_CUDA, "wadg_geofacs: launch", e);
  return WADG_OK;
}

size_t wadg_match_faces_workspace(int K, int NfqNf) {
  if (K <= 0 || NfqNf <= 0) return 0;
  return carve(nullptr, K, NfqNf).bytes;
}

int wadg_match_faces(const wadg_geo_ops *ops, int K, const double *xa, const double *lo,
                     const double *hi, int unpaired_self, void *work, size_t work_bytes,
                     uint32_t *mapPq, void *stream) {
  if (!ops || (ops->dim != 2 && ops->dim != 3) || !ops->Vfq || ops->Np <= 0 || ops->NfqNf <= 0)
    return gfail(WADG_ERR_INVALID, "wadg_match_faces: incomplete operator set");
  if (K < 0) return gfail(WADG_ERR_INVALID, "wadg_match_faces: K < 0");
  if (K == 0) return WADG_OK;
  if (!xa || !lo || !hi || !work || !mapPq)
    return gfail(WADG_ERR_INVALID, "wadg_match_faces: null pointer argument");
  const int dim = ops->dim, NF = ops->NfqNf, Np = ops->Np;
  if ((size_t)K * NF >= 0x7fffffffull)
    return gfail(WADG_ERR_INVALID, "wadg_match_faces: too many face points");
  Work w = carve(work, K, NF);
  if (work_bytes < w.bytes) return gfail(WADG_ERR_INVALID, "wadg_match_faces: workspace too small");
  Box box{};
  for (int d = 0; d < dim; ++d) {
    box.lo[d] = lo[d];
    box.L[d] = hi[d] - lo[d];
    if (!(box.L[d] > 0)) return gfail(WADG_ERR_INVALID, "wadg_match_faces: empty periodic box");
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int n = K * NF;
  cudaError_t e;
  if ((e = cudaMemsetAsync(w.tkey, 0xff, 8 * (size_t)w.tsize, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(w.tcnt, 0, 4 * (size_t)w.tsize, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(w.partner, 0xff, 4 * (size_t)n, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(w.flag, 0, 4, s)) != cudaSuccess)
    return gfail(WADG_ERR_CUDA, "wadg_match_faces: memset", e);
  face_keys_kernel<<<K, 64, sizeof(double) * dim * Np, s>>>(dim, Np, NF, ops->Vfq, xa, box, w.keys);
  insert_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, w.keys, w.tkey, w.tcnt, w.ta, w.tb,
                                                 w.tsize - 1, w.flag);
  pair_kernel<<<(w.tsize + 255) / 256, 256, 0, s>>>(w.tsize, unpaired_self, w.tcnt, w.ta, w.tb,
                                                     w.partner, w.flag);
  mapPq_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, NF, dim + 2, w.partner, mapPq, w.flag);
  if ((e = cudaGetLastError()) != cudaSuccess) return gfail(WADG_ERR_CUDA, "wadg_match_faces: launch", e);
  int flag = 0;
  if ((e = cudaMemcpyAsync(&flag, w.flag, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return gfail(WADG_ERR_CUDA, "wadg_match_faces: flag read-back", e);
  if (flag)
    return gfail(WADG_ERR_INVALID,
                 "wadg_match_faces: face points do not pair up (not a closed periodic mesh)");
  return WADG_OK;
}

}  // extern "C"
