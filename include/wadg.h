/*
 * wadg.h — C ABI of the B200-native entropy-stable flux-differencing RHS.
 *
 * Drop-in for the OCCA kernel launches of the reference's host driver
 * (`occaKernelRun(app->vol|surf|update, ...)`, euler.c:3610-3666).  Each
 * kernel entry point keeps the argument list and meaning of the OKL kernel
 * it replaces, with a leading context that carries what the reference passed
 * as OCCA compile-time defines (euler.c:2879-2950: degree and sizes, gamma,
 * tau) and the CUDA stream (the reference's `cmdx` stream, euler.c:2708-2710).
 *
 * Conventions (all entry points):
 *   - pointers are DEVICE pointers owned by the caller; layouts are the
 *     reference's (Q, rhsQ, resQ [K][Nfields][Nq]; Qf, rhsQf
 *     [K][Nfields][Nfq*Nfaces]; vgeo [K][Nvgeo][Nq]; vfgeo
 *     [K][Nvgeo][Nfq*Nfaces]; fgeo [K][Nfgeo][Nfq*Nfaces]; Jq [K][Nq];
 *     operators column-major; mapPq [K][Nfq*Nfaces], field-strided);
 *   - calls are asynchronous and ordered on the context's stream; nothing is
 *     allocated per call;
 *   - the return value is WADG_OK or an error code; wadg_last_error() gives a
 *     message for the calling thread.  The reference aborts on errors
 *     (ASD_ABORT); this library never aborts.
 *   - FP64 throughout (the reference's dfloat=double build, types.h:33).
 */
#ifndef WADG_H
#define WADG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum
{
  WADG_OK = 0,
  WADG_ERR_INVALID = 1,     /* bad argument (null pointer, K < 0, ...) */
  WADG_ERR_UNSUPPORTED = 2, /* (dim, N) not compiled, or sizes disagree */
  WADG_ERR_CUDA = 3,        /* a CUDA call or kernel launch failed */
  WADG_ERR_STATE = 4        /* non-physical state detected (check calls) */
};

typedef struct wadg_ctx wadg_ctx;

typedef struct
{
  int dim;      /* 2 (triangles, 4 fields) or 3 (tetrahedra, 5 fields) */
  int N;        /* polynomial degree; cubature degree M = 2N (euler.c:340) */
  int Nq;       /* volume cubature points   (p_Nq)  */
  int Nfq;      /* cubature points per face (p_Nfq) */
  int Nfaces;   /* faces per element        (p_Nfaces) */
  double gamma; /* p_gamma */
  double tau;   /* p_TAU: Lax-Friedrichs penalty scale (3D; the 2D surface
                   kernel of the reference hard-codes 1, Euler2D.okl:1423) */
  void *stream; /* cudaStream_t the kernels run on; NULL = default stream */
} wadg_params;

/* Create / destroy a context.  Fails with WADG_ERR_UNSUPPORTED when (dim, N)
 * is not compiled in or Nq/Nfq/Nfaces disagree with the compiled sizes. */
int wadg_ctx_create(const wadg_params *p, wadg_ctx **out);
int wadg_ctx_destroy(wadg_ctx *ctx);
int wadg_ctx_set_stream(wadg_ctx *ctx, void *stream);
/* Tiling of the pair volume kernel: warps per CTA (elements per CTA follow
 * from it; results do not depend on it).  wadg_vol_warps_candidates writes
 * the compiled shapes for the context's degree (at most 3; the first is the
 * default) and returns their number; wadg_ctx_set_vol_warps selects one
 * (0 = the default).  No counterpart in the reference (OCCA's inner-loop
 * sizes are fixed defines); wadg_app_autotune picks one by timing. */
int wadg_vol_warps_candidates(const wadg_ctx *ctx, int curved, int *out);
int wadg_ctx_set_vol_warps(wadg_ctx *ctx, int curved, int warps);
int wadg_ctx_get_vol_warps(const wadg_ctx *ctx);
/* Its node-to-thread map is a second axis: L lanes per element with R rows
 * each (by default about three rows per lane).  wadg_vol_shapes writes every
 * compiled (warps, rows) pair -- first those of wadg_vol_warps_candidates with
 * rows 0 (the default map), then the maps with half or twice the lanes per
 * element where they pad no more node slots, hold at most 4 rows per lane
 * and fit 4 warps (2D N=4: 4 lanes x 4 rows; 3D N=1: 4 lanes x 1 row) -- and
 * returns their number (at most WADG_MAX_VOL_SHAPES);
 * wadg_ctx_set_vol_shape selects one (rows 0: as wadg_ctx_set_vol_warps).
 * Results agree bit for bit across warp counts under one map and to
 * rounding across maps. */
#define WADG_MAX_VOL_SHAPES 5
int wadg_vol_shapes(const wadg_ctx *ctx, int curved, int *warps, int *rows);
int wadg_ctx_set_vol_shape(wadg_ctx *ctx, int curved, int warps, int rows);
int wadg_ctx_get_vol_rows(const wadg_ctx *ctx);
/* Launch shape of one kernel for K elements, the numbers its entry point
 * uses: elements per batch (one CTA pass) and CTAs launched.  The volume,
 * update and fused stage kernels are persistent: CTA b takes batches b,
 * b + grid, b + 2 grid, ..., so K > elems * grid makes CTAs run several
 * batches, and K not a multiple of elems leaves a partial last batch.  The
 * volume kernel's shape follows the context's wadg_ctx_set_vol_warps.  For
 * tests and tuning; no counterpart in the reference (OCCA launches one
 * work-group per Kblk elements, euler.c:2879-2950). */
enum
{
  WADG_KERNEL_VOL = 0,
  WADG_KERNEL_SURF = 1,
  WADG_KERNEL_UPDATE = 2,
  WADG_KERNEL_STAGE = 3,
  WADG_KERNEL_ADJ_PAIRS = 4, /* the adjoint's pair VJP kernel (persistent) */
  WADG_KERNEL_VOLSURF = 5    /* the volume + surface kernel (persistent) */
};
int wadg_kernel_shape(const wadg_ctx *ctx, int kernel, int curved, int K, int *elems_per_batch,
                      int *grid);
const char *wadg_last_error(void);
/* degrees compiled for `dim`, as a bit mask (bit N set = degree N) */
int wadg_supported_degrees(int dim);

/* ---------------------------------------------------------------- 3D kernels
 * euler_vol_3d: Euler3Daffine.okl:152 (geometric factors constant per
 * element, read at the first quadrature node).  rhsQ holds u(VqPq v) on entry
 * and the volume flux-differencing term on exit; rhsQf receives the face-row
 * block.  Drstq and Q are accepted and unused, as in the reference. */
int wadg_euler_vol_3d(wadg_ctx *ctx, int K, const double *vgeo,
                      const double *vfgeo, const double *nrJ,
                      const double *nsJ, const double *ntJ, const double *Drq,
                      const double *Dsq, const double *Dtq,
                      const double *Drstq, const double *VqLq,
                      const double *VfPq, const double *Q, const double *Qf,
                      double *rhsQ, double *rhsQf);

/* euler_vol_3d_curved: Euler3D.okl:2123 (pairwise averaged geometric
 * factors from vgeo and vfgeo). Same arguments. */
int wadg_euler_vol_3d_curved(wadg_ctx *ctx, int K, const double *vgeo,
                             const double *vfgeo, const double *nrJ,
                             const double *nsJ, const double *ntJ,
                             const double *Drq, const double *Dsq,
                             const double *Dtq, const double *Drstq,
                             const double *VqLq, const double *VfPq,
                             const double *Q, const double *Qf, double *rhsQ,
                             double *rhsQf);

/* euler_surf_3d: Euler3D.okl:3242 / Euler3Daffine.okl:421.  rhsQ += VqLq *
 * (rhsQf + 1/2 F_S(u-,u+).nJ - tau/4 max(lambda-,lambda+) sJ (u+ - u-)).
 * mapPq is the reference's uintloc_t array (declared int* in the OKL).
 * rhsQf is read only (the affine OKL file also overwrites it with rho+ as a
 * debug store that the next volume kernel discards; that store is not
 * reproduced). */
int wadg_euler_surf_3d(wadg_ctx *ctx, int K, const double *fgeo,
                       const uint32_t *mapPq, const double *VqLq,
                       const double *Qf, double *rhsQf, double *rhsQ);

/* euler_update_3d: Euler3Daffine.okl:555 (affine M^-1 = -2 VqPq / J, LSRK
 * stage, entropy projection).  euler_update_3d_curved: Euler3D.okl:2527
 * (weight-adjusted M^-1 and weight-adjusted entropy projection). */
int wadg_euler_update_3d(wadg_ctx *ctx, int K, const double *Jq,
                         const double *VqPq, const double *VfPq, double fa,
                         double fb, double fdt, double *rhsQ, double *resQ,
                         double *Q, double *Qf);
int wadg_euler_update_3d_curved(wadg_ctx *ctx, int K, const double *Jq,
                                const double *VqPq, const double *VfPq,
                                double fa, double fb, double fdt, double *rhsQ,
                                double *resQ, double *Q, double *Qf);

/* ---------------------------------------------------------------- 2D kernels
 * euler_vol_2d: Euler2D.okl:235 (affine); euler_vol_2d_curved: :773. */
int wadg_euler_vol_2d(wadg_ctx *ctx, int K, const double *vgeo,
                      const double *vfgeo, const double *nrJ,
                      const double *nsJ, const double *Drq, const double *Dsq,
                      const double *VqLq, const double *VfPq, const double *Q,
                      const double *Qf, double *rhsQ, double *rhsQf);
int wadg_euler_vol_2d_curved(wadg_ctx *ctx, int K, const double *vgeo,
                             const double *vfgeo, const double *nrJ,
                             const double *nsJ, const double *Drq,
                             const double *Dsq, const double *VqLq,
                             const double *VfPq, const double *Q,
                             const double *Qf, double *rhsQ, double *rhsQf);
/* euler_surf_2d: Euler2D.okl:1357 */
int wadg_euler_surf_2d(wadg_ctx *ctx, int K, const double *fgeo,
                       const uint32_t *mapPq, const double *VqLq,
                       const double *Qf, const double *rhsQf, double *rhsQ);
/* euler_update_2d: Euler2D.okl:1498; euler_update_2d_curved: :1729 */
int wadg_euler_update_2d(wadg_ctx *ctx, int K, const double *Jq,
                         const double *VqPq, const double *VfPq, double fa,
                         double fb, double fdt, double *rhsQ, double *resQ,
                         double *Q, double *Qf);
int wadg_euler_update_2d_curved(wadg_ctx *ctx, int K, const double *Jq,
                                const double *VqPq, const double *VfPq,
                                double fa, double fb, double fdt, double *rhsQ,
                                double *resQ, double *Q, double *Qf);

/* ------------------------------------------------------------ geometry
 * GPU builder of the geometric data the kernels read -- the work the
 * reference does on the host in host_operators_new_2D / _3D
 * (operators_c.cpp:39, 205: build_geofacs_2D / _3D, operators.cpp:343-719)
 * and in its neighbour maps with the periodic fix-up (operators.cpp:765-1025,
 * euler.c:3004-3175).  Inputs are the per-element nodal coordinates (the
 * reference maps each element's vertices to its nodes, operators.cpp:365-367,
 * 488-493; a curved mesh displaces them) and reference-element operators.
 * Every pointer in wadg_geo_ops and every array argument is device memory;
 * operators are column-major; the struct itself is read on the host. */
typedef struct {
  int dim, N;
  int Np, Nq, NfqNf; /* nodes; volume and face quadrature points */
  int Np2;           /* 3D: nodes of the degree N+1 element (curl form) */
  const double *Vq;  /* Nq x Np */
  const double *Vfq; /* NfqNf x Np */
  const double *VqDr, *VqDs, *VqDt; /* Nq x Np: Vq Dr, Vq Ds, Vq Dt */
  const double *VfDr, *VfDs, *VfDt; /* NfqNf x Np: Vfq Dr, ... */
  const double *VqPq;               /* Nq x Nq */
  const double *nrJ, *nsJ, *ntJ;    /* NfqNf reference normals (scaled) */
  const double *V12;                /* Np2 x Np: degree N -> N+1 nodes (3D) */
  const double *Dr2, *Ds2, *Dt2;    /* Np2 x Np2 derivatives at degree N+1 */
  const double *V21;                /* Np x Np2: degree N+1 -> N nodes */
} wadg_geo_ops;

/* x: nodal coordinates [K][dim][Np].  Out: vgeo [K][Nvgeo][Nq],
 * vfgeo [K][Nvgeo][NfqNf], fgeo [K][Nfgeo][NfqNf], Jq [K][Nq] (= VqPq J),
 * xyzq [K][3][Nq], xyzf [K][3][NfqNf] (2D: third row 0).  2D: the
 * cross-product form (operators.cpp:385-440); 3D: J and sJ from the
 * cross-product form, the metric terms from Kopriva's curl form at degree
 * N+1 (operators.cpp:542-719), so curved meshes keep the discrete GCL.
 * stream: a cudaStream_t (NULL: the legacy default stream). */
int wadg_geofacs(const wadg_geo_ops *ops, int K, const double *x, double *vgeo,
                 double *vfgeo, double *fgeo, double *Jq, double *xyzq,
                 double *xyzf, void *stream);
/* mapPq [K][NfqNf] of a mesh periodic in every direction of the box
 * [lo, hi] (host arrays of dim doubles): the neighbour face point of every
 * face quadrature point by physical coincidence, field-strided
 * (j + e NfqNf Nfields, euler.c:3156-3174).  xa: the nodal coordinates
 * that define the topology (a curved mesh's undisplaced ones) [K][dim][Np];
 * only ops->dim, Np, NfqNf and Vfq are read.  unpaired_self != 0: a face
 * point with no partner is a boundary point and its own neighbour
 * (mapPq(j) = j, the reference's idM == idP); 0: an error.  work: device
 * scratch of wadg_match_faces_workspace(K, NfqNf) bytes.  Synchronises the
 * stream; WADG_ERR_INVALID when the face points do not pair up across
 * elements. */
size_t wadg_match_faces_workspace(int K, int NfqNf);
int wadg_match_faces(const wadg_geo_ops *ops, int K, const double *xa,
                     const double *lo, const double *hi, int unpaired_self,
                     void *work, size_t work_bytes, uint32_t *mapPq,
                     void *stream);

/* ------------------------------------------------------------ partitions
 * Element partitioning with a face-trace halo (the exchange the reference's
 * partitioned mesh was to do, euler.c:2468-2605, never written there).  A
 * part keeps its neighbours' traces as ghost pseudo-elements appended to its
 * Qf array, so the surface kernel reads them through mapPq unchanged.
 * wadg_halo_pack fills a send buffer of n slots (a multiple of NfqNf): slot
 * g takes the trace at field-strided index src[g] of Qf (nQf doubles), all
 * fields, at face point g % NfqNf of pseudo-element g / NfqNf; padding slots
 * (src = 0xffffffff) get zeros.  The buffer's blocks then go to the other
 * parts' ghost regions (an all-to-all), between stages. */
int wadg_halo_pack(wadg_ctx *ctx, int n, const uint32_t *src, const double *Qf,
                   size_t nQf, double *buf);

/* Failure detection.  Scans the conserved state Q [K][Nfields][Nq] for
 * non-physical nodes: a field that is NaN or infinite, rho <= 0, or a
 * pressure (gamma-1)(E - |m|^2/(2 rho)) <= 0.  `work` is a caller-owned device
 * buffer of 2 ints.  Synchronous (waits for the context's stream).  Returns
 * WADG_OK when every node is physical; otherwise WADG_ERR_STATE, with
 * *nbad = the number of bad nodes, *first = the smallest bad node index
 * k*Nq + i, and wadg_last_error() naming it (nbad and first may be NULL).
 * The reference has no such check: a bad state runs on into NaNs, and its
 * only failure path is an abort (ASD_ABORT, asd.h:77-79); this call returns a
 * status instead. */
int wadg_check_state(wadg_ctx *ctx, int K, const double *Q, int *work, int *nbad, int *first);

/* ------------------------------------------------------------ mesh I/O
 * The host driver's mesh files.  wadg_mesh_read_gmsh reads ASCII gmsh 2.x as
 * host_mesh_read_msh does (euler.c:556-833): the nodes; the elements of type
 * 2 (dim 2, triangles) or 4 (dim 3, tetrahedra), others and all tags
 * skipped; $Periodic skipped.  Negatively oriented elements get vertices 1
 * and 2 swapped (counted in `flipped`).  The periodic box lo/hi is the
 * bounding box of the elements' vertices, the box modify_mapP matches
 * periodic faces on (euler.c:3013-3050).  wadg_mesh_write_mfem writes
 * "MFEM mesh v1.0" as host_mesh_write_mfem does (euler.c:1771-1857):
 * per-element vertex copies EToVX [K][dim+1][dim] and the faces flagged in
 * bface [K][dim+1] (faces whose points are their own neighbours) as
 * boundary elements.  wadg_mesh_write_gmsh writes ASCII gmsh 2.2 (VX
 * [Nv][dim], EToV [K][dim+1] 0-based) for the reference to read.  All host
 * memory; no CUDA call. */
typedef struct wadg_mesh wadg_mesh;
int wadg_mesh_read_gmsh(const char *path, int dim, wadg_mesh **out);
int wadg_mesh_sizes(const wadg_mesh *m, int *dim, int64_t *Nv, int64_t *K,
                    int64_t *flipped);
int wadg_mesh_get(const wadg_mesh *m, double *VX, int64_t *EToV, double *lo,
                  double *hi);
void wadg_mesh_destroy(wadg_mesh *m);
int wadg_mesh_write_gmsh(const char *path, int dim, int64_t Nv,
                         const double *VX, int64_t K, const int64_t *EToV);
int wadg_mesh_write_mfem(const char *path, int dim, int64_t K,
                         const double *EToVX, const uint8_t *bface);

/* ------------------------------------------------------------ diagnostics
 * euler_3d_compute_aux: Euler3D.okl:3888 -- aux[k] = sum_i 1/2 |m|^2/rho J w,
 * the kinetic energy of element k (the reference sums aux on the host; its
 * rk_run has the call compiled out, euler.c:3701-3710).  Also accepts a 2D
 * context (two momentum components).  wq: the volume cubature weights [Nq].
 * wadg_element_entropy: S[k] = sum_i w J (-rho s), s = log((gamma-1) rhoe /
 * rho^gamma) -- the per-element terms of the entropy the reference's driver
 * sums on the host (euler.c:4135-4156, 4276-4315). */
int wadg_euler_3d_compute_aux(wadg_ctx *ctx, int K, const double *Jq,
                              const double *wq, const double *Q, double *aux);
int wadg_element_entropy(wadg_ctx *ctx, int K, const double *Jq,
                         const double *wq, const double *Q, double *S);
/* The entropy balance of the RHS, per element: out[k] = sum_i wq_i v~_i .
 * rhs_i, with rhs [K][Nf][Nq] the RHS after the volume and surface kernels
 * (before the inverse mass) and v~ the projected entropy variables of the
 * state Q the stage started from (affine: VqPq V(Q); curved:
 * VqPq((VqPq(V(Q) J))/J), J = Jq, which only curved reads).  Summed over a
 * periodic mesh: 0 to round-off without the surface penalty (tau = 0),
 * positive with it.  The device-side form of the entropy checks the
 * reference runs on the host (euler.c:4135-4156). */
int wadg_entropy_rhs(wadg_ctx *ctx, int K, int curved, const double *wq,
                     const double *Jq, const double *VqPq, const double *Q,
                     const double *rhs, double *out);

/* ------------------------------------------------------------ fused stage
 * One LSRK stage -- vol, surf and update of the kernels above -- in a single
 * launch (rk_step, euler.c:3610-3666, with rhsQf kept on chip and each group
 * of 8 elements updated as soon as its right-hand side is complete).  No
 * single-kernel counterpart in the reference.  The entropy-projected state
 * is read from (rhsQ_in, Qf_in); rhsQ_out receives the RHS and then the next
 * stage's state, Qf_out the next traces.  Qf_out must differ from Qf_in
 * (WADG_ERR_INVALID otherwise: a neighbour's trace of the current stage is
 * still being read while the next stage's is written); rhsQ_out may equal
 * rhsQ_in.  Q and resQ are updated in place.  curved = 0: Euler3Daffine /
 * euler_vol_2d algebra; 1: Euler3D curved / WADG. */
int wadg_euler_stage_3d(wadg_ctx *ctx, int K, int curved, const double *vgeo,
                        const double *vfgeo, const double *fgeo,
                        const uint32_t *mapPq, const double *nrJ,
                        const double *nsJ, const double *ntJ, const double *Drq,
                        const double *Dsq, const double *Dtq,
                        const double *VqLq, const double *VfPq,
                        const double *VqPq, const double *Jq, double fa,
                        double fb, double fdt, const double *rhsQ_in,
                        const double *Qf_in, double *Q, double *resQ,
                        double *rhsQ_out, double *Qf_out);
int wadg_euler_stage_2d(wadg_ctx *ctx, int K, int curved, const double *vgeo,
                        const double *vfgeo, const double *fgeo,
                        const uint32_t *mapPq, const double *nrJ,
                        const double *nsJ, const double *Drq, const double *Dsq,
                        const double *VqLq, const double *VfPq,
                        const double *VqPq, const double *Jq, double fa,
                        double fb, double fdt, const double *rhsQ_in,
                        const double *Qf_in, double *Q, double *resQ,
                        double *rhsQ_out, double *Qf_out);

/* ------------------------------------------------------------ volume + surface
 * The first two launches of rk_step (euler_vol_* then euler_surf_*,
 * euler.c:3615-3640) in one: rhsQ holds u~ on entry and, on exit, the whole
 * right-hand side the surface kernel leaves (volume rows plus the lift of the
 * surface flux, penalty and face rows); the face rows stay on chip, so no
 * rhsQf buffer.  Qf (the traces of every element, read for the neighbour
 * gathers) is only read.  Arguments are those of the two kernels; the update
 * kernel follows as before.  Sums run in another order than the two kernels',
 * so results agree with them to rounding.  No single-kernel counterpart in
 * the reference. */
int wadg_euler_volsurf_3d(wadg_ctx *ctx, int K, int curved, const double *vgeo,
                          const double *vfgeo, const double *fgeo,
                          const uint32_t *mapPq, const double *nrJ,
                          const double *nsJ, const double *ntJ,
                          const double *Drq, const double *Dsq,
                          const double *Dtq, const double *VqLq,
                          const double *VfPq, const double *Qf, double *rhsQ);
int wadg_euler_volsurf_2d(wadg_ctx *ctx, int K, int curved, const double *vgeo,
                          const double *vfgeo, const double *fgeo,
                          const uint32_t *mapPq, const double *nrJ,
                          const double *nsJ, const double *Drq,
                          const double *Dsq, const double *VqLq,
                          const double *VfPq, const double *Qf, double *rhsQ);

/* ------------------------------------------------------------ host driver
 * The reference's app_t / rk_step / rk_run (euler.c:2607-2796, 3610-3738)
 * over device buffers owned by the library.  Host arrays are copied once at
 * creation (device_malloc, euler.c:2798-2877). */
typedef struct wadg_app wadg_app;

typedef struct
{
  /* geometry, per element (host pointers, reference layouts) */
  const double *vgeo, *vfgeo, *fgeo, *Jq;
  const uint32_t *mapPq;
  /* reference-element operators (host pointers, column-major) */
  const double *nrJ, *nsJ, *ntJ; /* ntJ ignored in 2D */
  const double *Drq, *Dsq, *Dtq; /* Dtq ignored in 2D */
  const double *VqLq, *VqPq, *VfPq;
} wadg_host_data;

/* curved = 0: affine kernels (vol/update without _curved); 1: curved/WADG */
int wadg_app_create(const wadg_params *p, int K, int curved,
                    const wadg_host_data *h, wadg_app **out);
int wadg_app_destroy(wadg_app *app);
/* Copy the solver state host -> device (any pointer may be NULL to skip). */
int wadg_app_set_state(wadg_app *app, const double *Q, const double *rhsQ,
                       const double *Qf, const double *resQ);
/* Copy the solver state device -> host (any pointer may be NULL to skip);
 * synchronises the app stream. */
int wadg_app_get_state(wadg_app *app, double *Q, double *rhsQ, double *Qf,
                       double *resQ);
/* rk_step (euler.c:3610): vol, surf, update for one LSRK stage. */
int wadg_rk_step(wadg_app *app, double rka, double rkb, double dt);
/* rk_run (euler.c:3672): nsteps LSRK-45 time steps of size dt.  With
 * use_graph != 0 one time step (15 launches) is captured once as a CUDA graph
 * and replayed. Asynchronous. */
int wadg_rk_run(wadg_app *app, double dt, int nsteps, int use_graph);
/* Failure detection in the time loop: with nsteps > 0, wadg_rk_run checks
 * the state (wadg_check_state) every nsteps steps and after the last one,
 * and stops with WADG_ERR_STATE at the first check that finds a bad node
 * (the message names the step); each check synchronises the stream.  0 (the
 * default) never checks.  wadg_app_check_state checks the app's Q now. */
int wadg_app_set_check_every(wadg_app *app, int nsteps);
int wadg_app_check_state(wadg_app *app, int *nbad, int *first);
/* The whole user-level solve with HOST buffers: copy the stage-0 state in,
 * run nsteps, copy Q out (and the other state arrays if non-NULL).
 * Synchronous. */
int wadg_app_solve_host(wadg_app *app, const double *Q0, const double *rhsQ0,
                        const double *Qf0, const double *resQ0, double dt,
                        int nsteps, double *Q, double *rhsQ, double *Qf,
                        double *resQ);
/* The entropy projection of the app's Q into the traces the next stage
 * reads (rhsQ = U(VqPq v), Qf = U(VfPq v), v = V(Q)), and resQ = 0: the
 * stage-0 state the reference's driver builds on the host
 * (euler.c:3958-4133).  As there, curved meshes are projected with VqPq
 * alone too (the weight-adjusted projection is the curved update kernel's,
 * applied from the first stage's update on).  Asynchronous. */
int wadg_app_project(wadg_app *app);
/* The user-level solve from the conserved state alone: copy Q0 in, project
 * (wadg_app_project), run nsteps, copy Q out.  Synchronous. */
int wadg_app_solve_host_q(wadg_app *app, const double *Q0, double dt,
                          int nsteps, double *Q);
int wadg_app_sync(wadg_app *app);
/* The stage variant wadg_rk_step / wadg_rk_run launch:
 * WADG_STAGE_THREE (0, the default): the three reference kernels;
 * WADG_STAGE_FUSED (1): the fused stage kernel (one launch per stage,
 * ping-pong state buffers); WADG_STAGE_VOLSURF (2): the volume + surface
 * kernel, then the update kernel.  Results agree to rounding. */
enum
{
  WADG_STAGE_THREE = 0,
  WADG_STAGE_FUSED = 1,
  WADG_STAGE_VOLSURF = 2
};
int wadg_app_set_fused(wadg_app *app, int variant);
/* device pointers of the state arrays (for zero-copy use and testing) */
int wadg_app_state_ptrs(wadg_app *app, double **Q, double **rhsQ, double **Qf,
                        double **resQ, double **rhsQf);
/* Time `nsteps` time steps on the app stream with CUDA events (after the
 * caller's warm-up); ms receives the elapsed device time. */
int wadg_app_time_run(wadg_app *app, double dt, int nsteps, int use_graph,
                      float *ms);
/* Time each of the three kernels over `nstages` stages with CUDA events
 * around every launch; ms[0..2] = total vol, surf, update time. */
int wadg_app_time_kernels(wadg_app *app, double dt, int nstages, float *ms);
/* Time `nstages` fused stage launches (CUDA events around the sequence);
 * ms receives the total. */
int wadg_app_time_stage(wadg_app *app, double dt, int nstages, float *ms);
/* Time `nstages` stages of the volume + surface variant with CUDA events
 * around every launch; ms[0..1] = total volume + surface, update time. */
int wadg_app_time_volsurf(wadg_app *app, double dt, int nstages, float *ms);

/* Autotuner: times `nstages` LSRK stages (CUDA events) with each compiled
 * CTA shape of the volume kernel -- or, in the volume + surface stage
 * variant, of the volume + surface kernel, which has the same shapes -- on
 * the app's own mesh and state, over every shape of wadg_vol_shapes (CTA
 * size and node-to-thread map), keeps the fastest (its warps written to
 * *warps, its rows to be read with wadg_ctx_get_vol_rows; times, if not NULL,
 * an array of WADG_MAX_VOL_SHAPES, receives that kernel's ms per launch for
 * each shape in the order of wadg_vol_shapes) and leaves it selected for the
 * app's kernels.  Advances the app's state: call it before set_state. */
int wadg_app_autotune(wadg_app *app, double dt, int nstages, int *warps,
                      float *times);

/* the app's CUDA stream (a cudaStream_t) */
void *wadg_app_stream(wadg_app *app);
/* the app's kernel context (for wadg_ctx_* settings such as the volume
 * kernel's CTA shape) */
wadg_ctx *wadg_app_ctx(wadg_app *app);
/* fused-stage ping-pong: which state buffer is current (0 or 1).  The state
 * accessors read the current buffer; set only to undo a capture. */
int wadg_app_set_parity(wadg_app *app, int parity);
int wadg_app_get_fused(wadg_app *app);

/* ------------------------------------------------------------ ensemble
 * Batched ensemble of independent solves, each instance with its own time
 * step.  A bin is one wadg_app holding the concatenation of instances of one
 * degree (neighbour maps offset per instance); instance i of a bin covers
 * elements [offsets[i], offsets[i+1]) and makes nsteps[i] LSRK-45 steps of
 * size dt[i] (per instance, e.g. the reference's dt = CFL hmin / C_N,
 * euler.c:4180-4193, rounded to reach the final time).  Every bin runs the volume + surface
 * kernel and the update kernel over work lists of the element batches that
 * hold a running instance (an instance done is frozen: its step becomes 0 and
 * the batches it alone occupied leave the lists); one CUDA graph per time step
 * covers all bins, each on its app's stream, concurrently.  The apps must not
 * use the fused stage variant.  The reference runs one instance per process;
 * no counterpart.
 *
 * wadg_ensemble_run advances up to nsteps time steps (fewer once every
 * instance is done); wadg_ensemble_steps reports the steps done and the
 * longest instance's count; wadg_ensemble_restart sets the step count and
 * the lists back to the start (the caller restores the apps' states). */
typedef struct wadg_ensemble wadg_ensemble;
typedef struct
{
  wadg_app *app;
  int ninst;
  const int *offsets;  /* ninst + 1 element offsets, from 0 to the app's K */
  const double *dt;    /* ninst steps, > 0 */
  const int *nsteps;   /* ninst step counts, >= 0 */
} wadg_ensemble_bin;
int wadg_ensemble_create(int nbins, const wadg_ensemble_bin *bins, wadg_ensemble **out);
int wadg_ensemble_destroy(wadg_ensemble *ens);
int wadg_ensemble_run(wadg_ensemble *ens, int nsteps);
int wadg_ensemble_restart(wadg_ensemble *ens);
int wadg_ensemble_steps(const wadg_ensemble *ens, int *done, int *max_steps);
int wadg_ensemble_sync(wadg_ensemble *ens);
int wadg_ensemble_time_run(wadg_ensemble *ens, int nsteps, float *ms);

/* ------------------------------------------------------------ no allocation
 * One LSRK stage -- vol, surf and update, exactly what wadg_rk_step does --
 * for callers that may not allocate device memory: a host program that owns
 * all GPU memory through its own pool and passes the library only its own
 * buffers (the way the reference's driver allocates everything up front with
 * device_malloc), or a time loop that must not call cudaMalloc/cudaFree,
 * which synchronise the device and can fail in the middle of a run.  No
 * counterpart in the reference.
 *
 * Arguments as for the three kernels; the face-row buffer they pass between
 * them (rhsQf) lives in a fixed device array of the library instead:
 * WADG_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB), resident on every GPU that
 * loads the library until the process exits.  Limit: K * Nfq*Nfaces *
 * Nfields must not exceed it (3D N=3: K <= 8738); larger K is rejected with
 * WADG_ERR_INVALID.  Each call outside a stream capture looks up the
 * array's device address on the current device (so a context made again
 * after cudaDeviceReset is followed); a call during a capture reuses the
 * address the last call on that device found, so make the first call on a
 * device before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race, so serialise them. */
#define WADG_NOALLOC_SCRATCH_DOUBLES (2 * 1024 * 1024)
int wadg_rk_stage_noalloc(wadg_ctx *ctx, int K, int curved, const double *vgeo,
                          const double *vfgeo, const double *fgeo,
                          const uint32_t *mapPq, const double *nrJ,
                          const double *nsJ, const double *ntJ,
                          const double *Drq, const double *Dsq,
                          const double *Dtq, const double *VqLq,
                          const double *VqPq, const double *VfPq,
                          const double *Jq, double fa, double fb, double fdt,
                          double *rhsQ, double *resQ, double *Q, double *Qf);

/* ------------------------------------------------------------ discrete adjoint
 * Vector-Jacobian products of the RHS and of the whole LSRK-45 run
 * (rk_run, euler.c:3672-3738) for an app, by hand-written adjoint kernels:
 * the log-mean flux derivative, the entropy-variable Jacobians, the
 * Lax-Friedrichs penalty with its wave-speed max differentiated along the
 * branch the forward evaluation took (the reference's `lamM > lamP ? lamM :
 * lamP`), the inverse mass and the entropy projection.  The reference has no
 * adjoint; no counterpart.
 *
 * All state arrays are DEVICE pointers in the [K][Nfields][Nq] layout of Q.
 * Calls are asynchronous on the app's stream.  The adjoint object borrows
 * the app (its operators, geometry and state buffers): destroy it before the
 * app, and do not step the app while a forward/reverse pair is in use.
 * Requires a conforming face pairing (mapPq(mapPq(j)) = j), checked at
 * creation. */
typedef struct wadg_adjoint wadg_adjoint;
/* Tape for `nsteps` time steps with a checkpoint every `every` steps:
 * device memory (nsteps/every + 1) Q-sized checkpoints plus two tapes of
 * 5*every stages of (Q, u~, uf~) (one when there is a single segment), and
 * a second CUDA stream on which the stage adjoints run beside the segment
 * recompute. */
int wadg_adjoint_create(wadg_app *app, int nsteps, int every,
                        wadg_adjoint **out);
int wadg_adjoint_destroy(wadg_adjoint *adj);
/* Forward run of nsteps steps of size dt from Q0 (copied into the app; the
 * projected traces are recomputed from it), storing the checkpoints, and the
 * stages of the last segment on its tape as they are computed (so that the
 * reverse sweep need not recompute that segment).  The app holds the final
 * state Q(T) afterwards; QT (may be NULL) receives a copy of it. */
int wadg_adjoint_forward(wadg_adjoint *adj, const double *Q0, double dt,
                         double *QT);
/* Reverse sweep: given QbarT = dJ/dQ(T), writes Qbar0 = dJ/dQ0 for the run
 * of the last wadg_adjoint_forward.  Recomputes each segment from its
 * checkpoint, except the last one while the forward run's tape of it is
 * intact (always for the first sweep after a forward run; for later sweeps
 * with at most two segments); leaves the app at Q(T). */
int wadg_adjoint_reverse(wadg_adjoint *adj, const double *QbarT,
                         double *Qbar0);
/* R(Q) = Minv rhs(u~(Q), uf~(Q)), the time derivative one stage applies
 * (the update kernel's r with the projected traces of Q). */
int wadg_adjoint_rhs(wadg_adjoint *adj, const double *Q, double *R);
/* Qbar = (dR/dQ)^T w at Q. */
int wadg_adjoint_rhs_vjp(wadg_adjoint *adj, const double *Q, const double *w,
                         double *Qbar);

/* ------------------------------------------------------------ measurement
 * FP64 FMA throughput of the current GPU (the denominator of the volume
 * kernel's FP64 roofline): a saturating FMA kernel timed with CUDA events on
 * `stream`; tflops = 2 * FMAs / time.  No counterpart in the reference. */
int wadg_probe_fp64_fma(void *stream, int iters, double *tflops, float *ms);

#ifdef __cplusplus
}
#endif

#endif
