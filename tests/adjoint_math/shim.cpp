// Host build of the adjoint's node-level derivative formulas
// (scratch_wadge_b200/csrc/wadg_adjoint_math.cuh) for the CPU tests: each
// entry point evaluates one forward map or its vector-Jacobian product on
// plain arrays, so that Python can compare it with central differences.
#include "../../scratch_wadge_b200/csrc/wadg_adjoint_math.cuh"

using namespace wadg::adj;

namespace {
Gas gas(double g) { return Gas{g, g - 1.0, 1.0 / (2.0 * (g - 1.0)), std::log(g - 1.0), 1.0 / (g - 1.0)}; }

template <int D> void flux(const double *A, const double *B, const double *n, double g, double *F) {
  flux_fwd<D>(prim<D>(A, gas(g)), prim<D>(B, gas(g)), n, gas(g), F);
}
template <int D>
void flux_vjp_cons(const double *A, const double *B, const double *n, const double *c, double g,
                   double *gA, double *gB) {
  PrimBar<D> ba, bb;
  zero(ba);
  zero(bb);
  flux_vjp<D>(prim<D>(A, gas(g)), prim<D>(B, gas(g)), n, gas(g), c, ba, bb);
  prim_vjp<D>(A, ba, gas(g), gA);
  prim_vjp<D>(B, bb, gas(g), gB);
}
}  // namespace

extern "C" {
void am_flux(int dim, const double *A, const double *B, const double *n, double g, double *F) {
  dim == 3 ? flux<3>(A, B, n, g, F) : flux<2>(A, B, n, g, F);
}
void am_flux_vjp(int dim, const double *A, const double *B, const double *n, const double *c,
                 double g, double *gA, double *gB) {
  dim == 3 ? flux_vjp_cons<3>(A, B, n, c, g, gA, gB) : flux_vjp_cons<2>(A, B, n, c, g, gA, gB);
}
double am_lambda(int dim, const double *U, double g, double *dl) {
  return dim == 3 ? lambda_d<3>(U, gas(g), dl) : lambda_d<2>(U, gas(g), dl);
}
void am_VU(int dim, const double *U, double g, double *V) {
  dim == 3 ? V_of_U<3>(U, gas(g), V) : V_of_U<2>(U, gas(g), V);
}
void am_UV(int dim, const double *V, double g, double *U) {
  dim == 3 ? U_of_V<3>(V, gas(g), U) : U_of_V<2>(V, gas(g), U);
}
void am_VU_vjp(int dim, const double *U, const double *Vb, double g, double *Ub) {
  dim == 3 ? VU_vjp<3>(U, Vb, gas(g), Ub) : VU_vjp<2>(U, Vb, gas(g), Ub);
}
void am_UV_vjp(int dim, const double *V, const double *Ub, double g, double *Vb) {
  dim == 3 ? UV_vjp<3>(V, Ub, gas(g), Vb) : UV_vjp<2>(V, Ub, gas(g), Vb);
}
void am_UV_vjp_U(int dim, const double *U, const double *Ub, double g, double *Vb) {
  dim == 3 ? UV_vjp_U<3>(U, Ub, gas(g), Vb) : UV_vjp_U<2>(U, Ub, gas(g), Vb);
}
}
